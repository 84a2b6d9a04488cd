"""Field drops in the reference's .arr layout and restartable state files."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim():
    from dtmaxwell4_b200 import Simulation, scenarios
    sc = scenarios.drude_sphere_tfsf(n=40, steps=80, pml=6, inset=5, radius=5, lambda0=12.0, nfreq=2)
    s = Simulation(sc["cfg"])
    scenarios.apply(s, sc)
    return s


def test_arr_layout(tmp_path):
    from dtmaxwell4_b200 import engine
    s = _sim()
    s.step(20)
    path = str(tmp_path / "ez.arr")
    s.write_arr(2, path)
    raw = np.fromfile(path, np.int32, count=9)
    assert list(raw) == [12, 0, 0, 0, 3, 4, 40, 40, 40]
    assert np.array_equal(engine.read_arr(path), s.get_field(2))
    s.close()


def test_state_file_resumes_bit_for_bit(tmp_path):
    from dtmaxwell4_b200 import DtmxError
    a = _sim()
    a.step(30)
    path = str(tmp_path / "run.state")
    a.save_state(path)
    a.step(25)
    b = _sim()
    b.load_state(path)
    b.step(25)
    for c in range(6):
        assert np.array_equal(a.get_field(c), b.get_field(c)), c
    from dtmaxwell4_b200 import Simulation, abi
    other = Simulation(abi.make_config(32, 32, 32))
    with pytest.raises(DtmxError):
        other.load_state(path)
    for q in (a, b, other):
        q.close()
