"""Runtime paths that must not change results: 16-step CUDA-graph replay of
the per-step launch sequence and the autotuner (every engine configuration
it may pick is bit-identical to the per-step engine)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _drude(n=48, steps=64):
    from dtmaxwell4_b200 import scenarios
    return scenarios.drude_sphere_tfsf(n=n, steps=steps, pml=6, inset=6, radius=6, lambda0=12.0, nfreq=3)


def _sim(sc):
    from dtmaxwell4_b200 import Simulation, scenarios
    s = Simulation(sc["cfg"])
    scenarios.apply(s, sc)
    return s


def test_graph_replay_matches_single_steps():
    sc = _drude()
    a, b = _sim(sc), _sim(sc)
    for _ in range(40):
        a.step(1)            # never aligned for a 16-step graph
    b.step(3)
    b.step(37)               # 3 single steps until the DFT staging realigns at 16, then a graph, then singles
    for c in range(6):
        assert np.array_equal(a.get_field(c), b.get_field(c)), c
    assert np.array_equal(a.read_probes(), b.read_probes())
    assert np.array_equal(a.read_dft(0), b.read_dft(0))
    a.close(); b.close()


def test_graph_replay_from_aligned_start():
    sc = _drude()
    a, b = _sim(sc), _sim(sc)
    for _ in range(48):
        a.step(1)
    b.step(48)               # three graph launches
    for c in range(6):
        assert np.array_equal(a.get_field(c), b.get_field(c)), c
    assert np.array_equal(a.read_dft(0), b.read_dft(0))
    a.close(); b.close()


def test_autotune_keeps_state_and_results():
    from dtmaxwell4_b200 import Simulation, abi
    cfg = abi.make_config(64, 64, 64, order=2, absorber=abi.ABS_CPML, pml=8)
    rng = np.random.default_rng(3)
    fields = [rng.standard_normal((64, 64, 64)).astype(np.float32) for _ in range(6)]
    a, b = Simulation(cfg), Simulation(cfg)
    for s in (a, b):
        for c in range(6):
            s.set_field(c, fields[c])
    eng, T, xc, ms = b.autotune(8)
    assert eng in (1, 2, 3) and ms > 0
    for c in range(6):
        assert np.array_equal(b.get_field(c), fields[c])
    a.step(20)
    b.step(20)
    for c in range(6):
        assert np.array_equal(a.get_field(c), b.get_field(c)), (c, eng, T, xc)
    a.close(); b.close()
