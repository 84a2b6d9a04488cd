"""Bounded device waits: a wait that runs out is reported, not hung on.

Every wait in the field kernels is bounded (staged-copy mbarriers of both
engines, the wavefront engine's neighbour counters).  dtmx_set_wait_limit
lowers the bound so that the waits run out in an ordinary launch: the CTA
then stops issuing copies, waits for those in flight and returns, the next
dtmx_sync reports DTMX_ERR_TIMEOUT, and the context stays usable -- with the
bound restored, a run from the same state gives the same fields as a context
that never timed out.  Nothing here faults or hangs a GPU: the kernels still
only touch their own buffers, and every wait, the drains included, ends.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(engine, T=0):
    from dtmaxwell4_b200 import Simulation, abi
    # no absorber: a run that timed out leaves no auxiliary state behind that set_field would not reset
    cfg = abi.make_config(48, 64, 80, dx=1.0, courant=0.5, order=2, absorber=abi.ABS_NONE)
    s = Simulation(cfg)
    rng = np.random.default_rng(3)
    fields = [rng.standard_normal(s.shape).astype(np.float32) for _ in range(6)]
    for c in range(6):
        s.set_field(c, fields[c])
    s.set_engine(engine, T)
    return s, fields


# The wavefront engine's neighbour waits run out deterministically with a
# one-poll bound (a neighbour tile is never that far ahead).  A staged-copy
# wait of the per-step engines does not: mbarrier.try_wait suspends the thread
# until the copy lands within its time slice, so one poll succeeds and those
# engines' give-up path is built but not exercised here.
@pytest.mark.parametrize("engine,T", [(2, 4), (2, 1)])
def test_wait_runs_out_reports_timeout_and_context_recovers(engine, T):
    from dtmaxwell4_b200 import abi, engine as eng
    ref, fields = _sim(engine, T)
    ref.step(8)
    ref.sync()
    want = [ref.get_field(c) for c in range(6)]
    ref.close()

    s, _ = _sim(engine, T)
    s.set_wait_limit(1)            # one poll: a staged copy or a neighbour is never that quick
    s.step(8)
    with pytest.raises(eng.DtmxError) as e:
        s.sync()
    assert e.value.code == abi.ERR_TIMEOUT
    # the context is usable again: default bound, same start state, same result
    s.set_wait_limit(0)
    s.sync()
    for c in range(6):
        s.set_field(c, fields[c])
    s.step(8)
    s.sync()
    for c in range(6):
        got = s.get_field(c)
        assert np.array_equal(got, want[c]), c
    s.close()
