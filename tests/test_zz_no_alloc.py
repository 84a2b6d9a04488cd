"""The allocation-free NaN/Inf count (dtmx_count_nonfinite_noalloc) against the
context's own check (dtmx_check_finite), on two calls in a row.

The entry point exists for callers that cannot allocate device memory (their
pool is owned by another allocator, or they run in a health-check thread that
must stay out of the allocator): they hand in their own device arrays and get
a host count back, while the reduction's scratch is a fixed array inside the
library.  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fields(sim):
    ptrs, n = [], None
    for c in range(6):
        p, st = sim.device_ptr(c)
        ptrs.append(p)
        n = sim.cfg.nx * st[0]          # padded storage of one component
    return ptrs, n


def test_noalloc_count_matches_check_finite_twice():
    from dtmaxwell4_b200 import Simulation, abi, engine
    cfg = abi.make_config(32, 24, 40, courant=0.5, order=2, pml=4)
    sim = Simulation(cfg)
    rng = np.random.default_rng(7)
    clean = [rng.standard_normal(sim.shape).astype(np.float32) for _ in range(6)]
    ptrs, n = _fields(sim)

    # call 1: 7 NaN in Ex and 3 +/-Inf in Hz
    bad_ex, bad_hz = clean[0].copy(), clean[5].copy()
    bad_ex.reshape(-1)[rng.choice(bad_ex.size, 7, replace=False)] = np.nan
    idx = rng.choice(bad_hz.size, 3, replace=False)
    bad_hz.reshape(-1)[idx] = [np.inf, -np.inf, np.inf]
    for c in range(6):
        sim.set_field(c, clean[c])
    sim.set_field(abi.EX, bad_ex)
    sim.set_field(abi.HZ, bad_hz)
    rc, count = engine.count_nonfinite_noalloc(ptrs, n)
    assert rc == abi.OK
    assert sim.check_finite() is False
    assert count == 10

    # call 2: every field finite again; the shared scratch keeps nothing from call 1
    for c in range(6):
        sim.set_field(c, clean[c])
    rc, count = engine.count_nonfinite_noalloc(ptrs, n)
    assert rc == abi.OK
    assert sim.check_finite() is True
    assert count == 0

    # sizes beyond the fixed scratch are rejected before any launch
    rc, _ = engine.count_nonfinite_noalloc(ptrs, abi.NOALLOC_MAX_ELEMS)
    assert rc == abi.ERR_TOO_LARGE
    sim.close()
