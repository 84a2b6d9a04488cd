"""The allocation-free NaN/Inf count (dtmx_count_nonfinite_noalloc) against the
context's own check (dtmx_check_finite), on two calls in a row, and its size
limit.

The entry point exists for callers that cannot allocate device memory (their
pool is owned by another allocator, or they run in a health-check thread that
must stay out of the allocator): they hand in their own device arrays and get
a host count back, while the reduction's scratch is a fixed array inside the
library.  This file is collected last so that a run stopping at the first
failure has already run every other test.

The limit cases run on the CPU: the size check comes before any CUDA call, so
the pointers handed in are never dereferenced and need not be device memory.
"""
import numpy as np
import pytest


def _fields(sim):
    ptrs, n = [], None
    for c in range(6):
        p, st = sim.device_ptr(c)
        ptrs.append(p)
        n = sim.cfg.nx * st[0]          # padded storage of one component
    return ptrs, n


def _lib_or_skip():
    from dtmaxwell4_b200 import engine
    try:
        engine.load()
    except OSError as e:
        pytest.skip(str(e))
    return engine


def test_noalloc_limit_counts_blocks_per_field():
    """Each field is rounded up to whole blocks on its own: 6 fields of
    2,796,202 floats are 16,777,212 floats in all (under 2^24) but need
    6 * 683 = 4098 blocks, more than the scratch holds -> TOO_LARGE."""
    from dtmaxwell4_b200 import abi
    engine = _lib_or_skip()
    fake = [0x1000 * (f + 1) for f in range(6)]          # never dereferenced: rejected first
    n = 2796202
    assert 6 * n <= abi.NOALLOC_MAX_ELEMS
    assert 6 * -(-n // abi.NOALLOC_BLOCK_ELEMS) > abi.NOALLOC_MAX_BLOCKS
    rc, _ = engine.count_nonfinite_noalloc(fake, n)
    assert rc == abi.ERR_TOO_LARGE
    # one block more than fits, spread over fields of whole blocks
    rc, _ = engine.count_nonfinite_noalloc(fake[:1], abi.NOALLOC_MAX_ELEMS + 1)
    assert rc == abi.ERR_TOO_LARGE
    rc, _ = engine.count_nonfinite_noalloc(fake[:2], abi.NOALLOC_MAX_ELEMS // 2 + 1)
    assert rc == abi.ERR_TOO_LARGE
    # sizes whose products overflow 64 bits are rejected, not wrapped
    rc, _ = engine.count_nonfinite_noalloc(fake[:2], 1 << 62)
    assert rc == abi.ERR_TOO_LARGE
    rc, _ = engine.count_nonfinite_noalloc(fake[:1], (1 << 63) - 1)
    assert rc == abi.ERR_TOO_LARGE


def test_noalloc_limit_accepts_exactly_the_maximum():
    """Exactly DTMX_NOALLOC_MAX_ELEMS in one field (4096 whole blocks), and 6
    fields of 682 whole blocks, pass the size check: without a GPU the call
    then stops at the device lookup, never at TOO_LARGE."""
    from dtmaxwell4_b200 import abi
    import torch
    if torch.cuda.is_available():
        pytest.skip("the accepted sizes would launch on real memory; covered by the GPU test")
    engine = _lib_or_skip()
    fake = [0x1000 * (f + 1) for f in range(6)]
    rc, _ = engine.count_nonfinite_noalloc(fake[:1], abi.NOALLOC_MAX_ELEMS)
    assert rc == abi.ERR_NODEVICE
    rc, _ = engine.count_nonfinite_noalloc(fake, 682 * abi.NOALLOC_BLOCK_ELEMS)
    assert rc == abi.ERR_NODEVICE


@pytest.mark.gpu
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
    sim.sync()
    rc, count = engine.count_nonfinite_noalloc(ptrs, n)
    assert rc == abi.OK
    assert sim.check_finite() is False
    assert count == 10

    # call 2: every field finite again; the shared scratch keeps nothing from call 1
    for c in range(6):
        sim.set_field(c, clean[c])
    sim.sync()
    rc, count = engine.count_nonfinite_noalloc(ptrs, n)
    assert rc == abi.OK
    assert sim.check_finite() is True
    assert count == 0

    # sizes beyond the fixed scratch are rejected before any launch
    rc, _ = engine.count_nonfinite_noalloc(ptrs, abi.NOALLOC_MAX_ELEMS)
    assert rc == abi.ERR_TOO_LARGE
    sim.close()
