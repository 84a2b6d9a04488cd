"""Batched forward + adjoint of independent instances of uneven sizes: the
interleaved batch returns exactly what separate runs return."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _make(sc):
    from dtmaxwell4_b200 import Simulation, scenarios
    s = Simulation(sc["cfg"])
    scenarios.apply(s, sc)
    s.set_design(*sc["design"])
    return s


@pytest.mark.parametrize("budget", [-1, 0])
def test_batch_equals_separate_runs(budget):
    """budget -1: recorded design histories; 0: checkpointed recompute in the batch."""
    from dtmaxwell4_b200 import engine, scenarios
    scs = [scenarios.design_block_instance(seed, edges=(40, 48, 56, 64), pml=6, design=6, steps=48, nblocks=3)
           for seed in range(5)]
    shapes = {(sc["cfg"].nx, sc["cfg"].ny, sc["cfg"].nz) for sc in scs}
    assert len(shapes) > 1
    sims = [_make(sc) for sc in scs]
    for s in sims:
        s.set_adjoint_memory(budget)
    J, G = engine.batch_forward_adjoint(sims, 48, [sc["plane_x"] for sc in scs], [sc["omega"] for sc in scs],
                                        checkpoint_every=20)
    for b, sc in enumerate(scs):
        s = _make(sc)
        Jb, gb = s.forward_adjoint(48, sc["plane_x"], sc["omega"], 20)
        assert J[b] == Jb and np.array_equal(G[b], gb), b
        for c in range(6):
            assert np.array_equal(s.get_field(c), sims[b].get_field(c))
        s.close()
        sims[b].close()
