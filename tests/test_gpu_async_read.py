"""The queued per-generation objective read equals the waiting one."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_read_objectives_async_matches(pe, gpu):
    import torch
    aa = pe.synthetic_protein(120, 3)
    with pe.Engine(aa, pe.dirichlet_table(3), 3, 48, 0.05, objectives=1, ref_p=3, seed=9) as eng:
        eng.init()
        ring = [torch.empty((96, 4), dtype=torch.float32, pin_memory=True) for _ in range(2)]
        snaps = []
        for g in range(4):
            eng.step(1)
            eng.read_objectives_async(ring[g & 1].data_ptr())
            if g & 1:                                   # both buffers filled: check them
                eng.synchronize()
                snaps.append([r.numpy().copy() for r in ring])
        want = eng.objectives()
        assert np.array_equal(snaps[-1][1].view(np.uint32), want.view(np.uint32))   # the last generation
        assert not np.array_equal(snaps[-1][0], snaps[-1][1])                      # the one before it differs
