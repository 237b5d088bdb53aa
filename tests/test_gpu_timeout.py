"""The bounded device wait's timeout path (the reference spins without a bound:
include/utils.cuh:873, include/sorting.cuh:939,949).  The stem scan's wait for its
staged planes is made to give up at once; pe_synchronize must report
PE_ERR_TIMEOUT, the GPU context must stay usable, and pe_init_population must
restart the instance as if it were new.  The wait returns: nothing faults or hangs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_wait_that_gives_up_reports_timeout_and_init_recovers(pe, gpu):
    tabc = pe.dirichlet_table(4)
    aa = pe.synthetic_protein(150, 4)
    with pe.Engine(aa, tabc, 3, 32, 0.05, objectives=1, ref_p=3, seed=4, sl_threads=128) as eng:
        eng.init()
        eng.set_wait_limit(-1)
        eng.step(1)
        with pytest.raises(pe.PeError) as e:
            eng.synchronize()
        assert e.value.code == 4
        # the status stays set until the instance restarts
        with pytest.raises(pe.PeError):
            eng.synchronize()
        eng.set_wait_limit(0)
        eng.init()
        eng.step(3)
        eng.synchronize()
        got = eng.population()
    with pe.Engine(aa, tabc, 3, 32, 0.05, objectives=1, ref_p=3, seed=4, sl_threads=128) as ref:
        ref.init()
        ref.step(3)
        want = ref.population()
    for a, b in zip(got, want):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
