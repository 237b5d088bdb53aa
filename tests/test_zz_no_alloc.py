"""pe_hairpin_noalloc: the allocation-free stem evaluation for callers that may not
allocate device memory, checked against the allocating evaluator
(pe_eval_objectives) on the same solutions, two calls in a row.  The test itself
allocates its input/output buffers (as such a caller's host application would)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(pe, seed, L, m, n):
    tabc = pe.dirichlet_table(seed)
    tab = tabc.arrays()
    aa = pe.synthetic_protein(L - 1, seed)
    rng = np.random.default_rng(seed)
    ids = np.stack([np.stack([tab["start"][aa] + (rng.random(L) * tab["count"][aa]).astype(np.int64)
                              for _ in range(m)]) for _ in range(n)]).astype(np.uint8)
    ids[1, 1] = ids[1, 0]
    nt = np.asarray(tab["nt"])[ids].reshape(n, m, 3 * L).astype(np.uint8)
    return aa, tabc, ids, nt


def _reference_values(pe, aa, tabc, ids):
    m = ids.shape[1]
    with pe.Engine(aa, tabc, m, 8, 0.05, objectives=pe.OBJ_BASE4, ref_p=2) as eng:
        obj, objidx, pql = eng.evaluate(ids)
    return obj[:, 3], objidx[:, 6], pql


def _noalloc(pe, torch, nt):
    n, m, n_nt = nt.shape
    dev = torch.device("cuda", 0)
    d_nt = torch.from_numpy(nt).to(dev)
    d_val = torch.zeros(n, dtype=torch.float32, device=dev)
    d_pql = torch.zeros((n, 3), dtype=torch.int32, device=dev)
    d_cds = torch.zeros(n, dtype=torch.int8, device=dev)
    stream = torch.cuda.current_stream(dev)
    pe.hairpin_noalloc(d_nt.data_ptr(), n, m, n_nt // 3, d_val.data_ptr(), d_pql.data_ptr(), d_cds.data_ptr(),
                       stream.cuda_stream)
    stream.synchronize()
    return d_val.cpu().numpy(), d_cds.cpu().numpy(), d_pql.cpu().numpy()


def test_noalloc_matches_allocating_evaluator_twice(pe, gpu):
    import torch
    for seed, L, m, n in ((3, 201, 2, 96), (4, 1001, 8, 24)):
        aa, tabc, ids, nt = _batch(pe, seed, L, m, n)
        want = _reference_values(pe, aa, tabc, ids)
        got = _noalloc(pe, torch, nt)
        assert np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32)), "stem values"
        assert np.array_equal(got[1], want[1]), "stem CDS"
        assert np.array_equal(got[2], want[2]), "stem p, q, length"


def test_noalloc_rejects_oversized_requests(pe, gpu):
    import torch
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.int32, device=dev)
    p = buf.data_ptr()
    with pytest.raises(pe.PeError) as e:
        pe.hairpin_noalloc(p, 100000, 8, 1001, p, p, p, torch.cuda.current_stream(dev).cuda_stream)
    assert e.value.code == 1 and "scratch" in str(e.value)
