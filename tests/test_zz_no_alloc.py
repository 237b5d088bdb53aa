"""pe_hairpin_noalloc: the allocation-free stem evaluation, for callers that may not
allocate device memory (a host application whose memory manager already holds
the GPU, or a loop that cannot pay cudaMalloc/cudaFree).

Checked through the C ABI against the allocating evaluator (pe_eval_objectives)
and the oracle's serial stem sweep on the same solutions, two calls in a row;
and, after the set-up call, that a call leaves the device's free memory
unchanged.  The test itself allocates the input and output buffers, as such a
caller's host application would.  This file is collected last."""
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


class _Buffers:
    def __init__(self, torch, nt):
        n, m, n_nt = nt.shape
        dev = torch.device("cuda", 0)
        self.n, self.m, self.L = n, m, n_nt // 3
        self.nt = torch.from_numpy(nt).to(dev)
        self.val = torch.zeros(n, dtype=torch.float32, device=dev)
        self.pql = torch.zeros((n, 3), dtype=torch.int32, device=dev)
        self.cds = torch.zeros(n, dtype=torch.int8, device=dev)
        self.stream = torch.cuda.current_stream(dev)

    def call(self, pe):
        pe.hairpin_noalloc(self.nt.data_ptr(), self.n, self.m, self.L, self.val.data_ptr(), self.pql.data_ptr(),
                           self.cds.data_ptr(), self.stream.cuda_stream)
        self.stream.synchronize()

    def result(self):
        return self.val.cpu().numpy(), self.cds.cpu().numpy(), self.pql.cpu().numpy()


def test_noalloc_matches_allocating_evaluator_and_oracle_twice(pe, orc, gpu):
    import torch
    # the set-up call: loads the code and reserves the fixed scratch on this device
    pe.hairpin_noalloc(0, 0, 2, 3, 0, 0, 0, 0)
    for seed, L, m, n in ((3, 201, 2, 96), (4, 1001, 8, 24)):
        aa, tabc, ids, nt = _batch(pe, seed, L, m, n)
        want = _reference_values(pe, aa, tabc, ids)
        buf = _Buffers(torch, nt)
        buf.call(pe)
        got = buf.result()
        assert np.array_equal(got[0].view(np.uint32), want[0].view(np.uint32)), "stem values"
        assert np.array_equal(got[1], want[1]), "stem CDS"
        assert np.array_equal(got[2], want[2]), "stem p, q, length"
        # the oracle's serial sweep of every CDS gives the same stem lengths
        longest = np.array([max(orc.sl_serial_one(nt[i, c]) for c in range(m)) for i in range(n)])
        assert np.array_equal(got[2][:, 2], longest)


def test_noalloc_call_leaves_free_device_memory_unchanged(pe, gpu):
    import torch
    aa, tabc, ids, nt = _batch(pe, 5, 301, 4, 64)
    buf = _Buffers(torch, nt)
    buf.call(pe)                      # first call on the device: the scratch is in place after it
    first = buf.result()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    buf.call(pe)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    second = buf.result()
    for a, b in zip(first, second):
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_noalloc_rejects_oversized_requests(pe, gpu):
    import torch
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.int32, device=dev)
    p = buf.data_ptr()
    with pytest.raises(pe.PeError) as e:
        pe.hairpin_noalloc(p, 100000, 8, 1001, p, p, p, torch.cuda.current_stream(dev).cuda_stream)
    assert e.value.code == 1 and "scratch" in str(e.value)
