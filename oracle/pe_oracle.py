"""ctypes binding of the CPU oracle (pe_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by the tests, the smoke entry and the CPU
baseline leg of the benchmark, never by the engine.  Build: ``make -C oracle``.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB = ORACLE_DIR / "_build" / "libpe_oracle.so"


class OrTable(C.Structure):
    _fields_ = [("nt", (C.c_uint8 * 3) * 64), ("weight", C.c_float * 64), ("cps", C.c_float * (61 * 61)),
                ("start", C.c_int8 * 21), ("count", C.c_int8 * 21), ("ref_gc3", C.c_float), ("ref_gc", C.c_float)]


class OrProblem(C.Structure):
    _fields_ = [("L", C.c_int), ("m", C.c_int), ("N", C.c_int), ("objset", C.c_int), ("gcmode", C.c_int),
                ("p", C.c_int), ("pm", C.c_float), ("seed", C.c_uint64), ("aa", C.c_void_p),
                ("tab", C.POINTER(OrTable)), ("slkind", C.c_int)]


class OrSelectInfo(C.Structure):
    _fields_ = [("rank_count", C.c_int32), ("last_front_size", C.c_int32), ("n_fronts", C.c_int32),
                ("cut", C.c_int32), ("hyp_exception", C.c_int32), ("ideal", C.c_float * 6),
                ("worst", C.c_float * 6), ("nadir", C.c_float * 6)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        P = C.c_void_p
        L.or_num_obj.argtypes = [C.c_int]
        L.or_slot_of.argtypes = [C.c_int, C.c_int]
        L.or_num_ref.argtypes = [C.c_int, C.c_int]
        L.or_auto_p.argtypes = [C.c_int, C.c_int]
        L.or_das_dennis.argtypes = [C.c_int, C.c_int, P]
        L.or_philox4x32_10.argtypes = [P, P, P]
        L.or_draw.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32]
        L.or_draw.restype = C.c_uint32
        L.or_det_exp.argtypes = [C.c_double]
        L.or_det_exp.restype = C.c_double
        L.or_gen_solution.argtypes = [C.POINTER(OrProblem), C.c_int, P]
        L.or_eval.argtypes = [C.POINTER(OrProblem), P, P, P, P]
        L.or_mutate.argtypes = [C.POINTER(OrProblem), C.c_uint32, C.c_int, P, P, P, P, P]
        L.or_sl_serial_one.argtypes = [P, C.c_int]
        L.or_lrcs.argtypes = [P, C.c_int, C.c_int, P]
        L.or_lrcs_pair.argtypes = [P, P, C.c_int, C.c_int, P]
        L.or_select.argtypes = [C.POINTER(OrProblem), C.c_uint32, P, P, P, C.c_int, P, P, C.POINTER(OrSelectInfo)]
        L.or_create.argtypes = [C.POINTER(OrProblem)]
        L.or_create.restype = C.c_void_p
        L.or_destroy.argtypes = [P]
        L.or_init.argtypes = [P, C.c_int]
        L.or_generation.argtypes = [P, C.c_int]
        L.or_get.argtypes = [P, P, P, P, P, P, P, P]
        L.or_eval_batch.argtypes = [C.POINTER(OrProblem), P, C.c_int, P, P, P, C.c_int]
        L.or_mutate_eval_batch.argtypes = [C.POINTER(OrProblem), C.c_uint32, P, C.c_int, P, P, P, P, P, P, P, P, P,
                                           C.c_int]
        L.or_sl_sample_batch.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P]
        L.or_mutate_eval_light_batch.argtypes = [C.POINTER(OrProblem), C.c_uint32, P, C.c_int, P, P, P, P, P, P, P,
                                                 P, C.c_int]
        L.or_synthetic_protein.argtypes = [C.c_int, C.c_uint64, P]
        L.or_dirichlet_table.argtypes = [C.c_uint64, C.POINTER(OrTable)]
        L.or_set_state.argtypes = [P, P, P, P, P, P, P, C.c_uint32]
        L.or_hypervolume.argtypes = [P, C.c_int, C.c_int, P]
        L.or_hypervolume.restype = C.c_double
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def make_table(arrays: dict) -> OrTable:
    t = OrTable()
    np.ctypeslib.as_array(t.nt).reshape(64, 3)[:] = np.asarray(arrays["nt"], np.uint8).reshape(64, 3)
    np.ctypeslib.as_array(t.weight)[:] = np.asarray(arrays["weight"], np.float32)
    np.ctypeslib.as_array(t.cps)[:] = np.asarray(arrays["cps"], np.float32).reshape(-1)
    np.ctypeslib.as_array(t.start)[:] = np.asarray(arrays["start"], np.int8)
    np.ctypeslib.as_array(t.count)[:] = np.asarray(arrays["count"], np.int8)
    t.ref_gc3 = arrays["ref_gc3"]
    t.ref_gc = arrays["ref_gc"]
    return t


class Problem:
    """A problem description shared by every oracle call."""

    def __init__(self, aa, table_arrays: dict, m: int, N: int, pm: float, objset: int = 1, gcmode: int = 0,
                 p: int = 0, seed: int = 0, slkind: int = 0):
        self.aa = np.ascontiguousarray(aa, np.int8)
        self.L = len(self.aa)
        self.m, self.N = m, N
        self.M = lib().or_num_obj(objset)
        if p <= 0:
            p = lib().or_auto_p(self.M, N)
        self.p = p
        self.R = lib().or_num_ref(self.M, p)
        self.tab = make_table(table_arrays)
        self.c = OrProblem(self.L, m, N, objset, gcmode, p, pm, seed, self.aa.ctypes.data_as(C.c_void_p),
                           C.pointer(self.tab), slkind)
        self.refpts = das_dennis(self.M, p)

    def slot(self, kind: int) -> int:
        return lib().or_slot_of(self.c.objset, kind)

    # --- operators
    def gen_solution(self, idx: int) -> np.ndarray:
        out = np.zeros((self.m, self.L), np.uint8)
        lib().or_gen_solution(C.byref(self.c), idx, _p(out))
        return out

    def evaluate(self, ids, threads: int = 0):
        ids = np.ascontiguousarray(ids, np.uint8).reshape(-1, self.m, self.L)
        n = ids.shape[0]
        obj = np.zeros((n, self.M), np.float32)
        objidx = np.zeros((n, 2 * self.M), np.int8)
        pql = np.zeros((n, 3), np.int32)
        lib().or_eval_batch(C.byref(self.c), _p(ids), n, _p(obj), _p(objidx), _p(pql), threads)
        return obj, objidx, pql

    def mutate(self, generation: int, idx, parents, pobj, pobjidx, ppql, threads: int = 0):
        parents = np.ascontiguousarray(parents, np.uint8).reshape(-1, self.m, self.L)
        n = parents.shape[0]
        idx = np.ascontiguousarray(idx, np.int32)
        child = np.zeros_like(parents)
        cobj = np.zeros((n, self.M), np.float32)
        cobjidx = np.zeros((n, 2 * self.M), np.int8)
        cpql = np.zeros((n, 3), np.int32)
        ops = np.zeros(n, np.int32)
        lib().or_mutate_eval_batch(C.byref(self.c), generation, _p(idx), n, _p(parents),
                                   _p(np.ascontiguousarray(pobj, np.float32)),
                                   _p(np.ascontiguousarray(pobjidx, np.int8)),
                                   _p(np.ascontiguousarray(ppql, np.int32)), _p(child), _p(cobj), _p(cobjidx),
                                   _p(cpql), _p(ops), threads)
        return child, ops, cobj, cobjidx, cpql

    def mutate_light(self, generation: int, idx, parents, pobj, pobjidx, ppql, threads: int = 0):
        """mutation + every objective except the hairpin stem (timing sample)"""
        parents = np.ascontiguousarray(parents, np.uint8).reshape(-1, self.m, self.L)
        n = parents.shape[0]
        idx = np.ascontiguousarray(idx, np.int32)
        child = np.zeros_like(parents)
        cobj = np.zeros((n, self.M), np.float32)
        cobjidx = np.zeros((n, 2 * self.M), np.int8)
        cpql = np.zeros((n, 3), np.int32)
        lib().or_mutate_eval_light_batch(C.byref(self.c), generation, _p(idx), n, _p(parents),
                                         _p(np.ascontiguousarray(pobj, np.float32)),
                                         _p(np.ascontiguousarray(pobjidx, np.int8)),
                                         _p(np.ascontiguousarray(ppql, np.int32)), _p(child), _p(cobj),
                                         _p(cobjidx), _p(cpql), threads)
        return child

    def select(self, generation: int, obj, extremes):
        obj = np.ascontiguousarray(obj, np.float32)
        ext = np.array(extremes, np.float32, copy=True).reshape(self.M, self.M)
        surv = np.zeros(self.N, np.int32)
        front = np.zeros(2 * self.N, np.int32)
        info = OrSelectInfo()
        lib().or_select(C.byref(self.c), generation, _p(obj), _p(ext), _p(self.refpts), self.R, _p(surv),
                        _p(front), C.byref(info))
        return surv, front, ext, info


class Run:
    """A whole oracle run (init + generations) on one problem."""

    def __init__(self, prob: Problem):
        self.prob = prob
        self.h = lib().or_create(C.byref(prob.c))

    def init(self, threads: int = 0):
        lib().or_init(self.h, threads)

    def generation(self, threads: int = 0):
        lib().or_generation(self.h, threads)

    def state(self):
        pr = self.prob
        N2 = 2 * pr.N
        ids = np.zeros((N2, pr.m, pr.L), np.uint8)
        obj = np.zeros((N2, pr.M), np.float32)
        objidx = np.zeros((N2, 2 * pr.M), np.int8)
        pql = np.zeros((N2, 3), np.int32)
        surv = np.zeros(pr.N, np.int32)
        ext = np.zeros((pr.M, pr.M), np.float32)
        gen = np.zeros(1, np.uint32)
        lib().or_get(self.h, _p(ids), _p(obj), _p(objidx), _p(pql), _p(surv), _p(ext), _p(gen))
        return ids, obj, objidx, pql, surv, ext, int(gen[0])

    def set_state(self, ids, obj, objidx, pql, survivors, extremes, generation: int):
        """Start the next generation from this 2N state (e.g. the CUDA engine's)."""
        pr = self.prob
        N2 = 2 * pr.N
        a = [np.ascontiguousarray(ids, np.uint8).reshape(N2, pr.m, pr.L),
             np.ascontiguousarray(obj, np.float32).reshape(N2, pr.M),
             np.ascontiguousarray(objidx, np.int8).reshape(N2, 2 * pr.M),
             np.ascontiguousarray(pql, np.int32).reshape(N2, 3),
             np.ascontiguousarray(survivors, np.int32).reshape(pr.N),
             np.ascontiguousarray(extremes, np.float32).reshape(pr.M, pr.M)]
        lib().or_set_state(self.h, *[_p(x) for x in a], generation)

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def synthetic_protein(L: int, seed: int) -> np.ndarray:
    """L amino indices uniform over the 20 standard letters, then the stop (index 20)."""
    out = np.zeros(L + 1, np.int8)
    lib().or_synthetic_protein(L, seed, _p(out))
    return out


def dirichlet_table(seed: int) -> dict:
    """Standard genetic code with Dirichlet(1) weights per amino acid (max 1, ascending
    inside each group) and seeded codon-pair scores, as the arrays Problem takes."""
    t = OrTable()
    lib().or_dirichlet_table(seed, C.byref(t))
    return {"nt": np.ctypeslib.as_array(t.nt).reshape(64, 3).astype(np.uint8).copy(),
            "weight": np.ctypeslib.as_array(t.weight).astype(np.float32).copy(),
            "cps": np.ctypeslib.as_array(t.cps).astype(np.float32).copy(),
            "start": np.ctypeslib.as_array(t.start).astype(np.int8).copy(),
            "count": np.ctypeslib.as_array(t.count).astype(np.int8).copy(),
            "ref_gc3": float(t.ref_gc3), "ref_gc": float(t.ref_gc)}


def das_dennis(M: int, p: int) -> np.ndarray:
    R = lib().or_num_ref(M, p)
    out = np.zeros((R, M), np.float32)
    lib().or_das_dennis(M, p, _p(out))
    return out


def philox(ctr, key) -> np.ndarray:
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    o = np.zeros(4, np.uint32)
    lib().or_philox4x32_10(_p(c), _p(k), _p(o))
    return o


def det_exp(x: float) -> float:
    return lib().or_det_exp(x)


def sl_serial_one(nt) -> int:
    nt = np.ascontiguousarray(nt, np.uint8)
    return lib().or_sl_serial_one(_p(nt), len(nt))


def lrcs(nt) -> tuple:
    """Longest repeated/common substring of m CDSs (rows of nt): (length, p, q, a, b)."""
    nt = np.ascontiguousarray(nt, np.uint8)
    out = np.zeros(5, np.int32)
    lib().or_lrcs(_p(nt), nt.shape[0], nt.shape[1], _p(out))
    return tuple(int(x) for x in out)


def lrcs_pair(sa, sb, self_pair: bool) -> tuple:
    """(length, delta, p) of one pair."""
    sa = np.ascontiguousarray(sa, np.uint8)
    sb = np.ascontiguousarray(sb, np.uint8)
    out = np.zeros(3, np.int32)
    lib().or_lrcs_pair(_p(sa), _p(sb), len(sa), int(self_pair), _p(out))
    return tuple(int(x) for x in out)


def sl_sample(nt_cds, offset: int, stride: int, threads: int = 0) -> np.ndarray:
    """serial stem sweep of each CDS (rows of nt_cds) on anti-diagonals offset, offset+stride, ..."""
    nt_cds = np.ascontiguousarray(nt_cds, np.uint8)
    out = np.zeros(nt_cds.shape[0], np.int32)
    lib().or_sl_sample_batch(_p(nt_cds), nt_cds.shape[0], nt_cds.shape[1], offset, stride, threads, _p(out))
    return out


def hypervolume(points, ref) -> float:
    pts = np.ascontiguousarray(points, np.float64)
    ref = np.ascontiguousarray(ref, np.float64)
    return lib().or_hypervolume(_p(pts), pts.shape[0], pts.shape[1], _p(ref))
