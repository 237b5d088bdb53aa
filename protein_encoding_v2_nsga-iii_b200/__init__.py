"""Python binding of the B200 NSGA-III codon-design engine (C ABI in include/pe_nsga3.h).

The reference (CAU-HPCL/Protein_encoding_v2_NSGA-III) is driven by its command
line ``Protein_NSGA3 <fasta> <N> <G> <m> <Pm>`` (src/main.cu:456-489) and by its
device-function signatures.  :class:`Engine` mirrors that run surface (one
protein, N solutions of m CDSs, G generations, mutation probability Pm); the
operator-level methods (:meth:`Engine.evaluate`, :meth:`Engine.mutate`,
:meth:`Engine.select`) expose the reference's evaluators, mutation dispatch and
sorting kernel one at a time.

The CUDA library is required: every compute call goes to ``lib/libpe_nsga3.so``;
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libpe_nsga3.so"
CLI_PATH = PKG_DIR / "lib" / "pe_nsga3"
HEADER = PKG_DIR.parent / "include" / "pe_nsga3.h"

AMINO = "ACDEFGHIKLMNPQRSTVWYZ"
NT = "ACGU"
OBJ_REF6, OBJ_BASE4 = 0, 1
GC3, GC_ALL = 0, 1
# string objective in the stem slot: the reference's hairpin stem, or the longest
# repeated/common substring (see pe_string_objective in the header)
SL_HAIRPIN, SL_LRCS = 0, 1
# slot layout per objective set (kinds: CAI CBP HSC HD GC SL)
OBJ_NAMES = {OBJ_REF6: ["mCAI", "mCBP", "mHSC", "mHD", "MGC", "MSL"], OBJ_BASE4: ["mCAI", "mHD", "MGC", "MSL"]}

STATUS = {0: "OK", 1: "bad argument", 2: "out of memory", 3: "CUDA error", 4: "device wait timed out",
          5: "call out of order", 6: "I/O error", 7: "no CUDA device"}


class PeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class CodonTable(C.Structure):
    _fields_ = [("nt", (C.c_uint8 * 3) * 64), ("weight", C.c_float * 64), ("cps", C.c_float * (61 * 61)),
                ("start", C.c_int8 * 21), ("count", C.c_int8 * 21), ("ref_gc3", C.c_float), ("ref_gc", C.c_float)]

    def arrays(self) -> dict:
        """numpy views of the table (copies)."""
        return {
            "nt": np.ctypeslib.as_array(self.nt).reshape(64, 3).astype(np.uint8).copy(),
            "weight": np.ctypeslib.as_array(self.weight).astype(np.float32).copy(),
            "cps": np.ctypeslib.as_array(self.cps).astype(np.float32).copy(),
            "start": np.ctypeslib.as_array(self.start).astype(np.int8).copy(),
            "count": np.ctypeslib.as_array(self.count).astype(np.int8).copy(),
            "ref_gc3": float(self.ref_gc3), "ref_gc": float(self.ref_gc),
        }

    @classmethod
    def from_arrays(cls, a: dict) -> "CodonTable":
        t = cls()
        np.ctypeslib.as_array(t.nt).reshape(64, 3)[:] = np.asarray(a["nt"], np.uint8).reshape(64, 3)
        np.ctypeslib.as_array(t.weight)[:] = np.asarray(a["weight"], np.float32)
        np.ctypeslib.as_array(t.cps)[:] = np.asarray(a["cps"], np.float32).reshape(-1)
        np.ctypeslib.as_array(t.start)[:] = np.asarray(a["start"], np.int8)
        np.ctypeslib.as_array(t.count)[:] = np.asarray(a["count"], np.int8)
        t.ref_gc3 = a["ref_gc3"]
        t.ref_gc = a["ref_gc"]
        return t

    def codon_strings(self) -> list[str]:
        nt = np.ctypeslib.as_array(self.nt).reshape(64, 3)
        return ["".join(NT[b] for b in row) for row in nt]


class Config(C.Structure):
    _fields_ = [("n_cds", C.c_int32), ("pop_size", C.c_int32), ("mutation_prob", C.c_float),
                ("objectives", C.c_int32), ("gc_mode", C.c_int32), ("ref_p", C.c_int32), ("seed", C.c_uint64),
                ("stream_priority", C.c_int32), ("sl_threads", C.c_int32), ("sl_kind", C.c_int32)]


class Info(C.Structure):
    _fields_ = [("L", C.c_int32), ("m", C.c_int32), ("N", C.c_int32), ("M", C.c_int32), ("R", C.c_int32),
                ("p", C.c_int32), ("generation", C.c_uint32), ("initialized", C.c_int32),
                ("device_bytes", C.c_uint64), ("sl_threads", C.c_int32)]


class ServerConfig(C.Structure):
    _fields_ = [("memory_budget", C.c_uint64), ("max_active", C.c_int32), ("tick", C.c_int32),
                ("hv_every", C.c_int32), ("order", C.c_int32), ("max_wait_s", C.c_double),
                ("priorities", C.c_int32)]


class JobSpec(C.Structure):
    _fields_ = [("cfg", Config), ("aa_idx", C.c_void_p), ("aa_len", C.c_int32), ("table", C.POINTER(CodonTable)),
                ("generations", C.c_int32), ("stall", C.c_int32), ("keep_codons", C.c_int32)]


class JobStatus(C.Structure):
    _fields_ = [("state", C.c_int32), ("reason", C.c_int32), ("generations_run", C.c_int32),
                ("priority", C.c_int32), ("hypervolume", C.c_double), ("submitted_s", C.c_double),
                ("started_s", C.c_double), ("finished_s", C.c_double), ("device_bytes", C.c_uint64),
                ("error", C.c_char * 256)]


class ServerStats(C.Structure):
    _fields_ = [("queued", C.c_int32), ("active", C.c_int32), ("peak_active", C.c_int32),
                ("used_bytes", C.c_uint64), ("peak_used_bytes", C.c_uint64), ("memory_budget", C.c_uint64)]


JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED, JOB_CANCELLED = range(5)
REASONS = {-1: None, 0: "budget", 1: "stall", 2: "error", 3: "cancelled"}
ORDER_ARRIVAL, ORDER_SHORTEST = 0, 1


class SelectInfo(C.Structure):
    _fields_ = [("rank_count", C.c_int32), ("last_front_size", C.c_int32), ("n_fronts", C.c_int32),
                ("cut", C.c_int32), ("hyp_exception", C.c_int32), ("ideal", C.c_float * 6),
                ("worst", C.c_float * 6), ("nadir", C.c_float * 6)]


_lib = None


def lib() -> C.CDLL:
    """Load the in-tree engine library (fails loudly when it is missing)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}`")
        L = C.CDLL(str(LIB_PATH))
        P = C.c_void_p
        sig = {
            "pe_create": [C.POINTER(Config), P, C.c_int32, C.POINTER(CodonTable), P, C.POINTER(P)],
            "pe_destroy": [P], "pe_get_info": [P, C.POINTER(Info)], "pe_init_population": [P],
            "pe_step": [P, C.c_int32], "pe_synchronize": [P],
            "pe_get_population": [P, P, P, P, P, P], "pe_get_objectives": [P, P],
            "pe_read_objectives_async": [P, P],
            "pe_eval_objectives": [P, P, C.c_int32, P, P, P],
            "pe_mutate": [P, C.c_uint32, P, C.c_int32, P, P, P, P, P, P],
            "pe_select": [P, C.c_uint32, P, P, P, P, C.POINTER(SelectInfo)],
            "pe_reference_points": [C.c_int32, C.c_int32, P, C.POINTER(C.c_int32)],
            "pe_parse_fasta": [C.c_char_p, P, C.c_int32, C.POINTER(C.c_int32)],
            "pe_synthetic_protein": [C.c_int32, C.c_uint64, P],
            "pe_dirichlet_table": [C.c_uint64, C.POINTER(CodonTable)],
            "pe_load_codon_table": [C.c_char_p, C.POINTER(CodonTable)],
            "pe_hypervolume": [P, C.c_int32, C.c_int32, P, C.POINTER(C.c_double)],
            "pe_set_profiling": [P, C.c_int32], "pe_stage_times": [P, P], "pe_scan_count": [P, P],
            "pe_scan_cells": [P, P], "pe_set_wait_limit": [P, C.c_int32],
            "pe_scan_fallbacks": [P, P], "pe_set_scan_method": [P, C.c_int32],
            "pe_hairpin_noalloc": [P, C.c_int32, C.c_int32, C.c_int32, P, P, P, P],
            "pe_batch_create": [P, C.c_int32, C.POINTER(P)], "pe_batch_step": [P, C.c_int32],
            "pe_batch_synchronize": [P], "pe_batch_destroy": [P], "pe_batch_set_scan_queue": [P, C.c_int32],
            "pe_instance_bytes": [C.POINTER(Config), C.c_int32, C.POINTER(C.c_uint64)],
            "pe_server_create": [C.POINTER(ServerConfig), C.POINTER(P)],
            "pe_batch_submit": [P, C.POINTER(JobSpec), C.POINTER(C.c_int64)],
            "pe_poll": [P, C.c_int64, C.POINTER(JobStatus)], "pe_job_result": [P, C.c_int64, P, P],
            "pe_cancel": [P, C.c_int64], "pe_server_clock": [P, C.POINTER(C.c_double)],
            "pe_server_get_stats": [P, C.POINTER(ServerStats)], "pe_server_drain": [P, C.c_double],
            "pe_server_destroy": [P],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.pe_last_error.restype = C.c_char_p
        L.pe_version.restype = C.c_char_p
        _lib = L
    return _lib


def _ck(code: int):
    if code != 0:
        raise PeError(code, lib().pe_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def declared_symbols() -> list[str]:
    """Function names declared in include/pe_nsga3.h."""
    import re
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(pe_[a-z_0-9]+)\s*\(", text, re.M)))


# ----------------------------------------------------------------- inputs

def synthetic_protein(L: int, seed: int) -> np.ndarray:
    """L amino acids i.i.d. uniform over the 20 standard letters, then the stop (index 20)."""
    out = np.zeros(L + 1, np.int8)
    _ck(lib().pe_synthetic_protein(L, seed, _ptr(out)))
    return out


def dirichlet_table(seed: int) -> CodonTable:
    t = CodonTable()
    _ck(lib().pe_dirichlet_table(seed, C.byref(t)))
    return t


def load_codon_table(path) -> CodonTable:
    t = CodonTable()
    _ck(lib().pe_load_codon_table(str(path).encode(), C.byref(t)))
    return t


def parse_fasta(path) -> np.ndarray:
    n = C.c_int32(0)
    _ck(lib().pe_parse_fasta(str(path).encode(), None, 0, C.byref(n)))
    out = np.zeros(n.value, np.int8)
    _ck(lib().pe_parse_fasta(str(path).encode(), _ptr(out), n.value, C.byref(n)))
    return out


def reference_points(M: int, p: int) -> np.ndarray:
    R = C.c_int32(0)
    _ck(lib().pe_reference_points(M, p, None, C.byref(R)))
    out = np.zeros((R.value, M), np.float32)
    _ck(lib().pe_reference_points(M, p, _ptr(out), C.byref(R)))
    return out


def hairpin_noalloc(d_nt: int, n_solutions: int, m: int, L: int, d_value: int, d_pql: int, d_cds: int,
                    stream: int = 0):
    """Allocation-free stem evaluation on device pointers (see pe_hairpin_noalloc)."""
    _ck(lib().pe_hairpin_noalloc(C.c_void_p(d_nt), n_solutions, m, L, C.c_void_p(d_value), C.c_void_p(d_pql),
                                 C.c_void_p(d_cds), C.c_void_p(stream) if stream else None))


def instance_bytes(aa_len: int, n_cds: int, pop_size: int, objectives: int = OBJ_BASE4, ref_p: int = 0,
                   sl_kind: int = SL_HAIRPIN) -> int:
    """Device bytes an Engine of this shape allocates (admission by memory footprint)."""
    cfg = Config(n_cds, pop_size, 0.0, objectives, GC3, ref_p, 0, 0, 0, sl_kind)
    out = C.c_uint64(0)
    _ck(lib().pe_instance_bytes(C.byref(cfg), aa_len, C.byref(out)))
    return out.value


def hypervolume(points, ref) -> float:
    pts = np.ascontiguousarray(points, np.float64)
    ref = np.ascontiguousarray(ref, np.float64)
    out = C.c_double(0.0)
    _ck(lib().pe_hypervolume(_ptr(pts), pts.shape[0], pts.shape[1], _ptr(ref), C.byref(out)))
    return out.value


# ----------------------------------------------------------------- engine

class Engine:
    """One protein-design instance resident on the current CUDA device."""

    def __init__(self, aa, table: CodonTable, n_cds: int, pop_size: int, mutation_prob: float,
                 objectives: int = OBJ_BASE4, gc_mode: int = GC3, ref_p: int = 0, seed: int = 0, stream=None,
                 stream_priority: int = 0, sl_threads: int = 0, sl_kind: int = SL_HAIRPIN):
        self.aa = np.ascontiguousarray(aa, np.int8)
        self.table = table
        self.sl_kind = sl_kind
        cfg = Config(n_cds, pop_size, mutation_prob, objectives, gc_mode, ref_p, seed, stream_priority, sl_threads,
                     sl_kind)
        h = C.c_void_p()
        _ck(lib().pe_create(C.byref(cfg), _ptr(self.aa), len(self.aa), C.byref(table),
                            None if stream is None else C.c_void_p(stream), C.byref(h)))
        self._h = h
        info = Info()
        _ck(lib().pe_get_info(h, C.byref(info)))
        self.L, self.m, self.N, self.M, self.R, self.p = info.L, info.m, info.N, info.M, info.R, info.p
        self.device_bytes = int(info.device_bytes)

    def close(self):
        if getattr(self, "_h", None):
            lib().pe_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def generation(self) -> int:
        info = Info()
        _ck(lib().pe_get_info(self._h, C.byref(info)))
        return info.generation

    @property
    def sl_threads(self) -> int:
        """Hairpin-scan CTA size in use (picked by timing at init unless forced)."""
        info = Info()
        _ck(lib().pe_get_info(self._h, C.byref(info)))
        return info.sl_threads

    def init(self):
        _ck(lib().pe_init_population(self._h))

    def step(self, generations: int = 1):
        _ck(lib().pe_step(self._h, generations))

    def synchronize(self):
        _ck(lib().pe_synchronize(self._h))

    def set_profiling(self, enable: bool = True):
        _ck(lib().pe_set_profiling(self._h, int(enable)))

    def stage_times(self):
        """Device ms of (variation + light evaluation, hairpin scan, selection) in the last generation."""
        out = np.zeros(3, np.float32)
        _ck(lib().pe_stage_times(self._h, _ptr(out)))
        return out

    def scan_count(self) -> int:
        """String-objective scans run so far: CDSs (hairpin) or CDS pairs (LRCS); a child's
        unchanged CDS (pair) keeps its parent's result."""
        v = C.c_uint64(0)
        _ck(lib().pe_scan_count(self._h, C.byref(v)))
        return v.value

    def set_wait_limit(self, polls: int):
        """Polls of the bounded device waits (0 default, < 0: give up at once; tests)."""
        _ck(lib().pe_set_wait_limit(self._h, polls))

    def scan_cells(self) -> int:
        """Counted cells of those scans (the string-objective kernel's unit of work)."""
        v = C.c_uint64(0)
        _ck(lib().pe_scan_cells(self._h, C.byref(v)))
        return v.value

    def scan_fallbacks(self) -> int:
        """Scans whose seeded first pass gave up on a repetitive CDS (the band scan ran)."""
        v = C.c_uint64(0)
        _ck(lib().pe_scan_fallbacks(self._h, C.byref(v)))
        return v.value

    def set_scan_method(self, method: int):
        """First pass of the string scan: 0 seeded (default), 1 band scan for every CDS."""
        _ck(lib().pe_set_scan_method(self._h, method))

    def population(self):
        N2 = 2 * self.N
        ids = np.zeros((N2, self.m, self.L), np.uint8)
        obj = np.zeros((N2, self.M), np.float32)
        objidx = np.zeros((N2, 2 * self.M), np.int8)
        pql = np.zeros((N2, 3), np.int32)
        surv = np.zeros(self.N, np.int32)
        _ck(lib().pe_get_population(self._h, _ptr(ids), _ptr(obj), _ptr(objidx), _ptr(pql), _ptr(surv)))
        return ids, obj, objidx, pql, surv

    def objectives(self, out=None):
        out = np.zeros((2 * self.N, self.M), np.float32) if out is None else out
        _ck(lib().pe_get_objectives(self._h, _ptr(out)))
        return out

    def read_objectives_async(self, out_ptr: int):
        """Queue the objective read (2N x M float32) into the host memory at out_ptr
        without waiting; it holds them after synchronize().  Page-locked memory (e.g.
        a pinned torch tensor's data_ptr()) lets the copy overlap the next generations."""
        _ck(lib().pe_read_objectives_async(self._h, C.c_void_p(out_ptr)))

    def survivor_objectives(self):
        """Objectives of the N solutions the last selection kept (the next parents)."""
        obj = np.zeros((2 * self.N, self.M), np.float32)
        surv = np.zeros(self.N, np.int32)
        _ck(lib().pe_get_population(self._h, None, _ptr(obj), None, None, _ptr(surv)))
        return obj[surv] if self.generation > 0 else obj[: self.N]

    def evaluate(self, ids):
        ids = np.ascontiguousarray(ids, np.uint8).reshape(-1, self.m, self.L)
        n = ids.shape[0]
        obj = np.zeros((n, self.M), np.float32)
        objidx = np.zeros((n, 2 * self.M), np.int8)
        pql = np.zeros((n, 3), np.int32)
        _ck(lib().pe_eval_objectives(self._h, _ptr(ids), n, _ptr(obj), _ptr(objidx), _ptr(pql)))
        return obj, objidx, pql

    def mutate(self, generation: int, idx, parents, pobj, pobjidx, ppql):
        parents = np.ascontiguousarray(parents, np.uint8).reshape(-1, self.m, self.L)
        n = parents.shape[0]
        idx = np.ascontiguousarray(idx, np.int32)
        pobj = np.ascontiguousarray(pobj, np.float32)
        pobjidx = np.ascontiguousarray(pobjidx, np.int8)
        ppql = np.ascontiguousarray(ppql, np.int32)
        child = np.zeros_like(parents)
        ops = np.zeros(n, np.int32)
        _ck(lib().pe_mutate(self._h, generation, _ptr(idx), n, _ptr(parents), _ptr(pobj), _ptr(pobjidx),
                            _ptr(ppql), _ptr(child), _ptr(ops)))
        return child, ops

    def select(self, generation: int, obj, extremes):
        obj = np.ascontiguousarray(obj, np.float32)
        ext = np.array(extremes, np.float32, copy=True).reshape(self.M, self.M)
        surv = np.zeros(self.N, np.int32)
        front = np.zeros(2 * self.N, np.int32)
        info = SelectInfo()
        _ck(lib().pe_select(self._h, generation, _ptr(obj), _ptr(ext), _ptr(surv), _ptr(front), C.byref(info)))
        return surv, front, ext, info


class Batch:
    """Independent design jobs advanced together: one CUDA graph launch per two
    generations, one concurrent branch per instance (pe_batch_* in the C ABI)."""

    def __init__(self, engines):
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e._h.value for e in self.engines])
        h = C.c_void_p()
        _ck(lib().pe_batch_create(arr, len(self.engines), C.byref(h)))
        self._h = h

    def step(self, generations: int = 1):
        _ck(lib().pe_batch_step(self._h, generations))

    def set_scan_queue(self, enable: bool = True):
        """Queued string scans for the whole batch, or (the default) one scan launch per member."""
        _ck(lib().pe_batch_set_scan_queue(self._h, int(enable)))

    def synchronize(self):
        _ck(lib().pe_batch_synchronize(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().pe_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
