"""Served design jobs on one GPU: continuous batching.

The reference runs one protein per process (src/main.cu:467-901).  Here design
requests arrive over time and share the device:

* admission by device footprint (pe_instance_bytes) against a memory budget and
  by a cap on resident jobs, in arrival order or shortest estimated work first
  (a job that has waited longer than `max_wait` seconds goes ahead of both); the
  chosen job waits until enough memory is released;
* every resident job keeps its population on the device, owns a stream and is
  driven by its own host thread, which replays the job's generation graphs
  `tick` generations at a time; the blocking calls release the interpreter
  lock, so the kernels of all resident jobs overlap on the GPU and a long job
  never holds back a short one;
* a job retires when it reaches its generation budget, or when the hypervolume
  of its survivors' normalised objectives (the measure of src/main.cu:789-858)
  has not improved for `stall` generations, checked every `hv_every`
  generations; the job waits for each check, so where it stops does not depend
  on timing;
* each job's stream gets a priority from its estimated work (counted cells of
  the stem scan over its generation budget): the block scheduler then serves
  the kernels of short jobs first and fills the rest of the GPU with long ones
  (shortest-job-first at CTA granularity), instead of slowing every job down
  equally;
* latency = time the result is on the host - arrival time; p50/p99 and designs/s.

A job's result does not depend on what else is resident: every draw is keyed by
(job seed, generation, individual, position) and each generation runs the same
kernels as a job alone.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass

import numpy as np

# normalisation constants: six objectives src/main.cu:23-24; four objectives
# src/auto_execution_experiments.py:47-48 (mCAI, mHD, MGC, MSL)
IDEAL = {0: np.array([1.0, 0.2, 0.4, 0.5, 0.0, 0.0], np.float32), 1: np.array([1.0, 0.4, 0.0, 0.0], np.float32)}
NADIR = {0: np.array([0.0, -0.15, 0.0, 0.0, 0.6, 1.0], np.float32), 1: np.array([0.0, 0.0, 0.6, 1.0], np.float32)}
N_MAXIMISED = {0: 4, 1: 2}


def normalised(obj: np.ndarray, objectives: int) -> np.ndarray:
    """Stored objectives -> the reference's normalised, clamped form."""
    v = np.array(obj, np.float32, copy=True)
    v[:, :N_MAXIMISED[objectives]] *= -1.0
    v = (v - IDEAL[objectives]) / (NADIR[objectives] - IDEAL[objectives])
    v = np.where(v >= 1.0, np.float32(0.999999), v)
    return np.where(v < 0.0, np.float32(0.0), v).astype(np.float32)


def estimated_cells(job) -> float:
    """Counted cells of the stem scan over the job's whole generation budget (the
    scan dominates a generation's device time)."""
    k = 3 * len(job.aa) - 5
    return float(job.pop_size) * job.n_cds * k * (k + 1) / 2 * job.generations


def work_priority(job, levels: int = 6) -> int:
    """Stream priority by estimated work: one level per decade of counted cells
    from 1e10 up; -(levels-1) (most urgent) for the smallest jobs, 0 for the largest."""
    decade = int(np.floor(np.log10(max(estimated_cells(job), 1.0)))) - 10
    return -(levels - 1) + min(max(decade, 0), levels - 1)


def front_hypervolume(pe, obj: np.ndarray, objectives: int) -> float:
    """Hypervolume of the normalised points w.r.t. (1, ..., 1) (pe_hypervolume drops
    the dominated ones itself)."""
    pts = normalised(obj, objectives).astype(np.float64)
    return pe.hypervolume(pts, np.ones(pts.shape[1]))


@dataclass(eq=False)
class Job:
    aa: np.ndarray
    table: object
    n_cds: int
    pop_size: int
    generations: int
    seed: int
    objectives: int = 1
    mutation_prob: float = 0.02
    stall: int = 50                 # 0 disables the stall rule
    arrival: float = 0.0            # seconds from the start of the run
    sl_kind: int = 0                # string objective: 0 hairpin stem, 1 longest repeated/common substring
    job_id: int = -1
    # filled by the server
    submitted: float | None = None
    start: float | None = None
    end: float | None = None
    generations_run: int = 0
    hv: float | None = None
    reason: str | None = None       # "budget", "stall" or "error"
    error: str | None = None
    survivors: np.ndarray | None = None    # survivors' objectives
    population: tuple | None = None
    priority: int = 0
    gpu_s: float = 0.0              # host time in generation launches + waits
    read_s: float = 0.0             # host time reading survivors for stall checks
    hv_s: float = 0.0               # host time computing their hypervolume
    _best_hv: float = -1.0
    _best_gen: int = 0


class Server:
    def __init__(self, pe, memory_budget: int, max_active: int = 64, tick: int = 10, hv_every: int = 25,
                 keep_population: bool = False, priority=work_priority, order: str = "arrival",
                 max_wait: float | None = None):
        if order not in ("arrival", "shortest"):
            raise ValueError("order must be 'arrival' or 'shortest'")
        self.pe = pe
        self.priority = priority      # job -> stream priority, or None for equal priorities
        self.order = order
        self.max_wait = max_wait
        self.memory_budget = int(memory_budget)
        self.max_active = max_active
        self.tick = tick
        self.hv_every = hv_every
        self.keep_population = keep_population
        self.queue: deque[Job] = deque()
        self.active: list[Job] = []
        self.done: list[Job] = []
        self.used = 0
        self.peak_used = 0
        self.peak_active = 0
        self._next_id = 0
        self._cv = threading.Condition()
        self._threads: list[threading.Thread] = []
        self.t0 = None

    # ------------------------------------------------------------ bookkeeping
    def now(self) -> float:
        return time.perf_counter() - self.t0

    def footprint(self, job: Job) -> int:
        return self.pe.instance_bytes(len(job.aa), job.n_cds, job.pop_size, job.objectives)

    def submit(self, job: Job) -> int:
        if self.t0 is None:
            self.t0 = time.perf_counter()
        if self.footprint(job) > self.memory_budget:
            raise ValueError("job needs more device memory than the whole budget")
        with self._cv:
            if job.job_id < 0:
                job.job_id = self._next_id
                self._next_id += 1
            job.submitted = self.now()
            self.queue.append(job)
            self._admit_locked()
        return job.job_id

    def _next_locked(self) -> Job:
        if self.max_wait is not None:
            now = self.now()
            for job in self.queue:  # arrival order
                if now - job.submitted > self.max_wait:
                    return job
        if self.order == "shortest":
            return min(self.queue, key=estimated_cells)
        return self.queue[0]

    def _admit_locked(self):
        while self.queue and len(self.active) < self.max_active:
            job = self._next_locked()
            need = self.footprint(job)
            if self.used + need > self.memory_budget:
                break  # the chosen job waits for memory
            self.queue.remove(job)
            self.used += need
            self.peak_used = max(self.peak_used, self.used)
            self.active.append(job)
            self.peak_active = max(self.peak_active, len(self.active))
            job.start = self.now()
            t = threading.Thread(target=self._serve, args=(job,), daemon=True)
            self._threads.append(t)
            t.start()

    # ------------------------------------------------------------ one job
    def _serve(self, job: Job):
        eng = None
        try:
            job.priority = self.priority(job) if self.priority else 0
            eng = self.pe.Engine(job.aa, job.table, job.n_cds, job.pop_size, job.mutation_prob,
                                 objectives=job.objectives, seed=job.seed, stream_priority=job.priority)
            eng.init()
            job.reason = "budget"
            while job.generations_run < job.generations:
                g = min(self.tick, job.generations - job.generations_run)
                if job.stall:
                    g = min(g, self.hv_every - job.generations_run % self.hv_every)
                t0 = time.perf_counter()
                eng.step(g)
                eng.synchronize()
                t1 = time.perf_counter()
                job.gpu_s += t1 - t0
                job.generations_run += g
                if job.stall and job.generations_run % self.hv_every == 0 and job.generations_run < job.generations:
                    surv = eng.survivor_objectives()
                    t2 = time.perf_counter()
                    hv = front_hypervolume(self.pe, surv, job.objectives)
                    job.read_s += t2 - t1
                    job.hv_s += time.perf_counter() - t2
                    if hv > job._best_hv + 1e-12:
                        job._best_hv, job._best_gen = hv, job.generations_run
                    elif job.generations_run - job._best_gen >= job.stall:
                        job.reason = "stall"
                        break
            job.survivors = eng.survivor_objectives()
            if self.keep_population:
                job.population = eng.population()
            job.end = self.now()
        except Exception as exc:  # the job fails alone; the server keeps serving
            job.reason, job.error, job.end = "error", repr(exc), self.now()
        finally:
            if eng is not None:
                eng.close()
            with self._cv:
                self.used -= self.footprint(job)
                self.active.remove(job)
                self.done.append(job)
                self._admit_locked()
                self._cv.notify_all()

    # ------------------------------------------------------------ driving
    def run(self, jobs: list[Job]) -> list[Job]:
        """Serve `jobs` with real-time arrivals (job.arrival seconds after the
        start); returns the finished jobs in completion order, each with the
        hypervolume of its final survivors."""
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        self.t0 = time.perf_counter()
        while pending:
            wait = pending[0].arrival - self.now()
            if wait > 0:
                time.sleep(wait)
            while pending and pending[0].arrival <= self.now():
                self.submit(pending.popleft())
        self.drain()
        for job in self.done:
            if job.survivors is not None and job.hv is None:
                job.hv = front_hypervolume(self.pe, job.survivors, job.objectives)
        return self.done

    def drain(self):
        """Block until every submitted job has finished."""
        with self._cv:
            while self.queue or self.active:
                self._cv.wait(timeout=1.0)
        for t in self._threads:
            t.join()
        self._threads.clear()


def latency_stats(done: list[Job]) -> dict:
    lat = np.array([j.end - j.arrival for j in done])
    span = max(j.end for j in done) - min(j.arrival for j in done)
    return {"jobs": len(done), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "designs_per_s": len(done) / span, "span_s": span,
            "stalled": sum(j.reason == "stall" for j in done), "failed": sum(j.reason == "error" for j in done),
"host_hv_s": float(sum(j.hv_s for j in done)), "host_read_s": float(sum(j.read_s for j in done)),
            "gpu_wait_s": float(sum(j.gpu_s for j in done))}



class NativeServer:
    """The same served mode run by the library's own serving core (pe_server_create,
    pe_batch_submit, pe_poll, pe_job_result, pe_cancel in include/pe_nsga3.h): this
    class only submits jobs at their arrival times and reads their status and
    results; admission, the per-job host threads, stall checks and retirement run in
    C++.  Same constructor arguments and run() contract as Server; `priority` is a
    switch here (the core derives each job's stream priority from its estimated work)."""

    def __init__(self, pe, memory_budget: int, max_active: int = 64, tick: int = 10, hv_every: int = 25,
                 keep_population: bool = False, priority=True, order: str = "arrival",
                 max_wait: float | None = None, poll_s: float = 0.001):
        if order not in ("arrival", "shortest"):
            raise ValueError("order must be 'arrival' or 'shortest'")
        self.pe = pe
        self.keep_population = keep_population
        self.poll_s = poll_s
        cfg = pe.ServerConfig(int(memory_budget), max_active, tick, hv_every,
                              pe.ORDER_SHORTEST if order == "shortest" else pe.ORDER_ARRIVAL,
                              float(max_wait or 0.0), 1 if priority else 0)
        h = pe.C.c_void_p()
        pe._ck(pe.lib().pe_server_create(pe.C.byref(cfg), pe.C.byref(h)))
        self._h = h
        self._jobs: dict[int, Job] = {}
        self._keep = []   # host buffers the core copies at submit (kept until then)
        self.peak_active = 0
        self.peak_used = 0
        self.used = 0

    def clock(self) -> float:
        v = self.pe.C.c_double(0.0)
        self.pe._ck(self.pe.lib().pe_server_clock(self._h, self.pe.C.byref(v)))
        return v.value

    def stats(self):
        st = self.pe.ServerStats()
        self.pe._ck(self.pe.lib().pe_server_get_stats(self._h, self.pe.C.byref(st)))
        return st

    def submit(self, job: Job) -> int:
        pe = self.pe
        aa = np.ascontiguousarray(job.aa, np.int8)
        cfg = pe.Config(job.n_cds, job.pop_size, job.mutation_prob, job.objectives, pe.GC3, 0, job.seed, 0, 0,
                        getattr(job, "sl_kind", 0))
        spec = pe.JobSpec(cfg, aa.ctypes.data_as(pe.C.c_void_p), len(aa), pe.C.pointer(job.table), job.generations,
                          job.stall, 1 if self.keep_population else 0)
        jid = pe.C.c_int64(0)
        pe._ck(pe.lib().pe_batch_submit(self._h, pe.C.byref(spec), pe.C.byref(jid)))
        job.job_id = int(jid.value)
        self._jobs[job.job_id] = job
        return job.job_id

    def cancel(self, job: Job):
        self.pe._ck(self.pe.lib().pe_cancel(self._h, job.job_id))

    def status(self, job: Job):
        st = self.pe.JobStatus()
        self.pe._ck(self.pe.lib().pe_poll(self._h, job.job_id, self.pe.C.byref(st)))
        return st

    def _collect(self, job: Job, st, t0: float):
        pe = self.pe
        job.generations_run = st.generations_run
        job.reason = pe.REASONS.get(st.reason)
        job.priority = st.priority
        job.submitted = st.submitted_s - t0
        job.start = st.started_s - t0 if st.started_s >= 0 else None
        job.end = st.finished_s - t0
        if st.state == pe.JOB_FAILED:
            job.error = st.error.decode()
        if st.state == pe.JOB_DONE:
            M = 4 if job.objectives == pe.OBJ_BASE4 else 6
            obj = np.zeros((job.pop_size, M), np.float32)
            codons = np.zeros((job.pop_size, job.n_cds, len(job.aa)), np.uint8) if self.keep_population else None
            pe._ck(pe.lib().pe_job_result(self._h, job.job_id, obj.ctypes.data_as(pe.C.c_void_p),
                                          None if codons is None else codons.ctypes.data_as(pe.C.c_void_p)))
            job.survivors = obj
            job.hv = st.hypervolume
            if codons is not None:
                job.population = (codons, obj)

    def run(self, jobs: list[Job]) -> list[Job]:
        """Serve `jobs` with real-time arrivals (job.arrival seconds after the start);
        returns the finished jobs in completion order."""
        pe = self.pe
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        t0 = self.clock()
        live: list[Job] = []
        done: list[Job] = []
        while pending or live:
            now = self.clock() - t0
            while pending and pending[0].arrival <= now:
                job = pending.popleft()
                self.submit(job)
                live.append(job)
            st_all = self.stats()
            self.peak_active = max(self.peak_active, st_all.peak_active)
            self.peak_used = max(self.peak_used, st_all.peak_used_bytes)
            still = []
            for job in live:
                st = self.status(job)
                if st.state in (pe.JOB_DONE, pe.JOB_FAILED, pe.JOB_CANCELLED):
                    self._collect(job, st, t0)
                    done.append(job)
                else:
                    still.append(job)
            live = still
            if pending or live:
                wait = self.poll_s
                if pending and not live:
                    wait = max(0.0, pending[0].arrival - (self.clock() - t0))
                time.sleep(min(wait, 0.05) if live else wait)
        st_all = self.stats()
        self.used = st_all.used_bytes
        return done

    def close(self):
        if getattr(self, "_h", None):
            self.pe.lib().pe_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
