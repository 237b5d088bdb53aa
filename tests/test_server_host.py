"""Scheduling logic of the served mode on CPU, with a fake engine standing in for the device."""
import threading

import numpy as np

from conftest import load_pkg_module


def _server_mod():
    return load_pkg_module("server")


class FakeEngine:
    lock = threading.Lock()
    live = 0
    peak = 0

    def __init__(self, aa, table, m, N, pm, objectives=1, seed=0, stream_priority=0):
        self.gen, self.N, self.seed = 0, N, seed
        with FakeEngine.lock:
            FakeEngine.live += 1
            FakeEngine.peak = max(FakeEngine.peak, FakeEngine.live)

    def init(self):
        pass

    def step(self, g):
        self.gen += g

    def synchronize(self):
        pass

    def survivor_objectives(self):
        # hypervolume rises until generation `seed`, then stays flat
        g = min(self.gen, self.seed)
        return np.full((self.N, 4), 0.5 + g * 1e-3, np.float32) * np.array([-1, -1, 0, 0], np.float32)

    def population(self):
        return (self.gen,)

    def close(self):
        with FakeEngine.lock:
            FakeEngine.live -= 1


class FakePe:
    Engine = FakeEngine

    @staticmethod
    def instance_bytes(L, m, N, objectives=1):
        return 1000 * m

    @staticmethod
    def hypervolume(pts, ref):
        return float(np.prod(ref - pts.min(0)))


def test_admission_budget_and_retirement():
    srv_mod = _server_mod()
    FakeEngine.live = FakeEngine.peak = 0
    srv = srv_mod.Server(FakePe, memory_budget=10000, max_active=3, tick=10, hv_every=25, keep_population=True)
    jobs = [srv_mod.Job(np.zeros(10, np.int8), None, n_cds=4, pop_size=8, generations=200, seed=s, stall=50)
            for s in (1000, 60, 1000, 30, 1000)]
    done = srv.run(jobs)
    assert len(done) == 5 and FakeEngine.live == 0
    assert srv.peak_used <= 10000 and srv.peak_active <= 2 and FakeEngine.peak <= 2    # 4000 B each
    by_id = {j.job_id: j for j in done}
    assert by_id[0].reason == "budget" and by_id[0].generations_run == 200 and by_id[0].population == (200,)
    # checks every 25 generations: the last rise is seen at 50 (seed 30) / 75 (seed 60)
    assert (by_id[3].reason, by_id[3].generations_run) == ("stall", 100)
    assert (by_id[1].reason, by_id[1].generations_run) == ("stall", 125)
    assert all(j.hv is not None and j.end >= j.start >= j.arrival for j in done)
    stats = srv_mod.latency_stats(done)
    assert stats["jobs"] == 5 and stats["p99_s"] >= stats["p50_s"] >= 0 and stats["stalled"] == 2


def test_admission_in_arrival_order():
    srv_mod = _server_mod()
    srv = srv_mod.Server(FakePe, memory_budget=8000, max_active=8)
    order = []
    big = srv_mod.Job(np.zeros(10, np.int8), None, n_cds=8, pop_size=8, generations=10, seed=1, stall=0)
    small = [srv_mod.Job(np.zeros(10, np.int8), None, n_cds=2, pop_size=8, generations=10, seed=1, stall=0)
             for _ in range(3)]
    srv.t0 = 0.0
    with srv._cv:   # hold the lock: nothing retires while the queue is built
        srv.t0 = __import__("time").perf_counter()
        srv.queue.extend([small[0], big, small[1]])
        srv._admit_locked()
        order = [j for j in srv.active]
    assert order == [small[0]]            # big (8000 B) waits behind small[0]; small[1] waits behind big
    srv.drain()
    assert srv.peak_used <= 8000 and {id(j) for j in srv.done} == {id(small[0]), id(big), id(small[1])}


def test_failed_job_does_not_stop_server():
    srv_mod = _server_mod()

    class Bad(FakePe):
        class Engine(FakeEngine):
            def step(self, g):
                raise RuntimeError("device error")

    srv = srv_mod.Server(Bad, memory_budget=1 << 20)
    done = srv.run([srv_mod.Job(np.zeros(4, np.int8), None, 2, 8, 30, 1)])
    assert done[0].reason == "error" and "device error" in done[0].error and srv.used == 0 and FakeEngine.live == 0


def test_normalisation():
    srv_mod = _server_mod()
    obj = np.array([[-0.8, -0.3, 0.1, 0.2], [-1.2, 0.1, 0.9, -0.1]], np.float32)
    v = srv_mod.normalised(obj, 1)
    # mCAI 0.8 -> (0.8-1)/(0-1) = 0.2; mHD 0.3 -> (0.3-0.4)/(0-0.4) = 0.25; MGC 0.1/0.6; MSL 0.2
    assert np.allclose(v[0], [0.2, 0.25, 0.1 / 0.6, 0.2], atol=1e-6)
    assert v[1, 0] == 0.0 and v[1, 1] == np.float32(0.999999) and v[1, 2] == np.float32(0.999999) and v[1, 3] == 0.0


def test_work_priority_orders_by_size():
    srv_mod = _server_mod()
    small = srv_mod.Job(np.zeros(51, np.int8), None, 2, 256, 200, 1)
    mid = srv_mod.Job(np.zeros(1001, np.int8), None, 8, 1024, 500, 1)
    big = srv_mod.Job(np.zeros(5001, np.int8), None, 10, 2048, 1000, 1)
    pr = [srv_mod.work_priority(j) for j in (small, mid, big)]
    assert pr[0] == -5 and pr[0] < pr[1] < pr[2] and pr[2] == 0
    assert srv_mod.estimated_cells(mid) == 1024 * 8 * 2998 * 2999 / 2 * 500


def test_shortest_first_admission_and_max_wait():
    srv_mod = _server_mod()
    srv = srv_mod.Server(FakePe, memory_budget=1 << 20, max_active=1, order="shortest")
    sizes = [400, 60, 200, 60]
    jobs = [srv_mod.Job(np.zeros(L, np.int8), None, 2, 8, 10, 1, stall=0) for L in sizes]
    import time
    srv.t0 = time.perf_counter()
    with srv._cv:   # queue all four before any is admitted
        for j in jobs:
            j.job_id = srv._next_id
            srv._next_id += 1
            j.submitted = srv.now()
            srv.queue.append(j)
        first = srv._next_locked()
    assert first is jobs[1]                      # smallest, earliest of the two smallest
    srv.max_wait = 0.0                           # everything has waited: arrival order wins
    with srv._cv:
        assert srv._next_locked() is jobs[0]
        srv.max_wait = None
        srv._admit_locked()
    srv.drain()
    order = [j.job_id for j in sorted(srv.done, key=lambda j: j.start)]
    assert order == [1, 3, 2, 0]
