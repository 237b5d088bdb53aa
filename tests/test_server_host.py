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

    def __init__(self, aa, table, m, N, pm, objectives=1, seed=0):
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


def test_nondominated_and_normalisation():
    srv_mod = _server_mod()
    pts = np.array([[0.1, 0.5], [0.2, 0.2], [0.3, 0.3], [0.1, 0.5], [0.6, 0.1]])
    nd = srv_mod.nondominated(pts)
    assert sorted(map(tuple, nd)) == [(0.1, 0.5), (0.2, 0.2), (0.6, 0.1)]
    obj = np.array([[-0.8, -0.3, 0.1, 0.2], [-1.2, 0.1, 0.9, -0.1]], np.float32)
    v = srv_mod.normalised(obj, 1)
    # mCAI 0.8 -> (0.8-1)/(0-1) = 0.2; mHD 0.3 -> (0.3-0.4)/(0-0.4) = 0.25; MGC 0.1/0.6; MSL 0.2
    assert np.allclose(v[0], [0.2, 0.25, 0.1 / 0.6, 0.2], atol=1e-6)
    assert v[1, 0] == 0.0 and v[1, 1] == np.float32(0.999999) and v[1, 2] == np.float32(0.999999) and v[1, 3] == 0.0
