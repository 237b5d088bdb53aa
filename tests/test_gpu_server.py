"""Served mode on the device: each job's result is the same alone and in the mix."""
import numpy as np
import pytest

from conftest import load_pkg_module

pytestmark = pytest.mark.gpu


def _server_mod():
    return load_pkg_module("server")


SPECS = [(180, 3, 64, 23, 101), (60, 2, 32, 37, 102), (400, 5, 128, 19, 103), (90, 8, 48, 31, 104), (250, 2, 96, 28, 105)]


@pytest.mark.parametrize("repeat", range(3))
def test_results_same_alone_and_in_mix(pe, gpu, repeat):
    srv_mod = _server_mod()
    jobs = []
    for L, m, N, G, seed in SPECS:
        jobs.append(srv_mod.Job(pe.synthetic_protein(L, seed), pe.dirichlet_table(seed), m, N, G, seed, stall=0,
                                arrival=0.0))
    budget = sum(pe.instance_bytes(len(j.aa), j.n_cds, j.pop_size) for j in jobs[:3])
    srv = srv_mod.Server(pe, memory_budget=budget, max_active=3, tick=7, keep_population=True)
    done = srv.run(jobs)
    assert len(done) == len(SPECS) and [j.error for j in done if j.error] == []
    assert srv.peak_active <= 3 and srv.peak_used <= budget and srv.used == 0
    for job in done:
        assert job.reason == "budget" and job.generations_run == job.generations, job.error
        with pe.Engine(job.aa, job.table, job.n_cds, job.pop_size, job.mutation_prob, objectives=job.objectives,
                       seed=job.seed) as e:
            e.init()
            e.step(job.generations)
            alone = e.population()
        for k in range(5):
            a, w = np.asarray(job.population[k]), np.asarray(alone[k])
            if a.dtype.kind == "f":
                a, w = a.view(np.uint32), w.view(np.uint32)
            assert np.array_equal(a, w), (job.job_id, k)
    stats = srv_mod.latency_stats(done)
    assert stats["p99_s"] >= stats["p50_s"] > 0


def test_stall_retirement(pe, gpu):
    srv_mod = _server_mod()
    job = srv_mod.Job(pe.synthetic_protein(12, 7), pe.dirichlet_table(7), 2, 16, 2000, 7, stall=50)
    srv = srv_mod.Server(pe, memory_budget=1 << 30, tick=25, hv_every=25)
    done = srv.run([job])
    j = done[0]
    assert j.reason in ("stall", "budget") and 0.0 < j.hv <= 1.0
    if j.reason == "stall":
        assert j.generations_run - j._best_gen >= 50 and j.generations_run < 2000


@pytest.mark.parametrize("L,m,N,obj,p", [(60, 2, 32, 1, 0), (1000, 8, 1024, 1, 8), (200, 3, 128, 0, 0), (3000, 4, 96, 0, 2)])
def test_instance_bytes_matches_allocation(pe, gpu, L, m, N, obj, p):
    aa = pe.synthetic_protein(L, 5)
    with pe.Engine(aa, pe.dirichlet_table(5), m, N, 0.02, objectives=obj, ref_p=p, seed=5) as e:
        assert e.device_bytes == pe.instance_bytes(len(aa), m, N, obj, ref_p=p)


def _alone_survivors(pe, job):
    with pe.Engine(job.aa, job.table, job.n_cds, job.pop_size, job.mutation_prob, objectives=job.objectives,
                   seed=job.seed) as e:
        e.init()
        e.step(job.generations)
        ids, obj, _, _, surv = e.population()
    return ids[surv], obj[surv]


def test_native_server_results_same_alone_and_in_mix(pe, gpu):
    """The C++ serving core (pe_batch_submit / pe_poll / pe_job_result): every job's
    survivors equal the same job run alone."""
    srv_mod = _server_mod()
    jobs = [srv_mod.Job(pe.synthetic_protein(L, seed), pe.dirichlet_table(seed), m, N, G, seed, stall=0,
                        arrival=0.01 * k)
            for k, (L, m, N, G, seed) in enumerate(SPECS)]
    budget = sum(pe.instance_bytes(len(j.aa), j.n_cds, j.pop_size) for j in jobs[:3])
    srv = srv_mod.NativeServer(pe, memory_budget=budget, max_active=3, tick=7, keep_population=True)
    done = srv.run(jobs)
    st = srv.stats()
    srv.close()
    assert len(done) == len(SPECS) and [j.error for j in done if j.error] == []
    assert 1 <= st.peak_active <= 3 and st.peak_used_bytes <= budget and st.used_bytes == 0
    for job in done:
        assert job.reason == "budget" and job.generations_run == job.generations
        ids, obj = _alone_survivors(pe, job)
        codons, sobj = job.population
        assert np.array_equal(codons, ids), job.job_id
        assert np.array_equal(sobj.view(np.uint32), obj.view(np.uint32)), job.job_id
        assert 0.0 < job.hv <= 1.0
    assert srv_mod.latency_stats(done)["p99_s"] > 0


def test_native_server_cancels_a_running_job(pe, gpu):
    srv_mod = _server_mod()
    srv = srv_mod.NativeServer(pe, memory_budget=1 << 32, max_active=2, tick=5)
    long_job = srv_mod.Job(pe.synthetic_protein(400, 3), pe.dirichlet_table(3), 4, 256, 100000, 3, stall=0)
    short = srv_mod.Job(pe.synthetic_protein(50, 4), pe.dirichlet_table(4), 2, 32, 20, 4, stall=0)
    srv.submit(long_job)
    srv.submit(short)
    import time
    t0 = time.time()
    while srv.status(long_job).generations_run < 10 and time.time() - t0 < 60:
        time.sleep(0.01)
    srv.cancel(long_job)
    while srv.status(long_job).state == pe.JOB_RUNNING and time.time() - t0 < 60:
        time.sleep(0.01)
    st = srv.status(long_job)
    assert st.state == pe.JOB_CANCELLED and pe.REASONS[st.reason] == "cancelled"
    assert 10 <= st.generations_run < 100000
    while srv.status(short).state in (pe.JOB_QUEUED, pe.JOB_RUNNING) and time.time() - t0 < 60:
        time.sleep(0.01)
    assert srv.status(short).state == pe.JOB_DONE
    assert srv.stats().used_bytes == 0
    srv.close()


def test_native_server_stall_retirement(pe, gpu):
    srv_mod = _server_mod()
    job = srv_mod.Job(pe.synthetic_protein(12, 7), pe.dirichlet_table(7), 2, 16, 2000, 7, stall=50)
    srv = srv_mod.NativeServer(pe, memory_budget=1 << 30, tick=25, hv_every=25)
    done = srv.run([job])
    srv.close()
    j = done[0]
    assert j.reason in ("stall", "budget") and 0.0 < j.hv <= 1.0
    if j.reason == "stall":
        assert j.generations_run < 2000 and j.generations_run % 25 == 0
