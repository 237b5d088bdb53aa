"""The library's serving core through its C ABI, on CPU: submission, polling and
cancellation of queued jobs (max_active = 0 admits nothing, so no device is
touched), the memory-budget check, and shutdown."""
import ctypes as C

import pytest

from conftest import load_pkg_module


def _server(pe, budget=1 << 30, max_active=0):
    cfg = pe.ServerConfig(budget, max_active, 10, 25, pe.ORDER_ARRIVAL, 0.0, 1)
    h = C.c_void_p()
    assert pe.lib().pe_server_create(C.byref(cfg), C.byref(h)) == 0
    return h


def _spec(pe, aa, table, m=2, N=16, G=30):
    cfg = pe.Config(m, N, 0.05, pe.OBJ_BASE4, pe.GC3, 0, 7, 0, 0, 0)
    return pe.JobSpec(cfg, aa.ctypes.data_as(C.c_void_p), len(aa), C.pointer(table), G, 0, 0)


def _status(pe, h, jid):
    st = pe.JobStatus()
    assert pe.lib().pe_poll(h, jid, C.byref(st)) == 0
    return st


def test_queued_jobs_poll_and_cancel(pe):
    aa = pe.synthetic_protein(40, 3)
    table = pe.dirichlet_table(3)
    h = _server(pe)
    ids = []
    for _ in range(3):
        jid = C.c_int64(0)
        assert pe.lib().pe_batch_submit(h, C.byref(_spec(pe, aa, table)), C.byref(jid)) == 0
        ids.append(jid.value)
    assert ids == [1, 2, 3]
    for jid in ids:
        st = _status(pe, h, jid)
        assert st.state == pe.JOB_QUEUED and st.reason == -1 and st.started_s < 0
        assert st.device_bytes == pe.instance_bytes(len(aa), 2, 16)
    stats = pe.ServerStats()
    assert pe.lib().pe_server_get_stats(h, C.byref(stats)) == 0
    assert stats.queued == 3 and stats.active == 0 and stats.used_bytes == 0
    # cancelling a queued job drops it at once
    assert pe.lib().pe_cancel(h, ids[1]) == 0
    st = _status(pe, h, ids[1])
    assert st.state == pe.JOB_CANCELLED and pe.REASONS[st.reason] == "cancelled" and st.finished_s >= st.submitted_s
    assert pe.lib().pe_server_get_stats(h, C.byref(stats)) == 0 and stats.queued == 2
    # no result for a job that did not finish; unknown ids are errors
    assert pe.lib().pe_job_result(h, ids[1], None, None) == 5
    assert pe.lib().pe_poll(h, 99, C.byref(pe.JobStatus())) == 1
    # a drain with a time limit reports the jobs still queued
    assert pe.lib().pe_server_drain(h, 0.01) == 4
    assert pe.lib().pe_server_destroy(h) == 0


def test_job_larger_than_the_budget_is_refused(pe):
    aa = pe.synthetic_protein(200, 3)
    table = pe.dirichlet_table(3)
    h = _server(pe, budget=1 << 20)
    jid = C.c_int64(0)
    assert pe.lib().pe_batch_submit(h, C.byref(_spec(pe, aa, table, m=4, N=512)), C.byref(jid)) == 1
    assert b"budget" in pe.lib().pe_last_error()
    assert pe.lib().pe_server_destroy(h) == 0


def test_native_server_client_cancels_queued_jobs(pe):
    srv_mod = load_pkg_module("server")
    srv = srv_mod.NativeServer(pe, memory_budget=1 << 30, max_active=0)
    job = srv_mod.Job(pe.synthetic_protein(30, 1), pe.dirichlet_table(1), 2, 16, 20, 1, stall=0)
    srv.submit(job)
    assert srv.status(job).state == pe.JOB_QUEUED
    srv.cancel(job)
    assert srv.status(job).state == pe.JOB_CANCELLED
    srv.close()
