// pe_server.cpp -- served design jobs on one GPU, behind the C ABI (no
// counterpart in the reference, which designs one protein per process,
// src/main.cu:467-901).
//
// Continuous batching: requests are submitted at any time and admitted by
// device footprint (pe_instance_bytes) against a memory budget and by a cap on
// resident jobs, in arrival order or shortest estimated work first (a job that
// has waited longer than max_wait_s goes ahead of both).  Every resident job
// keeps its population on the device, owns a stream and is driven by its own
// host thread, which replays the job's generation graphs `tick` generations at
// a time, so the kernels of all resident jobs overlap on the GPU.  A job
// retires at its generation budget, or when the hypervolume of its survivors'
// normalised objectives (the measure of src/main.cu:789-858) has not improved
// for `stall` generations, checked every `hv_every` generations (the job waits
// for each check, so where it stops does not depend on timing), or when it is
// cancelled (between two replays: no kernel of it is left in flight).  With
// priorities on, each job's stream gets a priority from its estimated work, so
// the block scheduler serves the kernels of short jobs first.
//
// A job's result does not depend on what else is resident: every draw is keyed
// by (job seed, generation, individual, position) and each generation runs the
// same kernels as the job alone.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "pe_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

// normalisation of the hypervolume: six objectives src/main.cu:23-24; four
// objectives src/auto_execution_experiments.py:47-48 (mCAI, mHD, MGC, MSL).  The
// first n_max objectives are stored negated (maximised ones, src/main.cu:789-795).
const float kIdeal6[6] = {1.0f, 0.2f, 0.4f, 0.5f, 0.0f, 0.0f};
const float kNadir6[6] = {0.0f, -0.15f, 0.0f, 0.0f, 0.6f, 1.0f};
const float kIdeal4[4] = {1.0f, 0.4f, 0.0f, 0.0f};
const float kNadir4[4] = {0.0f, 0.0f, 0.6f, 1.0f};

struct Job {
    int64_t id = 0;
    pe_config cfg{};
    std::vector<int8_t> aa;
    pe_codon_table table{};
    int32_t generations = 0, stall = 0, keep_codons = 0;
    int M = 4;
    uint64_t bytes = 0;
    double work = 0.0;  // estimated counted cells over the generation budget
    int priority = 0;
    // state (under the server lock, except what the job's own thread owns while running)
    int state = PE_JOB_QUEUED, reason = -1;
    int gens_run = 0;
    double hv = -1.0, best_hv = -1.0;
    int best_gen = 0;
    double t_submit = 0, t_start = -1, t_end = -1;
    std::atomic<bool> cancel{false};
    std::atomic<bool> exited{false};  // its thread has left serve() and can be joined
    std::vector<float> surv_obj;      // [N][M]
    std::vector<uint8_t> surv_codons; // [N][m][L] when kept
    std::string error;
};

double estimated_cells(const pe_config &cfg, int aa_len, int generations)
{
    const double n = 3.0 * aa_len, m = cfg.n_cds, N = cfg.pop_size;
    double per;
    if (cfg.sl_kind == PE_SL_LRCS) per = m * n * (n - 1) / 2 + m * (m - 1) / 2 * n * n;
    else per = m * std::max(0.0, (n - 5) * (n - 4) / 2);
    return N * per * generations;
}

// one stream-priority level per decade of counted cells from 1e10 up: -(levels-1)
// (most urgent) for the smallest jobs, 0 for the largest
int work_priority(double cells, int levels = 6)
{
    int decade = (int)std::floor(std::log10(std::max(cells, 1.0))) - 10;
    return -(levels - 1) + std::min(std::max(decade, 0), levels - 1);
}

}  // namespace

struct pe_server {
    pe_server_config cfg{};
    int device = 0;
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::shared_ptr<Job>> queue;
    std::vector<std::shared_ptr<Job>> active;
    std::map<int64_t, std::shared_ptr<Job>> jobs;
    std::vector<std::pair<std::thread, std::shared_ptr<Job>>> threads;
    uint64_t used = 0, peak_used = 0;
    int peak_active = 0;
    int64_t next_id = 1;
    bool closing = false;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    std::shared_ptr<Job> next_locked()
    {
        if (cfg.max_wait_s > 0) {
            const double t = now();
            for (auto &j : queue)
                if (t - j->t_submit > cfg.max_wait_s) return j;
        }
        if (cfg.order == PE_ORDER_SHORTEST)
            return *std::min_element(queue.begin(), queue.end(),
                                     [](const std::shared_ptr<Job> &a, const std::shared_ptr<Job> &b) {
                                         return a->work < b->work;
                                     });
        return queue.front();
    }

    void admit_locked()
    {
        // join the threads of jobs that have finished (they no longer take the lock)
        for (size_t k = 0; k < threads.size();) {
            if (threads[k].second->exited.load()) {
                threads[k].first.join();
                threads[k] = std::move(threads.back());
                threads.pop_back();
            } else {
                k++;
            }
        }
        while (!closing && !queue.empty() && (int)active.size() < cfg.max_active) {
            std::shared_ptr<Job> j = next_locked();
            if (used + j->bytes > cfg.memory_budget) break;  // the chosen job waits for memory
            queue.erase(std::find(queue.begin(), queue.end(), j));
            used += j->bytes;
            peak_used = std::max(peak_used, used);
            active.push_back(j);
            peak_active = std::max(peak_active, (int)active.size());
            j->state = PE_JOB_RUNNING;
            j->t_start = now();
            threads.emplace_back(std::thread([this, j] {
                                     serve(j);
                                     j->exited.store(true);
                                 }),
                                 j);
        }
    }

    double survivors_hv(const std::vector<float> &obj, int N, int M, int objectives)
    {
        const float *ideal = objectives == PE_OBJ_BASE4 ? kIdeal4 : kIdeal6;
        const float *nadir = objectives == PE_OBJ_BASE4 ? kNadir4 : kNadir6;
        const int nmax = objectives == PE_OBJ_BASE4 ? 2 : 4;
        std::vector<double> pts((size_t)N * M);
        for (int i = 0; i < N; i++)
            for (int k = 0; k < M; k++) {
                float v = obj[(size_t)i * M + k];
                if (k < nmax) v = -v;
                v = (v - ideal[k]) / (nadir[k] - ideal[k]);
                if (v >= 1.0f) v = 0.999999f;
                if (v < 0.0f) v = 0.0f;
                pts[(size_t)i * M + k] = v;
            }
        std::vector<double> ref(M, 1.0);
        double hv = 0.0;
        if (pe_hypervolume(pts.data(), N, M, ref.data(), &hv) != PE_OK) return -1.0;
        return hv;
    }

    // objectives of the N survivors of the last selection (the first N solutions before any)
    int read_survivors(pe_instance *inst, const Job &j, std::vector<float> &out, std::vector<uint8_t> *codons)
    {
        const int N = j.cfg.pop_size, M = j.M, m = j.cfg.n_cds, L = (int)j.aa.size();
        std::vector<float> obj((size_t)2 * N * M);
        std::vector<int32_t> surv(N);
        std::vector<uint8_t> ids;
        if (codons) ids.resize((size_t)2 * N * m * L);
        int rc = pe_get_population(inst, codons ? ids.data() : nullptr, obj.data(), nullptr, nullptr, surv.data());
        if (rc != PE_OK) return rc;
        out.resize((size_t)N * M);
        if (codons) codons->resize((size_t)N * m * L);
        for (int i = 0; i < N; i++) {
            const int s = j.gens_run > 0 ? surv[i] : i;
            memcpy(&out[(size_t)i * M], &obj[(size_t)s * M], sizeof(float) * M);
            if (codons) memcpy(&(*codons)[(size_t)i * m * L], &ids[(size_t)s * m * L], (size_t)m * L);
        }
        return PE_OK;
    }

    void serve(std::shared_ptr<Job> j)
    {
        pe_instance *inst = nullptr;
        int rc = cudaSetDevice(device) == cudaSuccess ? PE_OK : PE_ERR_CUDA;
        pe_config cfg = j->cfg;
        cfg.stream_priority = cfg_priorities() ? j->priority : 0;
        if (rc == PE_OK) rc = pe_create(&cfg, j->aa.data(), (int32_t)j->aa.size(), &j->table, nullptr, &inst);
        if (rc == PE_OK) rc = pe_init_population(inst);
        int reason = PE_REASON_BUDGET;
        while (rc == PE_OK && j->gens_run < j->generations) {
            if (j->cancel.load()) {
                reason = PE_REASON_CANCELLED;
                break;
            }
            int g = std::min(cfg_tick(), j->generations - j->gens_run);
            if (j->stall > 0) g = std::min(g, cfg_hv_every() - j->gens_run % cfg_hv_every());
            rc = pe_step(inst, g);
            if (rc == PE_OK) rc = pe_synchronize(inst);
            if (rc != PE_OK) break;
            j->gens_run += g;
            if (j->stall > 0 && j->gens_run % cfg_hv_every() == 0 && j->gens_run < j->generations) {
                std::vector<float> so;
                rc = read_survivors(inst, *j, so, nullptr);
                if (rc != PE_OK) break;
                const double hv = survivors_hv(so, j->cfg.pop_size, j->M, j->cfg.objectives);
                if (hv > j->best_hv + 1e-12) {
                    j->best_hv = hv;
                    j->best_gen = j->gens_run;
                } else if (j->gens_run - j->best_gen >= j->stall) {
                    reason = PE_REASON_STALL;
                    break;
                }
            }
        }
        std::vector<float> so;
        std::vector<uint8_t> sc;
        double hv = -1.0;
        if (rc == PE_OK && reason != PE_REASON_CANCELLED) {
            rc = read_survivors(inst, *j, so, j->keep_codons ? &sc : nullptr);
            if (rc == PE_OK) hv = survivors_hv(so, j->cfg.pop_size, j->M, j->cfg.objectives);
        }
        std::string err = rc == PE_OK ? std::string() : std::string(pe_last_error());
        if (inst) pe_destroy(inst);
        std::lock_guard<std::mutex> lock(mu);
        j->t_end = now();
        if (rc != PE_OK) {
            j->state = PE_JOB_FAILED;
            j->reason = PE_REASON_ERROR;
            j->error = err;
        } else if (reason == PE_REASON_CANCELLED) {
            j->state = PE_JOB_CANCELLED;
            j->reason = reason;
        } else {
            j->state = PE_JOB_DONE;
            j->reason = reason;
            j->hv = hv;
            j->surv_obj.swap(so);
            j->surv_codons.swap(sc);
        }
        used -= j->bytes;
        active.erase(std::find(active.begin(), active.end(), j));
        admit_locked();
        cv.notify_all();
    }

    int cfg_tick() const { return cfg.tick > 0 ? cfg.tick : 10; }
    int cfg_hv_every() const { return cfg.hv_every > 0 ? cfg.hv_every : 25; }
    bool cfg_priorities() const { return cfg.priorities != 0; }
};

using pe::set_error_text;

extern "C" int pe_server_create(const pe_server_config *cfg, pe_server **out)
{
    if (!cfg || !out) {
        set_error_text("pe_server_create: null argument");
        return PE_ERR_ARG;
    }
    *out = nullptr;
    if (cfg->max_active < 0 || (cfg->order != PE_ORDER_ARRIVAL && cfg->order != PE_ORDER_SHORTEST)) {
        set_error_text("pe_server_create: max_active must be >= 0 and order PE_ORDER_ARRIVAL or PE_ORDER_SHORTEST");
        return PE_ERR_ARG;
    }
    auto *s = new pe_server();
    s->cfg = *cfg;
    s->t0 = Clock::now();
    if (cudaGetDevice(&s->device) != cudaSuccess) s->device = 0;
    if (s->cfg.memory_budget == 0) {
        size_t free_b = 0, total = 0;
        if (cudaMemGetInfo(&free_b, &total) != cudaSuccess) {
            delete s;
            set_error_text("pe_server_create: no device to size the memory budget (give memory_budget)");
            return PE_ERR_NO_DEVICE;
        }
        s->cfg.memory_budget = (uint64_t)(0.8 * (double)free_b);
    }
    *out = s;
    return PE_OK;
}

extern "C" int pe_batch_submit(pe_server *s, const pe_job_spec *spec, int64_t *job_id)
{
    if (!s || !spec || !job_id || !spec->aa_idx || !spec->table) {
        set_error_text("pe_batch_submit: null argument");
        return PE_ERR_ARG;
    }
    if (spec->generations < 0 || spec->stall < 0 || spec->aa_len < 3) {
        set_error_text("pe_batch_submit: generations and stall must be >= 0 and the protein >= 3 positions");
        return PE_ERR_ARG;
    }
    auto j = std::make_shared<Job>();
    j->cfg = spec->cfg;
    j->aa.assign(spec->aa_idx, spec->aa_idx + spec->aa_len);
    j->table = *spec->table;
    j->generations = spec->generations;
    j->stall = spec->stall;
    j->keep_codons = spec->keep_codons;
    j->M = spec->cfg.objectives == PE_OBJ_BASE4 ? 4 : 6;
    int rc = pe_instance_bytes(&spec->cfg, spec->aa_len, &j->bytes);
    if (rc != PE_OK) return rc;
    j->work = estimated_cells(spec->cfg, spec->aa_len, spec->generations);
    j->priority = work_priority(j->work);
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->closing) {
        set_error_text("pe_batch_submit: the server is shutting down");
        return PE_ERR_STATE;
    }
    if (j->bytes > s->cfg.memory_budget) {
        set_error_text("pe_batch_submit: the job needs more device memory than the whole budget");
        return PE_ERR_ARG;
    }
    j->id = s->next_id++;
    j->t_submit = s->now();
    s->jobs[j->id] = j;
    s->queue.push_back(j);
    s->admit_locked();
    *job_id = j->id;
    return PE_OK;
}

extern "C" int pe_poll(pe_server *s, int64_t job_id, pe_job_status *st)
{
    if (!s || !st) {
        set_error_text("pe_poll: null argument");
        return PE_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) {
        set_error_text("pe_poll: unknown job id");
        return PE_ERR_ARG;
    }
    const Job &j = *it->second;
    memset(st, 0, sizeof *st);
    st->state = j.state;
    st->reason = j.reason;
    st->generations_run = j.gens_run;
    st->hypervolume = j.hv;
    st->submitted_s = j.t_submit;
    st->started_s = j.t_start;
    st->finished_s = j.t_end;
    st->device_bytes = j.bytes;
    st->priority = j.priority;
    snprintf(st->error, sizeof st->error, "%s", j.error.c_str());
    return PE_OK;
}

extern "C" int pe_job_result(pe_server *s, int64_t job_id, float *survivor_obj, uint8_t *survivor_codons)
{
    if (!s) {
        set_error_text("pe_job_result: null server");
        return PE_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) {
        set_error_text("pe_job_result: unknown job id");
        return PE_ERR_ARG;
    }
    const Job &j = *it->second;
    if (j.state != PE_JOB_DONE) {
        set_error_text("pe_job_result: the job has no result (not finished, failed or cancelled)");
        return PE_ERR_STATE;
    }
    if (survivor_obj) memcpy(survivor_obj, j.surv_obj.data(), j.surv_obj.size() * sizeof(float));
    if (survivor_codons) {
        if (!j.keep_codons) {
            set_error_text("pe_job_result: the job was submitted without keep_codons");
            return PE_ERR_STATE;
        }
        memcpy(survivor_codons, j.surv_codons.data(), j.surv_codons.size());
    }
    return PE_OK;
}

extern "C" int pe_cancel(pe_server *s, int64_t job_id)
{
    if (!s) {
        set_error_text("pe_cancel: null server");
        return PE_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) {
        set_error_text("pe_cancel: unknown job id");
        return PE_ERR_ARG;
    }
    Job &j = *it->second;
    if (j.state == PE_JOB_QUEUED) {
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), it->second));
        j.state = PE_JOB_CANCELLED;
        j.reason = PE_REASON_CANCELLED;
        j.t_end = s->now();
        s->admit_locked();
        s->cv.notify_all();
    } else if (j.state == PE_JOB_RUNNING) {
        j.cancel.store(true);  // honoured between two replays of its generations
    }
    return PE_OK;
}

extern "C" int pe_server_clock(pe_server *s, double *seconds)
{
    if (!s || !seconds) {
        set_error_text("pe_server_clock: null argument");
        return PE_ERR_ARG;
    }
    *seconds = s->now();
    return PE_OK;
}

extern "C" int pe_server_get_stats(pe_server *s, pe_server_stats *st)
{
    if (!s || !st) {
        set_error_text("pe_server_get_stats: null argument");
        return PE_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    st->queued = (int32_t)s->queue.size();
    st->active = (int32_t)s->active.size();
    st->peak_active = s->peak_active;
    st->used_bytes = s->used;
    st->peak_used_bytes = s->peak_used;
    st->memory_budget = s->cfg.memory_budget;
    return PE_OK;
}

extern "C" int pe_server_drain(pe_server *s, double timeout_s)
{
    if (!s) {
        set_error_text("pe_server_drain: null server");
        return PE_ERR_ARG;
    }
    std::unique_lock<std::mutex> lock(s->mu);
    auto idle = [s] { return s->queue.empty() && s->active.empty(); };
    if (timeout_s > 0) {
        if (!s->cv.wait_for(lock, std::chrono::duration<double>(timeout_s), idle)) {
            set_error_text("pe_server_drain: jobs still queued or running at the time limit");
            return PE_ERR_TIMEOUT;
        }
    } else {
        s->cv.wait(lock, idle);
    }
    return PE_OK;
}

extern "C" int pe_server_destroy(pe_server *s)
{
    if (!s) return PE_OK;
    std::vector<std::pair<std::thread, std::shared_ptr<Job>>> threads;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        s->closing = true;
        for (auto &j : s->queue) {
            j->state = PE_JOB_CANCELLED;
            j->reason = PE_REASON_CANCELLED;
        }
        s->queue.clear();
        for (auto &j : s->active) j->cancel.store(true);
        s->cv.wait(lock, [s] { return s->active.empty(); });
        threads.swap(s->threads);
    }
    for (auto &t : threads)
        if (t.first.joinable()) t.first.join();
    delete s;
    return PE_OK;
}
