// pe_api.cu -- C ABI (include/pe_nsga3.h): instances, the CUDA-graph
// generation loop, operator-level entry points and host-side input helpers.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include <cuda_runtime.h>

#include "pe_internal.h"

using namespace pe;

namespace {

thread_local std::string g_err;

// Instances may be driven from different host threads (one thread per instance).
// Nothing here calls cudaMalloc or cudaFree, which synchronise with the whole
// device: device memory comes from a stream-ordered pool per device
// (cudaMallocFromPoolAsync / cudaFreeAsync on the instance's stream), so one
// instance's create or destroy neither waits for nor disturbs the work and the
// stream captures of the others.  Captures still take this lock, one at a time.
std::mutex g_cuda_mu;
using CudaLock = std::lock_guard<std::mutex>;

// The pool keeps freed memory for the next instance (release threshold
// unlimited) and lives until the process exits.
cudaError_t device_pool(int dev, cudaMemPool_t *out)
{
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) {
        *out = it->second;
        return cudaSuccess;
    }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    cudaError_t e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
        cudaMemPoolDestroy(pool);
        return e;
    }
    pools[dev] = pool;
    *out = pool;
    return cudaSuccess;
}

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CK(call)                                                                                           \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            return fail(e_ == cudaErrorMemoryAllocation ? PE_ERR_OOM : PE_ERR_CUDA, "%s: %s (%s:%d)", #call, \
                        cudaGetErrorString(e_), __FILE__, __LINE__);                                       \
    } while (0)

const char kAmino[22] = "ACDEFGHIKLMNPQRSTVWYZ";

int amino_index(char c)
{
    // binary search over the sorted amino letters (findAminoIndex, include/utils.cuh:60-86)
    int lo = 0, hi = 20;
    while (lo <= hi) {
        int mid = (lo + hi) / 2;
        if (kAmino[mid] == c) return mid;
        if (kAmino[mid] > c) hi = mid - 1;
        else lo = mid + 1;
    }
    return -1;
}

uint64_t bincoef(int n, int r)
{
    if (r < 0 || n < r) return 0;
    if (2 * r > n) r = n - r;
    uint64_t res = 1;
    for (int i = 0; i < r; i++) res = (res * (uint64_t)(n - i)) / (uint64_t)(i + 1);
    return res;
}

// Das-Dennis points: rank -> multiset unranking (include/sorting.cuh:1285-1354)
void das_dennis(int M, int p, float *out)
{
    int R = (int)bincoef(M + p - 1, p);
    std::fill(out, out + (size_t)R * M, 0.0f);
    const int mm = M + p - 1;
    const float inc = 1.0f / (float)p;
    for (int r0 = 0; r0 < R; r0++) {
        int r = r0, x = 1;
        float *pt = out + (size_t)r0 * M;
        for (int i = 1; i <= p; i++) {
            uint64_t y = bincoef(mm - x - i + 1, p - i);
            bool stop = false;
            while (y <= (uint64_t)r) {
                r -= (int)y;
                x++;
                if (x > mm) {
                    stop = true;
                    break;
                }
                y = bincoef(mm - x - i + 1, p - i);
            }
            if (stop) break;
            pt[x - 1] += inc;
        }
    }
}

uint64_t splitmix64(uint64_t &x)
{
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace

void pe::set_error_text(const char *msg) { g_err = msg ? msg : ""; }

struct pe_instance {
    Shape s{};
    pe_config cfg{};
    int p = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaMemPool_t pool = nullptr;
    DevTables *d_tab = nullptr;
    int8_t *d_aa = nullptr;
    float *d_ref = nullptr;
    PopBuf buf[2]{};
    int32_t *d_surv = nullptr;
    int32_t *d_order = nullptr;  // [2][N] CTA order of the variation kernel, by generation parity
    SelectScratch sc{};
    int2 *d_part = nullptr;
    int32_t *d_counter = nullptr;
    int32_t *d_status = nullptr;
    unsigned long long *d_scanned = nullptr;  // [0] string-objective scans run, [1] LRCS self-pair scans,
                                              // [2] seeded scans handed to the band scan
    float *d_ext = nullptr;
    uint32_t *d_gen = nullptr;
    int cur = 0;
    bool initialized = false;
    uint32_t generation = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool profiling = false;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    std::vector<void *> allocs;
    uint64_t alloc_bytes = 0;  // requested sizes rounded to 512 B (what pe_instance_bytes predicts)

    template <class T> int alloc(T **p, size_t count)
    {
        void *v = nullptr;
        const size_t b = std::max<size_t>(count, 1) * sizeof(T);
        cudaError_t e = cudaMallocFromPoolAsync(&v, b, pool, stream);
        if (e != cudaSuccess) return fail(PE_ERR_OOM, "device allocation (%zu bytes): %s", b, cudaGetErrorString(e));
        allocs.push_back(v);
        alloc_bytes += (b + 511) & ~size_t(511);
        *p = (T *)v;
        return PE_OK;
    }
};

namespace {

int alloc_pop(pe_instance *in, PopBuf &b, int nsol)
{
    const Shape &s = in->s;
    int rc;
    if ((rc = in->alloc(&b.ids, (size_t)nsol * s.m * s.Lp))) return rc;
    if ((rc = in->alloc(&b.planes, (size_t)nsol * s.m * s.Wp))) return rc;
    if ((rc = in->alloc(&b.obj, (size_t)nsol * s.M))) return rc;
    if ((rc = in->alloc(&b.objidx, (size_t)nsol * 2 * s.M))) return rc;
    if ((rc = in->alloc(&b.pql, (size_t)nsol * 3))) return rc;
    if ((rc = in->alloc(&b.cds, (size_t)nsol * s.nres))) return rc;
    if ((rc = in->alloc(&b.aux, (size_t)nsol * s.naux))) return rc;
    CK(cudaMemsetAsync(b.ids, 0, (size_t)nsol * s.m * s.Lp, in->stream));
    CK(cudaMemsetAsync(b.planes, 0, (size_t)nsol * s.m * s.Wp * sizeof(uint2), in->stream));
    CK(cudaMemsetAsync(b.obj, 0, (size_t)nsol * s.M * sizeof(float), in->stream));
    CK(cudaMemsetAsync(b.objidx, 0, (size_t)nsol * 2 * s.M, in->stream));
    CK(cudaMemsetAsync(b.pql, 0, (size_t)nsol * 3 * sizeof(int32_t), in->stream));
    CK(cudaMemsetAsync(b.cds, 0xff, (size_t)nsol * s.nres * sizeof(int2), in->stream));  // x = -1: to scan
    CK(cudaMemsetAsync(b.aux, 0, (size_t)nsol * s.naux * sizeof(int32_t), in->stream));
    return PE_OK;
}

// temporary device buffers for the operator-level entry points, stream-ordered
// on the instance's stream
struct TempBufs {
    const pe_instance *in;
    std::vector<void *> v;
    explicit TempBufs(const pe_instance *in_) : in(in_) {}
    ~TempBufs()
    {
        for (void *p : v) cudaFreeAsync(p, in->stream);
    }
    template <class T> int get(T **p, size_t count)
    {
        void *q = nullptr;
        cudaError_t e = cudaMallocFromPoolAsync(&q, std::max<size_t>(count, 1) * sizeof(T), in->pool, in->stream);
        if (e != cudaSuccess) return fail(PE_ERR_OOM, "device allocation: %s", cudaGetErrorString(e));
        v.push_back(q);
        *p = (T *)q;
        return PE_OK;
    }
    int pop(const Shape &s, PopBuf &b, int nsol)
    {
        int rc;
        if ((rc = get(&b.ids, (size_t)nsol * s.m * s.Lp))) return rc;
        if ((rc = get(&b.planes, (size_t)nsol * s.m * s.Wp))) return rc;
        if ((rc = get(&b.obj, (size_t)nsol * s.M))) return rc;
        if ((rc = get(&b.objidx, (size_t)nsol * 2 * s.M))) return rc;
        if ((rc = get(&b.pql, (size_t)nsol * 3))) return rc;
        return PE_OK;
    }
};

int check_status(pe_instance *in)
{
    int32_t st = 0;
    CK(cudaMemcpyAsync(&st, in->d_status, sizeof st, cudaMemcpyDeviceToHost, in->stream));
    CK(cudaStreamSynchronize(in->stream));
    if (st) return fail(PE_ERR_TIMEOUT, "a bounded device wait gave up (status %d)", st);
    return PE_OK;
}

cudaError_t mark(pe_instance *in, int k)
{
    if (!in->profiling) return cudaSuccess;
    return cudaEventRecordWithFlags(in->ev[k], in->stream, cudaEventRecordExternal);
}

// the selection of a generation whose children sit in buf[dst]
cudaError_t enqueue_selection(pe_instance *in, int dst, bool pdl_first)
{
    (void)pdl_first;
    return launch_select(in->s, in->buf[dst].obj, in->d_ext, in->d_ref, in->sc, in->d_surv, in->d_gen, 1, in->stream);
}

cudaError_t enqueue_generation(pe_instance *in, int src)
{
    const Shape &s = in->s;
    int dst = 1 - src;
    cudaError_t e = mark(in, 0);
    if (e != cudaSuccess) return e;
    // the variation kernel presets each child's scan counter to the string results it
    // kept, so the scan's CTAs for those results leave at once
    e = launch_mutate(s, in->d_tab, in->d_aa, in->buf[src], in->buf[dst], in->d_surv, nullptr, s.N, 0, s.N, in->d_gen,
                      nullptr, in->d_order, in->stream, nullptr, nullptr, in->d_counter);
    if (e != cudaSuccess) return e;
    if ((e = mark(in, 1)) != cudaSuccess) return e;
    e = launch_sl(s, in->buf[dst], s.N, s.N, in->d_part, in->d_counter, in->d_status, in->stream, in->d_scanned, true);
    if (e != cudaSuccess) return e;
    if ((e = mark(in, 2)) != cudaSuccess) return e;
    e = launch_select(s, in->buf[dst].obj, in->d_ext, in->d_ref, in->sc, in->d_surv, in->d_gen, 1, in->stream);
    if (e != cudaSuccess) return e;
    return mark(in, 3);
}

int build_graphs(pe_instance *in)
{
    if (in->graph[0] && in->graph[1]) return PE_OK;
    CudaLock lock(g_cuda_mu);
    for (int src = 0; src < 2; src++) {
        if (in->graph[src]) continue;
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(in->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = enqueue_generation(in, src);
        cudaError_t e2 = cudaStreamEndCapture(in->stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return fail(PE_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        cudaError_t e3 = cudaGraphInstantiate(&in->graph[src], g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) return fail(PE_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e3));
    }
    return PE_OK;
}

// Hairpin-scan CTA sizes chosen at init, per (device, L, m, N): instances of a shape
// already tuned in this process skip the timing.
struct SlTuneKey {
    int dev, L, m, N, kind, method;
    bool operator<(const SlTuneKey &o) const
    {
        return std::tie(dev, L, m, N, kind, method) < std::tie(o.dev, o.L, o.m, o.N, o.kind, o.method);
    }
};
std::mutex g_tune_mu;
std::map<SlTuneKey, int> g_tuned;

int sl_tuned(const SlTuneKey &k)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tuned.find(k);
    return it == g_tuned.end() ? 0 : it->second;
}

void sl_remember(const SlTuneKey &k, int threads)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[k] = threads;
}

}  // namespace

extern "C" {

const char *pe_last_error(void) { return g_err.c_str(); }
const char *pe_version(void) { return "pe_nsga3 1.0 (sm_100a)"; }

int pe_reference_points(int32_t M, int32_t p, float *out, int32_t *R)
{
    if (M < 1 || M > PE_MAX_OBJ || p < 1 || !R) return fail(PE_ERR_ARG, "bad reference point request M=%d p=%d", M, p);
    uint64_t r = bincoef(M + p - 1, p);
    if (r > 1000000) return fail(PE_ERR_ARG, "too many reference points (%llu)", (unsigned long long)r);
    *R = (int32_t)r;
    if (out) das_dennis(M, p, out);
    return PE_OK;
}

int pe_create(const pe_config *cfg, const int8_t *aa_idx, int32_t aa_len, const pe_codon_table *table,
              void *cuda_stream, pe_instance **out)
{
    if (!cfg || !aa_idx || !table || !out) return fail(PE_ERR_ARG, "null argument");
    *out = nullptr;
    const int L = aa_len, m = cfg->n_cds, N = cfg->pop_size;
    if (L < 3) return fail(PE_ERR_ARG, "protein too short: %d positions (need >= 3 incl. stop)", L);
    if (m < 2 || m > kMaxCds) return fail(PE_ERR_ARG, "n_cds must be in [2, %d], got %d", kMaxCds, m);
    if (N < 1 || N > (1 << 20)) return fail(PE_ERR_ARG, "pop_size out of range: %d", N);
    if (!(cfg->mutation_prob >= 0.0f && cfg->mutation_prob <= 1.0f))
        return fail(PE_ERR_ARG, "mutation_prob must be in [0,1]");
    if (cfg->objectives != PE_OBJ_REF6 && cfg->objectives != PE_OBJ_BASE4) return fail(PE_ERR_ARG, "bad objective set");
    if (cfg->gc_mode != PE_GC3 && cfg->gc_mode != PE_GC_ALL) return fail(PE_ERR_ARG, "bad gc mode");
    if (cfg->sl_threads != 0 && cfg->sl_threads != 64 && cfg->sl_threads != 128 && cfg->sl_threads != 256)
        return fail(PE_ERR_ARG, "sl_threads must be 0, 64, 128 or 256, got %d", cfg->sl_threads);
    if (cfg->sl_kind != PE_SL_HAIRPIN && cfg->sl_kind != PE_SL_LRCS)
        return fail(PE_ERR_ARG, "sl_kind must be PE_SL_HAIRPIN or PE_SL_LRCS, got %d", cfg->sl_kind);
    // table validation
    {
        int expect = 0;
        for (int a = 0; a < PE_NUM_AMINO; a++) {
            if (table->start[a] != expect || table->count[a] < 1 || table->count[a] > 6)
                return fail(PE_ERR_ARG, "codon table: amino %d has start %d count %d", a, table->start[a], table->count[a]);
            expect += table->count[a];
        }
        if (expect != PE_NUM_CODON) return fail(PE_ERR_ARG, "codon table covers %d codons", expect);
        if (table->count[20] != 3) return fail(PE_ERR_ARG, "stop group must hold the last 3 codons");
        for (int c = 0; c < PE_NUM_CODON; c++) {
            for (int b = 0; b < 3; b++)
                if (table->nt[c][b] > 3) return fail(PE_ERR_ARG, "codon %d: bad nucleotide code", c);
            if (!(table->weight[c] >= 0.0f) || !std::isfinite(table->weight[c]))
                return fail(PE_ERR_ARG, "codon %d: weight must be finite and >= 0", c);
        }
    }
    for (int a = 0; a < L; a++)
        if (aa_idx[a] < 0 || aa_idx[a] >= PE_NUM_AMINO) return fail(PE_ERR_ARG, "amino index %d at %d", aa_idx[a], a);

    Shape s{};
    s.L = L;
    s.Lp = (L + 15) & ~15;
    s.m = m;
    s.N = N;
    s.objset = cfg->objectives;
    s.gcmode = cfg->gc_mode;
    s.M = cfg->objectives == PE_OBJ_BASE4 ? 4 : 6;
    s.n = 3 * L;
    s.W = (s.n + 31) / 32;
    s.Wp = (s.W + 2) & ~1;  // >= 1 zero guard word, even
    s.K = (s.n - 4) / 2;
    s.pm = cfg->mutation_prob;
    s.seed = cfg->seed;
    s.sl_threads = cfg->sl_threads;
    s.sl_kind = cfg->sl_kind;
    s.nres = s.sl_kind == PE_SL_LRCS ? m * (m + 1) / 2 : m;
    s.naux = AUX_HD(m) + m * (m - 1) / 2;
    {
        static const int ref6[6] = {K_CAI, K_CBP, K_HSC, K_HD, K_GC, K_SL};
        static const int base4[4] = {K_CAI, K_HD, K_GC, K_SL};
        for (int k = 0; k < 6; k++) s.slot[k] = -1;
        const int *kinds = s.M == 4 ? base4 : ref6;
        for (int i = 0; i < s.M; i++) s.slot[kinds[i]] = i;
    }
    int p = cfg->ref_p;
    if (p <= 0) {
        // src/main.cu:564-576: largest p with C(M+p-1, p) <= N
        p = 1;
        while ((int64_t)bincoef(s.M + p - 1, p) <= N) p++;
        p -= 1;
        if (p < 1) return fail(PE_ERR_ARG, "pop_size %d too small for the reference-point rule (M=%d)", N, s.M);
    }
    uint64_t R = bincoef(s.M + p - 1, p);
    if (R < 1 || R > 65536) return fail(PE_ERR_ARG, "reference points out of range (%llu)", (unsigned long long)R);
    s.R = (int)R;
    if ((size_t)m * L > 120000) return fail(PE_ERR_ARG, "m*L = %d exceeds the per-CTA solution limit (120000)", m * L);

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PE_ERR_NO_DEVICE, "no CUDA device");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    int smem_optin = 0;
    CK(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (sl_smem_bytes(s) > (size_t)smem_optin || var_smem_bytes(s) > (size_t)smem_optin ||
        select_smem_bytes(s) > (size_t)smem_optin || niche_smem_bytes(s) > (size_t)smem_optin)
        return fail(PE_ERR_ARG, "problem too large for one CTA (L=%d m=%d N=%d)", L, m, N);

    pe_instance *in = new pe_instance();
    in->s = s;
    in->cfg = *cfg;
    in->p = p;
    in->device = dev;
    if (cuda_stream) {
        in->stream = (cudaStream_t)cuda_stream;
    } else {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) least = greatest = 0;
        const int prio = std::min(least, std::max(greatest, (int)cfg->stream_priority));
        if (cudaStreamCreateWithPriority(&in->stream, cudaStreamNonBlocking, prio) != cudaSuccess) {
            delete in;
            return fail(PE_ERR_CUDA, "stream creation failed");
        }
        in->own_stream = true;
    }
    {
        cudaError_t e = device_pool(dev, &in->pool);
        if (e != cudaSuccess) {
            if (in->own_stream) cudaStreamDestroy(in->stream);
            delete in;
            return fail(PE_ERR_CUDA, "device memory pool: %s", cudaGetErrorString(e));
        }
    }
    int rc = PE_OK;
    auto cleanup = [&](int code) {
        pe_destroy(in);
        return code;
    };
    // tables
    DevTables ht;
    memset(&ht, 0, sizeof ht);
    for (int c = 0; c < 64; c++) {
        for (int b = 0; b < 3; b++) ht.nt[c][b] = table->nt[c][b];
        double w = (double)table->weight[c];
        ht.wzero[c] = !(w > 0.0);
        ht.lw[c] = w > 0.0 ? (int64_t)llrint(log(w) * 4294967296.0) : 0;
        ht.gc3[c] = table->nt[c][2] == 1 || table->nt[c][2] == 2;
        ht.gcn[c] = 0;
        for (int b = 0; b < 3; b++) ht.gcn[c] += table->nt[c][b] == 1 || table->nt[c][b] == 2;
    }
    for (int a = 0; a < 21; a++) {
        ht.start[a] = table->start[a];
        ht.count[a] = table->count[a];
        for (int j = 0; j < table->count[a]; j++) ht.aa_of[table->start[a] + j] = (int8_t)a;
    }
    auto is_stop = [&](int x, int y, int z) {
        for (int c = 61; c < 64; c++)
            if (table->nt[c][0] == x && table->nt[c][1] == y && table->nt[c][2] == z) return 1;
        return 0;
    };
    for (int x = 0; x < 64; x++)
        for (int y = 0; y < 64; y++)
            ht.hsc[x * 64 + y] = (uint8_t)(is_stop(table->nt[x][1], table->nt[x][2], table->nt[y][0]) +
                                           is_stop(table->nt[x][2], table->nt[y][0], table->nt[y][1]));
    for (int i = 0; i < 61 * 61; i++) {
        ht.cps[i] = table->cps[i];
        ht.cpsf[i] = (int64_t)llrint((double)table->cps[i] * 4294967296.0);
    }
    ht.ref_gc3 = table->ref_gc3;
    ht.ref_gc = table->ref_gc;
    for (int i = 0, pi = 0; i < m - 1; i++)
        for (int j = i + 1; j < m; j++, pi++) {
            ht.pair_i[pi] = (uint8_t)i;
            ht.pair_j[pi] = (uint8_t)j;
        }

    if ((rc = in->alloc(&in->d_tab, 1))) return cleanup(rc);
    if ((rc = in->alloc(&in->d_aa, (size_t)L))) return cleanup(rc);
    if ((rc = in->alloc(&in->d_ref, (size_t)s.R * s.M))) return cleanup(rc);
    for (int b = 0; b < 2; b++)
        if ((rc = alloc_pop(in, in->buf[b], 2 * N))) return cleanup(rc);
    const int N2 = 2 * N, words = (N2 + 31) / 32;
    if ((rc = in->alloc(&in->d_surv, (size_t)N))) return cleanup(rc);
    if ((rc = in->alloc(&in->d_order, (size_t)2 * N))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.dom, (size_t)N2 * words))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.np, (size_t)N2 * dom_tile_count(N2)))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.front, (size_t)N2))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.sorted, (size_t)N2))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.assoc, (size_t)N2))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.dist, (size_t)N2))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.rho, (size_t)s.R))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.ncand, (size_t)s.R))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.trank, (size_t)N2 + s.M))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.info, 8))) return cleanup(rc);
    if ((rc = in->alloc(&in->sc.finfo, 3 * PE_MAX_OBJ))) return cleanup(rc);
    if ((rc = in->alloc(&in->d_part, (size_t)N2 * s.nres))) return cleanup(rc);
    if ((rc = in->alloc(&in->d_counter, (size_t)N2))) return cleanup(rc);
    if ((rc = in->alloc(&in->d_scanned, 3))) return cleanup(rc);
    if ((rc = in->alloc(&in->d_status, 1))) return cleanup(rc);
    if ((rc = in->alloc(&in->d_ext, (size_t)s.M * s.M))) return cleanup(rc);
    if ((rc = in->alloc(&in->d_gen, 1))) return cleanup(rc);
    std::vector<float> ref((size_t)s.R * s.M);
    das_dennis(s.M, p, ref.data());
    std::vector<uint32_t> trank((size_t)N2 + s.M);
    tree_order_ranks(N2 + s.M, trank.data());
    std::vector<int32_t> ident((size_t)N2);  // both halves of d_order: children in index order
    for (int k = 0; k < N2; k++) ident[(size_t)k] = k % N;
    cudaStream_t st = in->stream;
#define CKC(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return cleanup(fail(PE_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_))); \
    } while (0)
    CKC(cudaMemcpyAsync(in->d_tab, &ht, sizeof ht, cudaMemcpyHostToDevice, st));
    CKC(cudaMemcpyAsync(in->d_aa, aa_idx, (size_t)L, cudaMemcpyHostToDevice, st));
    CKC(cudaMemcpyAsync(in->d_ref, ref.data(), ref.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    CKC(cudaMemcpyAsync(in->sc.trank, trank.data(), trank.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    CKC(cudaMemcpyAsync(in->d_order, ident.data(), ident.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    CKC(cudaMemsetAsync(in->d_counter, 0, (size_t)N2 * sizeof(int32_t), st));
    CKC(cudaMemsetAsync(in->d_scanned, 0, 3 * sizeof(unsigned long long), st));
    CKC(cudaMemsetAsync(in->d_status, 0, sizeof(int32_t), st));
    CKC(cudaMemsetAsync(in->d_ext, 0, (size_t)s.M * s.M * sizeof(float), st));
    CKC(cudaMemsetAsync(in->d_gen, 0, sizeof(uint32_t), st));
    CKC(cudaStreamSynchronize(st));
#undef CKC
    *out = in;
    return PE_OK;
}

// ---------------------------------------------------------------- batches

// a length class of the batch's queued scan: members with the same string objective
// and tuned scan CTA size, longest CDSs first
struct ScanClass {
    int fl = 0, nt = 128, ctas = 0;
    size_t smem = 0;
    std::vector<int> members;
    int32_t *ticket = nullptr;    // [2] device: next item, CTAs done
    SlJob *jobs[3][2] = {};       // device job tables per graph (generations 1, 2) and step
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
};

struct pe_batch {
    std::vector<pe_instance *> inst;
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};  // [generations] for 1 and 2
    std::vector<int> parity[3];                                // instance parities the graph was built for
    bool queue = false;                                        // queued stem scans (pe_batch_set_scan_queue)
    std::vector<int32_t *> q_items, q_count;                   // per member: its queue
    std::vector<ScanClass> classes;
};

static void free_scan_classes(pe_batch *b)
{
    for (ScanClass &c : b->classes) {
        for (auto &g : c.jobs)
            for (SlJob *&j : g)
                if (j) cudaFree(j), j = nullptr;
        if (c.ticket) cudaFree(c.ticket);
        if (c.done) cudaEventDestroy(c.done);
        if (c.stream) cudaStreamDestroy(c.stream);
    }
    b->classes.clear();
    for (int32_t *p : b->q_items)
        if (p) cudaFree(p);
    for (int32_t *p : b->q_count)
        if (p) cudaFree(p);
    b->q_items.clear();
    b->q_count.clear();
}

// Queues and length classes of the batch's queued scan.  A class is the members with
// the same string objective and the scan CTA size their init tuning chose; its wave
// of CTAs is its share of the device, by the members' scan cells per generation.
static cudaError_t setup_scan_queue(pe_batch *b)
{
    const int n = (int)b->inst.size();
    b->q_items.assign(n, nullptr);
    b->q_count.assign(n, nullptr);
    std::map<std::pair<int, int>, int> cls;
    std::vector<double> work;
    for (int i = 0; i < n; i++) {
        const Shape &s = b->inst[i]->s;
        cudaError_t e = cudaMalloc(&b->q_items[i], (size_t)s.N * s.nres * sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMalloc(&b->q_count[i], sizeof(int32_t));
        if (e == cudaSuccess) e = cudaMemset(b->q_count[i], 0, sizeof(int32_t));
        if (e != cudaSuccess) return e;
        const int fl = s.sl_kind == PE_SL_LRCS ? 1 : 0, nt = s.sl_threads ? s.sl_threads : 128;
        auto key = std::make_pair(fl, nt);
        if (!cls.count(key)) {
            cls[key] = (int)b->classes.size();
            b->classes.emplace_back();
            b->classes.back().fl = fl;
            b->classes.back().nt = nt;
            work.push_back(0.0);
        }
        const int c = cls[key];
        b->classes[c].members.push_back(i);
        b->classes[c].smem = std::max(b->classes[c].smem, sl_queue_smem_bytes(s, nt));
        work[c] += (double)s.N * s.nres * (double)s.n * s.n;
    }
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    double total = 0.0;
    for (double w : work) total += w;
    for (size_t c = 0; c < b->classes.size(); c++) {
        ScanClass &k = b->classes[c];
        if ((int)k.members.size() > kMaxBatchJobs) return cudaErrorInvalidValue;
        std::sort(k.members.begin(), k.members.end(),
                  [&](int x, int y) { return b->inst[x]->s.n > b->inst[y]->s.n; });
        const int per_sm = sl_queue_ctas_per_sm(k.nt, k.fl, k.smem);
        if (per_sm <= 0) return cudaErrorInvalidConfiguration;
        const double share = total > 0.0 ? work[c] / total : 1.0;
        k.ctas = std::max(1, (int)(share * sms * per_sm + 0.5));
        if ((e = cudaMalloc(&k.ticket, 2 * sizeof(int32_t))) != cudaSuccess) return e;
        if ((e = cudaMemset(k.ticket, 0, 2 * sizeof(int32_t))) != cudaSuccess) return e;
        if ((e = cudaStreamCreateWithFlags(&k.stream, cudaStreamNonBlocking)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&k.done, cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// the job table of class k for a step whose children go to each member's buffer dst
static cudaError_t scan_jobs(pe_batch *b, ScanClass &k, const std::vector<int> &dst, SlJob **out)
{
    std::vector<SlJob> h(k.members.size());
    for (size_t q = 0; q < k.members.size(); q++) {
        const int i = k.members[q];
        pe_instance *in = b->inst[i];
        SlJob &j = h[q];
        j.s = in->s;
        j.buf = in->buf[dst[i]];
        j.base = in->s.N;
        j.part = in->d_part;
        j.counter = in->d_counter;
        j.status = in->d_status;
        j.scanned = in->d_scanned;
        j.items = b->q_items[i];
        j.count = b->q_count[i];
    }
    if (!*out) {
        cudaError_t e = cudaMalloc(out, h.size() * sizeof(SlJob));
        if (e != cudaSuccess) return e;
    }
    return cudaMemcpy(*out, h.data(), h.size() * sizeof(SlJob), cudaMemcpyHostToDevice);
}

// fork every member's stream from the master, run f(member) on it, join them back
extern "C++" template <class F> cudaError_t batch_branches(pe_batch *b, F f)
{
    cudaError_t e = cudaEventRecord(b->fork, b->master);
    for (size_t i = 0; i < b->inst.size() && e == cudaSuccess; i++) {
        pe_instance *in = b->inst[i];
        e = cudaStreamWaitEvent(in->stream, b->fork, 0);
        if (e == cudaSuccess) e = f((int)i, in);
        if (e == cudaSuccess) e = cudaEventRecord(b->join[i], in->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->master, b->join[i], 0);
    }
    return e;
}

static int batch_capture(pe_batch *b, int gens, cudaGraphExec_t *out)
{
    const int n = (int)b->inst.size();
    std::vector<int> src(n);
    for (int i = 0; i < n; i++) src[i] = b->inst[i]->cur;
    if (b->queue && b->classes.empty()) {  // queues and classes on first use
        cudaError_t e0 = setup_scan_queue(b);
        if (e0 != cudaSuccess) {
            free_scan_classes(b);
            return fail(PE_ERR_CUDA, "batch scan queue setup: %s", cudaGetErrorString(e0));
        }
    }
    if (b->queue) {  // the job tables of each step, before the capture
        std::vector<int> s2 = src;
        for (int k = 0; k < gens; k++) {
            std::vector<int> dst(n);
            for (int i = 0; i < n; i++) dst[i] = 1 - s2[i];
            for (ScanClass &c : b->classes) CK(scan_jobs(b, c, dst, &c.jobs[gens][k]));
            s2 = dst;
        }
    }
    cudaGraph_t g = nullptr;
    CudaLock lock(g_cuda_mu);
    CK(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    if (!b->queue) {
        e = batch_branches(b, [&](int i, pe_instance *in) {
            cudaError_t e1 = cudaSuccess;
            int sr = src[i];
            for (int k = 0; k < gens && e1 == cudaSuccess; k++) {
                e1 = enqueue_generation(in, sr);
                sr = 1 - sr;
            }
            return e1;
        });
    }
    for (int k = 0; b->queue && k < gens && e == cudaSuccess; k++) {
        // variation of every member (queueing its scans), the batch's scans by class,
        // then every member's selection
        e = batch_branches(b, [&](int i, pe_instance *in) {
            const Shape &s = in->s;
            const int sr = src[i], ds = 1 - sr;
            return launch_mutate(s, in->d_tab, in->d_aa, in->buf[sr], in->buf[ds], in->d_surv, nullptr, s.N, 0, s.N,
                                 in->d_gen, nullptr, in->d_order, in->stream, b->q_items[i], b->q_count[i],
                                 in->d_counter);
        });
        if (e == cudaSuccess) e = cudaEventRecord(b->fork, b->master);
        for (ScanClass &c : b->classes) {
            if (e == cudaSuccess) e = cudaStreamWaitEvent(c.stream, b->fork, 0);
            if (e == cudaSuccess)
                e = launch_sl_queue(c.jobs[gens][k], (int)c.members.size(), c.ticket, c.nt, c.fl, c.smem, c.ctas,
                                    c.stream);
            if (e == cudaSuccess) e = cudaEventRecord(c.done, c.stream);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(b->master, c.done, 0);
        }
        if (e == cudaSuccess)
            e = batch_branches(b, [&](int i, pe_instance *in) { return enqueue_selection(in, 1 - src[i], false); });
        for (int i = 0; i < n; i++) src[i] = 1 - src[i];
    }
    cudaError_t e2 = cudaStreamEndCapture(b->master, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(PE_ERR_CUDA, "batch capture failed: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
    }
    cudaError_t e3 = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) return fail(PE_ERR_CUDA, "batch graph instantiate: %s", cudaGetErrorString(e3));
    return PE_OK;
}

int pe_batch_create(pe_instance *const *instances, int32_t count, pe_batch **out)
{
    if (!instances || count < 1 || !out) return fail(PE_ERR_ARG, "bad batch arguments");
    *out = nullptr;
    for (int i = 0; i < count; i++) {
        pe_instance *in = instances[i];
        if (!in) return fail(PE_ERR_ARG, "batch member %d is null", i);
        if (!in->initialized) return fail(PE_ERR_STATE, "batch member %d is not initialised", i);
        if (!in->own_stream) return fail(PE_ERR_ARG, "batch member %d must own its stream (create with NULL)", i);
        if (in->profiling) return fail(PE_ERR_STATE, "batch member %d has profiling on", i);
        for (int j = 0; j < i; j++)
            if (instances[j] == in) return fail(PE_ERR_ARG, "instance %d appears twice", i);
        if (in->device != instances[0]->device) return fail(PE_ERR_ARG, "batch members on different devices");
    }
    pe_batch *b = new pe_batch();
    b->inst.assign(instances, instances + count);
    b->join.resize(count, nullptr);
    auto bad = [&](cudaError_t e) {
        pe_batch_destroy(b);
        return fail(PE_ERR_CUDA, "batch setup: %s", cudaGetErrorString(e));
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bad(e);
    if ((e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess) return bad(e);
    for (int i = 0; i < count; i++)
        if ((e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming)) != cudaSuccess) return bad(e);
    // members' earlier work must be complete before the batch takes over their streams
    for (pe_instance *in : b->inst)
        if ((e = cudaStreamSynchronize(in->stream)) != cudaSuccess) return bad(e);
    *out = b;
    return PE_OK;
}

int pe_batch_step(pe_batch *b, int32_t generations)
{
    if (!b) return fail(PE_ERR_ARG, "null batch");
    if (generations < 0) return fail(PE_ERR_ARG, "negative generation count");
    if (generations == 0) return PE_OK;
    // order the batch after work already queued on the members' own streams ...
    for (size_t i = 0; i < b->inst.size(); i++) {
        CK(cudaEventRecord(b->join[i], b->inst[i]->stream));
        CK(cudaStreamWaitEvent(b->master, b->join[i], 0));
    }
    while (generations > 0) {
        const int g = generations >= 2 ? 2 : 1;
        std::vector<int> par(b->inst.size());
        for (size_t i = 0; i < b->inst.size(); i++) par[i] = b->inst[i]->cur;
        if (b->graph[g] && b->parity[g] != par) {
            cudaGraphExecDestroy(b->graph[g]);
            b->graph[g] = nullptr;
        }
        if (!b->graph[g]) {
            int rc = batch_capture(b, g, &b->graph[g]);
            if (rc) return rc;
            b->parity[g] = par;
        }
        CK(cudaGraphLaunch(b->graph[g], b->master));
        for (pe_instance *in : b->inst) {
            if (g == 1) in->cur = 1 - in->cur;
            in->generation += g;
        }
        generations -= g;
    }
    // ... and later calls on a member's stream (reads, pe_step) after the batch
    CK(cudaEventRecord(b->fork, b->master));
    for (pe_instance *in : b->inst) CK(cudaStreamWaitEvent(in->stream, b->fork, 0));
    return PE_OK;
}

int pe_batch_synchronize(pe_batch *b)
{
    if (!b) return fail(PE_ERR_ARG, "null batch");
    CK(cudaStreamSynchronize(b->master));
    for (pe_instance *in : b->inst) {
        int rc = check_status(in);
        if (rc) return rc;
    }
    return PE_OK;
}

int pe_batch_set_scan_queue(pe_batch *b, int32_t enable)
{
    if (!b) return fail(PE_ERR_ARG, "null batch");
    if ((enable != 0) != b->queue) {
        CK(cudaStreamSynchronize(b->master));
        for (auto &g : b->graph)
            if (g) cudaGraphExecDestroy(g), g = nullptr;
        for (auto &p : b->parity) p.clear();
        b->queue = enable != 0;
    }
    return PE_OK;
}

int pe_batch_destroy(pe_batch *b)
{
    if (!b) return PE_OK;
    if (b->master) cudaStreamSynchronize(b->master);
    for (auto &g : b->graph)
        if (g) cudaGraphExecDestroy(g);
    free_scan_classes(b);
    for (cudaEvent_t ev : b->join)
        if (ev) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->master) cudaStreamDestroy(b->master);
    delete b;
    return PE_OK;
}

int pe_set_profiling(pe_instance *in, int32_t enable)
{
    if (!in) return fail(PE_ERR_ARG, "null instance");
    CK(cudaStreamSynchronize(in->stream));
    for (int k = 0; k < 4; k++)
        if (!in->ev[k]) CK(cudaEventCreate(&in->ev[k]));
    if ((bool)enable != in->profiling) {
        for (int i = 0; i < 2; i++)
            if (in->graph[i]) {
                cudaGraphExecDestroy(in->graph[i]);
                in->graph[i] = nullptr;
            }
        in->profiling = enable != 0;
    }
    return PE_OK;
}

int pe_set_wait_limit(pe_instance *in, int32_t polls)
{
    if (!in) return fail(PE_ERR_ARG, "null instance");
    CK(cudaStreamSynchronize(in->stream));
    if (polls != in->s.wait_limit) {
        in->s.wait_limit = polls;
        for (int i = 0; i < 2; i++)
            if (in->graph[i]) {
                cudaGraphExecDestroy(in->graph[i]);
                in->graph[i] = nullptr;
            }
    }
    return PE_OK;
}

int pe_stage_times(pe_instance *in, float *ms3)
{
    if (!in || !ms3) return fail(PE_ERR_ARG, "null argument");
    if (!in->profiling) return fail(PE_ERR_STATE, "profiling is off");
    for (int k = 0; k < 3; k++) CK(cudaEventElapsedTime(&ms3[k], in->ev[k], in->ev[k + 1]));
    return PE_OK;
}

int pe_scan_count(pe_instance *in, uint64_t *count)
{
    if (!in || !count) return fail(PE_ERR_ARG, "null argument");
    unsigned long long v = 0;
    CK(cudaMemcpyAsync(&v, in->d_scanned, sizeof v, cudaMemcpyDeviceToHost, in->stream));
    CK(cudaStreamSynchronize(in->stream));
    *count = (uint64_t)v;
    return PE_OK;
}

int pe_scan_cells(pe_instance *in, uint64_t *cells)
{
    if (!in || !cells) return fail(PE_ERR_ARG, "null argument");
    unsigned long long v[2] = {0, 0};  // scans, LRCS scans of a CDS against itself
    CK(cudaMemcpyAsync(v, in->d_scanned, sizeof v, cudaMemcpyDeviceToHost, in->stream));
    CK(cudaStreamSynchronize(in->stream));
    const uint64_t n = (uint64_t)in->s.n;
    if (in->s.sl_kind == PE_SL_LRCS)
        *cells = (uint64_t)v[1] * (n * (n - 1) / 2) + (uint64_t)(v[0] - v[1]) * (n * n);
    else
        *cells = (uint64_t)v[0] * (n > 5 ? (n - 5) * (n - 4) / 2 : 0);
    return PE_OK;
}

int pe_scan_fallbacks(pe_instance *in, uint64_t *count)
{
    if (!in || !count) return fail(PE_ERR_ARG, "null argument");
    unsigned long long v = 0;
    CK(cudaMemcpyAsync(&v, in->d_scanned + 2, sizeof v, cudaMemcpyDeviceToHost, in->stream));
    CK(cudaStreamSynchronize(in->stream));
    *count = (uint64_t)v;
    return PE_OK;
}

int pe_set_scan_method(pe_instance *in, int32_t method)
{
    if (!in) return fail(PE_ERR_ARG, "null instance");
    if (method != 0 && method != 1) return fail(PE_ERR_ARG, "scan method must be 0 (seeded) or 1 (band scan), got %d", method);
    CK(cudaStreamSynchronize(in->stream));
    if (method != in->s.sl_method) {
        in->s.sl_method = method;
        for (int i = 0; i < 2; i++)
            if (in->graph[i]) {
                cudaGraphExecDestroy(in->graph[i]);
                in->graph[i] = nullptr;
            }
    }
    return PE_OK;
}

int pe_instance_bytes(const pe_config *cfg, int32_t aa_len, uint64_t *bytes)
{
    if (!cfg || !bytes || aa_len < 3 || cfg->pop_size < 1 || cfg->n_cds < 2) return fail(PE_ERR_ARG, "bad arguments");
    const uint64_t L = (uint64_t)aa_len, m = (uint64_t)cfg->n_cds, N = (uint64_t)cfg->pop_size, N2 = 2 * N;
    const uint64_t M = cfg->objectives == PE_OBJ_BASE4 ? 4 : 6;
    const uint64_t Lp = (L + 15) & ~uint64_t(15), n = 3 * L, W = (n + 31) / 32, Wp = (W + 2) & ~uint64_t(1);
    int p = cfg->ref_p;
    if (p <= 0) {
        p = 1;
        while ((int64_t)bincoef((int)M + p - 1, p) <= (int64_t)N) p++;
        p -= 1;
        if (p < 1) return fail(PE_ERR_ARG, "pop_size too small for the reference-point rule");
    }
    const uint64_t R = bincoef((int)M + p - 1, p), words = (N2 + 31) / 32;
    auto r = [](uint64_t b) { return (b + 511) & ~uint64_t(511); };  // allocation granularity
    uint64_t t = r(sizeof(DevTables)) + r(L) + r(R * M * 4);
    t += 2 * (r(N2 * m * Lp) + r(N2 * m * Wp * 8) + r(N2 * M * 4) + r(N2 * 2 * M) + r(N2 * 12));
    t += r(N * 4) + r(N2 * 4) + r(N2 * words * 4) + r(N2 * (uint64_t)dom_tile_count((int)N2) * 4) + 4 * r(N2 * 4) +
         2 * r(R * 4) + r((N2 + M) * 4) + r(32) + r(72);
    const uint64_t nres = cfg->sl_kind == PE_SL_LRCS ? m * (m + 1) / 2 : m;
    t += r(N2 * nres * 8) + r(N2 * 4) + r(4) + r(M * M * 4) + r(4);
    t += 2 * r(N2 * nres * 8) + r(24);  // per-CDS (per-pair) string results of both buffers, scan counts
    t += 2 * r(N2 * (5 * m + m * (m - 1) / 2) * 4);  // per-CDS sums of the light objectives, both buffers
    *bytes = t;
    return PE_OK;
}

int pe_destroy(pe_instance *in)
{
    if (!in) return PE_OK;
    if (in->stream) cudaStreamSynchronize(in->stream);
    for (int i = 0; i < 2; i++)
        if (in->graph[i]) cudaGraphExecDestroy(in->graph[i]);
    for (int k = 0; k < 4; k++)
        if (in->ev[k]) cudaEventDestroy(in->ev[k]);
    for (void *p : in->allocs) cudaFreeAsync(p, in->stream);
    if (in->stream) cudaStreamSynchronize(in->stream);
    if (in->own_stream && in->stream) cudaStreamDestroy(in->stream);
    delete in;
    return PE_OK;
}

int pe_get_info(const pe_instance *in, pe_info *info)
{
    if (!in || !info) return fail(PE_ERR_ARG, "null argument");
    info->L = in->s.L;
    info->m = in->s.m;
    info->N = in->s.N;
    info->M = in->s.M;
    info->R = in->s.R;
    info->p = in->p;
    info->generation = in->generation;
    info->initialized = in->initialized;
    info->device_bytes = in->alloc_bytes;
    info->sl_threads = in->s.sl_threads > 0 ? in->s.sl_threads : 128;
    return PE_OK;
}

int pe_init_population(pe_instance *in)
{
    if (!in) return fail(PE_ERR_ARG, "null instance");
    Shape &s = in->s;
    // a fresh start: clears a status left by a device wait that gave up, and the
    // per-solution counters of scans that did not finish
    CK(cudaMemsetAsync(in->d_status, 0, sizeof(int32_t), in->stream));
    CK(cudaMemsetAsync(in->d_counter, 0, (size_t)2 * s.N * sizeof(int32_t), in->stream));
    CK(launch_init(s, in->d_tab, in->d_aa, in->buf[0], in->d_surv, in->stream));
    bool scanned = false;
    if (in->cfg.sl_threads == 0 && s.sl_threads == 0) {
        const SlTuneKey key{in->device, s.L, s.m, s.N, s.sl_kind, s.sl_method};
        s.sl_threads = sl_tuned(key);
        if (s.sl_threads == 0) {
            // pick the string-scan CTA size: after one warm scan of the initial population,
            // time two scans with each size, in the orders 64, 128, 256 and 256, 128, 64
            // (they all give the same result), and keep the size with the fastest one;
            // the choice is remembered for this shape on this device.  The timed scans
            // cover a third of the population, about the share of CDSs a generation's
            // mutations change: the best size for few items per SM differs from the
            // best for a full scan (a fuller grid favours smaller CTAs)
            constexpr int kRuns = 6;
            cudaEvent_t ev[kRuns + 1] = {};
            cudaError_t e = cudaSuccess;
            for (int k = 0; k <= kRuns && e == cudaSuccess; k++) e = cudaEventCreate(&ev[k]);
            const int sizes[kRuns] = {64, 128, 256, 256, 128, 64};
            s.sl_threads = 128;
            // the warm scan stores the per-CDS results; the timed ones scan every CDS
            // (no carried results) and rewrite the same objectives
            PopBuf full = in->buf[0];
            full.cds = nullptr;
            if (e == cudaSuccess)
                e = launch_sl(s, in->buf[0], 0, s.N, in->d_part, in->d_counter, in->d_status, in->stream,
                              in->d_scanned);
            for (int k = 0; k < kRuns && e == cudaSuccess; k++) {
                s.sl_threads = sizes[k];
                e = cudaEventRecord(ev[k], in->stream);
                if (e == cudaSuccess)
                    e = launch_sl(s, full, 0, std::max(1, s.N / 3), in->d_part, in->d_counter, in->d_status,
                                  in->stream);
            }
            if (e == cudaSuccess) e = cudaEventRecord(ev[kRuns], in->stream);
            if (e == cudaSuccess) e = cudaEventSynchronize(ev[kRuns]);
            float best_ms = 0.0f;
            int best = 128;
            for (int k = 0; k < kRuns && e == cudaSuccess; k++) {
                float ms = 0.0f;
                e = cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
                if (e == cudaSuccess && (k == 0 || ms < best_ms)) {
                    best_ms = ms;
                    best = sizes[k];
                }
            }
            for (int k = 0; k <= kRuns; k++)
                if (ev[k]) cudaEventDestroy(ev[k]);
            s.sl_threads = best;
            if (e != cudaSuccess) return fail(PE_ERR_CUDA, "hairpin-scan tuning: %s", cudaGetErrorString(e));
            sl_remember(key, best);
            scanned = true;   // the timed scans left the initial population's stems in place
        }
        for (int i = 0; i < 2; i++)
            if (in->graph[i]) {
                cudaGraphExecDestroy(in->graph[i]);
                in->graph[i] = nullptr;
            }
    }
    if (!scanned)
        CK(launch_sl(s, in->buf[0], 0, s.N, in->d_part, in->d_counter, in->d_status, in->stream, in->d_scanned));
    // extreme points start as the objective vectors of solutions 0..M-1
    // (initializationKernel, src/main.cu:106-109)
    CK(cudaMemsetAsync(in->d_ext, 0, (size_t)s.M * s.M * sizeof(float), in->stream));
    int rows = std::min(s.M, s.N);
    CK(cudaMemcpyAsync(in->d_ext, in->buf[0].obj, (size_t)rows * s.M * sizeof(float), cudaMemcpyDeviceToDevice,
                       in->stream));
    CK(cudaMemsetAsync(in->d_gen, 0, sizeof(uint32_t), in->stream));
    in->cur = 0;
    in->generation = 0;
    in->initialized = true;
    return check_status(in);
}

int pe_step(pe_instance *in, int32_t generations)
{
    if (!in) return fail(PE_ERR_ARG, "null instance");
    if (!in->initialized) return fail(PE_ERR_STATE, "pe_step before pe_init_population");
    if (generations < 0) return fail(PE_ERR_ARG, "negative generation count");
    int rc = build_graphs(in);
    if (rc) return rc;
    for (int g = 0; g < generations; g++) {
        CK(cudaGraphLaunch(in->graph[in->cur], in->stream));
        in->cur = 1 - in->cur;
        in->generation++;
    }
    return PE_OK;
}

int pe_synchronize(pe_instance *in)
{
    if (!in) return fail(PE_ERR_ARG, "null instance");
    return check_status(in);   // queues the status read behind the stream's work and waits for it
}

int pe_get_population(pe_instance *in, uint8_t *codon_idx, float *obj, int8_t *objidx, int32_t *pql,
                      int32_t *survivors)
{
    if (!in) return fail(PE_ERR_ARG, "null instance");
    if (!in->initialized) return fail(PE_ERR_STATE, "population not initialised");
    const Shape &s = in->s;
    const PopBuf &b = in->buf[in->cur];
    // after init only the first N slots hold solutions
    const int nsol = in->generation == 0 ? s.N : 2 * s.N;
    if (codon_idx) {
        if (in->generation == 0) memset(codon_idx, 0, (size_t)2 * s.N * s.m * s.L);
        // rows are padded to Lp on the device: pack them there (a pitched device copy),
        // then make one contiguous copy to the host (a pitched copy into pageable host
        // memory goes row by row and is several times slower).  The packed rows go to
        // the codon ids of the other ping-pong buffer: between generations nothing
        // reads it, and the next generation writes all of it before reading any.
        const size_t rows = (size_t)nsol * s.m;
        const uint8_t *src = b.ids;
        if (s.Lp != s.L) {
            uint8_t *packed = in->buf[1 - in->cur].ids;
            CK(cudaMemcpy2DAsync(packed, (size_t)s.L, b.ids, (size_t)s.Lp, (size_t)s.L, rows, cudaMemcpyDeviceToDevice,
                                 in->stream));
            src = packed;
        }
        CK(cudaMemcpyAsync(codon_idx, src, rows * s.L, cudaMemcpyDeviceToHost, in->stream));
    }
    if (obj) CK(cudaMemcpyAsync(obj, b.obj, (size_t)2 * s.N * s.M * sizeof(float), cudaMemcpyDeviceToHost, in->stream));
    if (objidx) CK(cudaMemcpyAsync(objidx, b.objidx, (size_t)2 * s.N * 2 * s.M, cudaMemcpyDeviceToHost, in->stream));
    if (pql) CK(cudaMemcpyAsync(pql, b.pql, (size_t)2 * s.N * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, in->stream));
    if (survivors)
        CK(cudaMemcpyAsync(survivors, in->d_surv, (size_t)s.N * sizeof(int32_t), cudaMemcpyDeviceToHost, in->stream));
    return check_status(in);   // the status read queues behind the copies; one synchronisation
}

int pe_get_objectives(pe_instance *in, float *obj)
{
    return pe_get_population(in, nullptr, obj, nullptr, nullptr, nullptr);
}

int pe_read_objectives_async(pe_instance *in, float *obj)
{
    if (!in || !obj) return fail(PE_ERR_ARG, "bad arguments");
    if (!in->initialized) return fail(PE_ERR_STATE, "population not initialised");
    const Shape &s = in->s;
    CK(cudaMemcpyAsync(obj, in->buf[in->cur].obj, (size_t)2 * s.N * s.M * sizeof(float), cudaMemcpyDeviceToHost,
                       in->stream));
    return PE_OK;
}

int pe_eval_objectives(pe_instance *in, const uint8_t *codon_idx, int32_t n, float *obj, int8_t *objidx, int32_t *pql)
{
    if (!in || !codon_idx || n < 0) return fail(PE_ERR_ARG, "bad arguments");
    if (n == 0) return PE_OK;
    const Shape &s = in->s;
    for (size_t i = 0; i < (size_t)n * s.m * s.L; i++)
        if (codon_idx[i] >= PE_NUM_CODON) return fail(PE_ERR_ARG, "codon id out of range at %zu", i);
    TempBufs t(in);
    PopBuf b{};
    int2 *part;
    int32_t *counter;
    int rc;
    if ((rc = t.pop(s, b, n))) return rc;
    if ((rc = t.get(&part, (size_t)n * s.nres))) return rc;
    if ((rc = t.get(&counter, (size_t)n))) return rc;
    CK(cudaMemsetAsync(b.ids, 0, (size_t)n * s.m * s.Lp, in->stream));
    CK(cudaMemsetAsync(b.obj, 0, (size_t)n * s.M * sizeof(float), in->stream));
    CK(cudaMemsetAsync(b.objidx, 0, (size_t)n * 2 * s.M, in->stream));
    CK(cudaMemsetAsync(counter, 0, (size_t)n * sizeof(int32_t), in->stream));
    CK(cudaMemcpy2DAsync(b.ids, (size_t)s.Lp, codon_idx, (size_t)s.L, (size_t)s.L, (size_t)n * s.m,
                         cudaMemcpyHostToDevice, in->stream));
    CK(launch_light_eval(s, in->d_tab, in->d_aa, b, 0, n, in->stream));
    CK(launch_sl(s, b, 0, n, part, counter, in->d_status, in->stream, in->d_scanned));
    if (obj) CK(cudaMemcpyAsync(obj, b.obj, (size_t)n * s.M * sizeof(float), cudaMemcpyDeviceToHost, in->stream));
    if (objidx) CK(cudaMemcpyAsync(objidx, b.objidx, (size_t)n * 2 * s.M, cudaMemcpyDeviceToHost, in->stream));
    if (pql) CK(cudaMemcpyAsync(pql, b.pql, (size_t)n * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, in->stream));
    CK(cudaStreamSynchronize(in->stream));
    return check_status(in);
}

int pe_mutate(pe_instance *in, uint32_t generation, const int32_t *idx, int32_t n, const uint8_t *parents,
              const float *pobj, const int8_t *pobjidx, const int32_t *ppql, uint8_t *children, int32_t *ops)
{
    if (!in || !idx || !parents || !pobj || !pobjidx || !ppql || n < 0) return fail(PE_ERR_ARG, "bad arguments");
    if (n == 0) return PE_OK;
    const Shape &s = in->s;
    for (size_t i = 0; i < (size_t)n * s.m * s.L; i++)
        if (parents[i] >= PE_NUM_CODON) return fail(PE_ERR_ARG, "codon id out of range at %zu", i);
    TempBufs t(in);
    PopBuf src{}, dst{};
    int32_t *d_par, *d_idx, *d_ops;
    uint32_t *d_g;
    int rc;
    if ((rc = t.pop(s, src, n))) return rc;
    if ((rc = t.pop(s, dst, n))) return rc;
    if ((rc = t.get(&d_par, (size_t)n))) return rc;
    if ((rc = t.get(&d_idx, (size_t)n))) return rc;
    if ((rc = t.get(&d_ops, (size_t)n))) return rc;
    if ((rc = t.get(&d_g, 1))) return rc;
    std::vector<int32_t> ident(n);
    for (int i = 0; i < n; i++) ident[i] = i;
    CK(cudaMemsetAsync(src.ids, 0, (size_t)n * s.m * s.Lp, in->stream));
    CK(cudaMemcpy2DAsync(src.ids, (size_t)s.Lp, parents, (size_t)s.L, (size_t)s.L, (size_t)n * s.m,
                         cudaMemcpyHostToDevice, in->stream));
    CK(cudaMemcpyAsync(src.obj, pobj, (size_t)n * s.M * sizeof(float), cudaMemcpyHostToDevice, in->stream));
    CK(cudaMemcpyAsync(src.objidx, pobjidx, (size_t)n * 2 * s.M, cudaMemcpyHostToDevice, in->stream));
    CK(cudaMemcpyAsync(src.pql, ppql, (size_t)n * 3 * sizeof(int32_t), cudaMemcpyHostToDevice, in->stream));
    CK(cudaMemcpyAsync(d_par, ident.data(), (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, in->stream));
    CK(cudaMemcpyAsync(d_idx, idx, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, in->stream));
    CK(cudaMemcpyAsync(d_g, &generation, sizeof(uint32_t), cudaMemcpyHostToDevice, in->stream));
    CK(launch_mutate(s, in->d_tab, in->d_aa, src, dst, d_par, d_idx, n, -1, 0, d_g, d_ops, nullptr, in->stream));
    if (children)
        CK(cudaMemcpy2DAsync(children, (size_t)s.L, dst.ids, (size_t)s.Lp, (size_t)s.L, (size_t)n * s.m,
                             cudaMemcpyDeviceToHost, in->stream));
    if (ops) CK(cudaMemcpyAsync(ops, d_ops, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, in->stream));
    CK(cudaStreamSynchronize(in->stream));
    return PE_OK;
}

int pe_select(pe_instance *in, uint32_t generation, const float *obj, float *extremes, int32_t *survivors,
              int32_t *front, pe_select_info *info)
{
    if (!in || !obj || !extremes) return fail(PE_ERR_ARG, "bad arguments");
    const Shape &s = in->s;
    const int N2 = 2 * s.N;
    TempBufs t(in);
    float *d_obj, *d_ext;
    int32_t *d_sv;
    uint32_t *d_g;
    int rc;
    if ((rc = t.get(&d_obj, (size_t)N2 * s.M))) return rc;
    if ((rc = t.get(&d_ext, (size_t)s.M * s.M))) return rc;
    if ((rc = t.get(&d_sv, (size_t)s.N))) return rc;
    if ((rc = t.get(&d_g, 1))) return rc;
    CK(cudaMemcpyAsync(d_obj, obj, (size_t)N2 * s.M * sizeof(float), cudaMemcpyHostToDevice, in->stream));
    CK(cudaMemcpyAsync(d_ext, extremes, (size_t)s.M * s.M * sizeof(float), cudaMemcpyHostToDevice, in->stream));
    CK(cudaMemsetAsync(d_sv, 0xff, (size_t)s.N * sizeof(int32_t), in->stream));
    CK(cudaMemcpyAsync(d_g, &generation, sizeof(uint32_t), cudaMemcpyHostToDevice, in->stream));
    CK(launch_select(s, d_obj, d_ext, in->d_ref, in->sc, d_sv, d_g, 0, in->stream));
    CK(cudaMemcpyAsync(extremes, d_ext, (size_t)s.M * s.M * sizeof(float), cudaMemcpyDeviceToHost, in->stream));
    if (survivors) CK(cudaMemcpyAsync(survivors, d_sv, (size_t)s.N * sizeof(int32_t), cudaMemcpyDeviceToHost, in->stream));
    if (front) CK(cudaMemcpyAsync(front, in->sc.front, (size_t)N2 * sizeof(int32_t), cudaMemcpyDeviceToHost, in->stream));
    int32_t hi[8];
    float hf[3 * PE_MAX_OBJ];
    CK(cudaMemcpyAsync(hi, in->sc.info, sizeof hi, cudaMemcpyDeviceToHost, in->stream));
    CK(cudaMemcpyAsync(hf, in->sc.finfo, sizeof hf, cudaMemcpyDeviceToHost, in->stream));
    CK(cudaStreamSynchronize(in->stream));
    if (info) {
        memset(info, 0, sizeof *info);
        info->rank_count = hi[0];
        info->last_front_size = hi[1];
        info->n_fronts = hi[2];
        info->cut = hi[3];
        info->hyp_exception = hi[4];
        for (int k = 0; k < s.M; k++) {
            info->ideal[k] = hf[k];
            info->worst[k] = hf[s.M + k];
            info->nadir[k] = hf[2 * s.M + k];
        }
    }
    return PE_OK;
}

// ---------------------------------------------------------------- host inputs

int pe_parse_fasta(const char *path, int8_t *aa_out, int32_t capacity, int32_t *aa_len)
{
    // src/main.cu:491-523: first line (<= 255 chars) skipped, '\n' dropped,
    // the final read (EOF) replaced by the stop letter 'Z'
    if (!path || !aa_len) return fail(PE_ERR_ARG, "null argument");
    FILE *fp = fopen(path, "r");
    if (!fp) return fail(PE_ERR_IO, "cannot open %s", path);
    char buffer[256];
    if (!fgets(buffer, 256, fp)) {
        fclose(fp);
        return fail(PE_ERR_IO, "%s: empty file", path);
    }
    std::string seq;
    int ch;
    while ((ch = fgetc(fp)) != EOF)
        if (ch != '\n') seq.push_back((char)ch);
    fclose(fp);
    seq.push_back('Z');
    if (seq.size() < 3) return fail(PE_ERR_IO, "%s: sequence too short", path);
    *aa_len = (int32_t)seq.size();
    if (!aa_out) return PE_OK;
    if ((int32_t)seq.size() > capacity) return fail(PE_ERR_ARG, "capacity %d < %zu", capacity, seq.size());
    for (size_t i = 0; i < seq.size(); i++) {
        int a = amino_index(seq[i]);
        if (a < 0) return fail(PE_ERR_IO, "%s: unknown amino letter '%c' at %zu", path, seq[i], i);
        aa_out[i] = (int8_t)a;
    }
    return PE_OK;
}

int pe_synthetic_protein(int32_t L, uint64_t seed, int8_t *aa_out)
{
    if (L < 2 || !aa_out) return fail(PE_ERR_ARG, "bad arguments");
    uint64_t x = seed;
    for (int i = 0; i < L; i++) aa_out[i] = (int8_t)(((splitmix64(x) >> 32) * 20ull) >> 32);
    aa_out[L] = 20;
    return PE_OK;
}

static void standard_code(pe_codon_table *t)
{
    // the standard genetic code, grouped by amino acid in index order
    static const char *groups[21] = {"GCU GCC GCA GCG", "UGU UGC", "GAU GAC", "GAA GAG", "UUU UUC",
                                     "GGU GGC GGA GGG", "CAU CAC", "AUU AUC AUA", "AAA AAG",
                                     "UUA UUG CUU CUC CUA CUG", "AUG", "AAU AAC", "CCU CCC CCA CCG", "CAA CAG",
                                     "CGU CGC CGA CGG AGA AGG", "UCU UCC UCA UCG AGU AGC", "ACU ACC ACA ACG",
                                     "GUU GUC GUA GUG", "UGG", "UAU UAC", "UAA UAG UGA"};
    int id = 0;
    for (int a = 0; a < 21; a++) {
        t->start[a] = (int8_t)id;
        int k = 0;
        for (const char *p = groups[a]; *p; p += (p[3] ? 4 : 3)) {
            for (int b = 0; b < 3; b++) {
                char c = p[b];
                t->nt[id][b] = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : 3;
            }
            id++;
            k++;
            if (!p[3]) break;
        }
        t->count[a] = (int8_t)k;
    }
}

int pe_dirichlet_table(uint64_t seed, pe_codon_table *out)
{
    if (!out) return fail(PE_ERR_ARG, "null table");
    memset(out, 0, sizeof *out);
    pe_codon_table base;
    memset(&base, 0, sizeof base);
    standard_code(&base);
    uint64_t x = seed;
    for (int a = 0; a < 21; a++) {
        int k = base.count[a], st = base.start[a];
        double g[6], gmax = 0.0;
        for (int j = 0; j < k; j++) {
            double u = (double)((splitmix64(x) >> 11) + 1) * (1.0 / 9007199254740992.0);
            g[j] = -log(u);  // Gamma(1) draw; Dirichlet(1) after normalisation
            gmax = std::max(gmax, g[j]);
        }
        float w[6];
        int order[6];
        for (int j = 0; j < k; j++) {
            w[j] = (float)(g[j] / gmax);
            order[j] = j;
        }
        // ascending weight inside the group (the reference assumes the last codon is the best)
        std::stable_sort(order, order + k, [&](int p, int q) { return w[p] < w[q]; });
        out->start[a] = base.start[a];
        out->count[a] = base.count[a];
        for (int j = 0; j < k; j++) {
            for (int b = 0; b < 3; b++) out->nt[st + j][b] = base.nt[st + order[j]][b];
            out->weight[st + j] = w[order[j]];
        }
    }
    for (int i = 0; i < 61 * 61; i++) {
        double u = (double)(splitmix64(x) >> 11) * (1.0 / 9007199254740992.0);
        out->cps[i] = (float)(0.8 * u - 0.4);
    }
    out->ref_gc3 = 0.3810f;
    out->ref_gc = 0.3977f;
    return PE_OK;
}

int pe_load_codon_table(const char *path, pe_codon_table *out)
{
    if (!path || !out) return fail(PE_ERR_ARG, "null argument");
    FILE *fp = fopen(path, "r");
    if (!fp) return fail(PE_ERR_IO, "cannot open %s", path);
    memset(out, 0, sizeof *out);
    out->ref_gc3 = 0.3810f;
    out->ref_gc = 0.3977f;
    std::vector<char> linebuf(1 << 16);
    char *line = linebuf.data();
    int id = 0, last_aa = -1;
    int counts[21] = {0};
    int ncps = 0;
    bool in_cps = false;
    while (fgets(line, (int)linebuf.size(), fp)) {
        size_t len = strlen(line);
        if (len == linebuf.size() - 1 && line[len - 1] != '\n' && !feof(fp)) {
            fclose(fp);
            return fail(PE_ERR_IO, "%s: line longer than %zu characters", path, linebuf.size() - 2);
        }
        char *p = line;
        while (*p == ' ' || *p == '\t') p++;
        if (*p == '#' || *p == '\n' || *p == 0) continue;
        if (in_cps) {
            char *e = p;
            while (*e) {
                char *q;
                double v = strtod(e, &q);
                if (q == e) break;
                if (ncps < 61 * 61) out->cps[ncps++] = (float)v;
                e = q;
            }
            continue;
        }
        if (!strncmp(p, "cps", 3)) {
            in_cps = true;
            continue;
        }
        if (!strncmp(p, "gc3 ", 4)) {
            out->ref_gc3 = strtof(p + 4, nullptr);
            continue;
        }
        if (!strncmp(p, "gc ", 3)) {
            out->ref_gc = strtof(p + 3, nullptr);
            continue;
        }
        char cod[8], aa;
        float w;
        if (sscanf(p, "%7s %c %f", cod, &aa, &w) != 3 || strlen(cod) != 3) {
            fclose(fp);
            return fail(PE_ERR_IO, "%s: cannot parse line '%s'", path, p);
        }
        int a = amino_index(aa);
        if (a < 0 || id >= 64 || a < last_aa) {
            fclose(fp);
            return fail(PE_ERR_IO, "%s: codon %d (%s %c) out of order", path, id, cod, aa);
        }
        for (int b = 0; b < 3; b++) {
            char c = cod[b];
            if (c != 'A' && c != 'C' && c != 'G' && c != 'U') {
                fclose(fp);
                return fail(PE_ERR_IO, "%s: bad codon %s", path, cod);
            }
            out->nt[id][b] = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : 3;
        }
        out->weight[id] = w;
        counts[a]++;
        last_aa = a;
        id++;
    }
    fclose(fp);
    if (id != 64) return fail(PE_ERR_IO, "%s: %d codons (need 64)", path, id);
    if (in_cps && ncps != 61 * 61) return fail(PE_ERR_IO, "%s: %d CPS values (need %d)", path, ncps, 61 * 61);
    int st = 0;
    for (int a = 0; a < 21; a++) {
        out->start[a] = (int8_t)st;
        out->count[a] = (int8_t)counts[a];
        st += counts[a];
    }
    return PE_OK;
}

}  // extern "C"
