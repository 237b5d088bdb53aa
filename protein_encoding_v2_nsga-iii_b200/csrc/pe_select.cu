// pe_select.cu -- environmental selection (sortingKernel, src/main.cu:409-454).
//
//  k_dominance  one CTA per solution i: row i of the 2N x 2N dominance bit
//               matrix (bit j set when j dominates i) built with __ballot_sync,
//               and np[i] = popc(row) -- replaces the reference's two (2N)^2
//               bool matrices (include/sorting.cuh:974-1089).
//  k_select     one CTA: front peeling on the bit matrix, ideal / worst,
//               extreme points, hyperplane (Gaussian elimination) or MNDF nadir,
//               reference-point association and niche selection, stopping at
//               exactly N survivors (include/sorting.cuh:94-1282).
//
// Deterministic rules (the reference decides these by atomic order):
// fronts are listed in ascending solution index; each niche level visits
// reference points in ascending index; random niche picks come from Philox
// keyed by (generation, reference point, level).
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#include "pe_device.cuh"
#include "pe_internal.h"

namespace pe {

__device__ __forceinline__ bool dominates(const float *a, const float *b, int M)
{
    // dominate (include/sorting.cuh:94-130): |a-b| <= 1e-6 counts as equal
    int eq = 0;
    bool worse = false;
    for (int k = 0; k < M; k++) {
        float d = fabsf(__fsub_rn(a[k], b[k]));
        if (d > 1e-6f) {
            if (a[k] > b[k]) worse = true;
        } else {
            eq++;
        }
    }
    return eq != M && !worse;
}

__global__ void __launch_bounds__(256) k_dominance(Shape s, const float *__restrict__ obj, uint32_t *__restrict__ dom,
                                                   int32_t *__restrict__ np)
{
    __shared__ int wsum[8];
    const int N2 = 2 * s.N, words = (N2 + 31) >> 5;
    const int i = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float oi[kMaxObj];
    for (int k = 0; k < s.M; k++) oi[k] = obj[(size_t)i * s.M + k];
    int cnt = 0;
    for (int w = warp; w < words; w += 8) {
        int j = 32 * w + lane;
        bool bit = false;
        if (j < N2 && j != i) {
            float oj[kMaxObj];
            for (int k = 0; k < s.M; k++) oj[k] = __ldg(&obj[(size_t)j * s.M + k]);
            bit = dominates(oj, oi, s.M);
        }
        uint32_t word = __ballot_sync(0xffffffffu, bit);
        if (lane == 0) dom[(size_t)i * words + w] = word;
        cnt += __popc(word);
    }
    if (lane == 0) wsum[warp] = cnt;
    __syncthreads();
    if (tid == 0) {
        int t = 0;
        for (int w = 0; w < 8; w++) t += wsum[w];
        np[i] = t;
    }
}

struct SelSmem {
    int warp_tot[33];
    int i0, i1, i2, i3, i4;
    int rc, fstart, fsize, cut, nfront, count, level, hyp;
    float ideal[kMaxObj], worst[kMaxObj], nadir[kMaxObj];
    float red[64 * kMaxObj];
    float ext[kMaxObj * kMaxObj];  // extreme points while they are updated
};

// exclusive block scan of a 0/1 flag over kSelThreads threads; returns the
// prefix and leaves the total in *total (all threads)
__device__ __forceinline__ int block_scan_flag(int flag, SelSmem &sm, int *total)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    uint32_t b = __ballot_sync(0xffffffffu, flag);
    int wp = __popc(b & ((1u << lane) - 1u));
    if (lane == 0) sm.warp_tot[warp] = __popc(b);
    __syncthreads();
    if (warp == 0) {
        int v = lane < nwarps ? sm.warp_tot[lane] : 0;
        int inc = v;
        for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        sm.warp_tot[lane] = inc - v;
        if (lane == 31) sm.warp_tot[32] = inc;
    }
    __syncthreads();
    int res = sm.warp_tot[warp] + wp;
    *total = sm.warp_tot[32];
    __syncthreads();
    return res;
}

__device__ __forceinline__ float asf_val(const float *x, const float *ideal, int i, int M)
{
    // ASF (include/sorting.cuh:428-449) with weights 1 (objective i) / 1e-6
    float mx = -FLT_MAX;
    for (int k = 0; k < M; k++) {
        float tmp = __fsub_rn(x[k], ideal[k]);
        if ((double)tmp < 0.001) tmp = 0.0f;
        float q = __fdiv_rn(tmp, k == i ? 1.0f : 1e-6f);
        if (q > mx) mx = q;
    }
    return mx;
}

__global__ void __launch_bounds__(kSelThreads) k_select(Shape s, const float *__restrict__ obj, float *ext,
                                                        const float *__restrict__ refpts, SelectScratch sc,
                                                        int32_t *surv, uint32_t *d_gen, int bump_gen)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SelSmem &sm = *reinterpret_cast<SelSmem *>(smem_raw);
    const int N = s.N, N2 = 2 * N, M = s.M, R = s.R;
    const int words = (N2 + 31) >> 5;
    uint32_t *fmask = reinterpret_cast<uint32_t *>(smem_raw + ((sizeof(SelSmem) + 15) & ~size_t(15)));
    float *tbuf = reinterpret_cast<float *>(fmask + ((words + 3) & ~3));
    int32_t *tix = reinterpret_cast<int32_t *>(tbuf + ((N2 + M + 3) & ~3));
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
    (void)d_gen;
    (void)bump_gen;

    // ---------------- front 0 (np == 0), ascending index
    for (int i = tid; i < N2; i += nth) sc.front[i] = -1;
    if (tid == 0) sm.rc = 0;
    __syncthreads();
    for (int base = 0; base < N2; base += nth) {
        int i = base + tid;
        int flag = (i < N2) && sc.np[i] == 0;
        int tot;
        int pos = block_scan_flag(flag, sm, &tot);
        if (flag) {
            sc.front[i] = 0;
            sc.sorted[sm.rc + pos] = i;
        }
        __syncthreads();
        if (tid == 0) sm.rc += tot;
        __syncthreads();
    }
    const int f0 = sm.rc;
    if (tid == 0) {
        sm.fstart = 0;
        sm.fsize = f0;
        sm.cut = (f0 == N);
        sm.nfront = 1;
    }
    __syncthreads();
    // ---------------- later fronts (only while fewer than N are assigned)
    if (f0 < N) {
        for (int it = 0; it < N2 - 1; it++) {
            for (int w = tid; w < words; w += nth) fmask[w] = 0u;
            __syncthreads();
            for (int u = sm.fstart + tid; u < sm.fstart + sm.fsize; u += nth) {
                int j = sc.sorted[u];
                atomicOr(&fmask[j >> 5], 1u << (j & 31));
            }
            __syncthreads();
            const int rc0 = sm.rc;
            const int cf = sm.nfront;
            for (int base = 0; base < N2; base += nth) {
                int i = base + tid;
                int flag = 0;
                if (i < N2 && sc.front[i] < 0) {
                    const uint32_t *row = sc.dom + (size_t)i * words;
                    int dec = 0;
                    for (int w = 0; w < words; w++) {
                        uint32_t f = fmask[w];
                        if (f) dec += __popc(row[w] & f);
                    }
                    int v = sc.np[i] - dec;
                    sc.np[i] = v;
                    flag = (v == 0);
                }
                int tot;
                int pos = block_scan_flag(flag, sm, &tot);
                if (flag) {
                    sc.front[i] = cf;
                    sc.sorted[sm.rc + pos] = i;
                }
                __syncthreads();
                if (tid == 0) sm.rc += tot;
                __syncthreads();
            }
            if (tid == 0) {
                sm.fstart = rc0;
                sm.fsize = sm.rc - rc0;
                sm.nfront = cf + 1;
                if (sm.rc >= N) sm.cut = (sm.rc == N);
            }
            __syncthreads();
            if (sm.rc >= N) break;
        }
    }
    const int rc = sm.rc;
    const int last_size = sm.fsize;

    // ---------------- ideal / worst (exact min / max)
    {
        float mn[kMaxObj], mx[kMaxObj];
        for (int k = 0; k < M; k++) {
            mn[k] = FLT_MAX;
            mx[k] = -FLT_MAX;
        }
        for (int i = tid; i < N2; i += nth)
            for (int k = 0; k < M; k++) {
                float v = obj[(size_t)i * M + k];
                if (v < mn[k]) mn[k] = v;
                if (v > mx[k]) mx[k] = v;
            }
        for (int k = 0; k < M; k++) {
            for (int o = 16; o > 0; o >>= 1) {
                float a = __shfl_xor_sync(0xffffffffu, mn[k], o), b = __shfl_xor_sync(0xffffffffu, mx[k], o);
                if (a < mn[k]) mn[k] = a;
                if (b > mx[k]) mx[k] = b;
            }
        }
        if (lane == 0)
            for (int k = 0; k < M; k++) {
                sm.red[warp * kMaxObj + k] = mn[k];
                sm.red[32 * kMaxObj + warp * kMaxObj + k] = mx[k];
            }
        __syncthreads();
        if (tid < M) {
            float a = FLT_MAX, b = -FLT_MAX;
            for (int w = 0; w < (nth >> 5); w++) {
                float u = sm.red[w * kMaxObj + tid], v = sm.red[32 * kMaxObj + w * kMaxObj + tid];
                if (u < a) a = u;
                if (v > b) b = v;
            }
            sm.ideal[tid] = a;
            sm.worst[tid] = b;
        }
        __syncthreads();
    }

    // ---------------- extreme points (findExtremePoints, :601-683), tree order of findMinValue
    {
        const int B = N2 + M;
        for (int e = tid; e < M * M; e += nth) sm.ext[e] = ext[e];
        __syncthreads();
        auto value = [&](int t, int i, int &ix) {
            if (t < f0) {
                const int sol = sc.sorted[t];
                ix = sol;
                return asf_val(obj + (size_t)sol * M, sm.ideal, i, M);
            }
            if (t < f0 + M) {
                ix = N2 + (t - f0);
                return asf_val(sm.ext + (t - f0) * M, sm.ideal, i, M);
            }
            ix = -1;
            return FLT_MAX;
        };
        // tbuf[t] < tbuf[u] replaces t by u (strict: the lower position keeps ties)
        auto pair = [&](int t, int u) {
            if (tbuf[u] < tbuf[t]) {
                tbuf[t] = tbuf[u];
                tix[t] = tix[u];
            }
        };
        for (int i = 0; i < M; i++) {
            // first level fused with the ASF values: position t against t + B/2
            int h = B / 2;
            for (int t = tid; t < h; t += nth) {
                int i0, i1;
                const float v0 = value(t, i, i0), v1 = value(t + h, i, i1);
                tbuf[t] = v1 < v0 ? v1 : v0;
                tix[t] = v1 < v0 ? i1 : i0;
            }
            __syncthreads();
            // later levels; after an odd level its last position joins position 0,
            // done by the thread that handles position 0 next; levels of at most 32
            // pairs run in warp 0 alone
            while (h > 1) {
                const bool odd = h & 1;
                const int hp = h - 1;
                h >>= 1;
                if (h > 32) {
                    for (int t = tid; t < h; t += nth) {
                        if (t == 0 && odd) pair(0, hp);
                        pair(t, t + h);
                    }
                    __syncthreads();
                } else if (warp == 0) {
                    if (lane < h) {
                        if (lane == 0 && odd) pair(0, hp);
                        pair(lane, lane + h);
                    }
                    __syncwarp();
                }
            }
            if (tid == 0) {
                const int sel = tix[0];
                float tmp[kMaxObj];
                if (sel >= N2) {
                    for (int k = 0; k < M; k++) tmp[k] = sm.ext[(sel - N2) * M + k];
                } else if (sel >= 0) {
                    for (int k = 0; k < M; k++) tmp[k] = obj[(size_t)sel * M + k];
                }
                if (sel >= 0)
                    for (int k = 0; k < M; k++) {
                        sm.ext[i * M + k] = tmp[k];
                        ext[i * M + k] = tmp[k];
                    }
            }
            __syncthreads();
        }
    }

    // ---------------- hyperplane intercepts (GaussianElimination :555-599, check :929-956)
    if (tid == 0) {
        float AB[kMaxObj][kMaxObj + 1], x[kMaxObj];
        for (int i = 0; i < M; i++) {
            for (int j = 0; j < M; j++) AB[i][j] = sm.ext[i * M + j];
            AB[i][M] = 1.0f;
        }
        for (int c = 0; c < M; c++) {
            if ((double)fabsf(AB[c][c]) <= 1e-6) {
                int r = c;
                while (r < M && !((double)fabsf(AB[r][c]) > 1e-6)) r++;
                if (r < M)
                    for (int j = c; j <= M; j++) AB[c][j] = __fadd_rn(AB[c][j], AB[r][j]);
            }
            for (int r = c + 1; r < M; r++) {
                float f = __fdiv_rn(AB[r][c], AB[c][c]);
                for (int j = c; j <= M; j++) AB[r][j] = __fsub_rn(AB[r][j], __fmul_rn(f, AB[c][j]));
            }
        }
        for (int r = M - 1; r >= 0; r--) {
            float sacc = 0.0f;
            for (int j = r + 1; j < M; j++) sacc = __fadd_rn(sacc, __fmul_rn(AB[r][j], x[j]));
            x[r] = __fdiv_rn(__fsub_rn(AB[r][M], sacc), AB[r][r]);
        }
        int exc = 0;
        for (int k = 0; k < M; k++) {
            float res = 0.0f;
            for (int i = 0; i < M; i++) res = __fadd_rn(res, __fmul_rn(x[i], __fsub_rn(sm.ext[k * M + i], sm.ideal[i])));
            if (fabsf(__fsub_rn(res, 1.0f)) > 1e-6f || isnan(res) || isinf(res)) exc = 1;
            float icp = __fdiv_rn(1.0f, x[k]);
            if (icp <= 1e-6f || isnan(icp) || isinf(icp)) exc = 1;
            sm.nadir[k] = __fadd_rn(sm.ideal[k], icp);
        }
        sm.hyp = exc;
    }
    __syncthreads();
    if (sm.hyp) {
        // updateNadirValue_MNDF (:685-884): max over front 0, worst when too close to ideal
        float mx[kMaxObj];
        for (int k = 0; k < M; k++) mx[k] = -FLT_MAX;
        for (int t = tid; t < f0; t += nth) {
            int sol = sc.sorted[t];
            for (int k = 0; k < M; k++) {
                float v = obj[(size_t)sol * M + k];
                if (v > mx[k]) mx[k] = v;
            }
        }
        for (int k = 0; k < M; k++)
            for (int o = 16; o > 0; o >>= 1) {
                float b = __shfl_xor_sync(0xffffffffu, mx[k], o);
                if (b > mx[k]) mx[k] = b;
            }
        __syncthreads();
        if (lane == 0)
            for (int k = 0; k < M; k++) sm.red[warp * kMaxObj + k] = mx[k];
        __syncthreads();
        if (tid < M) {
            float b = -FLT_MAX;
            for (int w = 0; w < (nth >> 5); w++) {
                float v = sm.red[w * kMaxObj + tid];
                if (v > b) b = v;
            }
            sm.nadir[tid] = __fsub_rn(b, sm.ideal[tid]) > 1e-6f ? b : sm.worst[tid];
        }
        __syncthreads();
    }
    if (tid == 0) {
        sc.info[0] = rc;
        sc.info[1] = last_size;
        sc.info[2] = sm.nfront;
        sc.info[3] = sm.cut;
        sc.info[4] = sm.hyp;
        for (int k = 0; k < M; k++) {
            sc.finfo[k] = sm.ideal[k];
            sc.finfo[M + k] = sm.worst[k];
            sc.finfo[2 * M + k] = sm.nadir[k];
        }
    }
    if (sm.cut) {
        for (int t = tid; t < N; t += nth) surv[t] = sc.sorted[t];
        return;  // k_niche advances the generation counter
    }

    // niche counts are filled by k_assoc
    for (int j = tid; j < R; j += nth) {
        sc.rho[j] = 0;
        sc.ncand[j] = 0;
    }
    if (tid == 0) sc.info[5] = rc - last_size;
}

// referenceBasedSorting phase 1 (:1105-1180) on the whole grid: one warp per
// solution of fronts 0..last, lanes over reference points; perpendicular
// distance (include/utils.cuh:1149-1171), argmin with the lowest index on ties.
__global__ void __launch_bounds__(256) k_assoc(Shape s, const float *__restrict__ obj,
                                               const float *__restrict__ refpts, SelectScratch sc)
{
    if (sc.info[3]) return;  // fronts filled N exactly: no niching
    const int M = s.M, R = s.R;
    const int rc = sc.info[0], count0 = sc.info[5];
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    float ideal[kMaxObj], span[kMaxObj];
    for (int k = 0; k < M; k++) {
        ideal[k] = sc.finfo[k];
        span[k] = __fsub_rn(sc.finfo[2 * M + k], ideal[k]);
    }
    for (int t = gw; t < rc; t += nw) {
        const int sol = sc.sorted[t];
        float f[kMaxObj];
        for (int k = 0; k < M; k++) f[k] = __fdiv_rn(__fsub_rn(obj[(size_t)sol * M + k], ideal[k]), span[k]);
        float best = FLT_MAX;
        int bj = 0;
        for (int j = lane; j < R; j += 32) {
            const float *w = refpts + (size_t)j * M;
            float num = 0.0f, den = 0.0f;
            for (int k = 0; k < M; k++) {
                num = __fadd_rn(num, __fmul_rn(w[k], f[k]));
                den = __fadd_rn(den, __fmul_rn(w[k], w[k]));
            }
            float kk = __fdiv_rn(num, den);
            float d2 = 0.0f;
            for (int k = 0; k < M; k++) {
                float e = __fsub_rn(__fmul_rn(kk, w[k]), f[k]);
                d2 = __fadd_rn(d2, __fmul_rn(e, e));
            }
            float d = __fsqrt_rn(d2);
            if (d < best) {
                best = d;
                bj = j;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            float ob = __shfl_xor_sync(0xffffffffu, best, o);
            int oj = __shfl_xor_sync(0xffffffffu, bj, o);
            if (ob < best || (ob == best && oj < bj)) {
                best = ob;
                bj = oj;
            }
        }
        if (lane == 0) {
            sc.dist[sol] = best;
            sc.assoc[t] = bj;
            atomicAdd(t < count0 ? &sc.rho[bj] : &sc.ncand[bj], 1);
        }
    }
}

// exclusive block scan of an int over the CTA; returns the prefix and leaves
// the total in *total (all threads)
__device__ __forceinline__ int block_scan_value(int v, SelSmem &sm, int *total)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    int inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) sm.warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < nwarps ? sm.warp_tot[lane] : 0;
        int x = w;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane < nwarps) sm.warp_tot[lane] = x - w;
        if (lane == 31) sm.warp_tot[32] = x;
    }
    __syncthreads();
    const int r = sm.warp_tot[warp] + inc - v;
    *total = sm.warp_tot[32];
    __syncthreads();
    return r;
}

// referenceBasedSorting phase 2 (:1182-1279): candidate lists and niche levels.
//
// The reference visits levels 0, 1, 2, ... and, within a level, the reference
// points in ascending index; point j takes one candidate at every level from
// its niche count c_j on while it has candidates (n_j of them), until N are
// chosen.  So j picks at levels c_j .. c_j + n_j - 1, every level before the
// level L* at which the N-th pick falls is complete, and at L* the first K
// active points pick.  This kernel computes L* and K from a histogram over
// levels, lets every point draw its own picks (the draws of point j depend
// only on j, its levels and its list), and writes each level's picks to their
// positions with one warp per level: the same survivors, in the same order,
// as the level-by-level loop, in a fixed number of steps.
__global__ void __launch_bounds__(kSelThreads) k_niche(Shape s, SelectScratch sc, int32_t *surv, uint32_t *d_gen,
                                                       int bump_gen)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SelSmem &sm = *reinterpret_cast<SelSmem *>(smem_raw);
    const int N = s.N, N2 = 2 * N, R = s.R, Lsz = N2 + 4;
    int *cj = reinterpret_cast<int *>(smem_raw + ((sizeof(SelSmem) + 15) & ~size_t(15)));
    int *nj = cj + R;
    int *coff = nj + R;    // R + 1
    int *kq = coff + R + 1;
    int *lv = kq + R;      // Lsz: level histogram, then picks before each level
    int *las = lv + Lsz;   // 2N: reference point of each last-front member (position count0 + t)
    int *lsol = las + N2;  // 2N: the member itself
    int *cand = lsol + N2; // 2N: candidate lists (CSR by reference point)
    int *pofs = cand + N2; // R + 1: first pick of each point
    uint32_t *rnd = reinterpret_cast<uint32_t *>(pofs + R + 1);  // N: the raw draw of every pick
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nth >> 5;
    const uint32_t gen = *d_gen;
    if (sc.info[3]) {  // fronts filled N exactly; k_select wrote the survivors
        if (tid == 0 && bump_gen) *d_gen = gen + 1;
        return;
    }
    const int rc = sc.info[0], count0 = sc.info[5], need = N - count0;
    for (int j = tid; j < R; j += nth) {
        cj[j] = sc.rho[j];
        nj[j] = sc.ncand[j];
        kq[j] = 0;
    }
    for (int l = tid; l < Lsz; l += nth) lv[l] = 0;
    for (int t = count0 + tid; t < rc; t += nth) {
        las[t - count0] = sc.assoc[t];
        lsol[t - count0] = sc.sorted[t];
    }
    if (tid == 0) sm.i0 = 0;
    __syncthreads();
    // CSR offsets of the candidate lists; level histogram (+1 at c_j, -1 at c_j + n_j)
    for (int base = 0; base < R; base += nth) {
        const int j = base + tid;
        const int v = j < R ? nj[j] : 0;
        int tot;
        const int pos = block_scan_value(v, sm, &tot);
        if (j < R) {
            coff[j] = sm.i0 + pos;
            if (v > 0) {
                atomicAdd(&lv[min(cj[j], Lsz - 1)], 1);
                atomicAdd(&lv[min(cj[j] + v, Lsz - 1)], -1);
            }
        }
        __syncthreads();
        if (tid == 0) sm.i0 += tot;
        __syncthreads();
    }
    if (tid == 0) coff[R] = sm.i0;
    // candidate lists in ascending position (kq counts the fill)
    if (warp == 0) {
        for (int base = count0; base < rc; base += 32) {
            const int t = base + lane;
            const bool act = t < rc;
            const int j = act ? las[t - count0] : -1 - lane;
            const uint32_t peers = __match_any_sync(0xffffffffu, j);
            const int rank = __popc(peers & ((1u << lane) - 1u));
            const int f0v = act ? kq[j] : 0;
            __syncwarp();
            if (act) cand[coff[j] + f0v + rank] = lsol[t - count0];
            __syncwarp();
            if (act && rank == 0) kq[j] = f0v + __popc(peers);
            __syncwarp();
        }
    }
    // active points per level, then picks before each level: lv[l] = picks at levels < l
    if (tid == 0) {
        sm.i0 = 0;
        sm.i1 = 0;
    }
    __syncthreads();
    for (int base = 0; base < Lsz; base += nth) {
        const int l = base + tid;
        const int d = l < Lsz ? lv[l] : 0;
        int tot;
        const int act = sm.i0 + block_scan_value(d, sm, &tot) + d;  // active points at level l
        int tot2;
        const int before = sm.i1 + block_scan_value(l < Lsz ? act : 0, sm, &tot2);
        if (l < Lsz) lv[l] = before;
        __syncthreads();
        if (tid == 0) {
            sm.i0 += tot;
            sm.i1 += tot2;
        }
        __syncthreads();
    }
    // L*: the level of the last pick; K: picks at L*
    if (tid == 0) {
        sm.i2 = Lsz;
        sm.i3 = 0;
    }
    __syncthreads();
    for (int l = tid; l + 1 < Lsz; l += nth)
        if (lv[l] < need && lv[l + 1] >= need) {
            sm.i2 = l;
            sm.i3 = need - lv[l];
        }
    __syncthreads();
    const int Ls = sm.i2, K = sm.i3;
    // picks per point: every level in [c_j, min(c_j + n_j, L*)), plus L* for the first K active there
    if (tid == 0) sm.i0 = 0;
    __syncthreads();
    for (int base = 0; base < R; base += nth) {
        const int j = base + tid;
        const bool on = j < R && nj[j] > 0 && cj[j] <= Ls && Ls < cj[j] + nj[j];
        int tot;
        const int pos = sm.i0 + block_scan_flag(on, sm, &tot);
        if (j < R) kq[j] = (nj[j] > 0 ? max(0, min(cj[j] + nj[j], Ls) - cj[j]) : 0) + (on && pos < K ? 1 : 0);
        __syncthreads();
        if (tid == 0) sm.i0 += tot;
        __syncthreads();
    }
    // the raw draws of all picks, computed in parallel (each is keyed by its point and level)
    if (tid == 0) sm.i0 = 0;
    __syncthreads();
    for (int base = 0; base < R; base += nth) {
        const int j = base + tid;
        int tot;
        const int pos = sm.i0 + block_scan_value(j < R ? kq[j] : 0, sm, &tot);
        if (j < R) pofs[j] = pos;
        __syncthreads();
        if (tid == 0) sm.i0 += tot;
        __syncthreads();
    }
    if (tid == 0) pofs[R] = sm.i0;
    __syncthreads();
    for (int pk = tid; pk < pofs[R]; pk += nth) {
        int lo = 0, hi = R - 1;  // point: pofs[lo] <= pk < pofs[lo + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pofs[mid] <= pk) lo = mid;
            else hi = mid - 1;
        }
        const int level = cj[lo] + (pk - pofs[lo]);
        rnd[pk] = level == 0 ? 0u : draw(s.seed, TAG_NICHE, gen, (uint32_t)lo, (uint32_t)level, 0);
    }
    __syncthreads();
    // each point takes its picks; the q-th pick ends at list position n_j - 1 - q
    for (int j = tid; j < R; j += nth) {
        int *cl = cand + coff[j];
        int nc = nj[j];
        for (int q = 0; q < kq[j]; q++) {
            const int level = cj[j] + q;
            int slot = 0;
            if (level == 0) {
                float bd = sc.dist[cl[0]];
                for (int u = 1; u < nc; u++) {
                    const float dv = sc.dist[cl[u]];
                    if (dv < bd) {
                        bd = dv;
                        slot = u;
                    }
                }
            } else {
                slot = (int)rng_uint(rnd[pofs[j] + q], (uint32_t)nc);
            }
            const int pick = cl[slot];
            cl[slot] = cl[nc - 1];
            cl[nc - 1] = pick;
            nc--;
        }
    }
    for (int t = tid; t < count0; t += nth) surv[t] = sc.sorted[t];
    __syncthreads();
    // positions: level l's picks follow the picks of earlier levels, in ascending point index
    const int lmax = min(Ls, Lsz - 1);
    for (int l = warp; l <= lmax; l += nwarps) {
        int run = 0;
        for (int jb = 0; jb < R; jb += 32) {
            const int j = jb + lane;
            const bool act = j < R && nj[j] > 0 && cj[j] <= l && l < cj[j] + nj[j];
            const uint32_t bal = __ballot_sync(0xffffffffu, act);
            const int rank = run + __popc(bal & ((1u << lane) - 1u));
            if (act && (l < Ls || rank < K))
                surv[count0 + lv[l] + rank] = cand[coff[j] + nj[j] - 1 - (l - cj[j])];
            run += __popc(bal);
        }
    }
    __syncthreads();
    if (tid == 0 && bump_gen) *d_gen = gen + 1;
}

size_t niche_smem_bytes(const Shape &s)
{
    return ((sizeof(SelSmem) + 15) & ~size_t(15)) +
           (size_t)(4 * s.R + 1 + 2 * s.N + 4 + 3 * 2 * s.N + s.R + 1 + s.N) * sizeof(int);
}

size_t select_smem_bytes(const Shape &s)
{
    const int N2 = 2 * s.N, words = (N2 + 31) >> 5;
    return ((sizeof(SelSmem) + 15) & ~size_t(15)) + (size_t)((words + 3) & ~3) * 4 +
           (size_t)((N2 + s.M + 3) & ~3) * 4 + (size_t)(N2 + s.M) * 4;
}

cudaError_t launch_select(const Shape &s, const float *obj, float *ext, const float *refpts, SelectScratch sc,
                          int32_t *surv, uint32_t *d_gen, int bump_gen, cudaStream_t st)
{
    k_dominance<<<2 * s.N, 256, 0, st>>>(s, obj, sc.dom, sc.np);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t smem = select_smem_bytes(s);
    e = raise_smem_limit((const void *)k_select, smem);
    if (e != cudaSuccess) return e;
    k_select<<<1, kSelThreads, smem, st>>>(s, obj, ext, refpts, sc, surv, d_gen, bump_gen);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int warps_needed = 2 * s.N;
    k_assoc<<<std::min((warps_needed + 7) / 8, 148 * 8), 256, 0, st>>>(s, obj, refpts, sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t nsm = niche_smem_bytes(s);
    if ((e = raise_smem_limit((const void *)k_niche, nsm)) != cudaSuccess) return e;
    k_niche<<<1, kSelThreads, nsm, st>>>(s, sc, surv, d_gen, bump_gen);
    return cudaGetLastError();
}

}  // namespace pe
