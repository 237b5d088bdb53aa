// pe_select.cu -- environmental selection (sortingKernel, src/main.cu:409-454).
//
//  k_dominance  one CTA per solution i: row i of the 2N x 2N dominance bit
//               matrix (bit j set when j dominates i) built with __ballot_sync,
//               and np[i] = popc(row) -- replaces the reference's two (2N)^2
//               bool matrices (include/sorting.cuh:974-1089).
//  k_select     one CTA: front peeling on the bit matrix, ideal / worst,
//               extreme points, hyperplane (Gaussian elimination) or MNDF nadir
//               (include/sorting.cuh:94-972).
//  k_assoc      the whole grid, a warp per solution of fronts 0..last: nearest
//               reference point and its perpendicular distance (:1105-1180).
//  k_niche      one CTA: niche counts, candidate lists and the closed form of the
//               level-by-level niching, stopping at exactly N survivors (:1182-1279).
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
#include <cooperative_groups.h>

#include "pe_internal.h"

namespace pe {

__device__ __forceinline__ bool dominates(const float *a, const float *b, int M)
{
    // dominate (include/sorting.cuh:94-130): |a-b| <= 1e-6 counts as equal
    int eq = 0;
    bool worse = false;
#pragma unroll
    for (int k = 0; k < kMaxObj; k++) {
        if (k >= M) break;
        float d = fabsf(__fsub_rn(a[k], b[k]));
        if (d > 1e-6f) {
            if (a[k] > b[k]) worse = true;
        } else {
            eq++;
        }
    }
    return eq != M && !worse;
}

// MM: the objective count when known at compile time (4 or 6; 0: s.M at run time),
// so the two objective vectors stay in registers
template <int MM>
__global__ void __launch_bounds__(256) k_dominance(Shape s, const float *__restrict__ obj, uint32_t *__restrict__ dom,
                                                   int32_t *__restrict__ np)
{
    __shared__ int wsum[8];
    const int M = MM > 0 ? MM : s.M;
    const int N2 = 2 * s.N, words = (N2 + 31) >> 5;
    const int i = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float oi[kMaxObj];
#pragma unroll
    for (int k = 0; k < (MM > 0 ? MM : kMaxObj); k++)
        if (k < M) oi[k] = obj[(size_t)i * M + k];
    int cnt = 0;
#pragma unroll 2
    for (int w = warp; w < words; w += 8) {
        int j = 32 * w + lane;
        bool bit = false;
        if (j < N2 && j != i) {
            float oj[kMaxObj];
#pragma unroll
            for (int k = 0; k < (MM > 0 ? MM : kMaxObj); k++)
                if (k < M) oj[k] = __ldg(&obj[(size_t)j * M + k]);
            bit = dominates(oj, oi, M);
        }
        const uint32_t word = __ballot_sync(0xffffffffu, bit);
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

// The same rows, kDomRows per CTA (one warp per row), with every objective vector
// staged once per CTA in shared memory, objective-major so the lanes of a warp read
// 32 consecutive words: the matrix crosses L2 once per CTA instead of once per row.
constexpr int kDomRows = 16;
constexpr size_t kDomTiledSmemMax = 200 * 1024;  // the staged matrix must fit beside nothing else

template <int MM>
__global__ void __launch_bounds__(32 * kDomRows) k_dominance_tiled(Shape s, const float *__restrict__ obj,
                                                                   uint32_t *__restrict__ dom,
                                                                   int32_t *__restrict__ np)
{
    extern __shared__ float ot[];  // [M][N2]
    const int M = MM > 0 ? MM : s.M;
    const int N2 = 2 * s.N, words = (N2 + 31) >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < N2 * M; e += blockDim.x) {
        const int j = e / M, k = e - j * M;
        ot[k * N2 + j] = obj[e];
    }
    __syncthreads();
    const int i = blockIdx.x * kDomRows + warp;
    if (i >= N2) return;
    float oi[kMaxObj];
#pragma unroll
    for (int k = 0; k < (MM > 0 ? MM : kMaxObj); k++)
        if (k < M) oi[k] = ot[k * N2 + i];
    int cnt = 0;
    for (int w = 0; w < words; w++) {
        const int j = 32 * w + lane;
        bool bit = false;
        if (j < N2 && j != i) {
            float oj[kMaxObj];
#pragma unroll
            for (int k = 0; k < (MM > 0 ? MM : kMaxObj); k++)
                if (k < M) oj[k] = ot[k * N2 + j];
            bit = dominates(oj, oi, M);
        }
        const uint32_t word = __ballot_sync(0xffffffffu, bit);
        if (lane == 0) dom[(size_t)i * words + w] = word;
        cnt += __popc(word);
    }
    if (lane == 0) np[i] = cnt;
}

// Across the lanes of a warp, lane w holding v: the smallest (largest) value, the
// lowest lane among equal ones -- what a loop over w = 0, 1, ... keeping the first
// strictly better value returns (including which of -0 / +0).
__device__ __forceinline__ float warp_first_min(float v, int lane)
{
    int w = lane;
    for (int o = 16; o > 0; o >>= 1) {
        const float u = __shfl_xor_sync(0xffffffffu, v, o);
        const int x = __shfl_xor_sync(0xffffffffu, w, o);
        if (u < v || (u == v && x < w)) {
            v = u;
            w = x;
        }
    }
    return v;
}
__device__ __forceinline__ float warp_first_max(float v, int lane)
{
    int w = lane;
    for (int o = 16; o > 0; o >>= 1) {
        const float u = __shfl_xor_sync(0xffffffffu, v, o);
        const int x = __shfl_xor_sync(0xffffffffu, w, o);
        if (u > v || (u == v && x < w)) {
            v = u;
            w = x;
        }
    }
    return v;
}

// Extreme points: the reference finds, for each axis, the lowest ASF value with a
// tree reduction (findMinValue) over positions 0 .. B-1, B = 2N + M: front-0
// solutions first, then the current extreme points, then FLT_MAX fillers.  Level 1
// pairs position t with t + B/2; each later level, of h slots, pairs slot t with
// t + h/2 (h even) or, for odd h, slot 0 first with slot h-1 and then with (h-1)/2;
// a pair keeps its first slot on equal values.  So the winner is the lowest value,
// and among equal values the position first in a fixed order: the order of the
// merged lists, each merge listing its first slot, then (odd h) slot h-1, then the
// other.  tree_key gives a position's place in that order, the choice made at
// every level (0 first, 1 the odd slot, 2 the other), root level in the highest
// bits; positions that level 1 leaves out (odd B) never win and get ~0.
__device__ __forceinline__ uint64_t tree_key(int p, int B)
{
    int h = B >> 1;
    if (p >= 2 * h) return ~0ull;
    int slot = p < h ? p : p - h;
    uint64_t key = p < h ? 0u : 2u;
    int lvl = 1;
    while (h > 1) {
        const int hn = h >> 1;
        uint64_t d;
        if (slot < hn) {
            d = 0;
        } else if (slot < 2 * hn) {
            d = 2;
            slot -= hn;
        } else {  // odd h: the last slot joins slot 0 before slot hn does
            d = 1;
            slot = 0;
        }
        key |= d << (2 * lvl);
        lvl++;
        h = hn;
    }
    return key;
}

// candidate of the extreme-point search: ASF value bits (values are >= +0, so their
// bits order as the values do) and position (kNoPos: none yet).  Tree keys are only
// needed between equal values, so they are computed then.
constexpr uint32_t kNoPos = 0xffffffffu;
static_assert(kSelThreads == 1024, "the selection CTA's cross-warp steps use one lane per warp");
struct ExtCand {
    uint32_t v;
    uint32_t pos;
};

__device__ __forceinline__ bool ext_before(uint32_t v, uint32_t pos, const ExtCand &c, int B)
{
    if (v != c.v) return v < c.v;
    if (c.pos == kNoPos) return true;
    return tree_key((int)pos, B) < tree_key((int)c.pos, B);
}

struct SelSmem {
    int warp_tot[33];
    int i0, i1, i2, i3, i4;
    int rc, fstart, fsize, cut, nfront, count, level, hyp;
    float ideal[kMaxObj], worst[kMaxObj], nadir[kMaxObj];
    float red[64 * kMaxObj];
    float ext[kMaxObj * kMaxObj];  // extreme points while they are updated
};

// k_select's extreme-point workspace (after the front mask in its dynamic shared memory)
struct ExtSmem {
    ExtCand xc[32][kMaxObj];       // per-warp extreme-point candidates
    uint64_t xck[32][kMaxObj];     // their tree keys
    float xa[kMaxObj * kMaxObj];   // ASF of last generation's extreme points, per axis
    float xf[kMaxObj * kMaxObj];   // ASF of each axis' front-0 winner, per axis
    uint64_t xkey[kMaxObj];        // tree keys of the extreme-point positions
    uint64_t xfkey[kMaxObj];       // tree keys of the front-0 winners
    int xsrc[kMaxObj];             // source of each new extreme point
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

// ASF (include/sorting.cuh:428-449) of point x for every axis i: the largest of
// tmp_k / w_k with tmp_k = x_k - ideal_k (0 below 0.001), w_i = 1 and the other
// weights 1e-6.  Every tmp_k is >= 0 and a correctly rounded division is monotone in
// its dividend, so the largest tmp_k / 1e-6 over k != i is (the largest tmp_k over
// k != i) / 1e-6, and tmp_i / 1 is tmp_i: two divisions give all M values, equal to
// the reference's M * M.
__device__ __forceinline__ void asf_all(const float *x, const float *ideal, int M, float *out)
{
    float tmp[kMaxObj];
    float m1 = -1.0f, m2 = -1.0f;  // largest and second largest tmp_k
    int a1 = -1;
    for (int k = 0; k < M; k++) {
        float t = __fsub_rn(x[k], ideal[k]);
        if ((double)t < 0.001) t = 0.0f;
        tmp[k] = t;
        if (t > m1) {
            m2 = m1;
            m1 = t;
            a1 = k;
        } else if (t > m2) {
            m2 = t;
        }
    }
    const float q1 = m1 >= 0.0f ? __fdiv_rn(m1, 1e-6f) : -FLT_MAX;
    const float q2 = m2 >= 0.0f ? __fdiv_rn(m2, 1e-6f) : -FLT_MAX;
    for (int i = 0; i < M; i++) {
        const float q = i == a1 ? q2 : q1;  // largest over k != i
        out[i] = tmp[i] > q ? tmp[i] : q;
    }
}

// the same for one axis i: one division
__device__ __forceinline__ float asf_axis(const float *x, const float *ideal, int i, int M)
{
    float ti = 0.0f, m = -1.0f;  // tmp_i and the largest tmp_k over k != i
    for (int k = 0; k < M; k++) {
        float t = __fsub_rn(x[k], ideal[k]);
        if ((double)t < 0.001) t = 0.0f;
        if (k == i) ti = t;
        else if (t > m) m = t;
    }
    const float q = m >= 0.0f ? __fdiv_rn(m, 1e-6f) : -FLT_MAX;
    return ti > q ? ti : q;
}

// element j of a row held in registers (j known only at run time)
__device__ __forceinline__ float row_at(const float (&row)[kMaxObj + 1], int j)
{
    float v = row[0];
#pragma unroll
    for (int q = 1; q <= kMaxObj; q++)
        if (j == q) v = row[q];
    return v;
}

// Hyperplane through the extreme points by Gaussian elimination
// (GaussianElimination, include/sorting.cuh:555-599) and its check (:929-956), by
// one warp: lane r < M holds row r of [ext | 1] and does that row's share of every
// step, with the same operations in the same order as the serial loops.  Writes
// nadir = ideal + intercepts; returns 1 (all lanes) when the hyperplane is unusable.
__device__ int hyperplane_nadir(int M, const float *ext, const float *ideal, float *nadir, int lane)
{
    const unsigned full = 0xffffffffu;
    const bool mine = lane < M;
    float row[kMaxObj + 1];
#pragma unroll
    for (int j = 0; j <= kMaxObj; j++) row[j] = (mine && j < M) ? ext[lane * M + j] : (j == M ? 1.0f : 0.0f);
    for (int c = 0; c < M; c++) {
        const float pcc = __shfl_sync(full, row_at(row, c), c);
        if ((double)fabsf(pcc) <= 1e-6) {
            // add the first later row with a usable entry in column c
            const unsigned cand = __ballot_sync(full, mine && lane > c && (double)fabsf(row_at(row, c)) > 1e-6);
            if (cand) {
                const int r = __ffs(cand) - 1;
#pragma unroll
                for (int j = 0; j <= kMaxObj; j++) {
                    const float vr = __shfl_sync(full, row[j], r);
                    if (lane == c && j >= c && j <= M) row[j] = __fadd_rn(row[j], vr);
                }
            }
        }
        const float pc = __shfl_sync(full, row_at(row, c), c);
        const float f = __fdiv_rn(row_at(row, c), pc);
        const bool elim = mine && lane > c;
#pragma unroll
        for (int j = 0; j <= kMaxObj; j++) {
            const float vc = __shfl_sync(full, row[j], c);
            if (elim && j >= c && j <= M) row[j] = __fsub_rn(row[j], __fmul_rn(f, vc));
        }
    }
    // back substitution: lane r finds x[r] once x[r+1 .. M-1] are known
    float xr = 0.0f;
    for (int r = M - 1; r >= 0; r--) {
        float sacc = 0.0f;
        for (int j = r + 1; j < M; j++) sacc = __fadd_rn(sacc, __fmul_rn(row_at(row, j), __shfl_sync(full, xr, j)));
        const float xv = __fdiv_rn(__fsub_rn(row_at(row, M), sacc), row_at(row, r));
        if (lane == r) xr = xv;
    }
    int exc = 0;
    float res = 0.0f;
    for (int i = 0; i < M; i++) {
        const float xi = __shfl_sync(full, xr, i);
        if (mine) res = __fadd_rn(res, __fmul_rn(xi, __fsub_rn(ext[lane * M + i], ideal[i])));
    }
    if (mine) {
        if (fabsf(__fsub_rn(res, 1.0f)) > 1e-6f || isnan(res) || isinf(res)) exc = 1;
        const float icp = __fdiv_rn(1.0f, xr);
        if (icp <= 1e-6f || isnan(icp) || isinf(icp)) exc = 1;
        nadir[lane] = __fadd_rn(ideal[lane], icp);
    }
    return __any_sync(full, exc) ? 1 : 0;
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

// nonDominatedSorting (include/sorting.cuh:974-1089): fronts peeled on the
// dominance bit matrix by a cluster of kFrontCtas CTAs.  CTA c owns the rows
// [c*RR, c*RR + RR) (RR a multiple of 32, so each CTA's rows are whole mask
// words).  Per front: every CTA puts its rows that joined the front into its
// slice of the front mask (in its shared memory); after one cluster barrier each
// CTA assembles the whole mask from the slices (distributed shared memory),
// lists its own members in ascending index (prefix popcounts over the mask), and
// tests each of its unassigned rows against the mask -- one warp per row,
// coalesced loads of the row, dominators in the front subtracted from the row's
// count -- to fill its slice of the next front.  Slices are double-buffered, so
// one barrier per front suffices.  Every CTA sees the same masks and counts, so
// they stop together: when fronts 0..f hold N or more solutions, or when a front
// comes out empty (a cycle of the epsilon-dominance relation leaves the rest
// unassigned; the reference's loop would then run out its 2N-1 rounds on empty
// fronts, which the recorded front count reproduces).
constexpr int kFrontCtas = 8;
constexpr int kFrontThreads = 1024;

__host__ __device__ __forceinline__ int front_rows_per_cta(int N2)
{
    return ((N2 + kFrontCtas - 1) / kFrontCtas + 31) & ~31;
}

__global__ void __cluster_dims__(kFrontCtas, 1, 1) __launch_bounds__(kFrontThreads, 1)
    k_fronts(Shape s, SelectScratch sc)
{
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char fsm_raw[];
    __shared__ int s_warp[32];
    const int c = (int)cluster.block_rank();
    const int N = s.N, N2 = 2 * N, words = (N2 + 31) >> 5;
    const int RR = front_rows_per_cta(N2), sw = RR >> 5;
    const int r0 = c * RR, nrow = max(0, min(N2, r0 + RR) - r0);
    uint32_t *fmask = reinterpret_cast<uint32_t *>(fsm_raw);          // words: the current front
    uint32_t *slice = fmask + ((words + 3) & ~3);                      // [2][sw]: own rows joining a front
    int *npr = reinterpret_cast<int *>(slice + 2 * ((sw + 3) & ~3));   // [RR]: unassigned dominators
    int *wpre = npr + RR;                                              // [words]: members before each word
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nth >> 5;
    const int swp = (sw + 3) & ~3;

    for (int q = tid; q < RR; q += nth) {
        const int v = q < nrow ? sc.np[r0 + q] : -1;
        npr[q] = v;
        if (q < nrow) sc.front[r0 + q] = -1;
    }
    for (int w = tid; w < 2 * swp; w += nth) slice[w] = 0u;
    __syncthreads();
    for (int q = tid; q < nrow; q += nth)
        if (npr[q] == 0) atomicOr(&slice[q >> 5], 1u << (q & 31));
    int rc = 0, fstart = 0, fsize = 0, nfront = 0, cut = 0, f0 = 0, par = 0;
    for (int it = 0; it < N2; it++) {
        cluster.sync();  // every slice of this front is complete
        // the whole mask from the slices (one remote load per thread and word), then
        // warp 0 takes the exclusive prefix of the words' popcounts (lane l: words
        // [l*per, l*per + per))
        for (int w = tid; w < words; w += nth) {
            const int owner = w / sw, off = w - owner * sw;
            const uint32_t *rs = cluster.map_shared_rank(slice + par * swp, owner);
            fmask[w] = rs[off];
        }
        __syncthreads();
        if (warp == 0) {
            const int per = (words + 31) >> 5, w0 = lane * per;
            int sum = 0;
            for (int w = w0; w < min(words, w0 + per); w++) {
                wpre[w] = sum;
                sum += __popc(fmask[w]);
            }
            int inc = sum;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            const int before = inc - sum;
            for (int w = w0; w < min(words, w0 + per); w++) wpre[w] += before;
            if (lane == 31) s_warp[0] = inc;
        }
        __syncthreads();
        const int tot = s_warp[0];
        // own members of front `it`, in ascending index
        for (int w = (r0 >> 5) + tid; w < min(words, (r0 >> 5) + sw); w += nth) {
            uint32_t x = fmask[w];
            int pos = rc + wpre[w];
            while (x) {
                const int b = __ffs(x) - 1;
                x &= x - 1;
                const int i = 32 * w + b;
                sc.front[i] = it;
                sc.sorted[pos++] = i;
            }
        }
        fstart = rc;
        fsize = tot;
        rc += tot;
        nfront = it + 1;
        if (it == 0) f0 = tot;
        if (rc >= N) {
            cut = rc == N;
            break;
        }
        if (tot == 0) {
            nfront = N2;
            break;
        }
        // the next front: own unassigned rows whose remaining dominators are all in this one
        const int nx = par ^ 1;
        for (int w = tid; w < sw; w += nth) slice[nx * swp + w] = 0u;
        __syncthreads();
        // eight rows per warp at a time, so their loads are in flight together
        for (int q0 = warp; q0 < nrow; q0 += 8 * nwarps) {
            const uint32_t *base = sc.dom + (size_t)(r0 + q0) * words;
            const size_t step = (size_t)nwarps * words;  // between the warp's rows u and u+1
            unsigned act = 0u;
            int dec[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int q = q0 + u * nwarps;
                if (q < nrow && npr[q] > 0) act |= 1u << u;  // rows assigned already are skipped
                dec[u] = 0;
            }
            if (!act) continue;
            for (int w = lane; w < words; w += 32) {
                const uint32_t f = fmask[w];
                if (!f) continue;
#pragma unroll
                for (int u = 0; u < 8; u++)
                    if (act & (1u << u)) dec[u] += __popc(__ldg(base + u * step + w) & f);
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                int d = dec[u];
                for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
                const int q = q0 + u * nwarps;
                if (lane == 0 && (act & (1u << u)) && d) {
                    const int v = npr[q] - d;
                    npr[q] = v;
                    if (v == 0) atomicOr(&slice[nx * swp + (q >> 5)], 1u << (q & 31));
                }
            }
        }
        par = nx;
        __syncthreads();
    }
    if (c == 0 && tid == 0) {
        sc.info[0] = rc;
        sc.info[1] = fsize;
        sc.info[2] = nfront;
        sc.info[3] = cut;
        sc.info[6] = fstart;
        sc.info[7] = f0;
    }
    cluster.sync();  // no CTA leaves while another may still read its slices
}

size_t fronts_smem_bytes(const Shape &s)
{
    const int N2 = 2 * s.N, words = (N2 + 31) >> 5, RR = front_rows_per_cta(N2), sw = RR >> 5;
    return (size_t)((words + 3) & ~3) * 4 + (size_t)2 * ((sw + 3) & ~3) * 4 + (size_t)RR * 4 + (size_t)words * 4;
}

__global__ void __launch_bounds__(kSelThreads, 1) k_select(Shape s, const float *__restrict__ obj, float *ext,
                                                        const float *__restrict__ refpts, SelectScratch sc,
                                                        int32_t *surv, uint32_t *d_gen, int bump_gen)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SelSmem &sm = *reinterpret_cast<SelSmem *>(smem_raw);
    const int N = s.N, N2 = 2 * N, M = s.M, R = s.R;
    const int words = (N2 + 31) >> 5;
    ExtSmem &xs = *reinterpret_cast<ExtSmem *>(smem_raw + ((sizeof(SelSmem) + 15) & ~size_t(15)));
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5;
    (void)d_gen;
    (void)bump_gen;
    (void)words;

    // fronts 0..last: peeled by k_fronts (front[], sorted[] and the counts in info)
    const int rc = sc.info[0];
    const int last_size = sc.info[1];
    const int f0 = sc.info[7];
    if (tid == 0) {
        sm.rc = rc;
        sm.fsize = last_size;
        sm.fstart = sc.info[6];
        sm.nfront = sc.info[2];
        sm.cut = sc.info[3];
    }
    __syncthreads();

    // ---------------- ideal / worst (exact min / max), objective by objective
    for (int k = 0; k < M; k++) {
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (int i = tid; i < N2; i += nth) {
            const float v = obj[(size_t)i * M + k];
            if (v < mn) mn = v;
            if (v > mx) mx = v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float a = __shfl_xor_sync(0xffffffffu, mn, o), b = __shfl_xor_sync(0xffffffffu, mx, o);
            if (a < mn) mn = a;
            if (b > mx) mx = b;
        }
        if (lane == 0) {
            sm.red[warp * kMaxObj + k] = mn;
            sm.red[32 * kMaxObj + warp * kMaxObj + k] = mx;
        }
    }
    __syncthreads();
    if (warp < M) {  // warp k: objective k over the per-warp results, in warp order
        const float a = warp_first_min(sm.red[lane * kMaxObj + warp], lane);
        const float b = warp_first_max(sm.red[32 * kMaxObj + lane * kMaxObj + warp], lane);
        if (lane == 0) {
            sm.ideal[warp] = a;
            sm.worst[warp] = b;
        }
    }
    __syncthreads();

    // ---------------- extreme points (findExtremePoints, :601-683), tree order of findMinValue
    // Front 0 does not change between axes: a parallel pass finds, axis by axis, its
    // first solution in (value, tree order).  The current extreme points, which change
    // as the axes are done in turn, and the FLT_MAX fillers are then weighed against
    // it axis by axis.  The pass also takes the maximum of front 0 (MNDF nadir).
    {
        const int B = N2 + M;
        for (int e = tid; e < M * M; e += nth) sm.ext[e] = ext[e];
        for (int i = 0; i < M; i++) {
            ExtCand best{0xffffffffu, kNoPos};
            float fmx = -FLT_MAX;
            for (int t = tid; t < f0; t += nth) {
                const float *x = obj + (size_t)sc.sorted[t] * M;
                const uint32_t v = __float_as_uint(asf_axis(x, sm.ideal, i, M));
                if (ext_before(v, (uint32_t)t, best, B)) best = ExtCand{v, (uint32_t)t};
                const float xi = x[i];
                if (xi > fmx) fmx = xi;
            }
            uint64_t bkey = best.pos != kNoPos ? tree_key((int)best.pos, B) : ~0ull;
            for (int o = 16; o > 0; o >>= 1) {
                const uint32_t v2 = __shfl_xor_sync(0xffffffffu, best.v, o), p2 = __shfl_xor_sync(0xffffffffu, best.pos, o);
                const uint64_t k2 = __shfl_xor_sync(0xffffffffu, bkey, o);
                if (v2 < best.v || (v2 == best.v && k2 < bkey)) {
                    best = ExtCand{v2, p2};
                    bkey = k2;
                }
                const float b = __shfl_xor_sync(0xffffffffu, fmx, o);
                if (b > fmx) fmx = b;
            }
            if (lane == 0) {
                xs.xc[warp][i] = best;
                xs.xck[warp][i] = bkey;
                sm.red[warp * kMaxObj + i] = fmx;
            }
        }
        __syncthreads();
        if (warp < M) {  // warp i: axis i over the per-warp candidates
            const ExtCand d = xs.xc[lane][warp];
            uint32_t v = d.v, pos = d.pos;
            uint64_t key = xs.xck[lane][warp];
            for (int o = 16; o > 0; o >>= 1) {
                const uint32_t v2 = __shfl_xor_sync(0xffffffffu, v, o), p2 = __shfl_xor_sync(0xffffffffu, pos, o);
                const uint64_t k2 = __shfl_xor_sync(0xffffffffu, key, o);
                if (v2 < v || (v2 == v && k2 < key)) {
                    v = v2;
                    pos = p2;
                    key = k2;
                }
            }
            const float b = warp_first_max(sm.red[lane * kMaxObj + warp], lane);
            if (lane == 0) {
                xs.xc[0][warp] = ExtCand{v, pos};
                xs.xfkey[warp] = key;
                sm.red[32 * kMaxObj + warp] = b;  // max of front 0 (MNDF)
            }
            if (lane == 1) xs.xkey[warp] = tree_key(f0 + warp, B);
        }
        __syncthreads();
        // The current extreme point r, as the axes are done in turn, is a copy of an
        // extreme point of the last generation (source r' < M) or of the front-0 winner
        // of an earlier axis j (source M + j): its ASF values come from two small tables.
        if (tid < 2 * M) {
            const int r = tid % M;
            float a[kMaxObj];
            if (tid < M) {
                asf_all(sm.ext + r * M, sm.ideal, M, a);
                for (int i = 0; i < M; i++) xs.xa[r * M + i] = a[i];
            } else {
                const uint32_t pos = xs.xc[0][r].pos;
                if (pos < (uint32_t)f0) asf_all(obj + (size_t)sc.sorted[pos] * M, sm.ideal, M, a);
                for (int i = 0; i < M; i++) xs.xf[r * M + i] = pos < (uint32_t)f0 ? a[i] : 0.0f;
            }
        }
        __syncthreads();
        if (warp == 0) {  // the axes in turn; lane r < M holds extreme point r's source
            const uint32_t vmax = __float_as_uint(FLT_MAX);
            // the FLT_MAX fillers can only come first on an axis whose front-0 value is
            // not below FLT_MAX: the first filler in tree order, only then
            uint64_t fkey = ~0ull;
            if (__any_sync(0xffffffffu, lane < M && xs.xc[0][lane].v >= vmax)) {
                for (int t = f0 + M + lane; t < B; t += 32) fkey = min(fkey, tree_key(t, B));
                for (int o = 16; o > 0; o >>= 1) fkey = min(fkey, __shfl_xor_sync(0xffffffffu, fkey, o));
            }
            int src = lane;
            const uint64_t rkey = lane < M ? xs.xkey[lane] : ~0ull;
            for (int i = 0; i < M; i++) {
                uint32_t cv = xs.xc[0][i].v;
                uint64_t ck = xs.xfkey[i];
                int win = ck != ~0ull ? M + i : -1;  // -1: a filler, the point stays
                if (fkey != ~0ull && (vmax < cv || (vmax == cv && fkey < ck))) {
                    cv = vmax;
                    ck = fkey;
                    win = -1;
                }
                // the extreme points as they stand, lowest (value, key) over the lanes
                uint32_t v = 0xffffffffu;
                uint64_t key = ~0ull;
                int q = src;
                if (lane < M && rkey != ~0ull) {
                    v = __float_as_uint(src < M ? xs.xa[src * M + i] : xs.xf[(src - M) * M + i]);
                    key = rkey;
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const uint32_t v2 = __shfl_xor_sync(0xffffffffu, v, o);
                    const uint64_t k2 = __shfl_xor_sync(0xffffffffu, key, o);
                    const int q2 = __shfl_xor_sync(0xffffffffu, q, o);
                    if (v2 < v || (v2 == v && k2 < key)) {
                        v = v2;
                        key = k2;
                        q = q2;
                    }
                }
                if (key != ~0ull && (v < cv || (v == cv && key < ck))) win = q;
                if (win >= 0 && lane == i) src = win;
            }
            if (lane < M) xs.xsrc[lane] = src;
        }
        __syncthreads();
        for (int e = tid; e < M * M; e += nth) {
            const int i = e / M, k = e - i * M, q = xs.xsrc[i];
            xs.xa[e] = q < M ? sm.ext[q * M + k] : obj[(size_t)sc.sorted[xs.xc[0][q - M].pos] * M + k];
        }
        __syncthreads();
        for (int e = tid; e < M * M; e += nth) {
            sm.ext[e] = xs.xa[e];
            ext[e] = xs.xa[e];
        }
        __syncthreads();
    }

    // ---------------- hyperplane intercepts (GaussianElimination :555-599, check :929-956)
    if (warp == 0) {
        const int exc = hyperplane_nadir(M, sm.ext, sm.ideal, sm.nadir, lane);
        if (lane == 0) sm.hyp = exc;
        if (exc && lane < M) {
            // updateNadirValue_MNDF (:685-884): max over front 0, worst when too close to ideal
            const float b = sm.red[32 * kMaxObj + lane];
            sm.nadir[lane] = __fsub_rn(b, sm.ideal[lane]) > 1e-6f ? b : sm.worst[lane];
        }
    }
    __syncthreads();
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
// MM: the objective count when known at compile time (0: s.M at run time)
template <int MM>
__global__ void __launch_bounds__(256) k_assoc(Shape s, const float *__restrict__ obj,
                                               const float *__restrict__ refpts, SelectScratch sc)
{
    if (sc.info[3]) return;  // fronts filled N exactly: no niching
    const int M = MM > 0 ? MM : s.M, R = s.R;
    constexpr int KU = MM > 0 ? MM : kMaxObj;  // unrolled loop bound (k < M guards the rest)
    const int rc = sc.info[0], count0 = sc.info[5];
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    float ideal[kMaxObj], span[kMaxObj];
#pragma unroll
    for (int k = 0; k < KU; k++) {
        if (k >= M) break;
        ideal[k] = sc.finfo[k];
        span[k] = __fsub_rn(sc.finfo[2 * M + k], ideal[k]);
    }
    for (int t = gw; t < rc; t += nw) {
        const int sol = sc.sorted[t];
        float f[kMaxObj];
#pragma unroll
        for (int k = 0; k < KU; k++) {
            if (k >= M) break;
            f[k] = __fdiv_rn(__fsub_rn(obj[(size_t)sol * M + k], ideal[k]), span[k]);
        }
        float best = FLT_MAX;
        int bj = 0;
        for (int j = lane; j < R; j += 32) {
            const float *w = refpts + (size_t)j * M;
            float num = 0.0f, den = 0.0f;
#pragma unroll
            for (int k = 0; k < KU; k++) {
                if (k >= M) break;
                num = __fadd_rn(num, __fmul_rn(w[k], f[k]));
                den = __fadd_rn(den, __fmul_rn(w[k], w[k]));
            }
            float kk = __fdiv_rn(num, den);
            float d2 = 0.0f;
#pragma unroll
            for (int k = 0; k < KU; k++) {
                if (k >= M) break;
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
    // candidate lists in ascending position: one warp walks the last front's members
    // in order, 32 at a time; __match_any_sync groups the lanes of the same point,
    // each lane's place is its point's fill so far plus the lanes of its group below
    // it, and the group's lowest lane advances the fill (kq counts it).  las[t] then
    // holds the member's place in the lists.
    const int nm = rc - count0;
    if (warp == 0) {
        for (int t0 = 0; t0 < nm; t0 += 32) {
            const int t = t0 + lane;
            const int j = t < nm ? las[t] : -1 - lane;  // lanes past the end match nobody
            const unsigned peers = __match_any_sync(0xffffffffu, j);
            if (t < nm) {
                const int leader = __ffs(peers) - 1;
                const int below = __popc(peers & ((1u << lane) - 1u));
                const int pos = coff[j] + kq[j] + below;
                cand[pos] = lsol[t];
                las[t] = pos;
                __syncwarp(peers);
                if (lane == leader) kq[j] += __popc(peers);
            }
            __syncwarp();
        }
    }
    __syncthreads();
    // the nearest member of a point with niche count 0 (the first in list order among
    // equal distances) is its pick at level 0, which is the point's first pick whenever
    // it has one: found with two atomicMin passes over the members (distance bits,
    // then place) and moved to the list's end (a point that ends up picking nothing
    // never reads its list).  pofs and kq serve as scratch.
    for (int j = tid; j < R; j += nth) {
        pofs[j] = 0x7fffffff;
        kq[j] = 0x7fffffff;
    }
    __syncthreads();
    for (int t = tid; t < nm; t += nth) {
        const int j = sc.assoc[count0 + t];
        // distances are >= +0 (or FLT_MAX), so their bits order as the values do
        if (cj[j] == 0) atomicMin(&pofs[j], __float_as_int(sc.dist[lsol[t]]));
    }
    __syncthreads();
    for (int t = tid; t < nm; t += nth) {
        const int j = sc.assoc[count0 + t];
        if (cj[j] == 0 && __float_as_int(sc.dist[lsol[t]]) == pofs[j]) atomicMin(&kq[j], las[t] - coff[j]);
    }
    __syncthreads();
    for (int j = tid; j < R; j += nth)
        if (cj[j] == 0 && nj[j] > 0) {
            int *cl = cand + coff[j];
            const int slot = kq[j], last = nj[j] - 1, pick = cl[slot];
            cl[slot] = cl[last];
            cl[last] = pick;
        }
    __syncthreads();
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
                slot = nc - 1;  // made while the lists were built: already at the end
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
    (void)s;
    return ((sizeof(SelSmem) + 15) & ~size_t(15)) + sizeof(ExtSmem);
}

cudaError_t launch_select(const Shape &s, const float *obj, float *ext, const float *refpts, SelectScratch sc,
                          int32_t *surv, uint32_t *d_gen, int bump_gen, cudaStream_t st)
{
    cudaError_t e;
    const size_t dsm = (size_t)2 * s.N * s.M * sizeof(float);
    if (dsm <= kDomTiledSmemMax) {
        const int g = (2 * s.N + kDomRows - 1) / kDomRows;
        if (s.M == 4) {
            if ((e = raise_smem_limit((const void *)k_dominance_tiled<4>, dsm)) != cudaSuccess) return e;
            k_dominance_tiled<4><<<g, 32 * kDomRows, dsm, st>>>(s, obj, sc.dom, sc.np);
        } else if (s.M == 6) {
            if ((e = raise_smem_limit((const void *)k_dominance_tiled<6>, dsm)) != cudaSuccess) return e;
            k_dominance_tiled<6><<<g, 32 * kDomRows, dsm, st>>>(s, obj, sc.dom, sc.np);
        } else {
            if ((e = raise_smem_limit((const void *)k_dominance_tiled<0>, dsm)) != cudaSuccess) return e;
            k_dominance_tiled<0><<<g, 32 * kDomRows, dsm, st>>>(s, obj, sc.dom, sc.np);
        }
    } else if (s.M == 4) {
        k_dominance<4><<<2 * s.N, 256, 0, st>>>(s, obj, sc.dom, sc.np);
    } else if (s.M == 6) {
        k_dominance<6><<<2 * s.N, 256, 0, st>>>(s, obj, sc.dom, sc.np);
    } else {
        k_dominance<0><<<2 * s.N, 256, 0, st>>>(s, obj, sc.dom, sc.np);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t fsm = fronts_smem_bytes(s);
    if ((e = raise_smem_limit((const void *)k_fronts, fsm)) != cudaSuccess) return e;
    k_fronts<<<kFrontCtas, kFrontThreads, fsm, st>>>(s, sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    size_t smem = select_smem_bytes(s);
    e = raise_smem_limit((const void *)k_select, smem);
    if (e != cudaSuccess) return e;
    k_select<<<1, kSelThreads, smem, st>>>(s, obj, ext, refpts, sc, surv, d_gen, bump_gen);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int warps_needed = 2 * s.N;
    const int ag = std::min((warps_needed + 7) / 8, 148 * 8);
    if (s.M == 4) k_assoc<4><<<ag, 256, 0, st>>>(s, obj, refpts, sc);
    else if (s.M == 6) k_assoc<6><<<ag, 256, 0, st>>>(s, obj, refpts, sc);
    else k_assoc<0><<<ag, 256, 0, st>>>(s, obj, refpts, sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t nsm = niche_smem_bytes(s);
    if ((e = raise_smem_limit((const void *)k_niche, nsm)) != cudaSuccess) return e;
    k_niche<<<1, kSelThreads, nsm, st>>>(s, sc, surv, d_gen, bump_gen);
    return cudaGetLastError();
}

}  // namespace pe
