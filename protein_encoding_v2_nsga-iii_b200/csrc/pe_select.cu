// pe_select.cu -- environmental selection (sortingKernel, src/main.cu:409-454).
//
//  k_dominance  32 x 256 tiles of the 2N x 2N dominance bit matrix (bit j of row
//               i set when j dominates i) and each row's dominator count per tile
//               -- replaces the reference's two (2N)^2 bool matrices
//               (include/sorting.cuh:974-1089).
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
#include <vector>

#include "pe_device.cuh"
#include <cooperative_groups.h>

#include "pe_internal.h"

namespace pe {

// dominate (include/sorting.cuh:94-130): |a-b| <= 1e-6 counts as equal, and a
// dominates b when it is not worse on any objective and not equal on all of them --
// that is, some a_k - b_k < -1e-6 and no a_k - b_k > 1e-6.  The rounded difference is
// 0 only when a_k == b_k (subnormals are kept), so its sign is that of a_k - b_k, and
// a NaN difference (inf - inf) is neither, as the reference's equal branch takes it.
__device__ __forceinline__ bool dominates(const float *a, const float *b, int M)
{
    bool better = false, worse = false;
#pragma unroll
    for (int k = 0; k < kMaxObj; k++) {
        if (k >= M) break;
        const float d = __fsub_rn(a[k], b[k]);
        better |= d < -1e-6f;
        worse |= d > 1e-6f;
    }
    return better && !worse;
}

// The dominance matrix in 32 x 256 tiles: CTA (x, y) takes rows 32x .. 32x+31 (one
// per lane) and columns 256y .. 256y+255 (32 per warp, one matrix word), with the
// tile's column objectives staged in shared memory (every lane reads the same
// column: a broadcast) and each lane's row in registers.  A warp builds its 32
// rows' words bit by bit; the tile is written row by row in 32-byte runs, and each
// row's dominator count over the tile goes to np[y][row] (k_fronts adds the y's).
// MM: the objective count when known at compile time (4 or 6; 0: s.M at run time).
constexpr int kDomTileWords = 8;
template <int MM>
__global__ void __launch_bounds__(32 * kDomTileWords) k_dominance(Shape s, const float *__restrict__ obj,
                                                                  uint32_t *__restrict__ dom, int32_t *__restrict__ np)
{
    __shared__ __align__(16) float oc[32 * kDomTileWords * kMaxObj];  // tile columns, objective vectors in column order
    __shared__ uint32_t tw[32][kDomTileWords + 1];       // the tile's words by row
    constexpr int KU = MM > 0 ? MM : kMaxObj;
    const int M = MM > 0 ? MM : s.M;
    const int N2 = 2 * s.N, words = (N2 + 31) >> 5;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i = blockIdx.x * 32 + lane, j0 = blockIdx.y * 32 * kDomTileWords;
    const int ncol = min(32 * kDomTileWords, N2 - j0);
    for (int e = tid; e < ncol * M; e += blockDim.x) oc[e] = obj[(size_t)j0 * M + e];
    float oi[kMaxObj];
#pragma unroll
    for (int k = 0; k < KU; k++)
        if (k < M) oi[k] = i < N2 ? obj[(size_t)i * M + k] : 0.0f;
    __syncthreads();
    const int wd = blockIdx.y * kDomTileWords + warp;
    uint32_t word = 0;
    if (wd < words) {
        const int b1 = min(32, N2 - 32 * wd);
        for (int b = 0; b < b1; b++) {
            const int jl = 32 * warp + b, j = j0 + jl;
            float oj[kMaxObj];
            if (MM == 4) {  // one 16-byte broadcast load
                const float4 v = reinterpret_cast<const float4 *>(oc)[jl];
                oj[0] = v.x;
                oj[1] = v.y;
                oj[2] = v.z;
                oj[3] = v.w;
            } else {
#pragma unroll
                for (int k = 0; k < KU; k++)
                    if (k < M) oj[k] = oc[jl * M + k];
            }
            if (j != i && dominates(oj, oi, M)) word |= 1u << b;
        }
    }
    tw[lane][warp] = word;
    __syncthreads();
    {
        const int r = tid / kDomTileWords, w = tid % kDomTileWords;
        const int row = blockIdx.x * 32 + r, wd2 = blockIdx.y * kDomTileWords + w;
        if (row < N2 && wd2 < words) dom[(size_t)row * words + wd2] = tw[r][w];
    }
    if (tid < 32) {
        int cnt = 0;
#pragma unroll
        for (int w = 0; w < kDomTileWords; w++) cnt += __popc(tw[tid][w]);
        const int row = blockIdx.x * 32 + tid;
        if (row < N2) np[(size_t)blockIdx.y * N2 + row] = cnt;
    }
}

// column tiles of the dominance matrix (np holds this many counts per row)
__host__ __device__ inline int dom_tiles(int N2) { return (((N2 + 31) >> 5) + kDomTileWords - 1) / kDomTileWords; }

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
// bits; positions that level 1 leaves out (odd B) never win and get ~0.  The
// kernels read a position's place in that order from a table made once per shape
// (tree_order_ranks), so a tie costs one load.
__host__ __device__ inline uint64_t tree_key(int p, int B)
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

void tree_order_ranks(int B, uint32_t *rank)
{
    std::vector<std::pair<uint64_t, int>> k((size_t)B);
    for (int p = 0; p < B; p++) k[(size_t)p] = {tree_key(p, B), p};
    std::sort(k.begin(), k.end());
    for (int r = 0; r < B; r++) rank[k[(size_t)r].second] = k[(size_t)r].first == ~0ull ? 0xffffffffu : (uint32_t)r;
}

// place of position p in tree order, as a key (~0: never wins)
__device__ __forceinline__ uint64_t tree_rank(const uint32_t *trank, int p)
{
    const uint32_t r = __ldg(&trank[p]);
    return r == 0xffffffffu ? ~0ull : (uint64_t)r;
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

// asf_all for a row held in registers (fixed-size arrays, M <= kMaxObj live entries)
__device__ __forceinline__ void asf_rows(const float (&x)[kMaxObj], const float (&ideal)[kMaxObj], int M,
                                         float (&out)[kMaxObj])
{
    float tmp[kMaxObj] = {};
    float m1 = -1.0f, m2 = -1.0f;  // largest and second largest tmp_k
    int a1 = -1;
#pragma unroll
    for (int k = 0; k < kMaxObj; k++) {
        if (k >= M) break;
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
#pragma unroll
    for (int i = 0; i < kMaxObj; i++) {
        const float q = i == a1 ? q2 : q1;  // largest over k != i
        out[i] = i < M && tmp[i] > q ? tmp[i] : q;
    }
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

// Hyperplane intercepts (GaussianElimination, include/sorting.cuh:555-599, and the
// check of :929-956) by one thread, MM known at compile time so the augmented matrix
// stays in registers.  Row r of [E | 1] is extreme point r; every element
// goes through the reference's operations in its order: a near-zero pivot takes the
// first later row with a usable entry added to its row, each later row subtracts
// (its entry / pivot) times the pivot row, back substitution sums in ascending
// column order.  Returns 1 when the intercepts are unusable (residual off by more
// than 1e-6, or an intercept not above 1e-6, NaN or infinite), else writes
// nadir = ideal + intercepts and returns 0.
template <int MM>
__device__ int hyperplane_nadir(const float *ext, const float *ideal, float *nadir)
{
    float a[MM][MM + 1];
#pragma unroll
    for (int r = 0; r < MM; r++) {
#pragma unroll
        for (int j = 0; j < MM; j++) a[r][j] = ext[r * MM + j];
        a[r][MM] = 1.0f;
    }
#pragma unroll
    for (int c = 0; c < MM; c++) {
        if ((double)fabsf(a[c][c]) <= 1e-6) {
            bool added = false;
#pragma unroll
            for (int r = c + 1; r < MM; r++) {
                if (!added && (double)fabsf(a[r][c]) > 1e-6) {
#pragma unroll
                    for (int j = c; j <= MM; j++) a[c][j] = __fadd_rn(a[c][j], a[r][j]);
                    added = true;
                }
            }
        }
        const float pc = a[c][c];
#pragma unroll
        for (int r = c + 1; r < MM; r++) {
            const float f = __fdiv_rn(a[r][c], pc);
#pragma unroll
            for (int j = c; j <= MM; j++) a[r][j] = __fsub_rn(a[r][j], __fmul_rn(f, a[c][j]));
        }
    }
    float x[MM];
#pragma unroll
    for (int r = MM - 1; r >= 0; r--) {
        float sacc = 0.0f;
#pragma unroll
        for (int j = r + 1; j < MM; j++) sacc = __fadd_rn(sacc, __fmul_rn(a[r][j], x[j]));
        x[r] = __fdiv_rn(__fsub_rn(a[r][MM], sacc), a[r][r]);
    }
    int exc = 0;
#pragma unroll
    for (int r = 0; r < MM; r++) {
        float res = 0.0f;
#pragma unroll
        for (int i = 0; i < MM; i++) res = __fadd_rn(res, __fmul_rn(x[i], __fsub_rn(ext[r * MM + i], ideal[i])));
        if (fabsf(__fsub_rn(res, 1.0f)) > 1e-6f || isnan(res) || isinf(res)) exc = 1;
        const float icp = __fdiv_rn(1.0f, x[r]);
        if (icp <= 1e-6f || isnan(icp) || isinf(icp)) exc = 1;
        nadir[r] = __fadd_rn(ideal[r], icp);
    }
    return exc;
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

// Compare-exchange of bitonic stage (k, jj) on a 64-key block held in registers: lane
// l holds the keys at base + l (e0) and base + l + 32 (e1).  jj <= 32.
__device__ __forceinline__ void bitonic_reg_stage(uint32_t &e0, uint32_t &e1, int base, int lane, int k, int jj)
{
    if (jj == 32) {  // both keys of the pair in this lane
        const bool asc = ((base + lane) & k) == 0;
        const uint32_t lo = min(e0, e1), hi = max(e0, e1);
        e0 = asc ? lo : hi;
        e1 = asc ? hi : lo;
    } else {
        const uint32_t o0 = __shfl_xor_sync(0xffffffffu, e0, jj), o1 = __shfl_xor_sync(0xffffffffu, e1, jj);
        const bool lower = (lane & jj) == 0;
        const bool asc0 = ((base + lane) & k) == 0, asc1 = ((base + lane + 32) & k) == 0;
        e0 = lower == asc0 ? min(e0, o0) : max(e0, o0);
        e1 = lower == asc1 ? min(e1, o1) : max(e1, o1);
    }
}

// Ascending bitonic sort of keys[0, P) (P a power of two) by the whole CTA, called by
// every thread after the keys are written.  Stages that compare keys 32 or fewer
// apart run in registers, each warp on its own 64-key blocks; the wider stages go
// through shared memory with a barrier each.  Returns after a barrier.
__device__ void block_bitonic_sort(uint32_t *keys, int P, int tid, int nth)
{
    const int lane = tid & 31, warp = tid >> 5, nwarps = nth >> 5;
    __syncthreads();
    if (P < 64) {  // one warp, through shared memory
        if (warp == 0)
            for (int k = 2; k <= P; k <<= 1)
                for (int jj = k >> 1; jj > 0; jj >>= 1) {
                    for (int q = lane; q < (P >> 1); q += 32) {
                        const int i = ((q & ~(jj - 1)) << 1) | (q & (jj - 1)), ixj = i + jj;
                        const uint32_t a = keys[i], b = keys[ixj];
                        if ((a > b) == ((i & k) == 0)) {
                            keys[i] = b;
                            keys[ixj] = a;
                        }
                    }
                    __syncwarp();
                }
        __syncthreads();
        return;
    }
    const int nblk = P >> 6;
    for (int b = warp; b < nblk; b += nwarps) {  // phases k <= 64: inside each block
        const int base = b << 6;
        uint32_t e0 = keys[base + lane], e1 = keys[base + lane + 32];
        for (int k = 2; k <= 64; k <<= 1)
            for (int jj = k >> 1; jj > 0; jj >>= 1) bitonic_reg_stage(e0, e1, base, lane, k, jj);
        keys[base + lane] = e0;
        keys[base + lane + 32] = e1;
    }
    for (int k = 128; k <= P; k <<= 1) {
        for (int jj = k >> 1; jj >= 64; jj >>= 1) {
            __syncthreads();
            for (int q = tid; q < (P >> 1); q += nth) {
                const int i = ((q & ~(jj - 1)) << 1) | (q & (jj - 1)), ixj = i + jj;
                const uint32_t a = keys[i], b = keys[ixj];
                if ((a > b) == ((i & k) == 0)) {
                    keys[i] = b;
                    keys[ixj] = a;
                }
            }
        }
        __syncthreads();
        for (int b = warp; b < nblk; b += nwarps) {
            const int base = b << 6;
            uint32_t e0 = keys[base + lane], e1 = keys[base + lane + 32];
            for (int jj = 32; jj > 0; jj >>= 1) bitonic_reg_stage(e0, e1, base, lane, k, jj);
            keys[base + lane] = e0;
            keys[base + lane + 32] = e1;
        }
    }
    __syncthreads();
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

    const int gy = dom_tiles(N2);
    for (int q = tid; q < RR; q += nth) {
        int v = -1;
        if (q < nrow) {
            v = 0;
            for (int y = 0; y < gy; y++) v += sc.np[(size_t)y * N2 + r0 + q];
        }
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

// MM: the objective count (4 or 6)
template <int MM>
__global__ void __launch_bounds__(kSelThreads, 1) k_select(Shape s, const float *__restrict__ obj, float *ext,
                                                        const float *__restrict__ refpts, SelectScratch sc,
                                                        int32_t *surv, uint32_t *d_gen, int bump_gen)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SelSmem &sm = *reinterpret_cast<SelSmem *>(smem_raw);
    const int N = s.N, N2 = 2 * N, R = s.R;
    constexpr int M = MM;
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

    // ---------------- ideal / worst (exact min / max): each thread reads its rows once
    {
        float mn[kMaxObj], mx[kMaxObj];
#pragma unroll
        for (int k = 0; k < kMaxObj; k++) {
            mn[k] = FLT_MAX;
            mx[k] = -FLT_MAX;
        }
        for (int i = tid; i < N2; i += nth) {
            const float *x = obj + (size_t)i * M;
#pragma unroll
            for (int k = 0; k < kMaxObj; k++) {
                if (k < M) {
                    const float v = x[k];
                    if (v < mn[k]) mn[k] = v;
                    if (v > mx[k]) mx[k] = v;
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kMaxObj; k++) {
            if (k >= M) break;
            for (int o = 16; o > 0; o >>= 1) {
                const float a = __shfl_xor_sync(0xffffffffu, mn[k], o), b = __shfl_xor_sync(0xffffffffu, mx[k], o);
                if (a < mn[k]) mn[k] = a;
                if (b > mx[k]) mx[k] = b;
            }
            if (lane == 0) {
                sm.red[warp * kMaxObj + k] = mn[k];
                sm.red[32 * kMaxObj + warp * kMaxObj + k] = mx[k];
            }
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
        // one pass over front 0 for every axis: each member's row is read once.  The
        // objectives take few distinct values, so ASF ties are common: tree places are
        // looked up only for ties, at most once per member and once per running best.
        constexpr uint64_t kUnset = ~0ull;
        ExtCand bests[kMaxObj];
        uint64_t bks[kMaxObj];  // tree key of each running best (kUnset: not computed yet)
        float fmxs[kMaxObj], id[kMaxObj];
#pragma unroll
        for (int i = 0; i < kMaxObj; i++) {
            bests[i] = ExtCand{0xffffffffu, kNoPos};
            bks[i] = kUnset;
            fmxs[i] = -FLT_MAX;
            id[i] = i < M ? sm.ideal[i] : 0.0f;
        }
        for (int t = tid; t < f0; t += nth) {
            const float *x = obj + (size_t)sc.sorted[t] * M;
            float xv[kMaxObj], a[kMaxObj];
#pragma unroll
            for (int k = 0; k < kMaxObj; k++) xv[k] = k < M ? x[k] : 0.0f;
            asf_rows(xv, id, M, a);
            uint64_t tk = kUnset;  // this member's tree key, once needed
#pragma unroll
            for (int i = 0; i < kMaxObj; i++) {
                if (i < M) {
                    const uint32_t v = __float_as_uint(a[i]);
                    bool take = v < bests[i].v || bests[i].pos == kNoPos;
                    if (!take && v == bests[i].v) {  // tie: the earlier position in tree order
                        if (tk == kUnset) tk = tree_rank(sc.trank, t);
                        if (bks[i] == kUnset) bks[i] = tree_rank(sc.trank, (int)bests[i].pos);
                        take = tk < bks[i];
                    }
                    if (take) {
                        bests[i] = ExtCand{v, (uint32_t)t};
                        bks[i] = tk;
                    }
                    if (xv[i] > fmxs[i]) fmxs[i] = xv[i];
                }
            }
        }
#pragma unroll
        for (int i = 0; i < kMaxObj; i++) {
            if (i >= M) break;
            ExtCand best = bests[i];
            float fmx = fmxs[i];
            uint64_t bkey = best.pos == kNoPos ? ~0ull : (bks[i] != kUnset ? bks[i] : tree_rank(sc.trank, (int)best.pos));
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
            if (lane == 1) xs.xkey[warp] = tree_rank(sc.trank, f0 + warp);
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
                for (int t = f0 + M + lane; t < B; t += 32) fkey = min(fkey, tree_rank(sc.trank, t));
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
    if (tid == 0) {
        const int exc = hyperplane_nadir<MM>(sm.ext, sm.ideal, sm.nadir);
        sm.hyp = exc;
        if (exc) {
            // updateNadirValue_MNDF (:685-884): max over front 0, worst when too close to ideal
#pragma unroll
            for (int k = 0; k < MM; k++) {
                const float b = sm.red[32 * kMaxObj + k];
                sm.nadir[k] = __fsub_rn(b, sm.ideal[k]) > 1e-6f ? b : sm.worst[k];
            }
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

// reference points staged in k_assoc's shared memory up to this size (larger sets are
// read from global memory, so the CTAs stay small)
constexpr size_t kAssocSmemMax = 16 * 1024;

// referenceBasedSorting phase 1 (:1105-1180) on the whole grid: one warp per
// solution of fronts 0..last, lanes over reference points; perpendicular
// distance (include/utils.cuh:1149-1171), argmin with the lowest index on ties.
// MM: the objective count when known at compile time (0: s.M at run time)
template <int MM>
__global__ void __launch_bounds__(256) k_assoc(Shape s, const float *__restrict__ obj,
                                               const float *__restrict__ refpts, SelectScratch sc)
{
    if (sc.info[3]) return;  // fronts filled N exactly: no niching (uniform over the grid)
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
    // the reference points in shared memory when they fit (every warp of the CTA reads them)
    extern __shared__ __align__(16) float rsm[];
    const bool staged = (size_t)R * M * sizeof(float) <= kAssocSmemMax;
    if (staged)
        for (int e = threadIdx.x; e < R * M; e += blockDim.x) rsm[e] = refpts[e];
    __syncthreads();
    const float *rp = staged ? rsm : refpts;
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
#pragma unroll 2
        for (int j = lane; j < R; j += 32) {
            const float *w = rp + (size_t)j * M;
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
// k_niche's shared memory without and with the counting sort's [32][R] table; the
// candidate lists are counted when R <= kCountSortMaxR and the table still fits in
// the 227 KB a CTA may use
constexpr int kCountSortMaxR = 512;
__host__ __device__ inline size_t niche_base_bytes(const Shape &s)
{
    // cj, nj, coff, kq | lv | keys (4N) | lsol (2N) | pofs | rnd
    return ((sizeof(SelSmem) + 15) & ~size_t(15)) +
           (size_t)(4 * s.R + 1 + 2 * s.N + 4 + 4 * s.N + 2 * s.N + s.R + 1 + s.N) * sizeof(int);
}
__host__ __device__ inline bool niche_counting(const Shape &s)
{
    return s.R <= kCountSortMaxR && niche_base_bytes(s) + (size_t)32 * s.R * sizeof(int) <= 232448;
}

__global__ void __launch_bounds__(kSelThreads, 1) k_niche(Shape s, SelectScratch sc, int32_t *surv, uint32_t *d_gen,
                                                       int bump_gen)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SelSmem &sm = *reinterpret_cast<SelSmem *>(smem_raw);
    const int N = s.N, N2 = 2 * N, R = s.R, Lsz = N2 + 4;
    int *cj = reinterpret_cast<int *>(smem_raw + ((sizeof(SelSmem) + 15) & ~size_t(15)));
    int *nj = cj + R;
    int *coff = nj + R;    // R + 1
    int *kq = coff + R + 1;
    int *lv = kq + R;      // Lsz: member distances (bits) for the lists, level histogram, picks before each level
    // 4N: sort keys (point, member) of the last front's members, then in place the
    // candidate lists (CSR by reference point)
    uint32_t *keys = reinterpret_cast<uint32_t *>(lv + Lsz);
    int *cand = reinterpret_cast<int *>(keys);
    int *lsol = cand + 2 * N2;  // 2N: the solution of each last-front member (position count0 + t)
    int *pofs = lsol + N2;      // R + 1: first pick of each point
    uint32_t *rnd = reinterpret_cast<uint32_t *>(pofs + R + 1);  // N: the list slot of every pick
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nth >> 5;
    const uint32_t gen = *d_gen;
    if (sc.info[3]) {  // fronts filled N exactly; k_select wrote the survivors
        if (tid == 0 && bump_gen) *d_gen = gen + 1;
        return;
    }
    const int rc = sc.info[0], count0 = sc.info[5], need = N - count0;
    const int nm = rc - count0;  // members of the last front
    for (int j = tid; j < R; j += nth) {
        cj[j] = sc.rho[j];
        nj[j] = sc.ncand[j];
        kq[j] = 0;
    }
    // member t of the last front: its point (a sort key (point, then t) for the sort;
    // the point itself, in the second half of the keys region, for the count), the
    // solution, and (in lv, free until the level histogram) its perpendicular distance
    // as bits.  Keys past the members pad the sort to a power of two.
    const bool counting = niche_counting(s);
    int *pj = cand + N2;
    int *hist = reinterpret_cast<int *>(rnd + N);  // [32][R] when counting
    const int tb = 32 - __clz(max(nm - 1, 1));  // bits of a member index
    int P = 1;
    while (P < nm) P <<= 1;
    for (int t = tid; t < (counting ? nm : P); t += nth) {
        if (t < nm) {
            const int sol = sc.sorted[count0 + t], j = sc.assoc[count0 + t];
            if (counting) pj[t] = j;
            else keys[t] = ((uint32_t)j << tb) | (uint32_t)t;
            lsol[t] = sol;
            lv[t] = __float_as_int(sc.dist[sol]);
        } else {
            keys[t] = 0xffffffffu;
        }
    }
    if (counting)
        for (int e = tid; e < 32 * R; e += nth) hist[e] = 0;
    if (tid == 0) sm.i0 = 0;
    __syncthreads();
    // CSR offsets of the candidate lists
    for (int base = 0; base < R; base += nth) {
        const int j = base + tid;
        const int v = j < R ? nj[j] : 0;
        int tot;
        const int pos = block_scan_value(v, sm, &tot);
        if (j < R) coff[j] = sm.i0 + pos;
        __syncthreads();
        if (tid == 0) sm.i0 += tot;
        __syncthreads();
    }
    if (tid == 0) coff[R] = sm.i0;
    // candidate lists in ascending member order: point j's list is positions coff[j] ..
    // coff[j] + n_j - 1.  With few points, a counting sort: warp w counts the points of
    // its chunk of members, each chunk's place in a list follows the earlier chunks',
    // and one lane per warp places its chunk in order.  Otherwise a sort of the keys
    // (point, member).
    if (counting) {
        const int C = (nm + 31) >> 5, t0 = warp * C, t1 = min(nm, t0 + C);
        for (int t = t0 + lane; t < t1; t += 32) atomicAdd(&hist[warp * R + pj[t]], 1);
        __syncthreads();
        for (int j = tid; j < R; j += nth) {
            int run = coff[j];
            for (int w = 0; w < 32; w++) {
                const int c = hist[w * R + j];
                hist[w * R + j] = run;
                run += c;
            }
        }
        __syncthreads();
        if (lane == 0)
            for (int t = t0; t < t1; t++) cand[hist[warp * R + pj[t]]++] = t;
    } else {
        block_bitonic_sort(keys, P, tid, nth);
        for (int q = tid; q < nm; q += nth) cand[q] = (int)(keys[q] & ((1u << tb) - 1u));  // member indices t
    }
    __syncthreads();
    // the nearest member of a point with niche count 0 (the first in list order among
    // equal distances) is its pick at level 0, which is the point's first pick whenever
    // it has one: it is moved to the list's end (a point that ends up picking nothing
    // never reads its list).  Distances are >= +0 (or FLT_MAX), so their bits order as
    // the values do.  Lists of up to kShortList members are scanned by one thread;
    // longer ones are queued (in pofs, free until the picks) for one warp each.
    constexpr int kShortList = 64;
    if (tid == 0) sm.i1 = 0;
    __syncthreads();
    for (int j = tid; j < R; j += nth) {
        const int n = nj[j];
        if (cj[j] != 0 || n == 0) continue;
        if (n > kShortList) {
            pofs[atomicAdd(&sm.i1, 1)] = j;
            continue;
        }
        int *cl = cand + coff[j];
        uint32_t bd = 0xffffffffu;
        int slot = 0;
        for (int q = 0; q < n; q++) {
            const uint32_t d = (uint32_t)lv[cl[q]];
            if (d < bd) {
                bd = d;
                slot = q;
            }
        }
        const int pick = cl[slot];
        cl[slot] = cl[n - 1];
        cl[n - 1] = pick;
    }
    __syncthreads();
    for (int u = warp; u < sm.i1; u += nwarps) {
        const int j = pofs[u], n = nj[j];
        int *cl = cand + coff[j];
        uint64_t best = ~0ull;
        for (int q = lane; q < n; q += 32) {
            const uint64_t key = ((uint64_t)(uint32_t)lv[cl[q]] << 32) | (uint32_t)q;
            best = key < best ? key : best;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const uint64_t other = __shfl_xor_sync(0xffffffffu, best, o);
            best = other < best ? other : best;
        }
        if (lane == 0) {
            const int slot = (int)(uint32_t)best, pick = cl[slot];
            cl[slot] = cl[n - 1];
            cl[n - 1] = pick;
        }
    }
    __syncthreads();
    // member indices to solutions; then the level histogram (+1 at c_j, -1 at c_j + n_j)
    for (int q = tid; q < nm; q += nth) cand[q] = lsol[cand[q]];
    for (int l = tid; l < Lsz; l += nth) lv[l] = 0;
    if (tid == 0) sm.i4 = 0;
    __syncthreads();
    for (int base = 0; base < R; base += nth) {
        const int j = base + tid;
        const int v = j < R ? nj[j] : 0;
        const int l0 = min(j < R ? cj[j] : 0, Lsz - 1), l1 = min((j < R ? cj[j] : 0) + v, Lsz - 1);
        // most points start at level 0: one add per warp there
        const unsigned z = __ballot_sync(0xffffffffu, v > 0 && l0 == 0);
        if (lane == 0 && z) atomicAdd(&lv[0], __popc(z));
        if (v > 0 && l0 != 0) atomicAdd(&lv[l0], 1);
        if (v > 0) atomicAdd(&lv[l1], -1);
        const int top = __reduce_max_sync(0xffffffffu, v > 0 ? l1 : 0);
        if (lane == 0) atomicMax(&sm.i4, top);
    }
    __syncthreads();
    // every pick falls below level max_j(c_j + n_j): the scans stop there
    const int Lscan = min(Lsz, sm.i4 + 1);
    // active points per level, then picks before each level: lv[l] = picks at levels < l
    if (tid == 0) {
        sm.i0 = 0;
        sm.i1 = 0;
    }
    __syncthreads();
    for (int base = 0; base < Lscan; base += nth) {
        const int l = base + tid;
        const int d = l < Lscan ? lv[l] : 0;
        int tot;
        const int act = sm.i0 + block_scan_value(d, sm, &tot) + d;  // active points at level l
        int tot2;
        const int before = sm.i1 + block_scan_value(l < Lscan ? act : 0, sm, &tot2);
        if (l < Lscan) lv[l] = before;
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
    for (int l = tid; l + 1 < Lscan; l += nth)
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
    // the slot of every pick, computed in parallel (each draw is keyed by its point and level)
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
    // Each pick also gets the key (level, point) of its place among the survivors: the
    // picks of a level follow those of earlier levels, in ascending point index.  The
    // keys sit in the second half of the keys region (the lists use the first).
    const int npick = pofs[R];  // = need
    // survivor order: a warp per level over the points' activity when levels x point
    // words are few, else a sort of the picks' keys
    const int lmax = min(Ls, Lsz - 1);
    const bool by_levels = (lmax + 1) * ((R + 31) >> 5) <= 32 * 24;
    uint32_t *pkeys = keys + N2;
    const int pb = 32 - __clz(max(R - 1, 1));  // bits of a point index
    int P2 = 1;
    while (P2 < npick) P2 <<= 1;
    for (int pk = tid; pk < P2; pk += nth) {
        if (pk >= npick) {
            if (!by_levels) pkeys[pk] = 0xffffffffu;
            continue;
        }
        int lo = 0, hi = R - 1;  // point: pofs[lo] <= pk < pofs[lo + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (pofs[mid] <= pk) lo = mid;
            else hi = mid - 1;
        }
        const int q = pk - pofs[lo], level = cj[lo] + q, nc = nj[lo] - q;  // nc: candidates left
        // level 0: the nearest member, already at the list's end
        rnd[pk] = level == 0 ? (uint32_t)(nc - 1)
                             : rng_uint(draw(s.seed, TAG_NICHE, gen, (uint32_t)lo, (uint32_t)level, 0), (uint32_t)nc);
        if (!by_levels) pkeys[pk] = ((uint32_t)level << pb) | (uint32_t)lo;
    }
    __syncthreads();
    // each point takes its picks (rnd now holds each pick's slot); the q-th pick ends
    // at list position n_j - 1 - q.  The chain is serial per point: the next slot is
    // read before this pick's swap is stored.
    for (int j = tid; j < R; j += nth) {
        const int npk = kq[j];
        if (npk == 0) continue;
        int *cl = cand + coff[j];
        const uint32_t *sl = rnd + pofs[j];
        int last = nj[j] - 1, slot = (int)sl[0];
        for (int q = 0; q < npk; q++, last--) {
            const int nxt = q + 1 < npk ? (int)sl[q + 1] : 0;
            const int pick = cl[slot];
            cl[slot] = cl[last];
            cl[last] = pick;
            slot = nxt;
        }
    }
    for (int t = tid; t < count0; t += nth) surv[t] = sc.sorted[t];
    if (by_levels) {
        __syncthreads();
        for (int l = warp; l <= lmax; l += nwarps) {
            int run = 0;
            for (int jb = 0; jb < R; jb += 32) {
                const int j = jb + lane;
                const bool act = j < R && nj[j] > 0 && cj[j] <= l && l < cj[j] + nj[j];
                const uint32_t bal = __ballot_sync(0xffffffffu, act);
                const int rank = run + __popc(bal & ((1u << lane) - 1u));
                if (act && (l < Ls || rank < K)) surv[count0 + lv[l] + rank] = cand[coff[j] + nj[j] - 1 - (l - cj[j])];
                run += __popc(bal);
            }
        }
    } else {
        block_bitonic_sort(pkeys, P2, tid, nth);
        for (int p = tid; p < npick; p += nth) {
            const uint32_t key = pkeys[p];
            const int j = (int)(key & ((1u << pb) - 1u)), level = (int)(key >> pb);
            surv[count0 + p] = cand[coff[j] + nj[j] - 1 - (level - cj[j])];
        }
    }
    __syncthreads();
    if (tid == 0 && bump_gen) *d_gen = gen + 1;
}

size_t niche_smem_bytes(const Shape &s)
{
    return niche_base_bytes(s) + (niche_counting(s) ? (size_t)32 * s.R * sizeof(int) : 0);
}

int dom_tile_count(int N2) { return dom_tiles(N2); }

size_t select_smem_bytes(const Shape &s)
{
    (void)s;
    return ((sizeof(SelSmem) + 15) & ~size_t(15)) + sizeof(ExtSmem);
}

cudaError_t launch_select(const Shape &s, const float *obj, float *ext, const float *refpts, SelectScratch sc,
                          int32_t *surv, uint32_t *d_gen, int bump_gen, cudaStream_t st)
{
    cudaError_t e;
    const dim3 dgrid((2 * s.N + 31) / 32, dom_tiles(2 * s.N));
    if (s.M == 4) {
        k_dominance<4><<<dgrid, 32 * kDomTileWords, 0, st>>>(s, obj, sc.dom, sc.np);
    } else if (s.M == 6) {
        k_dominance<6><<<dgrid, 32 * kDomTileWords, 0, st>>>(s, obj, sc.dom, sc.np);
    } else {
        k_dominance<0><<<dgrid, 32 * kDomTileWords, 0, st>>>(s, obj, sc.dom, sc.np);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t fsm = fronts_smem_bytes(s);
    if ((e = raise_smem_limit((const void *)k_fronts, fsm)) != cudaSuccess) return e;
    k_fronts<<<kFrontCtas, kFrontThreads, fsm, st>>>(s, sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    size_t smem = select_smem_bytes(s);
    if (s.M == 4) {
        if ((e = raise_smem_limit((const void *)k_select<4>, smem)) != cudaSuccess) return e;
        k_select<4><<<1, kSelThreads, smem, st>>>(s, obj, ext, refpts, sc, surv, d_gen, bump_gen);
    } else {
        if ((e = raise_smem_limit((const void *)k_select<6>, smem)) != cudaSuccess) return e;
        k_select<6><<<1, kSelThreads, smem, st>>>(s, obj, ext, refpts, sc, surv, d_gen, bump_gen);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int warps_needed = 2 * s.N;
    const int ag = std::min((warps_needed + 7) / 8, 148 * 8);
    const size_t rb = (size_t)s.R * s.M * sizeof(float), asm_ = rb <= kAssocSmemMax ? rb : 0;
    if (s.M == 4) k_assoc<4><<<ag, 256, asm_, st>>>(s, obj, refpts, sc);
    else if (s.M == 6) k_assoc<6><<<ag, 256, asm_, st>>>(s, obj, refpts, sc);
    else k_assoc<0><<<ag, 256, asm_, st>>>(s, obj, refpts, sc);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t nsm = niche_smem_bytes(s);
    if ((e = raise_smem_limit((const void *)k_niche, nsm)) != cudaSuccess) return e;
    k_niche<<<1, kSelThreads, nsm, st>>>(s, sc, surv, d_gen, bump_gen);
    return cudaGetLastError();
}

}  // namespace pe
