// pe_eval.cu -- variation and objective-evaluation kernels for sm_100a.
//
//  k_variation<MODE>  one CTA per solution: initialise (initializationKernel,
//                     src/main.cu:26-119), mutate (mutationKernel,
//                     src/main.cu:121-240) or just re-evaluate a supplied
//                     solution; then packs the nucleotide bit planes and
//                     evaluates every objective except the hairpin stem.
//  k_sl               one CTA per (solution, CDS): the hairpin-stem scan
//                     (calMaximumSL, include/utils.cuh:712-888) on bit planes;
//                     the last CTA of a solution combines its CDSs.
#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include <cuda_runtime.h>

#include "pe_device.cuh"
#include "pe_internal.h"

namespace pe {

enum { MODE_INIT = 0, MODE_EVAL = 1, MODE_MUTATE = 2 };

// small per-CTA copies of the codon tables
struct SmemTab {
    uint8_t nt[64][4];
    uint8_t pat[64];  // the codon's three nucleotides as plane bits: lo bits 0..2, hi bits 4..6
    int64_t lw[64];
    uint8_t wzero[64];
    uint8_t gc3[64];
    uint8_t gcn[64];
    int8_t start[21];
    int8_t count[21];
    int8_t pad[2];
};

__device__ __forceinline__ void load_tab(SmemTab &st, const DevTables *gt, int tid, int nth)
{
    for (int i = tid; i < 64; i += nth) {
        *(uint32_t *)st.nt[i] = *(const uint32_t *)gt->nt[i];
        uint32_t pt = 0;
        for (int b = 0; b < 3; b++) pt |= ((gt->nt[i][b] & 1u) << b) | ((gt->nt[i][b] >> 1) << (4 + b));
        st.pat[i] = (uint8_t)pt;
        st.lw[i] = gt->lw[i];
        st.wzero[i] = gt->wzero[i];
        st.gc3[i] = gt->gc3[i];
        st.gcn[i] = gt->gcn[i];
    }
    for (int i = tid; i < 21; i += nth) {
        st.start[i] = gt->start[i];
        st.count[i] = gt->count[i];
    }
}

__device__ __forceinline__ int nt_at(const SmemTab &st, const uint8_t *row, int x)
{
    int a = x / 3;
    return st.nt[row[a]][x - 3 * a];
}

// Pack codon ids of every CDS into (lo, hi) nucleotide bit planes:
// bit b of word w holds nucleotide 32w+b (A=00, C=01, G=10, U=11).
__device__ void pack_planes(const Shape &s, const SmemTab &st, const uint8_t *ids, uint2 *planes, int tid, int nth,
                            const uint32_t *only = nullptr)
{
    // word w holds nucleotides 32w .. 32w+31: the codons a0 = floor(32w/3) .. that
    // overlap it contribute their 3-bit patterns at bit offset 3a - 32w.  With
    // `only`, just the words whose bit is set there are packed (the others hold
    // their values already).
    const int total = s.m * s.Wp;
    for (int e = tid; e < total; e += nth) {
        if (only && !((only[e >> 5] >> (e & 31)) & 1u)) continue;
        int c = e / s.Wp, w = e - c * s.Wp;
        uint32_t lo = 0, hi = 0;
        if (w < s.W) {
            const uint8_t *row = ids + c * s.Lp;
            const int base = 32 * w;
            const int a0 = base / 3, a1 = min((base + 31) / 3, s.L - 1);
            for (int a = a0; a <= a1; a++) {
                const uint32_t pt = st.pat[row[a]];
                const int off = 3 * a - base;  // -2 .. 31
                const uint32_t l3 = pt & 7u, h3 = (pt >> 4) & 7u;
                lo |= off >= 0 ? (l3 << off) : (l3 >> -off);
                hi |= off >= 0 ? (h3 << off) : (h3 >> -off);
            }
        }
        planes[e] = make_uint2(lo, hi);
    }
}

// True when the CDS holds a stem of length K = (n-4)/2 with a loop of >= 4
// nucleotides: the only case in which mutationSL's undo branch runs
// (include/mutation.cuh:843).  Uniform result for the CTA.
__device__ bool cta_full_hairpin(const Shape &s, const SmemTab &st, const uint8_t *row, int tid, int nth)
{
    const int n = s.n, K = s.K;
    if (K <= 0) return false;
    bool found = false;
    // (ri, ci) pairs exist only for ri <= n - K - 5 (ci in [ri + 5, n - K])
    for (int ri = K - 1; ri <= n - K - 5 && !found; ri++) {
        for (int ci = ri + 5; ci + K - 1 <= n - 1 && !found; ci++) {
            int ok = 1;
            for (int u = tid; u < K; u += nth) ok &= (nt_at(st, row, ri - u) ^ nt_at(st, row, ci + u)) == 3;
            found = __syncthreads_and(ok) != 0;
        }
    }
    return found;
}

// CDS pair of LRCS result r: (0,0), (0,1), .., (0,m-1), (1,1), (1,2), ..
__host__ __device__ __forceinline__ void lrcs_pair_of(int m, int r, int &a, int &b)
{
    a = 0;
    while (r >= m - a) {
        r -= m - a;
        a++;
    }
    b = a + r;
}

struct VarSmem {
    SmemTab tab;
    float pobj[kMaxObj];
    int8_t pobjidx[2 * kMaxObj];
    int32_t ppql[3];
    int32_t sl_old;
    int32_t sl_mut;
    int32_t op;
    unsigned long long changed;  // CDSs whose planes the mutation changed (bit c)
    int32_t ntask;               // entries of the evaluation's task list
};

// Across a warp whose lanes hold (value, index) with index -1 for none: the largest
// value, the highest index among equal ones, left in every lane; returns the lane
// that held it.  Values are never NaN.
__device__ __forceinline__ int warp_last_max(float &v, int &idx)
{
    int src = threadIdx.x & 31;
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o), os = __shfl_xor_sync(0xffffffffu, src, o);
        if (oi >= 0 && (idx < 0 || ov > v || (ov == v && oi > idx))) {
            v = ov;
            idx = oi;
            src = os;
        }
    }
    return src;
}

// the same for the smallest count, the highest index among equal ones
__device__ __forceinline__ void warp_last_min(int &v, int &idx)
{
    for (int o = 16; o > 0; o >>= 1) {
        const int ov = __shfl_xor_sync(0xffffffffu, v, o), oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (oi >= 0 && (idx < 0 || ov < v || (ov == v && oi > idx))) {
            v = ov;
            idx = oi;
        }
    }
}

// Every objective except the string objective, for the solution in smem.
// Reference evaluators: include/utils.cuh:271-710.  Per-CDS sums are exact
// integers (fixed-point log weights for CAI, fixed-point CPS), so the result
// does not depend on the reduction order.
//
// The per-CDS (per-pair) sums sit in `ax` in the aux layout (AUX_* offsets): CAI
// value bits, CBP sum halves, HSC count, GC count per CDS, then the HD count of
// every CDS pair.  Only the CDSs in `changed` (and the pairs touching one) are
// summed; the others are taken from the parent's aux `pax`, bit for bit what the
// sums give for an unchanged CDS (pax == nullptr: `changed` holds every CDS).  The
// warps share one list of tasks: for each changed CDS, one per enabled per-CDS
// objective, then its HD pairs.  After one barrier the sums go to `cax` (the
// child's aux) and one thread per objective (each in its own warp) reduces over the
// CDSs in CDS order, as the reference's loops do.
__device__ void light_eval(const Shape &s, const DevTables *gt, const SmemTab &st, const uint8_t *ids,
                           const uint2 *planes, int32_t *ax, int32_t *tl, int *ntl, unsigned long long changed,
                           const int32_t *pax, int32_t *cax, float *obj, int8_t *objidx, int tid, int nth)
{
    const int warp = tid >> 5, lane = tid & 31, nwarps = nth >> 5;
    const int L = s.L, m = s.m;
    const int sCAI = s.slot[K_CAI], sCBP = s.slot[K_CBP], sHSC = s.slot[K_HSC], sHD = s.slot[K_HD],
              sGC = s.slot[K_GC];
    const int npairs = m * (m - 1) / 2;
    const int kinds[4] = {sCAI >= 0 ? 0 : -1, sCBP >= 0 ? 1 : -1, sHSC >= 0 ? 2 : -1, sGC >= 0 ? 3 : -1};
    // the task list (warp 0): one entry (kind << 16 | CDS) per changed CDS and enabled
    // per-CDS objective, then (4 << 16 | pair) per CDS pair with a changed member
    if (warp == 0) {
        int n = 0;
        for (int cb = 0; cb < m; cb += 32) {
            const int c = cb + lane;
            const bool on = c < m && ((changed >> c) & 1ull);
            const unsigned bal = __ballot_sync(0xffffffffu, on);
            const int r = __popc(bal & ((1u << lane) - 1u));
            int kk = 0;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (kinds[q] < 0) continue;
                if (on) tl[n + r + kk * __popc(bal)] = (kinds[q] << 16) | c;
                kk++;
            }
            n += kk * __popc(bal);
        }
        if (sHD >= 0) {
            for (int pb = 0; pb < npairs; pb += 32) {
                const int pi = pb + lane;
                const bool on = pi < npairs && (((changed >> gt->pair_i[pi]) | (changed >> gt->pair_j[pi])) & 1ull);
                const unsigned bal = __ballot_sync(0xffffffffu, on);
                if (on) tl[n + __popc(bal & ((1u << lane) - 1u))] = (4 << 16) | pi;
                n += __popc(bal);
            }
        }
        if (lane == 0) *ntl = n;
    }
    if (pax) {  // the unchanged CDSs' sums, and the pairs of two unchanged CDSs, from the parent
        for (int q = 0; q < 5; q++)
            for (int c = tid; c < m; c += nth)
                if (!((changed >> c) & 1ull)) ax[q * m + c] = pax[q * m + c];
        if (sHD >= 0)
            for (int pi = tid; pi < npairs; pi += nth)
                if (!(((changed >> gt->pair_i[pi]) | (changed >> gt->pair_j[pi])) & 1ull))
                    ax[AUX_HD(m) + pi] = pax[AUX_HD(m) + pi];
    }
    __syncthreads();
    const int ntask = *ntl;
    for (int task = warp; task < ntask; task += nwarps) {
        const int ent = tl[task], kind = ent >> 16;
        if (kind < 4) {
            const int c = ent & 0xffff;
            const uint8_t *row = ids + c * s.Lp;
            if (kind == 0) {  // CAI: exp(mean log w)
                long long S = 0;
                int z = 0;
#pragma unroll 4
                for (int a = lane; a < L; a += 32) {
                    int id = row[a];
                    S += st.lw[id];
                    z |= st.wzero[id];
                }
                S = warp_sum(S);
                z = __any_sync(0xffffffffu, z);
                if (lane == 0) {
                    double x = __ddiv_rn(__dmul_rn((double)S, 1.0 / 4294967296.0), (double)L);
                    float cai = z ? 0.0f : (float)det_exp(x);
                    ax[AUX_CAI(m) + c] = __float_as_int(cai);
                }
            } else if (kind == 1) {  // CBP: codon-pair score sum over pairs a in [0, L-3]
                long long S = 0;
                for (int a = lane; a < L - 2; a += 32) {
                    int c1 = row[a], c2 = row[a + 1];
                    if (c1 < 61 && c2 < 61) S += __ldg(&gt->cpsf[c1 * 61 + c2]);
                }
                S = warp_sum(S);
                if (lane == 0) {
                    ax[AUX_CBP_LO(m) + c] = (int32_t)(uint32_t)(unsigned long long)S;
                    ax[AUX_CBP_HI(m) + c] = (int32_t)(uint32_t)((unsigned long long)S >> 32);
                }
            } else if (kind == 2) {  // HSC: hidden stop codons in the +1/+2 frames per boundary
                int cnt = 0;
                for (int a = lane; a < L - 1; a += 32) cnt += __ldg(&gt->hsc[row[a] * 64 + row[a + 1]]);
                cnt = warp_sum(cnt);
                if (lane == 0) ax[AUX_HSC(m) + c] = cnt;
            } else {  // GC3 (or whole-CDS GC) count
                int cnt = 0;
                if (s.gcmode == PE_GC3) {
#pragma unroll 4
                    for (int a = lane; a < L; a += 32) cnt += st.gc3[row[a]];
                } else {
                    const uint2 *A = planes + c * s.Wp;
                    for (int w = lane; w < s.W; w += 32) cnt += __popc(A[w].x ^ A[w].y);
                }
                cnt = warp_sum(cnt);
                if (lane == 0) ax[AUX_GC(m) + c] = cnt;
            }
        } else {  // HD: nucleotide mismatches of a pair with a changed CDS, XOR/popcount of planes
            const int pi = ent & 0xffff;
            const uint2 *A = planes + gt->pair_i[pi] * s.Wp, *B = planes + gt->pair_j[pi] * s.Wp;
            int cnt = 0;
            for (int w = lane; w < s.W; w += 32) {
                uint2 x = A[w], y = B[w];
                cnt += __popc((x.x ^ y.x) | (x.y ^ y.y));
            }
            cnt = warp_sum(cnt);
            if (lane == 0) ax[AUX_HD(m) + pi] = cnt;
        }
    }
    __syncthreads();
    if (cax)
        for (int e = tid; e < AUX_HD(m) + npairs; e += nth) cax[e] = ax[e];
    if (warp >= 5) return;
    // The reductions over CDSs, one objective per warp.  The reference's loops keep the
    // last CDS whose value reaches the extreme (`>=`); no value is NaN, so that is the
    // highest index holding the extreme, found here with the lanes over CDSs (pairs).
    // HD and HSC divide counts by a constant: a correctly rounded quotient of counts
    // below 2^23 by the same divisor is strictly increasing in the count, so their
    // extremes are found on the counts and divided once.
    if (warp == 0 && sCAI >= 0) {
        float best = 0.0f;
        int bi = -1;
        for (int c = lane; c < m; c += 32) {
            const float v = -__int_as_float(ax[AUX_CAI(m) + c]);
            if (bi < 0 || v >= best) {
                best = v;
                bi = c;
            }
        }
        warp_last_max(best, bi);
        if (lane == 0) {
            obj[sCAI] = best;
            objidx[2 * sCAI] = (int8_t)bi;
            objidx[2 * sCAI + 1] = 0;
        }
    }
    if (warp == 1 % nwarps && sCBP >= 0) {
        float best = 0.0f;
        int bi = -1;
        for (int c = lane; c < m; c += 32) {
            const long long S = (long long)(((unsigned long long)(uint32_t)ax[AUX_CBP_HI(m) + c] << 32) |
                                            (uint32_t)ax[AUX_CBP_LO(m) + c]);
            const double x = __ddiv_rn(__dmul_rn((double)S, 1.0 / 4294967296.0), (double)(L - 2));
            const float v = -(float)x;
            if (bi < 0 || v >= best) {
                best = v;
                bi = c;
            }
        }
        warp_last_max(best, bi);
        if (lane == 0) {
            obj[sCBP] = best;
            objidx[2 * sCBP] = (int8_t)bi;
            objidx[2 * sCBP + 1] = 0;
        }
    }
    if (warp == 2 % nwarps && sHSC >= 0) {  // the largest -count/(L-1): the last smallest count
        int bc = 0, bi = -1;
        for (int c = lane; c < m; c += 32) {
            const int cnt = ax[AUX_HSC(m) + c];
            if (bi < 0 || cnt <= bc) {
                bc = cnt;
                bi = c;
            }
        }
        warp_last_min(bc, bi);
        if (lane == 0) {
            obj[sHSC] = -__fdiv_rn((float)bc, (float)(L - 1));
            objidx[2 * sHSC] = (int8_t)bi;
            objidx[2 * sHSC + 1] = 0;
        }
    }
    if (warp == 3 % nwarps && sHD >= 0) {  // the largest -count/n: the last pair with the smallest count
        int bc = 0, bp = -1;
        for (int pi = lane; pi < npairs; pi += 32) {
            const int cnt = ax[AUX_HD(m) + pi];
            if (bp < 0 || cnt <= bc) {
                bc = cnt;
                bp = pi;
            }
        }
        warp_last_min(bc, bp);
        if (lane == 0) {
            obj[sHD] = -__fdiv_rn((float)bc, (float)s.n);
            objidx[2 * sHD] = (int8_t)gt->pair_i[bp];
            objidx[2 * sHD + 1] = (int8_t)gt->pair_j[bp];
        }
    }
    if (warp == 4 % nwarps && sGC >= 0) {
        float best = 0.0f;
        int bi = -1, dir = 1;
        for (int c = lane; c < m; c += 32) {
            float dev, diff;
            const int cnt = ax[AUX_GC(m) + c];
            if (s.gcmode == PE_GC3) {
                diff = __fsub_rn(__fdiv_rn((float)cnt, (float)L), gt->ref_gc3);
                dev = fabsf(diff);
            } else {
                const float refGC = __fmul_rn((float)s.n, gt->ref_gc);
                diff = __fsub_rn((float)cnt, refGC);
                dev = __fdiv_rn(fabsf(diff), refGC);
            }
            if (bi < 0 || dev >= best) {
                best = dev;
                bi = c;
                dir = diff < 0.0f ? 1 : -1;
            }
        }
        const int w = warp_last_max(best, bi);
        dir = __shfl_sync(0xffffffffu, dir, w);
        if (lane == 0) {
            obj[sGC] = best;
            objidx[2 * sGC] = (int8_t)bi;
            objidx[2 * sGC + 1] = (int8_t)dir;
        }
    }
}

// ---------------------------------------------------------------------------
// mutation operators (include/mutation.cuh), each thread owns one codon
// ---------------------------------------------------------------------------

#define MDRAW(pos, j) draw(s.seed, TAG_MUT, gen, ridx, (uint32_t)(pos), (uint32_t)(j))

// The probability tests of codon positions 4q .. 4q+3: one Philox4x32-10 block with
// counter (TAG_MUTP, gen, idx, q), word p % 4 for position p.  Each thread takes four
// consecutive positions, so a block is computed once for four tests.
__device__ __forceinline__ uint4 pdraw4(const Shape &s, uint32_t gen, uint32_t ridx, int q)
{
    return philox4x32_10(make_uint4(TAG_MUTP, gen, ridx, (uint32_t)q),
                         make_uint2((uint32_t)s.seed, (uint32_t)(s.seed >> 32)));
}
__device__ __forceinline__ uint32_t word4(const uint4 &w, int u)
{
    return u == 0 ? w.x : u == 1 ? w.y : u == 2 ? w.z : w.w;
}

// indexArrayShuffling (include/utils.cuh:203-218) of 0 .. k-1 with the draws
// MDRAW(pos, 1 .. k-1), as a packed array (entry u in bits 3u .. 3u+2).  Draws 1..3
// are words 1..3 of one Philox block and draws 4, 5 words 0, 1 of the next, so at
// most two blocks are computed.
__device__ __forceinline__ uint32_t shuffle_k(const Shape &s, uint32_t gen, uint32_t ridx, int pos, int k)
{
    uint32_t arr = 0;
#pragma unroll
    for (int u = 0; u < 6; u++) arr |= (uint32_t)u << (3 * u);
    if (k < 2) return arr;
    const uint2 key = make_uint2((uint32_t)s.seed, (uint32_t)(s.seed >> 32));
    const uint4 b0 = philox4x32_10(make_uint4(TAG_MUT, gen, ridx, (uint32_t)pos * 8u), key);
    uint4 b1 = make_uint4(0u, 0u, 0u, 0u);
    if (k > 4) b1 = philox4x32_10(make_uint4(TAG_MUT, gen, ridx, (uint32_t)pos * 8u + 1u), key);
    const uint32_t w[5] = {b0.y, b0.z, b0.w, b1.x, b1.y};  // draws 1 .. 5
#pragma unroll
    for (int d = 1; d <= 5; d++) {
        const int i = k - d;  // i = k-1 down to 1
        if (i < 1) break;
        const int j = (int)rng_uint(w[d - 1], (uint32_t)(i + 1));
        const uint32_t ai = (arr >> (3 * i)) & 7u, aj = (arr >> (3 * j)) & 7u;
        arr = (arr & ~(7u << (3 * i)) & ~(7u << (3 * j))) | (aj << (3 * i)) | (ai << (3 * j));
    }
    return arr;
}

// mismatching nucleotides of two codons from their plane patterns
__device__ __forceinline__ int codon_mismatch(uint32_t pa, uint32_t pb)
{
    const uint32_t x = pa ^ pb;
    return __popc((x | (x >> 4)) & 7u);
}

// Marks the plane words codon a of CDS c covers (nucleotides 3a .. 3a+2: one or two
// words) as changed: bit c * Wp + w of `dirty`.  Every operator marks each codon it
// leaves different from the parent's, so the marked words are exactly the words
// whose packed nucleotides differ (distinct codon ids are distinct triplets).
__device__ __forceinline__ void mark_codon(const Shape &s, uint32_t *dirty, int c, int a)
{
    const int w0 = (3 * a) >> 5, w1 = min((3 * a + 2) >> 5, s.W - 1);
    for (int w = w0; w <= w1; w++) {
        const int bit = c * s.Wp + w;
        atomicOr(&dirty[bit >> 5], 1u << (bit & 31));
    }
}

__device__ void mutate_solution(const Shape &s, const DevTables *gt, VarSmem &sm, const int8_t *aa, uint8_t *ids,
                                uint32_t *dirty, uint32_t gen, uint32_t ridx, int tid, int nth)
{
    const SmemTab &st = sm.tab;
    const int L = s.L, m = s.m;
    const float pm = s.pm;
    const int op = sm.op;
    switch (op) {
    case 0: {  // mutationRandom (:16-63)
        for (int q = tid; 4 * q < m * L; q += nth) {
            const uint4 w4 = pdraw4(s, gen, ridx, q);
            const int c0 = (4 * q) / L, a0 = 4 * q - c0 * L;  // CDS and codon of position 4q
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int pos = 4 * q + u;
                if (pos >= m * L) break;
                const bool wrap = a0 + u >= L;  // L >= 3, so a quad crosses at most one CDS boundary
                const int c = c0 + (wrap ? 1 : 0), a = a0 + u - (wrap ? L : 0);
                int am = aa[a];
                int k = st.count[am];
                if (rng_u01(word4(w4, u)) > pm || k == 1) continue;
                uint8_t *cell = ids + c * s.Lp + a;
                int cur = *cell - st.start[am];
                int nw = (int)rng_uint(MDRAW(pos, 1), (uint32_t)(k - 1));
                if (nw >= cur) nw++;
                *cell = (uint8_t)(st.start[am] + nw);
                mark_codon(s, dirty, c, a);
            }
        }
        break;
    }
    case 1: {  // mutationCAI, SELECT_UPPER_RANDOM (:65-142)
        int c = sm.pobjidx[2 * s.slot[K_CAI]];
        for (int q = tid; 4 * q < L; q += nth) {
            const uint4 w4 = pdraw4(s, gen, ridx, q);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int a = 4 * q + u;
                if (a >= L) break;
                int am = aa[a];
                int k = st.count[am];
                if (rng_u01(word4(w4, u)) > pm || k == 1) continue;
                uint8_t *cell = ids + c * s.Lp + a;
                int cur = *cell - st.start[am];
                if (cur == k - 1) continue;
                int nw = cur + 1 + (int)rng_uint(MDRAW(a, 1), (uint32_t)(k - 1 - cur));
                *cell = (uint8_t)(st.start[am] + nw);
                mark_codon(s, dirty, c, a);
            }
        }
        break;
    }
    case 2: {  // mutationCBP, SELECT_UPPER_RANDOM, prob 2Pm, positions of parity gen%2 (:144-262)
        int c = sm.pobjidx[2 * s.slot[K_CBP]];
        float pm2 = __fmul_rn(pm, 2.0f);
        int parity = (int)(gen & 1u);
        uint8_t *row = ids + c * s.Lp;
        for (int q = tid; 4 * q < L - 1; q += nth) {
          const uint4 w4 = pdraw4(s, gen, ridx, q);
          for (int u = 0; u < 4; u++) {
            const int a = 4 * q + u;
            if (a >= L - 1) break;
            if ((a & 1) != parity) continue;
            int am = aa[a];
            int k = st.count[am];
            if (rng_u01(word4(w4, u)) > pm2 || k == 1) continue;
            int curg = row[a];
            int cur = curg - st.start[am];
            int left = a > 0 ? row[a - 1] : -1;
            int right = row[a + 1];
            float curs = 0.0f;
            if (left >= 0 && left < 61 && curg < 61) curs = __ldg(&gt->cps[left * 61 + curg]);
            if (right < 61 && curg < 61) curs = __fadd_rn(curs, __ldg(&gt->cps[curg * 61 + right]));
            uint32_t up = 0;  // the better synonyms, packed 3 bits each
            int nup = 0;
            for (int j = 0; j < k; j++) {
                if (j == cur) continue;
                int g = st.start[am] + j;
                float ns = 0.0f;
                if (left >= 0 && left < 61 && g < 61) ns = __fadd_rn(ns, __ldg(&gt->cps[left * 61 + g]));
                if (right < 61 && g < 61) ns = __fadd_rn(ns, __ldg(&gt->cps[g * 61 + right]));
                if (ns > curs) up |= (uint32_t)j << (3 * nup++);
            }
            if (nup > 0) {
                const int pick = (int)rng_uint(MDRAW(a, 1), (uint32_t)nup);
                row[a] = (uint8_t)(st.start[am] + ((up >> (3 * pick)) & 7u));
                mark_codon(s, dirty, c, a);
            }
          }
        }
        break;
    }
    case 3: {  // mutationHSC, SELECT_UPPER_RANDOM, prob 2Pm, parity gen%2 (:264-388)
        int c = sm.pobjidx[2 * s.slot[K_HSC]];
        float pm2 = __fmul_rn(pm, 2.0f);
        int parity = (int)(gen & 1u);
        uint8_t *row = ids + c * s.Lp;
        for (int q = tid; 4 * q < L; q += nth) {
          const uint4 w4 = pdraw4(s, gen, ridx, q);
          for (int u = 0; u < 4; u++) {
            const int a = 4 * q + u;
            if (a >= L) break;
            if ((a & 1) != parity) continue;
            int am = aa[a];
            int k = st.count[am];
            if (rng_u01(word4(w4, u)) > pm2 || k == 1) continue;
            int cur = row[a] - st.start[am];
            bool hl = a > 0, hr = a < L - 1;
            int lft = hl ? row[a - 1] : 0, rgt = hr ? row[a + 1] : 0;
            int curs = (hl ? __ldg(&gt->hsc[lft * 64 + row[a]]) : 0) + (hr ? __ldg(&gt->hsc[row[a] * 64 + rgt]) : 0);
            uint32_t up = 0;  // the better synonyms, packed 3 bits each
            int nup = 0;
            for (int j = 0; j < k; j++) {
                if (j == cur) continue;
                int g = st.start[am] + j;
                int ns = (hl ? __ldg(&gt->hsc[lft * 64 + g]) : 0) + (hr ? __ldg(&gt->hsc[g * 64 + rgt]) : 0);
                if (ns > curs) up |= (uint32_t)j << (3 * nup++);
            }
            if (nup > 0) {
                const int pick = (int)rng_uint(MDRAW(a, 1), (uint32_t)nup);
                row[a] = (uint8_t)(st.start[am] + ((up >> (3 * pick)) & 7u));
                mark_codon(s, dirty, c, a);
            }
          }
        }
        break;
    }
    case 4: {  // mutationHD (:390-534)
        int hs = s.slot[K_HD];
        int c1 = sm.pobjidx[2 * hs], c2 = sm.pobjidx[2 * hs + 1];
        for (int q = tid; 4 * q < L; q += nth) {
          const uint4 w4 = pdraw4(s, gen, ridx, q);
          for (int u = 0; u < 4; u++) {
            const int a = 4 * q + u;
            if (a >= L) break;
            int am = aa[a];
            int k = st.count[am];
            if (rng_u01(word4(w4, u)) > pm || k == 1) continue;
            const uint32_t arr = shuffle_k(s, gen, ridx, a, k);
            const int x = ids[c1 * s.Lp + a];
            const int cur = x - st.start[am];
            // mismatches of every synonym sh against CDS c2 (np) and its fewest against the
            // other CDSs (nm), the current codon's too, one pass over the CDSs
            const uint32_t px = st.pat[x], p2 = st.pat[ids[c2 * s.Lp + a]];
            uint32_t pg[6];
            int nmv[6];
#pragma unroll
            for (int sh = 0; sh < 6; sh++) {
                pg[sh] = sh < k ? st.pat[st.start[am] + sh] : 0u;
                nmv[sh] = 127;
            }
            int cur_m = 127;
            for (int j = 0; j < m; j++) {
                if (j == c1) continue;
                const uint32_t py = st.pat[ids[j * s.Lp + a]];
                cur_m = min(cur_m, codon_mismatch(px, py));
#pragma unroll
                for (int sh = 0; sh < 6; sh++)
                    if (sh < k) nmv[sh] = min(nmv[sh], codon_mismatch(pg[sh], py));
            }
            const int cur_pair = codon_mismatch(px, p2);
            int best_pair = -1, best_m = -1, best = -1;
#pragma unroll
            for (int u = 0; u < 6; u++) {
                if (u >= k) break;
                const int sh = (arr >> (3 * u)) & 7u;
                if (sh == cur) continue;
                int np = 0, nm = 0;
#pragma unroll
                for (int q = 0; q < 6; q++)
                    if (q == sh) {
                        np = codon_mismatch(pg[q], p2);
                        nm = nmv[q];
                    }
                if (nm > cur_m && nm > best_m) {
                    best_m = nm;
                    best = sh;
                } else if (best_m == -1 && nm == cur_m && np > cur_pair && np > best_pair) {
                    best_pair = np;
                    best = sh;
                }
            }
            if (best_m != -1 || best_pair != -1) {
                ids[c1 * s.Lp + a] = (uint8_t)(st.start[am] + best);
                mark_codon(s, dirty, c1, a);
            }
          }
        }
        break;
    }
    case 5: {  // mutationGC3 (:536-653) / mutationGC (:655-773), direction from objidx
        int gs = s.slot[K_GC];
        int c = sm.pobjidx[2 * gs];
        int dir = sm.pobjidx[2 * gs + 1];
        if (dir != 1 && dir != -1) break;
        float prob;
        if (s.gcmode == PE_GC3) {
            prob = sm.pobj[gs];
        } else {
            float refGC = __fmul_rn((float)(3 * L), gt->ref_gc);
            prob = __fdiv_rn(__fmul_rn(sm.pobj[gs], refGC), (float)L);
        }
        uint8_t *row = ids + c * s.Lp;
        for (int q = tid; 4 * q < L; q += nth) {
          const uint4 w4 = pdraw4(s, gen, ridx, q);
          for (int u = 0; u < 4; u++) {
            const int a = 4 * q + u;
            if (a >= L) break;
            int am = aa[a];
            int k = st.count[am];
            if (rng_u01(word4(w4, u)) > prob || k == 1) continue;
            const uint32_t arr = shuffle_k(s, gen, ridx, a, k);
            int curg = row[a];
            int cur = curg - st.start[am];
            int cgc = s.gcmode == PE_GC3 ? st.gc3[curg] : st.gcn[curg];
            for (int u = 0; u < k; u++) {
                int sh = (arr >> (3 * u)) & 7u;
                if (sh == cur) continue;
                int g = st.start[am] + sh;
                int ngc = s.gcmode == PE_GC3 ? st.gc3[g] : st.gcn[g];
                if ((dir == 1 && ngc > cgc) || (dir == -1 && ngc < cgc)) {
                    row[a] = (uint8_t)g;
                    mark_codon(s, dirty, c, a);
                    break;
                }
            }
          }
        }
        break;
    }
    case 6: {  // mutationSL (:775-969): attempts at the stem's centre codons
        int ss = s.slot[K_SL];
        if (s.sl_kind == PE_SL_LRCS) {
            // LRCS flavour (no reference counterpart): walk outward from the middle codon
            // of the repeat's second occurrence (CDS b, nucleotides q .. q+l-1), mutating
            // each codon with prob Pm, and stop at the first codon changed
            if (tid == 0) {
                const int b = sm.pobjidx[2 * ss + 1], q = sm.ppql[1], l = sm.ppql[2];
                if (l > 0 && q >= 0 && b >= 0 && b < s.m) {
                    const int a0 = q / 3, a1 = (q + l - 1) / 3, mid = (a0 + a1) / 2;
                    uint8_t *row = ids + b * s.Lp;
                    int attempt = 0;
                    for (int u = 0; u <= 2 * (a1 - a0); u++) {
                        const int a = (u & 1) ? mid - (u + 1) / 2 : mid + u / 2;
                        if (a < a0 || a > a1 || a >= L) continue;
                        const int am = aa[a], k = st.count[am];
                        const uint32_t r0 = draw(s.seed, TAG_SLMUT, gen, ridx, (uint32_t)attempt, 0);
                        const uint32_t r1 = draw(s.seed, TAG_SLMUT, gen, ridx, (uint32_t)attempt, 1);
                        attempt++;
                        if (rng_u01(r0) <= pm && k > 1) {
                            const int cur = row[a] - st.start[am];
                            int nw = (int)rng_uint(r1, (uint32_t)(k - 1));
                            if (nw == cur) nw++;
                            row[a] = (uint8_t)(st.start[am] + nw);
                            mark_codon(s, dirty, b, a);
                            break;
                        }
                    }
                }
            }
            __syncthreads();
            break;
        }
        int c = sm.pobjidx[2 * ss];
        float v = sm.pobj[ss];
        int P = sm.ppql[0], Ls = sm.ppql[2];
        int l_idx = P / 3;
        int r_idx = (P + Ls - 1) / 3;
        int mid = (r_idx + l_idx) / 2;
        int stem = r_idx - l_idx + 1;
        int half = stem / 2;
        int odd = (stem % 2) == 1;
        int npos = odd + 2 * min(half, 4096);
        uint8_t *row = ids + c * s.Lp;
        for (int u = 0; u < npos; u++) {
            int a;
            if (odd && u == 0) {
                a = mid;
            } else {
                int v2 = u - odd;
                a = (v2 & 1) ? (mid + 1 + (v2 >> 1)) : ((odd ? mid - 1 : mid) - (v2 >> 1));
            }
            if (a < 0 || a >= L) break;
            if (tid == 0) {
                int am = aa[a];
                int k = st.count[am];
                uint32_t r0 = draw(s.seed, TAG_SLMUT, gen, ridx, (uint32_t)u, 0);
                uint32_t r1 = draw(s.seed, TAG_SLMUT, gen, ridx, (uint32_t)u, 1);
                sm.sl_mut = 0;
                if (rng_u01(r0) <= pm && k > 1) {
                    int old = row[a];
                    int cur = old - st.start[am];
                    int nw = (int)rng_uint(r1, (uint32_t)(k - 1));
                    if (nw == cur) nw++;
                    row[a] = (uint8_t)(st.start[am] + nw);
                    sm.sl_old = old;
                    sm.sl_mut = 1;
                }
            }
            __syncthreads();
            bool full = cta_full_hairpin(s, st, row, tid, nth);
            float thr = full ? 1.0f : 0.0f;
            if (s.K > 0 && v > thr) {  // keep the change
                if (tid == 0 && sm.sl_mut) mark_codon(s, dirty, c, a);
                break;
            }
            if (tid == 0 && sm.sl_mut) row[a] = (uint8_t)sm.sl_old;
            __syncthreads();
        }
        break;
    }
    default:
        break;
    }
}

// The operator of a child (src/main.cu:172-211): uniform over the seven, or over the
// five kept with four objectives.
__device__ __forceinline__ int operator_of(const Shape &s, uint32_t gen, uint32_t ridx)
{
    const uint32_t r = draw(s.seed, TAG_OP, gen, ridx, 0, 0);
    if (s.objset == PE_OBJ_REF6) return (int)rng_uint(r, 7);
    const int k = (int)rng_uint(r, 5);  // 0, 1, 4, 5, 6
    return k < 2 ? k : k + 2;
}

// The children 0 .. n-1 of generation gen in the order their CTAs should start:
// by operator, the ones that take longest first (random, HD, GC, CBP, HSC, CAI, stem).
// Any order gives the same results (each CTA writes only its own child); this one
// leaves the short CTAs for the last wave.  One CTA; the order within an operator
// is arbitrary.
__device__ void order_children(const Shape &s, uint32_t gen, int n, int32_t *out, int tid, int nth)
{
    __shared__ int cnt[8], cur[8];
    const int lane = tid & 31;
    const int cls_of_op[7] = {0, 5, 3, 4, 1, 2, 6};
    if (tid < 8) cnt[tid] = 0;
    __syncthreads();
    for (int base = 0; base < n; base += nth) {
        const int c = base + tid;
        const int cls = c < n ? cls_of_op[operator_of(s, gen, (uint32_t)c)] : -1;
        for (int k = 0; k < 7; k++) {
            const unsigned b = __ballot_sync(0xffffffffu, cls == k);
            if (lane == 0 && b) atomicAdd(&cnt[k], __popc(b));
        }
    }
    __syncthreads();
    if (tid == 0) {
        int run = 0;
        for (int k = 0; k < 7; k++) {
            cur[k] = run;
            run += cnt[k];
        }
    }
    __syncthreads();
    for (int base = 0; base < n; base += nth) {
        const int c = base + tid;
        const int cls = c < n ? cls_of_op[operator_of(s, gen, (uint32_t)c)] : -1;
        for (int k = 0; k < 7; k++) {
            const unsigned b = __ballot_sync(0xffffffffu, cls == k);
            int pos = 0;
            if (lane == 0 && b) pos = atomicAdd(&cur[k], __popc(b));
            pos = __shfl_sync(0xffffffffu, pos, 0);
            if (cls == k) out[pos + __popc(b & ((1u << lane) - 1u))] = c;
        }
    }
}

// ---------------------------------------------------------------------------
// k_variation: one CTA (kVarThreads) per solution
// ---------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(kVarThreads, 4) k_variation(Shape s, const DevTables *__restrict__ gt,
                                                           const int8_t *__restrict__ aa_g, PopBuf src, PopBuf dst,
                                                           const int32_t *__restrict__ parent_of,
                                                           const int32_t *__restrict__ rng_idx, int copy_base,
                                                           int child_base, const uint32_t *__restrict__ d_gen,
                                                           int32_t *ops, int32_t *surv, int32_t *order,
                                                           int32_t *q_items, int32_t *q_count, int32_t *q_counter)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    VarSmem &sm = *reinterpret_cast<VarSmem *>(smem_raw);
    uint8_t *ids = smem_raw + ((sizeof(VarSmem) + 15) & ~size_t(15));
    uint2 *planes = reinterpret_cast<uint2 *>(ids + (size_t)s.m * s.Lp);
    int8_t *aa = reinterpret_cast<int8_t *>(planes + (size_t)s.m * s.Wp);
    // MODE_MUTATE: plane words the mutation touched (bit c * Wp + w)
    uint32_t *dirty = reinterpret_cast<uint32_t *>(aa + ((s.L + 15) & ~15));
    // the per-CDS (per-pair) sums of the light objectives, aux layout; then the
    // evaluation's task list (4m + m(m-1)/2 entries)
    int32_t *ax = reinterpret_cast<int32_t *>(dirty + (s.m * s.Wp + 31) / 32);
    int32_t *tl = ax + s.naux;

    const int tid = threadIdx.x, nth = blockDim.x;
    // MODE_MUTATE with an order: CTA b makes child order[gen parity][b] (heaviest
    // operators first, so the CTAs of the last wave are the short ones); CTA 0, which
    // starts first, writes the next generation's order
    const uint32_t gen0 = MODE == MODE_MUTATE ? *d_gen : 0u;
    const int i = MODE == MODE_MUTATE && order ? order[(gen0 & 1u) * gridDim.x + blockIdx.x] : (int)blockIdx.x;
    if (MODE == MODE_MUTATE && order && blockIdx.x == 0)
        order_children(s, gen0 + 1u, (int)gridDim.x, order + ((gen0 + 1u) & 1u) * gridDim.x, tid, nth);
    const size_t sol_bytes = (size_t)s.m * s.Lp;
    const size_t sol_words = (size_t)s.m * s.Wp;

    load_tab(sm.tab, gt, tid, nth);
    for (int a = tid; a < s.L; a += nth) aa[a] = aa_g[a];

    uint32_t gen = 0, ridx = (uint32_t)i;
    int out_slot = i;
    if (MODE == MODE_INIT) {
        __syncthreads();
        for (int pos = tid; pos < s.m * s.L; pos += nth) {
            int c = pos / s.L, a = pos - c * s.L;
            int am = aa[a];
            int k = sm.tab.count[am];
            int choice = (i == 0) ? k - 1 : (int)rng_uint(draw(s.seed, TAG_INIT, 0, (uint32_t)i, (uint32_t)pos, 0), k);
            ids[c * s.Lp + a] = (uint8_t)(sm.tab.start[am] + choice);
        }
        for (int c = 0; c < s.m; c++)
            for (int a = s.L + tid; a < s.Lp; a += nth) ids[c * s.Lp + a] = 0;
        if (tid == 0 && surv) surv[i] = i;
        if (dst.cds)
            for (int c = tid; c < s.nres; c += nth) dst.cds[(size_t)i * s.nres + c] = make_int2(-1, 0);
    } else if (MODE == MODE_EVAL) {
        const uint4 *g = reinterpret_cast<const uint4 *>(dst.ids + (size_t)i * sol_bytes);
        uint4 *d = reinterpret_cast<uint4 *>(ids);
        for (size_t e = tid; e < sol_bytes / 16; e += nth) d[e] = g[e];
        if (dst.cds)
            for (int c = tid; c < s.nres; c += nth) dst.cds[(size_t)i * s.nres + c] = make_int2(-1, 0);
    } else {  // MODE_MUTATE
        gen = gen0;
        ridx = rng_idx ? (uint32_t)rng_idx[i] : (uint32_t)i;
        int par = parent_of[i];
        // the parent's codon ids and planes into shared memory (the child's planes differ
        // only in the words its mutation touches) and, when the parent survives, into
        // its slot of the next population.  Each thread issues up to four 16-byte loads
        // before their stores, so the loads of a pass are in flight together.
        {
            const uint4 *g = reinterpret_cast<const uint4 *>(src.ids + (size_t)par * sol_bytes);
            const uint4 *ps = reinterpret_cast<const uint4 *>(src.planes + (size_t)par * sol_words);
            uint4 *d = reinterpret_cast<uint4 *>(ids);
            uint4 *pd = reinterpret_cast<uint4 *>(planes);
            const size_t dslot = (size_t)(copy_base + i);
            uint4 *gd = copy_base >= 0 ? reinterpret_cast<uint4 *>(dst.ids + dslot * sol_bytes) : nullptr;
            uint4 *pdd = copy_base >= 0 ? reinterpret_cast<uint4 *>(dst.planes + dslot * sol_words) : nullptr;
            const int nid = (int)(sol_bytes / 16), ntot = nid + (int)(sol_words / 2);
            for (int e0 = tid; e0 < ntot; e0 += 4 * nth) {
                uint4 v[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int e = e0 + u * nth;
                    if (e < ntot) v[u] = e < nid ? g[e] : ps[e - nid];
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int e = e0 + u * nth;
                    if (e < nid) {
                        d[e] = v[u];
                        if (gd) gd[e] = v[u];
                    } else if (e < ntot) {
                        pd[e - nid] = v[u];
                        if (pdd) pdd[e - nid] = v[u];
                    }
                }
            }
            for (int e = tid; e < (int)((sol_words + 31) / 32); e += nth) dirty[e] = 0u;
        }
        if (tid < s.M) sm.pobj[tid] = src.obj[(size_t)par * s.M + tid];
        if (tid < 2 * s.M) sm.pobjidx[tid] = src.objidx[(size_t)par * 2 * s.M + tid];
        if (tid < 3) sm.ppql[tid] = src.pql[(size_t)par * 3 + tid];
        if (copy_base >= 0) {
            // the surviving parent keeps its slot: its objectives and per-CDS results too
            const size_t dslot = (size_t)(copy_base + i);
            if (tid < s.M) dst.obj[dslot * s.M + tid] = src.obj[(size_t)par * s.M + tid];
            if (tid < 2 * s.M) dst.objidx[dslot * 2 * s.M + tid] = src.objidx[(size_t)par * 2 * s.M + tid];
            if (tid < 3) dst.pql[dslot * 3 + tid] = src.pql[(size_t)par * 3 + tid];
            if (dst.aux)
                for (int e = tid; e < s.naux; e += nth) dst.aux[dslot * s.naux + e] = src.aux[(size_t)par * s.naux + e];
            if (dst.cds)
                for (int c = tid; c < s.nres; c += nth)
                    dst.cds[dslot * s.nres + c] = src.cds ? src.cds[(size_t)par * s.nres + c] : make_int2(-1, 0);
        }
        out_slot = child_base + i;
        if (tid == 0) {
            const int op = operator_of(s, gen, ridx);
            sm.op = op;
            if (ops) ops[i] = op;
        }
        __syncthreads();
        mutate_solution(s, gt, sm, aa, ids, dirty, gen, ridx, tid, nth);
    }
    __syncthreads();
    pack_planes(s, sm.tab, ids, planes, tid, nth, MODE == MODE_MUTATE ? dirty : nullptr);
    // CDSs the mutation changed (bit c); every CDS outside MODE_MUTATE
    unsigned long long chmask = s.m == 64 ? ~0ull : (1ull << s.m) - 1ull;
    if (MODE == MODE_MUTATE && (dst.cds || src.aux)) {
        if (tid == 0) sm.changed = 0ull;
        __syncthreads();
        for (int c = tid; c < s.m; c += nth) {
            bool changed = false;
            const int b0 = c * s.Wp, b1 = b0 + s.Wp;  // this CDS's bits [b0, b1)
            for (int wd = b0 >> 5; wd <= (b1 - 1) >> 5 && !changed; wd++) {
                const int lo = max(b0, 32 * wd) - 32 * wd, hi = min(b1, 32 * wd + 32) - 32 * wd;
                const uint32_t mask = hi - lo == 32 ? ~0u : ((1u << (hi - lo)) - 1u) << lo;
                changed = (dirty[wd] & mask) != 0u;
            }
            if (changed) atomicOr(&sm.changed, 1ull << c);
        }
        __syncthreads();
        const unsigned long long ch = sm.changed;
        if (src.aux) chmask = ch;
        if (dst.cds) {
            // a CDS none of whose plane words changed keeps its parent's hairpin result;
            // an LRCS pair of two such CDSs keeps its parent's pair result
            const int par = parent_of[i];
            for (int c = tid; c < s.nres; c += nth) {
                bool changed;
                if (src.cds == nullptr) {
                    changed = true;
                } else if (s.sl_kind == PE_SL_LRCS) {
                    int a, b;
                    lrcs_pair_of(s.m, c, a, b);
                    changed = ((ch >> a) | (ch >> b)) & 1ull;
                } else {
                    changed = (ch >> c) & 1ull;
                }
                dst.cds[(size_t)out_slot * s.nres + c] = changed ? make_int2(-1, 0) : src.cds[(size_t)par * s.nres + c];
            }
        }
        if (q_counter) {
            // The results this child's mutation invalidated are the only ones the scan
            // will count: the solution's counter starts at the results kept, so the
            // combine runs after the last scanned one and a carried result takes no count.
            // A child with none keeps its parent's string objective, as the combine of the
            // parent's results gives.  With a queue (batches) the invalidated results are
            // also appended to it, in result order.
            const int par = parent_of[i], nres = s.nres, lane = tid & 31;
            // results invalidated: the changed CDSs (hairpin), or the CDS pairs with a
            // changed member (LRCS: all pairs but those of the u unchanged CDSs)
            const int nch = __popcll(ch), u = s.m - nch;
            const int nq = s.sl_kind == PE_SL_LRCS ? nres - u * (u + 1) / 2 : nch;
            if (q_count && tid < 32) {
                auto invalid = [&](int r) {
                    if (r >= nres) return false;
                    if (s.sl_kind == PE_SL_LRCS) {
                        int a, b;
                        lrcs_pair_of(s.m, r, a, b);
                        return (((ch >> a) | (ch >> b)) & 1ull) != 0ull;
                    }
                    return ((ch >> r) & 1ull) != 0ull;
                };
                int qb = 0;
                if (lane == 0 && nq > 0) qb = atomicAdd(q_count, nq);
                qb = __shfl_sync(0xffffffffu, qb, 0);
                int run = 0;
                for (int rb = 0; rb < nres; rb += 32) {
                    const bool on = invalid(rb + lane);
                    const unsigned bal = __ballot_sync(0xffffffffu, on);
                    if (on) q_items[qb + run + __popc(bal & ((1u << lane) - 1u))] = i * nres + rb + lane;
                    run += __popc(bal);
                }
            }
            if (tid == 0) {
                // (with nothing invalidated the counter stays 0, ready for a full scan later)
                if (nq > 0) q_counter[i] = nres - nq;
                if (nq == 0) {
                    const int sl = s.slot[K_SL];
                    dst.obj[(size_t)out_slot * s.M + sl] = src.obj[(size_t)par * s.M + sl];
                    dst.objidx[(size_t)out_slot * 2 * s.M + 2 * sl] = src.objidx[(size_t)par * 2 * s.M + 2 * sl];
                    dst.objidx[(size_t)out_slot * 2 * s.M + 2 * sl + 1] = src.objidx[(size_t)par * 2 * s.M + 2 * sl + 1];
                    for (int k = 0; k < 3; k++) dst.pql[(size_t)out_slot * 3 + k] = src.pql[(size_t)par * 3 + k];
                }
            }
        }
    }
    __syncthreads();
    // write the (new) solution
    if (MODE != MODE_EVAL) {
        uint4 *gd = reinterpret_cast<uint4 *>(dst.ids + (size_t)out_slot * sol_bytes);
        const uint4 *d = reinterpret_cast<const uint4 *>(ids);
        for (size_t e = tid; e < sol_bytes / 16; e += nth) gd[e] = d[e];
    }
    {
        uint4 *pd = reinterpret_cast<uint4 *>(dst.planes + (size_t)out_slot * sol_words);
        const uint4 *ps = reinterpret_cast<const uint4 *>(planes);
        for (size_t e = tid; e < sol_words / 2; e += nth) pd[e] = ps[e];
    }
    const int32_t *pax = MODE == MODE_MUTATE && src.aux ? src.aux + (size_t)parent_of[i] * s.naux : nullptr;
    int32_t *cax = dst.aux ? dst.aux + (size_t)out_slot * s.naux : nullptr;
    light_eval(s, gt, sm.tab, ids, planes, ax, tl, &sm.ntask, chmask, pax, cax, dst.obj + (size_t)out_slot * s.M,
               dst.objidx + (size_t)out_slot * 2 * s.M, tid, nth);
}

size_t var_smem_bytes(const Shape &s)
{
    return ((sizeof(VarSmem) + 15) & ~size_t(15)) + (size_t)s.m * s.Lp + (size_t)s.m * s.Wp * sizeof(uint2) +
           (size_t)((s.L + 15) & ~15) + (size_t)((s.m * s.Wp + 31) / 32) * sizeof(uint32_t) +
           (size_t)(s.naux + 4 * s.m + s.m * (s.m - 1) / 2) * sizeof(int32_t);
}

cudaError_t raise_smem_limit(const void *func, size_t bytes)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t &cur = limit[{dev, func}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

template <int MODE> static cudaError_t set_var_attr(size_t smem)
{
    return raise_smem_limit((const void *)k_variation<MODE>, smem);
}

cudaError_t launch_init(const Shape &s, const DevTables *tab, const int8_t *aa, PopBuf dst, int32_t *surv,
                        cudaStream_t st)
{
    size_t smem = var_smem_bytes(s);
    cudaError_t e = set_var_attr<MODE_INIT>(smem);
    if (e != cudaSuccess) return e;
    k_variation<MODE_INIT><<<s.N, kVarThreads, smem, st>>>(s, tab, aa, dst, dst, nullptr, nullptr, -1, 0, nullptr,
                                                            nullptr, surv, nullptr, nullptr, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_light_eval(const Shape &s, const DevTables *tab, const int8_t *aa, PopBuf buf, int base, int count,
                              cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    size_t smem = var_smem_bytes(s);
    cudaError_t e = set_var_attr<MODE_EVAL>(smem);
    if (e != cudaSuccess) return e;
    PopBuf b = buf;
    size_t sol_bytes = (size_t)s.m * s.Lp, sol_words = (size_t)s.m * s.Wp;
    b.ids += (size_t)base * sol_bytes;
    b.planes += (size_t)base * sol_words;
    b.obj += (size_t)base * s.M;
    b.objidx += (size_t)base * 2 * s.M;
    b.pql += (size_t)base * 3;
    k_variation<MODE_EVAL><<<count, kVarThreads, smem, st>>>(s, tab, aa, b, b, nullptr, nullptr, -1, 0, nullptr,
                                                              nullptr, nullptr, nullptr, nullptr, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_mutate(const Shape &s, const DevTables *tab, const int8_t *aa, PopBuf src, PopBuf dst,
                          const int32_t *parent_of, const int32_t *rng_idx, int count, int copy_base, int child_base,
                          const uint32_t *d_gen, int32_t *ops, int32_t *order, cudaStream_t st, int32_t *q_items,
                          int32_t *q_count, int32_t *q_counter)
{
    if (count <= 0) return cudaSuccess;
    // a queued scan needs the parents' results to carry the unchanged ones
    if ((q_count || q_counter) && (src.cds == nullptr || dst.cds == nullptr)) return cudaErrorInvalidValue;
    if (q_count && !q_counter) return cudaErrorInvalidValue;
    // a child reuses its parent's per-CDS sums only when both buffers carry them
    if ((src.aux == nullptr) != (dst.aux == nullptr)) return cudaErrorInvalidValue;
    size_t smem = var_smem_bytes(s);
    cudaError_t e = set_var_attr<MODE_MUTATE>(smem);
    if (e != cudaSuccess) return e;
    k_variation<MODE_MUTATE><<<count, kVarThreads, smem, st>>>(s, tab, aa, src, dst, parent_of, rng_idx, copy_base,
                                                                child_base, d_gen, ops, nullptr, order, q_items,
                                                                q_count, q_counter);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// k_sl: hairpin-stem scan on bit planes
// ---------------------------------------------------------------------------
//
// For one CDS s (n nucleotides) with reverse complement t (t[i] = comp(s[n-1-i]))
// the cell (r, c) of the reference's anti-diagonal sweep pairs iff
// s[r] == t[r + delta] with delta = n-1-(r+c).  The counted cells of
// anti-diagonal d = r+c are r in [max(0, d-n+1), floor((d-5)/2)] (upper
// triangle, loop of >= 4 nucleotides); their longest run of pairing cells is
// that anti-diagonal's stem length, and the lower triangle never exceeds it
// (include/utils.cuh:743-774).
//
// Two passes.  The band scan (below) finds every run of >= 8 pairing cells and
// measures those exactly; for random-like sequences of a few hundred
// nucleotides or more the longest stem is >= 8 and that pass is the whole scan.
// Otherwise the exact word scan runs: each lane owns one shift delta and walks
// its cells 32 at a time,
//     match word = ~((S.lo ^ T.lo) | (S.hi ^ T.hi)),
// with runs carried across words by ffs/clz and the longest run inside each
// word counted; T is then kept as 32 pre-shifted copies, transposed so that the
// 32 lanes of a warp read 32 consecutive 8-byte words.

__device__ __forceinline__ uint32_t fshr(uint32_t lo, uint32_t hi, int sh) { return __funnelshift_r(lo, hi, sh); }

// The same scan serves the longest repeated/common substring (LRCS flavour):
// for CDSs a and b, T is b's own planes (not a reverse complement), so a cell
// (r, delta) matches iff s_a[r] == s_b[r + delta] and the runs along a fixed
// delta are common substrings.  Its diagonals are every delta in (-n, n) for
// a != b and delta >= 1 for a == b (a substring at two different starts), each
// over all rows r in [max(0, -delta), min(n-1, n-1-delta)].  FL selects the
// flavour at compile time: 0 hairpin, 1 LRCS.
struct SlGeo {
    int n;
    int dlo, dhi;  // diagonals (shifts delta) scanned
    int D0;        // first band's shift (a multiple of 32, <= dlo)
    int ng;        // band groups
};

template <int FL> __host__ __device__ __forceinline__ SlGeo sl_geo(int n, bool self_pair)
{
    SlGeo g;
    g.n = n;
    if (FL == 0) {
        g.dlo = -(n - 6);
        g.dhi = n - 6;
    } else {
        g.dlo = self_pair ? 1 : -(n - 1);
        g.dhi = n - 1;
    }
    g.D0 = g.dlo >= 0 ? (g.dlo & ~31) : -((-g.dlo + 31) & ~31);
    const int nb = g.dhi >= g.dlo ? (g.dhi - g.D0) / 32 + 1 : 0;
    g.ng = (nb + 2) / 3;
    return g;
}

// counted rows of diagonal delta
template <int FL> __device__ __forceinline__ void sl_diag_rows(int n, int delta, int &r_lo, int &r_hi)
{
    r_lo = max(0, -delta);
    r_hi = FL == 0 ? ((n - 6 - delta) >> 1) : min(n - 1, n - 1 - delta);
}

// order key of a diagonal among equally long runs (smaller wins): the hairpin
// keeps the smallest anti-diagonal d = n-1-delta, LRCS the smallest delta
template <int FL> __device__ __forceinline__ int sl_key(int n, int delta) { return FL == 0 ? n - 1 - delta : delta + n; }

template <bool MASKED>
__device__ __forceinline__ void sl_word(uint2 sv, uint2 tv, int k, int r_lo, int r_hi, int &cur, int &dbest)
{
    uint32_t m = ~((sv.x ^ tv.x) | (sv.y ^ tv.y));
    if (MASKED) {
        int lo_b = r_lo - 32 * k, hi_b = r_hi - 32 * k;
        uint32_t mk = (lo_b > 31 || hi_b < 0 || lo_b > hi_b)
                          ? 0u
                          : ((0xffffffffu << max(lo_b, 0)) & (0xffffffffu >> (31 - min(hi_b, 31))));
        m &= mk;
    }
    if (m == 0xffffffffu) {
        cur += 32;  // the run goes on through the whole word
    } else {
        const uint32_t z = ~m;
        dbest = max(dbest, cur + __ffs(z) - 1);  // run carried in + ones at the low end
        cur = __clz(z);                          // ones at the high end carry out
        uint32_t y = m;                          // longest run inside the word
        int len = 0;
        while (y) {
            y &= y >> 1;
            len++;
        }
        dbest = max(dbest, len);
    }
}

template <int FL>
__device__ void sl_scan(const uint2 *__restrict__ S, const uint32_t *__restrict__ Tlo, const uint32_t *__restrict__ Thi,
                        const SlGeo &geo, int *next_chunk, int lane, int &best, int &bestd)
{
    const int n = geo.n;
    if (geo.dhi < geo.dlo) return;
    const int ndiag = geo.dhi - geo.dlo + 1;
    const int nchunks = (ndiag + 31) >> 5;
    const int c0 = nchunks >> 1;
    for (;;) {
        // warps take chunks of 32 anti-diagonals from the centre outwards (longest
        // first), so the CTA's warps finish together
        int t = 0;
        if (lane == 0) t = atomicAdd(next_chunk, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= nchunks) break;
        const int ch = (t & 1) ? c0 - 1 - (t >> 1) : c0 + (t >> 1);
        const int delta = geo.dlo + 32 * ch + lane;
        const bool valid = delta <= geo.dhi;
        int r_lo = 1, r_hi = 0;
        if (valid) sl_diag_rows<FL>(n, delta, r_lo, r_hi);
        const int klo = r_lo >> 5, khi = r_hi >> 5;
        const int kmin = warp_min_i(valid ? klo : 0x7fffffff);
        const int kmax = warp_max_i(valid ? khi : -1);
        // words fully inside every valid lane's range need no mask
        const int full_lo = (r_lo + 31) >> 5, full_hi = ((r_hi + 1) >> 5) - 1;
        const bool allvalid = __all_sync(0xffffffffu, valid);
        int kf_lo = warp_max_i(full_lo), kf_hi = warp_min_i(full_hi);
        if (!allvalid) {
            kf_lo = kmax + 1;
            kf_hi = kmax;
        }
        kf_lo = max(kf_lo, kmin);
        kf_hi = min(kf_hi, kmax);
        // T bits [32k + delta, +31]: words row, row + 1 of T at bit offset delta mod 32
        const int row = (delta >> 5) + kSlGuardRows, sh = delta & 31;
        auto tw = [&](int k) {
            return make_uint2(fshr(Tlo[row + k], Tlo[row + k + 1], sh), fshr(Thi[row + k], Thi[row + k + 1], sh));
        };
        int cur = 0, dbest = 0;
        int k = kmin;
        for (; k < kf_lo; k++) sl_word<true>(S[k], tw(k), k, r_lo, r_hi, cur, dbest);
#pragma unroll 4
        for (; k <= kf_hi; k++) sl_word<false>(S[k], tw(k), k, r_lo, r_hi, cur, dbest);
        for (; k <= kmax; k++) sl_word<true>(S[k], tw(k), k, r_lo, r_hi, cur, dbest);
        dbest = max(dbest, cur);
        if (valid) {
            int d = sl_key<FL>(n, delta);
            if (dbest > best) {
                best = dbest;
                bestd = d;
            } else if (dbest == best && d < bestd) {
                bestd = d;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Band scan: the first pass, which finds every run of >= 8 pairing cells.
//
// Shifts are grouped in bands of 32 (delta0 .. delta0+31, delta0 a multiple of
// 32).  A lane takes one item = (group of kBandGroup adjacent bands, segment of
// 32 consecutive rows r = 32s..32s+31).  Row r's match word over a band (bit j:
// s[r] pairs with t[r + delta0 + j]) is a window of T's equality plane for the
// nucleotide s[r]:
//     m_r = E_{s[r]} bits [r + delta0, r + delta0 + 32),
// at bit offset r mod 32, a constant of the unrolled step; one 16-byte load of
// four consecutive plane words gives the windows of all bands of the group.
// The rows are cut into blocks: rows 29..31 of the previous segment, then
// 3k..3k+2 (k = 0..9) and 30..31 of the segment.  The AND of two consecutive
// blocks' match words gives the diagonals pairing on those 6 (or 5) rows: a
// window.  Window starts are never more than 3 rows apart, so a run of >= 8 rows
// always covers one window, first the one starting at the run's start or within
// 2 rows after.  Such a run is longer than its 6-row window, so it also pairs on
// the row just before or just after the window: a diagonal is marked when a
// 6-row window and one of its two neighbouring rows pair (the row before the
// first window, in the previous segment, is not needed: the runs this segment
// owns that cover that window reach the row after it), and on the last, 5-row
// window alone.  The marks catch every run of 8 or more; the neighbour test
// drops the exact 6-row runs, two thirds of the shorter runs the windows alone
// would mark.  Per band and row that is one funnel shift and 4/3 of a 3-input
// logic op.  Marked diagonals are rare: the lane ORs the marks into one mask
// per band and queues (mask, band, segment); each warp measures its queued
// runs exactly, 32 at a time, one per lane (sl_band_entry), which keeps the
// runs that start at rows
// 32s-4 .. 32s+27, the ones whose first covering window lies in segment s, so
// each run is measured once.
//
// Cells outside a diagonal's counted range: rows below it read T outside
// [0, n) (zero planes) or a row outside [0, n) (the zero plane 4), so they
// never match; rows past its top end may match, which only extends a run
// beyond the range, and sl_band_entry clips every run to the range.  So every
// counted run of length >= 8 is measured exactly once, and runs that are
// shorter inside the range never win against it.
constexpr int kBandGroup = 3;            // bands per item (one 4-word load)
constexpr int kEqGuard = kBandGroup + 3; // guard words on each side of the equality planes
constexpr int kSegPitch = 17;            // row-entry table: 16 words (two rows each) per segment + 1 (bank spread)
constexpr int kBandQueue = 64;

__host__ __device__ __forceinline__ int sl_plane_stride(int W) { return (W + 2 * kEqGuard + 4 + 31) & ~31; }
__host__ __device__ __forceinline__ int sl_band_base(int n) { return -(((n - 6) + 31) & ~31); }
__host__ __device__ __forceinline__ int sl_num_bands(int n) { return n - 6 >= 0 ? ((n - 6) - sl_band_base(n)) / 32 + 1 : 0; }
__host__ __device__ __forceinline__ int sl_num_groups(int n) { return (sl_num_bands(n) + kBandGroup - 1) / kBandGroup; }

// Segments of the rows a group of bands starting at shift d0 covers (rows of
// the counted triangle: r >= -delta, 2r + delta <= n - 6): from the lowest
// first row of its bands (the last band) to the highest last row (the first).
__host__ __device__ __forceinline__ void sl_group_segments(int n, int d0, int &s_lo, int &s_hi)
{
    s_lo = max(0, -(d0 + 32 * (kBandGroup - 1)) - 31) >> 5;
    s_hi = ((n - 6 - d0) >> 1) >> 5;
}

// Exact measurement of the runs queued for one (band, segment): for each
// diagonal j of the mask, the rows where its run reached 8 inside segment s are
// found again from 64 rows of match bits (same cells as the band scan), and
// each run is followed to its end and clipped to the diagonal's counted range.
template <int FL>
__device__ void sl_band_entry(uint32_t mask, int d0, int s, const SlGeo &geo, const uint2 *__restrict__ S,
                              const uint32_t *__restrict__ Tlo, const uint32_t *__restrict__ Thi, int &best, int &bestd)
{
    const int n = geo.n;
    const int R0 = 32 * (s - 1);
    const uint2 SA = s >= 1 ? S[s - 1] : make_uint2(0u, 0u), SB = S[s];
    while (mask) {
        const int j = __ffs(mask) - 1;
        mask &= mask - 1;
        const int delta = d0 + j;
        if (delta < geo.dlo || delta > geo.dhi) continue;
        int r_lo_d, r_hi;
        sl_diag_rows<FL>(n, delta, r_lo_d, r_hi);
        // match bits of rows R0 .. R0+63 on this diagonal, zero where the row or
        // its T index falls outside [0, n)
        const int i0 = R0 + delta, w0 = (i0 >> 5) + kSlGuardRows, sh = i0 & 31;
        const uint32_t tlA = fshr(Tlo[w0], Tlo[w0 + 1], sh), thA = fshr(Thi[w0], Thi[w0 + 1], sh);
        const uint32_t tlB = fshr(Tlo[w0 + 1], Tlo[w0 + 2], sh), thB = fshr(Thi[w0 + 1], Thi[w0 + 2], sh);
        const uint32_t eA = ~((SA.x ^ tlA) | (SA.y ^ thA)), eB = ~((SB.x ^ tlB) | (SB.y ^ thB));
        const int lo = max(max(0, -delta), R0) - R0, hi = min(min(n, n - delta) - 1, R0 + 63) - R0;
        if (lo > hi) continue;
        const uint64_t valid = (~0ull >> (63 - hi)) & (~0ull << lo);
        const uint64_t X = (((uint64_t)eB << 32) | eA) & valid;
        uint64_t R8 = X & (X >> 1);
        R8 &= R8 >> 2;
        R8 &= R8 >> 4;
        // segment s owns the runs of >= 8 that start at rows 32s-4 .. 32s+27 (bits 28 .. 59):
        // the first window covering such a run (window starts ... 32s-5 | 32s-3, 32s, ...,
        // 32s+24, 32s+27 | 32s+29 ...) belongs to segment s.  Runs starting at bits 57 .. 59
        // reach past the 64 rows when all their bits up to 63 pair.
        const uint64_t starts = X & ~(X << 1) & (((1ull << 32) - 1) << 28);
        uint64_t open_end = 0;
#pragma unroll
        for (int b = 57; b <= 59; b++)
            if ((X >> b) == (~0ull >> b)) open_end |= 1ull << b;
        uint64_t edges = starts & (R8 | open_end);
        while (edges) {
            const int b = __ffsll((long long)edges) - 1;
            edges &= edges - 1;
            const int a = R0 + b;  // first row of the run
            if (a > r_hi) continue;
            int e;                 // last row known to pair
            if ((R8 >> b) & 1) {
                e = a + 7;
            } else {               // a run from bit b to bit 63 at least; shorter than 8 so far
                e = R0 + 63;
            }
            while (e < r_hi) {
                const int p = e + 1, i = p + delta;
                const int ws = p >> 5, wt = (i >> 5) + kSlGuardRows;
                const uint32_t sl = fshr(S[ws].x, S[ws + 1].x, p & 31), sh2 = fshr(S[ws].y, S[ws + 1].y, p & 31);
                const uint32_t tl = fshr(Tlo[wt], Tlo[wt + 1], i & 31), th = fshr(Thi[wt], Thi[wt + 1], i & 31);
                const uint32_t mm = ~((sl ^ tl) | (sh2 ^ th));
                if (mm == 0xffffffffu) {
                    e += 32;
                    continue;
                }
                e += __ffs(~mm) - 1;
                break;
            }
            const int L = min(e, r_hi) - a + 1;
            const int d = sl_key<FL>(n, delta);
            if (L > best || (L == best && d < bestd)) {
                best = L;
                bestd = d;
            }
        }
    }
}

// read-only table loads from the shared window (free to reorder: nothing
// writes the tables during the scan)
__device__ __forceinline__ uint32_t lds_u32(uint32_t a)
{
    uint32_t v;
    asm("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ uint4 lds_v4(uint32_t a)
{
    uint4 v;
    asm("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ uint32_t word_of(const uint4 &w, int i)
{
    return i == 0 ? w.x : i == 1 ? w.y : i == 2 ? w.z : w.w;
}

// segments of the rows a group of bands starting at shift d0 covers
template <int FL> __device__ __forceinline__ void sl_group_rows(int n, int d0, int &s_lo, int &s_hi)
{
    if (FL == 0) {
        sl_group_segments(n, d0, s_lo, s_hi);
    } else {
        s_lo = max(0, -(d0 + 32 * kBandGroup - 1)) >> 5;
        s_hi = min(n - 1, n - 1 - d0) >> 5;
    }
}

template <int FL>
__device__ void sl_band_scan(const uint4 *__restrict__ E4, const int *__restrict__ poffT,
                             const int *__restrict__ gstart, const SlGeo &geo, const uint2 *__restrict__ S,
                             const uint32_t *__restrict__ Tlo, const uint32_t *__restrict__ Thi,
                             int2 *__restrict__ queue, int *next_chunk, int lane, int &best, int &bestd)
{
    const int ng = geo.ng, n = geo.n;
    if (ng <= 0) return;
    const int D0 = geo.D0;
    const int nitems = gstart[ng];
    const int nchunks = (nitems + 31) >> 5;
    const unsigned lt = (1u << lane) - 1u;
    int qn = 0;  // entries in this warp's queue (warp-uniform)
    for (;;) {
        int ch = 0;
        if (lane == 0) ch = atomicAdd(next_chunk, 1);
        ch = __shfl_sync(0xffffffffu, ch, 0);
        if (ch >= nchunks) break;
        const int item = ch * 32 + lane;
        uint32_t pend[kBandGroup];
#pragma unroll
        for (int g = 0; g < kBandGroup; g++) pend[g] = 0;
        int grp = 0, s = 0;
        if (item < nitems) {
            int lo = 0, hi = ng - 1;  // group: gstart[grp] <= item < gstart[grp + 1]
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (gstart[mid] <= item) lo = mid;
                else hi = mid - 1;
            }
            grp = lo;
            const int d0 = D0 + 32 * kBandGroup * grp;
            int s_lo, s_hi;
            sl_group_rows<FL>(n, d0, s_lo, s_hi);
            s = s_lo + (item - gstart[grp]);
            // E4 entry x holds T words x-kEqGuard .. x+3-kEqGuard; row 32u + t reads entry
            // u + d0/32 + kEqGuard of the row's plane, words g, g+1 for band g, at bit offset t;
            // the row-entry table gives the entry of two rows per 32-bit word
            const uint32_t qa = (uint32_t)__cvta_generic_to_shared(E4 + (d0 / 32 + kEqGuard));
            const uint32_t pa = (uint32_t)__cvta_generic_to_shared(poffT + s * kSegPitch);
            // blocks of rows: 29..31 of segment s-1, then 3k..3k+2 (k = 0..9) and 30..31
            // of segment s; two consecutive blocks and a neighbouring row pairing on a
            // diagonal mark it
            uint32_t bprev[kBandGroup], win[kBandGroup], l1[kBandGroup], l2[kBandGroup];
            uint32_t pw = 0;  // the table word holding the current row's entry (two rows per word)
#pragma unroll
            for (int k = -1; k <= 10; k++) {
                const int r0 = k < 0 ? 29 : 3 * k, nr = k == 10 ? 2 : 3;
                uint32_t b[kBandGroup], f[kBandGroup], l[kBandGroup];
#pragma unroll
                for (int u = 0; u < nr; u++) {
                    const int t = r0 + u;
                    if (k < 0 ? (t == 29 || t == 30) : (t & 1) == 0)
                        pw = lds_u32(pa + 4 * ((k < 0 ? 0 : kSegPitch) + (t >> 1)));
                    const uint32_t pv = ((t & 1) ? (pw >> 16) : (pw & 0xffffu)) * 16u;
                    const uint4 w = lds_v4(qa + pv);
#pragma unroll
                    for (int g = 0; g < kBandGroup; g++) {
                        const uint32_t m = fshr(word_of(w, g), word_of(w, g + 1), t);
                        b[g] = u == 0 ? m : (b[g] & m);
                        if (u == 0) f[g] = m;
                        l[g] = m;
                    }
                }
                // window (k-2, k-1) closes with the first row of block k; window (k-1, k)
                // opens with the last row of block k-2 (none for k = 0); the last window
                // (rows 27..31) is kept as it is
#pragma unroll
                for (int g = 0; g < kBandGroup; g++) {
                    if (k >= 1) pend[g] |= win[g] & f[g];
                    if (k >= 0) {
                        win[g] = bprev[g] & b[g];
                        if (k == 10) pend[g] |= win[g];
                        else if (k >= 1) pend[g] |= win[g] & l2[g];
                    }
                    l2[g] = l1[g];
                    l1[g] = l[g];
                    bprev[g] = b[g];
                }
            }
        }
        if (FL == 1) {
            // LRCS: drop the diagonals below the first one scanned (delta <= 0 of a self pair)
            const int d0 = D0 + 32 * kBandGroup * grp;
#pragma unroll
            for (int g = 0; g < kBandGroup; g++) {
                const int below = geo.dlo - (d0 + 32 * g);
                if (below > 0) pend[g] &= below >= 32 ? 0u : (0xffffffffu << below);
            }
        }
        // queue the (band, segment) pairs with rising edges; measure 32 at a time
#pragma unroll
        for (int g = 0; g < kBandGroup; g++) {
            const unsigned has = __ballot_sync(0xffffffffu, pend[g] != 0);
            if (has) {
                if (pend[g]) queue[qn + __popc(has & lt)] = make_int2((int)pend[g], ((kBandGroup * grp + g) << 16) | s);
                qn += __popc(has);
                __syncwarp();
                if (qn >= 32) {
                    const int2 q = queue[lane];
                    sl_band_entry<FL>((uint32_t)q.x, D0 + 32 * (q.y >> 16), q.y & 0xffff, geo, S, Tlo, Thi, best,
                                      bestd);
                    __syncwarp();
                    if (lane < qn - 32) queue[lane] = queue[32 + lane];
                    qn -= 32;
                    __syncwarp();
                }
            }
        }
    }
    if (lane < qn) {
        const int2 q = queue[lane];
        sl_band_entry<FL>((uint32_t)q.x, D0 + 32 * (q.y >> 16), q.y & 0xffff, geo, S, Tlo, Thi, best, bestd);
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------
// Seeded scan: the first pass for CDSs short enough for a table of their words.
//
// A cell (r, delta) pairs exactly when S's nucleotide r equals T's r + delta (T is
// the reverse complement for the hairpin, the other CDS for LRCS).  With words of K
// nucleotides looked up at rows that are multiples of t = 9 - K, a counted run of
// >= 8 pairing rows st .. st+L-1 on shift delta holds, at its row e in
// [st, st + t - 1] with e a multiple of t, K pairing rows e .. e+K-1: S's K-word at
// e equals T's at e + delta.  T's n-K+1 words (every position) go into a chained
// table and S's words at rows that are multiples of t walk their chains.  An equal
// word whose shift is scanned and whose row e+K-1 is counted joins its warp's
// queue; the warp measures queued words 32 at a time, one per lane.  The run's
// start is found by walking back at most t-1 rows (the first row that does not
// pair or is not counted ends the walk); when rows e-1 .. e-t all pair, the run is
// the one found from row e-t and this word is dropped.  The run is followed 32 rows
// at a time to its end and clipped to the diagonal's counted range, as the band
// scan measures its marked runs.  Every counted run of >= 8 is measured exactly
// once, so (longest, smallest key) is the band scan's when the longest reaches 8
// (shorter ones may be measured too; a result below 8 sends the CDS to the exact
// word scan).  Each lane walks two chains at once, and the lanes of a warp walk in
// step and meet in the queue, so neither the uneven chain lengths nor the dependent
// loads of a chain split the warp for long.
//
// The hairpin uses K = 6, t = 3: a 6-word has 4096 values and indexes the table's
// heads directly (no hash, no word compare, every node an equal word; 16-bit nodes
// holding the next position).  LRCS compares CDSs that encode the same protein and
// share many short words, so it uses K = 7, t = 2 with fewer equal words: hashed
// 32-bit heads (the power of two >= n, at most 4096) and 32-bit nodes holding the
// word (high half) and the next position (low half).
//
// For random-like CDSs the chains hold about n/4096 nodes and the work is linear in
// n instead of the n^2/2 cells.  A repetitive CDS makes long chains (many equal
// words): each thread bounds the nodes and run words it visits, and when any
// thread passes its bound the CTA drops the partial result and the band scan runs.
constexpr int kSeedMaxN = 12288;  // longest CDS (nucleotides) with a seeded scan
constexpr uint32_t kSeedEnd = 0xffffu;
template <int FL> struct Seed {
    static constexpr int K = FL == 0 ? 6 : 7;  // word length
    static constexpr int step = 9 - K;         // rows between looked-up words
    static constexpr bool direct = FL == 0;    // the word indexes the heads
};

__host__ __device__ __forceinline__ int sl_seed_bits(int n, bool direct)
{
    if (direct) return 12;
    int b = 6;
    while ((1 << b) < n && b < 12) b++;
    return b;
}
__host__ __device__ __forceinline__ bool sl_seeded(const Shape &s) { return s.sl_method == 0 && s.n >= 8 && s.n <= kSeedMaxN; }
// 32-bit heads, then the nodes (16-bit next positions, or 32-bit word and next)
__host__ __device__ __forceinline__ size_t sl_seed_head_bytes(int n, bool direct)
{
    return ((size_t)1 << sl_seed_bits(n, direct)) * 4;
}
__host__ __device__ __forceinline__ size_t sl_seed_bytes(int n, bool direct)
{
    return sl_seed_head_bytes(n, direct) + (((size_t)n * (direct ? 2 : 4) + 15) & ~size_t(15));
}

// The K-nucleotide word from bit sh of (w0, w1) of both planes: for the direct table
// its 12-bit index (plane-0 bits low); else the 7-bit plane bytes twice (plane 0 in
// bytes 0 and 2, plane 1 in bytes 1 and 3), which the hash and the node compare use.
template <int FL>
__device__ __forceinline__ uint32_t seed_word(uint32_t lo0, uint32_t lo1, uint32_t hi0, uint32_t hi1, int sh)
{
    if (Seed<FL>::direct) return (fshr(lo0, lo1, sh) & 63u) | ((fshr(hi0, hi1, sh) & 63u) << 6);
    return __byte_perm(fshr(lo0, lo1, sh), fshr(hi0, hi1, sh), 0x4040) & 0x7f7f7f7fu;
}
template <int FL> __device__ __forceinline__ uint32_t seed_bucket(uint32_t w, int hb)
{
    return Seed<FL>::direct ? w : (w * 0x9E3779B1u) >> (32 - hb);
}

// row p pairs on shift delta (p and p + delta inside [0, n))
__device__ __forceinline__ bool seed_pairs(const uint2 *__restrict__ S, const uint32_t *__restrict__ Tlo,
                                           const uint32_t *__restrict__ Thi, int p, int i)
{
    const int G = kSlGuardRows;
    const uint32_t tl = Tlo[(i >> 5) + G] >> (i & 31), th = Thi[(i >> 5) + G] >> (i & 31);
    const uint2 sp = S[p >> 5];
    return ((((sp.x >> (p & 31)) ^ tl) | ((sp.y >> (p & 31)) ^ th)) & 1u) == 0u;
}

// Measures the queued equal word q = e | i << 16 (rows e .. e+K-1 pair on delta = i - e,
// e+K-1 is counted): the run it belongs to, when this word is the one that owns it,
// against (best, bestd).  Adds the run words it read to work.
template <int FL>
__device__ __forceinline__ void seed_measure(uint32_t q, const SlGeo &geo, const uint2 *__restrict__ S,
                                             const uint32_t *__restrict__ Tlo, const uint32_t *__restrict__ Thi,
                                             int &work, int &best, int &bestd)
{
    constexpr int t = Seed<FL>::step, K = Seed<FL>::K;
    const int n = geo.n, G = kSlGuardRows;
    const int e = (int)(q & 0xffffu), j = (int)(q >> 16), delta = j - e;
    int r_lo, r_hi;
    sl_diag_rows<FL>(n, delta, r_lo, r_hi);
    int st = e, last = e + K - 1;  // first row of the run; last row known to pair
    if (e >= t && j >= t) {
        // one window of 32 rows from e-t: bit k pairs row e-t+k (rows below r_lo cleared);
        // the ones below bit t walk the run back, the first zero from bit t+K ends it
        const int p0 = e - t, i0 = j - t, ws = p0 >> 5, wt = (i0 >> 5) + G;
        const uint32_t sl = fshr(S[ws].x, S[ws + 1].x, p0 & 31), sh2 = fshr(S[ws].y, S[ws + 1].y, p0 & 31);
        const uint32_t tl = fshr(Tlo[wt], Tlo[wt + 1], i0 & 31), th = fshr(Thi[wt], Thi[wt + 1], i0 & 31);
        uint32_t m = ~((sl ^ tl) | (sh2 ^ th));
        if (r_lo > p0) m &= 0xffffffffu << (r_lo - p0);  // r_lo - p0 <= t
        const int back = __clz(~(m << (32 - t)));        // pairing rows e-1, e-2, ... (at most t)
        if (back >= t) return;                           // rows e-t .. e pair: the word at e-t owns the run
        st = e - back;
        const uint32_t ahead = ~(m >> (t + K));          // zeros of rows e+K .. e-t+31 (ones above them)
        const int runs = __ffs(ahead) - 1;               // pairing rows from e+K on
        last = e + K - 1 + runs;
        if (runs < 32 - t - K) {                         // the run ends inside the window
            if (st + 7 > r_hi) return;
            const int L = min(last, r_hi) - st + 1, d = sl_key<FL>(n, delta);
            if (L > best || (L == best && d < bestd)) {
                best = L;
                bestd = d;
            }
            return;
        }
    } else {
        while (st > e - t && st - 1 >= r_lo && seed_pairs(S, Tlo, Thi, st - 1, st - 1 + delta)) st--;
        if (st == e - t) return;  // rows e-t .. e pair: the word at e-t owns the run
    }
    if (st + 7 > r_hi) return;  // fewer than 8 counted rows from st
    while (last < r_hi) {
        work++;
        const int p = last + 1, i = p + delta;
        const int ws = p >> 5, wt = (i >> 5) + G;
        const uint32_t sl = fshr(S[ws].x, S[ws + 1].x, p & 31), sh2 = fshr(S[ws].y, S[ws + 1].y, p & 31);
        const uint32_t tl = fshr(Tlo[wt], Tlo[wt + 1], i & 31), th = fshr(Thi[wt], Thi[wt + 1], i & 31);
        const uint32_t mm = ~((sl ^ tl) | (sh2 ^ th));
        if (mm != 0xffffffffu) {
            last += __ffs(~mm) - 1;
            break;
        }
        last += 32;
    }
    const int L = min(last, r_hi) - st + 1, d = sl_key<FL>(n, delta);
    if (L > best || (L == best && d < bestd)) {
        best = L;
        bestd = d;
    }
}

// Returns false (CTA-uniform) when some thread passed its bound; (best, bestd) then
// hold a partial result that the caller discards.  table: the heads, then the nodes;
// q: this warp's queue, 64 words.
template <int FL>
__device__ bool sl_seed_scan(const SlGeo &geo, const uint2 *__restrict__ S, const uint32_t *__restrict__ Tlo,
                             const uint32_t *__restrict__ Thi, unsigned char *table, uint32_t *q, int tid, int nth,
                             int &best, int &bestd)
{
    constexpr int K = Seed<FL>::K, t = Seed<FL>::step;
    constexpr bool direct = Seed<FL>::direct;
    const int n = geo.n, G = kSlGuardRows, lane = tid & 31;
    const int hb = sl_seed_bits(n, direct), npos = n - K + 1;  // word starts 0 .. n-K
    uint32_t *heads = reinterpret_cast<uint32_t *>(table);
    unsigned short *next16 = reinterpret_cast<unsigned short *>(table + sl_seed_head_bytes(n, direct));
    uint32_t *node32 = reinterpret_cast<uint32_t *>(table + sl_seed_head_bytes(n, direct));
    uint4 *h4 = reinterpret_cast<uint4 *>(heads);
    for (int h = tid; h < (1 << hb) / 4; h += nth) h4[h] = make_uint4(kSeedEnd, kSeedEnd, kSeedEnd, kSeedEnd);
    __syncthreads();
    // two positions per thread and step, so their exchanges are in flight together
    for (int i = tid; i < npos; i += 2 * nth) {
        const int i2 = i + nth;
        const bool two = i2 < npos;
        const int w = (i >> 5) + G, sh = i & 31, w2 = (i2 >> 5) + G, sh2 = i2 & 31;
        const uint32_t c = seed_word<FL>(Tlo[w], Tlo[w + 1], Thi[w], Thi[w + 1], sh);
        const uint32_t c2 = two ? seed_word<FL>(Tlo[w2], Tlo[w2 + 1], Thi[w2], Thi[w2 + 1], sh2) : 0u;
        const uint32_t old = atomicExch(&heads[seed_bucket<FL>(c, hb)], (uint32_t)i);
        const uint32_t old2 = two ? atomicExch(&heads[seed_bucket<FL>(c2, hb)], (uint32_t)i2) : 0u;
        if (direct) {
            next16[i] = (unsigned short)old;
            if (two) next16[i2] = (unsigned short)old2;
        } else {
            node32[i] = (c & 0xffff0000u) | old;
            if (two) node32[i2] = (c2 & 0xffff0000u) | old2;
        }
    }
    __syncthreads();
    // nodes and run words a thread may visit: about where the band scan, whose work per
    // thread grows as n^2, becomes the cheaper pass (n/32 per word looked up, at least 16)
    const int nlook = (npos + t - 1) / t;  // starts that are multiples of t
    const int budget = max(16, n >> 5) * ((nlook + nth - 1) / nth) + 64;
    const unsigned lt = (1u << lane) - 1u;
    int work = 0, qn = 0;  // qn: entries in this warp's queue (warp-uniform)
    bool over = false;
    // an equal word (rows a .. a+K-1 pair on shift jc - a) joins the warp's queue when
    // its shift is scanned and row a+K-1 is counted; 32 queued words are measured at once
    auto push = [&](bool equal, uint32_t jc, int a) {
        bool hit = false;
        if (equal) {
            const int delta = (int)jc - a;
            int r_lo, r_hi;
            sl_diag_rows<FL>(n, delta, r_lo, r_hi);
            hit = delta >= geo.dlo && delta <= geo.dhi && a + K - 1 <= r_hi;
        }
        const unsigned hm = __ballot_sync(0xffffffffu, hit);
        if (hm) {
            if (hit) q[qn + __popc(hm & lt)] = (uint32_t)a | (jc << 16);
            qn += __popc(hm);
            __syncwarp();
            if (qn >= 32) {
                seed_measure<FL>(q[lane], geo, S, Tlo, Thi, work, best, bestd);
                __syncwarp();
                if (lane < qn - 32) q[lane] = q[32 + lane];
                qn -= 32;
                __syncwarp();
            }
        }
    };
    // one chain step: the node at jc (kSeedEnd: none); returns the next position and
    // whether jc holds the word c
    auto step = [&](uint32_t jc, uint32_t c, bool &equal) -> uint32_t {
        equal = false;
        if (jc == kSeedEnd) return kSeedEnd;
        uint32_t nx;
        if (direct) {
            nx = next16[jc];
            equal = true;
        } else {
            const uint32_t node = node32[jc];
            nx = node & 0xffffu;
            equal = (node ^ c) < 0x10000u;
        }
        return ++work > budget ? kSeedEnd : nx;  // past the bound: stop walking
    };
    // two words per lane and step (rows a and a + t*nth), their chains walked together
    for (int k0 = tid - lane; k0 < nlook; k0 += 2 * nth) {
        const int a = t * (k0 + lane), a2 = a + t * nth;
        uint32_t c = 0, j = kSeedEnd, c2 = 0, j2 = kSeedEnd;
        if (a < npos) {
            const int w = a >> 5, sh = a & 31;
            const uint2 s0 = S[w], s1 = S[w + 1];
            c = seed_word<FL>(s0.x, s1.x, s0.y, s1.y, sh);
            j = heads[seed_bucket<FL>(c, hb)];
        }
        if (a2 < npos) {
            const int w = a2 >> 5, sh = a2 & 31;
            const uint2 s0 = S[w], s1 = S[w + 1];
            c2 = seed_word<FL>(s0.x, s1.x, s0.y, s1.y, sh);
            j2 = heads[seed_bucket<FL>(c2, hb)];
        }
        while (__any_sync(0xffffffffu, j != kSeedEnd || j2 != kSeedEnd)) {
            const uint32_t jc = j, jc2 = j2;
            bool eq, eq2;
            j = step(jc, c, eq);
            j2 = step(jc2, c2, eq2);
            push(eq, jc, a);
            push(eq2, jc2, a2);
        }
        over = over || work > budget;
        if (__any_sync(0xffffffffu, over)) break;
    }
    if (lane < qn) seed_measure<FL>(q[lane], geo, S, Tlo, Thi, work, best, bestd);
    over = over || work > budget;
    return !__syncthreads_or(over);
}

// T's equality plane for nucleotide v (4 = the zero plane) at T word w, zero
// outside [0, n)
__device__ __forceinline__ uint32_t eq_word(const uint32_t *Tlo, const uint32_t *Thi, int W, int n, int v, int w)
{
    if (v > 3 || w < 0 || w >= W) return 0u;
    const uint32_t lo = Tlo[w + kSlGuardRows], hi = Thi[w + kSlGuardRows];
    const uint32_t valid = n - 32 * w >= 32 ? 0xffffffffu : ((1u << (n - 32 * w)) - 1u);
    const uint32_t x = (v & 1) ? lo : ~lo, y = (v & 2) ? hi : ~hi;
    return x & y & valid;
}

__device__ __forceinline__ void pair_reduce(int &best, int &bestd, int ob, int od)
{
    if (ob > best || (ob == best && od < bestd)) {
        best = ob;
        bestd = od;
    }
}

template <int NT> struct SlSmem {
    int2 queue[NT / 32][kBandQueue];  // band-scan items waiting for exact measurement
    int wbest[NT / 32];
    int wbestd[NT / 32];
    int last;
    int res[3];
    int next_chunk;
};

__device__ __forceinline__ int plane_nt(const uint2 *P, int x)
{
    uint2 w = P[x >> 5];
    int b = x & 31;
    return (int)(((w.x >> b) & 1u) | (((w.y >> b) & 1u) << 1));
}

template <int FL> __device__ void lrcs_combine(const Shape &s, PopBuf &buf, size_t gsol, const int2 *res,
                                               unsigned char *tab, int tid, int lane, int warp, int *shared_res);

// Warp-wide: the result with the longest run among res[0 .. count-1], read in
// parallel (one L2 round trip for up to 32 results); ties go to the largest index
// (last_on_tie) or to the smallest.  Every lane returns it.
__device__ __forceinline__ void warp_pick_result(const int2 *res, int count, bool last_on_tie, int lane, int &L, int &idx,
                                                 int &y)
{
    L = -1;
    idx = -1;
    y = 0;
    for (int r = lane; r < count; r += 32) {  // r rises within a lane
        const int2 v = __ldcg(&res[r]);
        if (v.x > L || (last_on_tie && v.x == L)) {
            L = v.x;
            idx = r;
            y = v.y;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const int L2 = __shfl_xor_sync(0xffffffffu, L, o), i2 = __shfl_xor_sync(0xffffffffu, idx, o),
                  y2 = __shfl_xor_sync(0xffffffffu, y, o);
        if (L2 > L || (L2 == L && (last_on_tie ? i2 > idx : i2 < idx))) {
            L = L2;
            idx = i2;
            y = y2;
        }
    }
}

// One scan item: result `item` = sol * nres + c of solution base + sol (CDS c, or CDS
// pair c for LRCS), then, in the last of the solution's items to finish, the combine.
// Called by the whole CTA with the CTA's dynamic shared memory.
// preset: the variation kernel set each child's counter to the results it kept, so a
// CTA whose result is carried over has nothing to count and leaves at once.
template <int NT, int FL>
__device__ void sl_item(const Shape &s, PopBuf buf, int base, int2 *part, int32_t *counter, int32_t *status,
                        unsigned long long *scanned, int item, unsigned char *smem_raw, bool preset = false)
{
    SlSmem<NT> &sm = *reinterpret_cast<SlSmem<NT> *>(smem_raw);
    const int G = kSlGuardRows;
    const int W = s.W, n = s.n;
    uint2 *S = reinterpret_cast<uint2 *>(smem_raw + ((sizeof(SlSmem<NT>) + 15) & ~size_t(15)));  // W + 2
    uint32_t *Tlo = reinterpret_cast<uint32_t *>(S + (W + 2));                               // W + 2G + 1
    uint32_t *Thi = Tlo + (W + 2 * G + 1);
    unsigned char *tab = reinterpret_cast<unsigned char *>(Thi + (W + 2 * G + 1));
    tab = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(tab) + 15) & ~uintptr_t(15));

    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nth >> 5;
    const int nres = FL == 0 ? s.m : s.nres;
    const int sol = item / nres, c = item - sol * nres;
    const size_t gsol = (size_t)(base + sol);
    // hairpin: CDS c against its reverse complement; LRCS: pair c = (pa, pb)
    int pa = c, pb = c;
    if (FL == 1) lrcs_pair_of(s.m, c, pa, pb);
    const uint2 *P = buf.planes + (gsol * s.m + pa) * s.Wp;

    // this CDS's (pair's) result: carried over from the parent when the mutation left
    // the CDS (both CDSs) as it was, else found by the scan below
    int2 *res = buf.cds ? buf.cds + gsol * nres : part + (size_t)sol * nres;
    const bool reuse = buf.cds != nullptr && res[c].x >= 0;
    if (reuse && preset) return;
    if (!reuse) {
        // stage S (the CDS planes) with one bulk async copy (TMA engine)
        {
            __shared__ __align__(8) uint64_t bar;
            const uint32_t bytes = (uint32_t)(s.Wp * sizeof(uint2));
            uint32_t bar_a = (uint32_t)__cvta_generic_to_shared(&bar);
            if (tid == 0) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
            __syncthreads();
            if (tid == 0) {
                uint32_t dst_a = (uint32_t)__cvta_generic_to_shared(S);
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes) : "memory");
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst_a),
                    "l"(P), "r"(bytes), "r"(bar_a)
                    : "memory");
            }
            // bounded wait on phase 0
            int done = 0;
            const int polls = wait_polls(s.wait_limit);
            for (int it = 0; it < polls && !done; it++) {
                uint32_t ok;
                asm volatile(
                    "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                    : "=r"(ok)
                    : "r"(bar_a), "r"(0u)
                    : "memory");
                done = (int)ok;
            }
            // the copy engine never completed: flag it, give the copy a second
            // bounded window to land, and leave this CTA (the host reports PE_ERR_TIMEOUT)
            if (__syncthreads_or(!done)) {
                if (tid == 0) atomicOr(status, 1);
                for (int it = 0; it < (1 << 20) && !done; it++) {
                    uint32_t ok;
                    asm volatile(
                        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                        : "=r"(ok)
                        : "r"(bar_a), "r"(0u)
                        : "memory");
                    done = (int)ok;
                }
                return;
            }
            if (tid == 0) asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar_a));
            for (int w = s.Wp + tid; w < W + 2; w += nth) S[w] = make_uint2(0u, 0u);
        }
        __syncthreads();
        // T: reverse complement planes (hairpin) or CDS pb's own planes (LRCS), zero outside [0, W)
        const uint2 *Pb = buf.planes + (gsol * s.m + pb) * s.Wp;
        for (int e = tid; e < W + 2 * G + 1; e += nth) {
            int w = e - G;
            uint32_t lo = 0, hi = 0;
            if (FL == 1) {
                if (w >= 0 && w < W) {
                    const uint2 v = pa == pb ? S[w] : Pb[w];
                    lo = v.x;
                    hi = v.y;
                }
            } else if (w >= 0 && w < W) {
                int start = n - 32 - 32 * w;  // source bit of T bit 31 ... bit 0 is source n-1-32w
                int q = start >> 5, sh = start & 31;
                uint32_t a0 = (q >= 0 && q < W) ? S[q].x : 0u, a1 = (q + 1 >= 0 && q + 1 < W) ? S[q + 1].x : 0u;
                uint32_t b0 = (q >= 0 && q < W) ? S[q].y : 0u, b1 = (q + 1 >= 0 && q + 1 < W) ? S[q + 1].y : 0u;
                lo = ~__brev(fshr(a0, a1, sh));
                hi = ~__brev(fshr(b0, b1, sh));
            }
            Tlo[e] = lo;
            Thi[e] = hi;
        }
        __syncthreads();
        const SlGeo geo = sl_geo<FL>(n, pa == pb);
        int best = 0, bestd = 0x7fffffff;
        // the seeded scan where the CDS fits its table, else (or when it gives up on a
        // repetitive CDS) the band scan
        bool band = true;
        if (sl_seeded(s)) {
            band = !sl_seed_scan<FL>(geo, S, Tlo, Thi, tab, reinterpret_cast<uint32_t *>(sm.queue[warp]), tid, nth, best,
                                     bestd);
            if (band) {
                best = 0;
                bestd = 0x7fffffff;
                if (tid == 0 && scanned) atomicAdd(&scanned[2], 1ull);
            }
        }
        if (band) {
            // band-scan tables (their space is free again: the seeded scan's last reads
            // came before its closing barrier):
            //   E4[v][x]      E_v words x-kEqGuard .. x+3-kEqGuard, v = 0..3 nucleotides, 4 the zero plane
            //   poffT[sp][i]  rows r = 32(sp-1)+2i, r+1: E4 entries v(r)*PS + sp-1 in the low and high
            //                 16 bits (v(r) = 4 outside [0, n); 5*PS < 65536 since E4's 80*PS bytes fit in
            //                 shared memory); pitch 17 words
            //   gstart[g]     first item of band group g (items: the group's 32-row segments)
            const int PS = sl_plane_stride(W), NSP = W + 2;
            const int ng = geo.ng, D0 = geo.D0;
            uint4 *E4 = reinterpret_cast<uint4 *>(tab);
            int *poffT = reinterpret_cast<int *>(E4 + 5 * PS);
            int *gstart = poffT + kSegPitch * NSP;
            // each equality word once, stored into the four entries that hold it (entry x holds
            // words x - kEqGuard .. x + 3 - kEqGuard, word j of the entry being word x - kEqGuard + j)
            uint32_t *E4w = reinterpret_cast<uint32_t *>(E4);
            for (int e = tid; e < 5 * (PS + 3); e += nth) {
                const int v = e / (PS + 3), w = e - v * (PS + 3) - kEqGuard;
                const uint32_t word = eq_word(Tlo, Thi, W, n, v, w);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int x = w + kEqGuard - j;
                    if (x >= 0 && x < PS) E4w[(v * PS + x) * 4 + j] = word;
                }
            }
            for (int e = tid; e < kSegPitch * NSP; e += nth) {
                const int sp = e / kSegPitch, i = e - sp * kSegPitch;
                int word = (4 * PS + sp - 1) * 0x10001;  // both rows outside [0, n): the zero plane
                if (i < 16 && sp >= 1 && sp - 1 < W) {   // rows r = 32(sp-1) + 2i and r + 1
                    const uint2 sw = S[sp - 1];
                    const int b = 2 * i, r = 32 * (sp - 1) + b;
                    const int v0 = r < n ? (int)(((sw.x >> b) & 1u) | (((sw.y >> b) & 1u) << 1)) : 4;
                    const int v1 = r + 1 < n ? (int)(((sw.x >> (b + 1)) & 1u) | (((sw.y >> (b + 1)) & 1u) << 1)) : 4;
                    word = (v0 * PS + sp - 1) | ((v1 * PS + sp - 1) << 16);  // E4 entries of rows r, r + 1
                }
                poffT[e] = word;
            }
            if (warp == 0) {
                int carry = 0;
                for (int g0 = 0; g0 < ng; g0 += 32) {
                    const int g = g0 + lane;
                    int x = 0;
                    if (g < ng) {
                        int s_lo, s_hi;
                        sl_group_rows<FL>(n, D0 + 32 * kBandGroup * g, s_lo, s_hi);
                        x = max(0, s_hi - s_lo + 1);
                    }
                    for (int o = 1; o < 32; o <<= 1) {
                        const int y = __shfl_up_sync(0xffffffffu, x, o);
                        if (lane >= o) x += y;
                    }
                    if (g < ng) gstart[g + 1] = carry + x;
                    carry += __shfl_sync(0xffffffffu, x, 31);
                }
                if (lane == 0) gstart[0] = 0;
            }
            if (tid == 0) sm.next_chunk = 0;
            __syncthreads();
            sl_band_scan<FL>(E4, poffT, gstart, geo, S, Tlo, Thi, sm.queue[warp], &sm.next_chunk, lane, best, bestd);
        }
        // CTA reduction of (best, smallest anti-diagonal)
        for (int o = 16; o > 0; o >>= 1) {
            int ob = __shfl_xor_sync(0xffffffffu, best, o), od = __shfl_xor_sync(0xffffffffu, bestd, o);
            pair_reduce(best, bestd, ob, od);
        }
        if (lane == 0) {
            sm.wbest[warp] = best;
            sm.wbestd[warp] = bestd;
        }
        __syncthreads();
        if (tid == 0) {
            int b = sm.wbest[0], d = sm.wbestd[0];
            for (int w = 1; w < nwarps; w++) pair_reduce(b, d, sm.wbest[w], sm.wbestd[w]);
            sm.res[0] = b;
            sm.res[1] = d;
            sm.next_chunk = 0;
        }
        __syncthreads();
        if (sm.res[0] < 8) {
            // no run reaches 8: exact per-word runs
            best = 0;
            bestd = 0x7fffffff;
            sl_scan<FL>(S, Tlo, Thi, geo, &sm.next_chunk, lane, best, bestd);
            for (int o = 16; o > 0; o >>= 1) {
                int ob = __shfl_xor_sync(0xffffffffu, best, o), od = __shfl_xor_sync(0xffffffffu, bestd, o);
                pair_reduce(best, bestd, ob, od);
            }
            __syncthreads();
            if (lane == 0) {
                sm.wbest[warp] = best;
                sm.wbestd[warp] = bestd;
            }
            __syncthreads();
            if (tid == 0) {
                int b = sm.wbest[0], d = sm.wbestd[0];
                for (int w = 1; w < nwarps; w++) pair_reduce(b, d, sm.wbest[w], sm.wbestd[w]);
                sm.res[0] = b;
                sm.res[1] = d;
            }
            __syncthreads();
        }
    }
    if (tid == 0) {
        if (!reuse) res[c] = make_int2(sm.res[0], sm.res[1]);
        // a scan's result must be visible before the count says it is there (a carried
        // result wrote nothing); the solution's last CTA fences again before it reads
        if (!reuse) __threadfence();
        int old = atomicAdd(&counter[sol], 1);
        sm.last = (old == nres - 1);
        if (!reuse && scanned) {
            // scans, and the LRCS scans of a CDS against itself (the host derives the
            // counted cells from them); after the counter, so the fence does not wait
            // for these adds that every scanning CTA makes to the same words
            atomicAdd(&scanned[0], 1ull);
            if (FL == 1 && pa == pb) atomicAdd(&scanned[1], 1ull);
        }
    }
    __syncthreads();
    if (!sm.last) return;
    __threadfence();
    if (FL == 1) {
        if (tid == 0) counter[sol] = 0;
        lrcs_combine<FL>(s, buf, gsol, res, tab, tid, lane, warp, sm.res);
        return;
    }
    // ---- last CTA of this solution: combine CDSs (largest CDS index on ties)
    if (warp == 0) {
        int Lb, cb, db;
        warp_pick_result(res, s.m, true, lane, Lb, cb, db);
        if (lane == 0) {
            sm.res[0] = Lb;
            sm.res[1] = cb;
            sm.res[2] = db;
            counter[sol] = 0;
        }
    }
    __syncthreads();
    const int Lb = sm.res[0], cb = sm.res[1], d = sm.res[2];
    const int slot = s.slot[K_SL];
    float *obj = buf.obj + gsol * s.M;
    int8_t *objidx = buf.objidx + gsol * 2 * s.M;
    int32_t *pql = buf.pql + gsol * 3;
    if (Lb <= 0) {
        if (tid == 0) {
            obj[slot] = 0.0f;
            objidx[2 * slot] = 0;
            objidx[2 * slot + 1] = 0;
            pql[0] = pql[1] = pql[2] = 0;
        }
        return;
    }
    // Position of the stem the reference's serial sweep records last on
    // anti-diagonal d: the outermost stem of exactly Lb pairs closed on both
    // sides inside the counted cells (recorded again, later, from the lower
    // triangle), else the run cut at the loop limit.
    if (warp == 0) {
        // the winning CDS's planes, staged in shared memory (the tables' space is free)
        uint2 *Q = reinterpret_cast<uint2 *>(tab);
        const uint2 *Qg = buf.planes + (gsol * s.m + cb) * s.Wp;
        for (int w = lane; w < s.Wp; w += 32) Q[w] = Qg[w];
        __syncwarp();
        const int r_lo = max(0, d - (n - 1)), r_hi = (d - 5) >> 1;
        // Pairing rows r_lo .. r_hi of anti-diagonal d, 32 per lane: every counted run
        // on d is at most Lb long (Lb is the CDS's longest), so a run of Lb starts
        // wherever Lb consecutive rows pair.  Each lane takes the runs whose last row
        // lies in its word; a run that enters from the words below carries their
        // length (a scan over the lanes).  The first run of Lb closed by a row that
        // does not pair gives (p, q); one ending at r_hi is closed by row r_hi + 1
        // (outside the counted range), and if that row pairs too the stem is cut at
        // the loop limit (typeII).
        const int nwords = (r_hi - r_lo + 1 + 31) >> 5;
        const int beyond = ((plane_nt(Q, r_hi + 1) ^ plane_nt(Q, d - r_hi - 1)) == 3);
        // rows r .. r+31 of diagonal d: s[r+b] against s[d-r-b]
        auto diag_word = [&](int r) -> uint32_t {
            const int ws = r >> 5, bs = r & 31;
            const uint32_t slo = fshr(Q[ws].x, Q[ws + 1].x, bs), shi = fshr(Q[ws].y, Q[ws + 1].y, bs);
            const int t0 = d - r - 31;  // partner of row r + 31; bit 31 - b of the window is s[d - r - b]
            const int wt = t0 >> 5, bt = t0 & 31;  // wt may be -1 when high rows fall outside
            const uint2 qa = wt >= 0 ? Q[wt] : make_uint2(0u, 0u), qb = Q[wt + 1];
            const uint32_t tlo = __brev(fshr(qa.x, qb.x, bt)), thi = __brev(fshr(qa.y, qb.y, bt));
            return (slo ^ tlo) & (shi ^ thi);  // complementary in both bits
        };
        int first = 0x7fffffff, typeII = 0;
        uint32_t carry = 0;  // run length ending at the last row of the previous pass
        for (int k0 = 0; k0 < nwords; k0 += 32) {
            const int k = k0 + lane, r0 = r_lo + 32 * k;
            uint32_t X = 0u, nb = 0u;  // this word's in-range bits; bit 0 of the next word
            if (k < nwords) {
                X = diag_word(r0);
                const int rows = r_hi - r0 + 1;
                if (rows < 32) X &= (1u << rows) - 1u;
                if (lane == 31 && r0 + 32 <= r_hi)
                    nb = (plane_nt(Q, r0 + 32) ^ plane_nt(Q, d - r0 - 32)) == 3;
            }
            const uint32_t nb_lane = __shfl_down_sync(0xffffffffu, X & 1u, 1);
            if (lane < 31) nb = nb_lane;
            // run length ending at this word's top: all ones ? 32 + previous : trailing ones
            uint32_t A = X == 0xffffffffu, Bv = A ? 32u : (uint32_t)__clz((int)~X);
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t A2 = __shfl_up_sync(0xffffffffu, A, o), B2 = __shfl_up_sync(0xffffffffu, Bv, o);
                if (lane >= o) {
                    Bv = A * B2 + Bv;
                    A &= A2;
                }
            }
            const uint32_t E = A * carry + Bv;
            uint32_t cin = __shfl_up_sync(0xffffffffu, E, 1);
            if (lane == 0) cin = carry;
            carry = __shfl_sync(0xffffffffu, E, 31);
            // runs ending in this word: a one followed by a zero (or by the range's end)
            const uint32_t ends = X & ~((X >> 1) | (nb << 31));
            const uint32_t starts = X & ~((X << 1) | (cin ? 1u : 0u));
            int cand = 0x7fffffff, cand2 = 0;
            uint32_t e_bits = ends;
            while (e_bits && cand == 0x7fffffff) {
                const int e = __ffs((int)e_bits) - 1;
                e_bits &= e_bits - 1;
                const uint32_t sm_ = starts & (e == 31 ? ~0u : ((2u << e) - 1u));
                const int len = sm_ ? e - (31 - __clz((int)sm_)) + 1 : e + 1 + (int)cin;
                if (len >= Lb) {
                    const int pstart = r0 + e - len + 1;
                    if (r0 + e == r_hi && beyond) cand2 = 1;  // cut at the loop limit
                    else cand = pstart;
                }
            }
            // lowest lane with a closed run of Lb holds the first one
            const unsigned has = __ballot_sync(0xffffffffu, cand != 0x7fffffff);
            if (has && first == 0x7fffffff) first = __shfl_sync(0xffffffffu, cand, __ffs((int)has) - 1);
            if (__any_sync(0xffffffffu, cand2)) typeII = 1;
            if (first != 0x7fffffff) break;
        }
        if (first == 0x7fffffff) first = -1;
        if (lane == 0) {
            int p, q;
            if (first >= 0) {
                p = first;
                q = d - (first + Lb - 1);
            } else if (typeII) {
                p = r_hi - Lb + 1;
                q = d - r_hi;
            } else {
                p = -1;
                q = -1;
            }
            obj[slot] = __fdiv_rn((float)Lb, (float)s.K);
            objidx[2 * slot] = (int8_t)cb;
            objidx[2 * slot + 1] = 0;
            pql[0] = p;
            pql[1] = q;
            pql[2] = Lb;
        }
    }
}

// one CTA per result of solutions base .. base + count - 1
template <int NT, int FL>
__global__ void __launch_bounds__(NT) k_sl(Shape s, PopBuf buf, int base, int2 *part, int32_t *counter,
                                                 int32_t *status, unsigned long long *scanned, int preset)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    sl_item<NT, FL>(s, buf, base, part, counter, status, scanned, (int)blockIdx.x, smem_raw, preset != 0);
}

// The scan items of a whole batch: the variation kernels of the batch's instances
// queue the results their children's mutations invalidated (SlJob.items, .count), and
// one wave of CTAs takes them by ticket, the jobs in the order given (longest CDSs
// first), until all are done.  The last CTA to leave clears the tickets and the
// counts for the next generation.
template <int NT, int FL>
__global__ void __launch_bounds__(NT) k_sl_queue(const SlJob *__restrict__ jobs, int njobs, int32_t *ticket)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int qpre[kMaxBatchJobs + 1];
    __shared__ int cur_job, cur_item;
    const int tid = threadIdx.x;
    if (tid == 0) {
        int run = 0;
        for (int k = 0; k < njobs; k++) {
            qpre[k] = run;
            run += *jobs[k].count;
        }
        qpre[njobs] = run;
    }
    __syncthreads();
    const int total = qpre[njobs];
    for (;;) {
        if (tid == 0) {
            const int t = atomicAdd(&ticket[0], 1);
            int k = -1, it = 0;
            if (t < total) {
                k = 0;
                while (qpre[k + 1] <= t) k++;
                it = jobs[k].items[t - qpre[k]];
            }
            cur_job = k;
            cur_item = it;
        }
        __syncthreads();
        const int k = cur_job, it = cur_item;
        if (k < 0) break;
        const SlJob &J = jobs[k];
        sl_item<NT, FL>(J.s, J.buf, J.base, J.part, J.counter, J.status, J.scanned, it, smem_raw);
        __syncthreads();  // the next item reuses the shared memory
    }
    if (tid == 0) {
        __threadfence();
        if (atomicAdd(&ticket[1], 1) == (int)gridDim.x - 1) {
            for (int q = 0; q < njobs; q++) *jobs[q].count = 0;
            ticket[0] = 0;
            ticket[1] = 0;
        }
    }
}

// LRCS combine (last CTA of a solution): the pair with the longest run (the
// first pair on ties), its diagonal (the smallest delta reaching that length),
// and on it the first run of that length.  Every run of the pair is at most Lb
// long, so a run of Lb starts wherever Lb consecutive rows match; one warp takes
// 32 rows per lane from the two CDSs' planes staged in shared memory, carries run
// lengths across lanes with a scan, and the lowest lane holding a run of Lb that
// ends in its word gives the start.
template <int FL> __device__ void lrcs_combine(const Shape &s, PopBuf &buf, size_t gsol, const int2 *res,
                                               unsigned char *tab, int tid, int lane, int warp, int *shared_res)
{
    if (warp == 0) {  // the first pair on ties; no pair with a run: length 0 (nothing else is read)
        int Lb, rb, kb;
        warp_pick_result(res, s.nres, false, lane, Lb, rb, kb);
        if (lane == 0) {
            shared_res[0] = Lb;
            shared_res[1] = rb;
            shared_res[2] = kb;
        }
    }
    __syncthreads();
    const int Lb = shared_res[0], n = s.n, delta = shared_res[2] - n;
    int a, b;
    lrcs_pair_of(s.m, shared_res[1], a, b);
    const int slot = s.slot[K_SL];
    float *obj = buf.obj + gsol * s.M;
    int8_t *objidx = buf.objidx + gsol * 2 * s.M;
    int32_t *pql = buf.pql + gsol * 3;
    if (Lb <= 0) {
        if (tid == 0) {
            obj[slot] = 0.0f;
            objidx[2 * slot] = 0;
            objidx[2 * slot + 1] = 0;
            pql[0] = pql[1] = pql[2] = 0;
        }
        return;
    }
    if (warp != 0) return;
    uint2 *Qa = reinterpret_cast<uint2 *>(tab), *Qb = Qa + s.Wp;
    const uint2 *Ga = buf.planes + (gsol * s.m + a) * s.Wp, *Gb = buf.planes + (gsol * s.m + b) * s.Wp;
    for (int w = lane; w < s.Wp; w += 32) {
        Qa[w] = Ga[w];
        Qb[w] = Gb[w];
    }
    __syncwarp();
    const int r_lo = max(0, -delta), r_hi = min(n - 1, n - 1 - delta);
    const int nwords = (r_hi - r_lo + 1 + 31) >> 5;
    // rows r .. r+31 of the diagonal: s_a[r + j] against s_b[r + delta + j]
    auto diag_word = [&](int r) -> uint32_t {
        const int ws = r >> 5, bs = r & 31, i = r + delta, wt = i >> 5, bt = i & 31;
        const uint32_t alo = fshr(Qa[ws].x, Qa[ws + 1].x, bs), ahi = fshr(Qa[ws].y, Qa[ws + 1].y, bs);
        const uint32_t blo = fshr(Qb[wt].x, Qb[wt + 1].x, bt), bhi = fshr(Qb[wt].y, Qb[wt + 1].y, bt);
        return ~((alo ^ blo) | (ahi ^ bhi));
    };
    int first = -1;
    uint32_t carry = 0;  // run length ending at the last row of the previous pass
    for (int k0 = 0; k0 < nwords && first < 0; k0 += 32) {
        const int k = k0 + lane, r0 = r_lo + 32 * k;
        uint32_t X = 0u, nb = 0u;
        if (k < nwords) {
            X = diag_word(r0);
            const int rows = r_hi - r0 + 1;
            if (rows < 32) X &= (1u << rows) - 1u;
            if (lane == 31 && r0 + 32 <= r_hi) nb = diag_word(r0 + 32) & 1u;
        }
        const uint32_t nb_lane = __shfl_down_sync(0xffffffffu, X & 1u, 1);
        if (lane < 31) nb = nb_lane;
        uint32_t A = X == 0xffffffffu, Bv = A ? 32u : (uint32_t)__clz((int)~X);
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t A2 = __shfl_up_sync(0xffffffffu, A, o), B2 = __shfl_up_sync(0xffffffffu, Bv, o);
            if (lane >= o) {
                Bv = A * B2 + Bv;
                A &= A2;
            }
        }
        const uint32_t E = A * carry + Bv;
        uint32_t cin = __shfl_up_sync(0xffffffffu, E, 1);
        if (lane == 0) cin = carry;
        carry = __shfl_sync(0xffffffffu, E, 31);
        const uint32_t ends = X & ~((X >> 1) | (nb << 31));
        const uint32_t starts = X & ~((X << 1) | (cin ? 1u : 0u));
        int cand = -1;
        uint32_t e_bits = ends;
        while (e_bits && cand < 0) {
            const int e = __ffs((int)e_bits) - 1;
            e_bits &= e_bits - 1;
            const uint32_t sm_ = starts & ((2u << e) - 1u);
            const int len = sm_ ? e - (31 - __clz((int)sm_)) + 1 : e + 1 + (int)cin;
            if (len >= Lb) cand = r0 + e - len + 1;
        }
        const unsigned has = __ballot_sync(0xffffffffu, cand >= 0);
        if (has) first = __shfl_sync(0xffffffffu, cand, __ffs((int)has) - 1);
    }
    if (lane == 0) {
        obj[slot] = __fdiv_rn((float)Lb, (float)n);
        objidx[2 * slot] = (int8_t)a;
        objidx[2 * slot + 1] = (int8_t)b;
        pql[0] = first;
        pql[1] = first >= 0 ? first + delta : -1;
        pql[2] = Lb;
    }
}

static size_t sl_smem_bytes_nt(const Shape &s, size_t head)
{
    const int G = kSlGuardRows, W = s.W;
    size_t b = (head + 15) & ~size_t(15);
    b += (size_t)(W + 2) * sizeof(uint2);
    b += 2 * (size_t)(W + 2 * G + 1) * sizeof(uint32_t);
    b += 16;  // alignment of the band-scan tables
    const int ng = s.sl_kind == PE_SL_LRCS ? sl_geo<1>(s.n, false).ng : sl_num_groups(s.n);
    const size_t band = (size_t)5 * sl_plane_stride(W) * sizeof(uint4) + (size_t)kSegPitch * (W + 2) * sizeof(int) +
                        (size_t)(ng + 1) * sizeof(int);
    // the two passes share the space
    b += sl_seeded(s) ? std::max(band, sl_seed_bytes(s.n, s.sl_kind != PE_SL_LRCS)) : band;
    return b;
}

size_t sl_smem_bytes(const Shape &s) { return sl_smem_bytes_nt(s, sizeof(SlSmem<kSlThreadsMax>)); }

// the queued scan's shared memory for a job at CTA size nt
size_t sl_queue_smem_bytes(const Shape &s, int nt)
{
    switch (nt) {
    case 64: return sl_smem_bytes_nt(s, sizeof(SlSmem<64>));
    case 256: return sl_smem_bytes_nt(s, sizeof(SlSmem<256>));
    default: return sl_smem_bytes_nt(s, sizeof(SlSmem<128>));
    }
}

template <int NT, int FL> static const void *sl_queue_fn() { return (const void *)k_sl_queue<NT, FL>; }
static const void *sl_queue_kernel(int nt, int fl)
{
    if (fl == 1) return nt == 64 ? sl_queue_fn<64, 1>() : nt == 256 ? sl_queue_fn<256, 1>() : sl_queue_fn<128, 1>();
    return nt == 64 ? sl_queue_fn<64, 0>() : nt == 256 ? sl_queue_fn<256, 0>() : sl_queue_fn<128, 0>();
}

int sl_queue_ctas_per_sm(int nt, int fl, size_t smem)
{
    const void *fn = sl_queue_kernel(nt, fl);
    if (raise_smem_limit(fn, smem) != cudaSuccess) return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, nt == 64 || nt == 256 ? nt : 128, smem) != cudaSuccess) return 0;
    return n;
}

cudaError_t launch_sl_queue(const SlJob *jobs, int njobs, int32_t *ticket, int nt, int fl, size_t smem, int ctas,
                            cudaStream_t st)
{
    if (njobs <= 0 || njobs > kMaxBatchJobs || ctas <= 0) return cudaErrorInvalidValue;
    const void *fn = sl_queue_kernel(nt, fl);
    cudaError_t e = raise_smem_limit(fn, smem);
    if (e != cudaSuccess) return e;
    if (fl == 1) {
        if (nt == 64) k_sl_queue<64, 1><<<ctas, 64, smem, st>>>(jobs, njobs, ticket);
        else if (nt == 256) k_sl_queue<256, 1><<<ctas, 256, smem, st>>>(jobs, njobs, ticket);
        else k_sl_queue<128, 1><<<ctas, 128, smem, st>>>(jobs, njobs, ticket);
    } else {
        if (nt == 64) k_sl_queue<64, 0><<<ctas, 64, smem, st>>>(jobs, njobs, ticket);
        else if (nt == 256) k_sl_queue<256, 0><<<ctas, 256, smem, st>>>(jobs, njobs, ticket);
        else k_sl_queue<128, 0><<<ctas, 128, smem, st>>>(jobs, njobs, ticket);
    }
    return cudaGetLastError();
}

template <int NT>
static cudaError_t launch_sl_nt(const Shape &s, PopBuf buf, int base, int count, int2 *part, int32_t *counter,
                                int32_t *status, cudaStream_t st, unsigned long long *scanned, bool preset)
{
    const size_t smem = sl_smem_bytes_nt(s, sizeof(SlSmem<NT>));
    if (s.sl_kind == PE_SL_LRCS) {
        cudaError_t e = raise_smem_limit((const void *)k_sl<NT, 1>, smem);
        if (e != cudaSuccess) return e;
        k_sl<NT, 1><<<count * s.nres, NT, smem, st>>>(s, buf, base, part, counter, status, scanned, (int)preset);
        return cudaGetLastError();
    }
    cudaError_t e = raise_smem_limit((const void *)k_sl<NT, 0>, smem);
    if (e != cudaSuccess) return e;
    k_sl<NT, 0><<<count * s.m, NT, smem, st>>>(s, buf, base, part, counter, status, scanned, (int)preset);
    return cudaGetLastError();
}

cudaError_t launch_sl(const Shape &s, PopBuf buf, int base, int count, int2 *part, int32_t *counter, int32_t *status,
                      cudaStream_t st, unsigned long long *scanned, bool preset)
{
    if (count <= 0) return cudaSuccess;
    switch (s.sl_threads) {
    case 64: return launch_sl_nt<64>(s, buf, base, count, part, counter, status, st, scanned, preset);
    case 256: return launch_sl_nt<256>(s, buf, base, count, part, counter, status, st, scanned, preset);
    default: return launch_sl_nt<128>(s, buf, base, count, part, counter, status, st, scanned, preset);
    }
}

}  // namespace pe
