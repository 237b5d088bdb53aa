/*
 * pe_oracle.c -- CPU oracle (test infrastructure, see pe_oracle.h).
 *
 * Build with -ffp-contract=off: every float/double operation here is one IEEE
 * operation, in the order written, so the CUDA engine (built with --fmad=false
 * where it mirrors these formulas) reproduces the same bits.
 */
#include "pe_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* objective slots                                                          */
/* ------------------------------------------------------------------------ */

static const int kinds_ref6[6] = {OR_K_CAI, OR_K_CBP, OR_K_HSC, OR_K_HD, OR_K_GC, OR_K_SL};
static const int kinds_base4[4] = {OR_K_CAI, OR_K_HD, OR_K_GC, OR_K_SL};

int or_num_obj(int objset) { return objset == OR_OBJSET_BASE4 ? 4 : 6; }

int or_slot_of(int objset, int kind)
{
    const int *k = objset == OR_OBJSET_BASE4 ? kinds_base4 : kinds_ref6;
    int M = or_num_obj(objset);
    for (int i = 0; i < M; i++)
        if (k[i] == kind) return i;
    return -1;
}

/* ------------------------------------------------------------------------ */
/* Das-Dennis reference points: include/sorting.cuh:1285-1354 (bincoef,     */
/* NUnrank, combinationRepetition) and the p rule of src/main.cu:564-576.   */
/* ------------------------------------------------------------------------ */

static uint64_t bincoef(int n, int r)
{
    if (r < 0 || n < r) return 0;
    if (2 * r > n) r = n - r;
    uint64_t res = 1;
    for (int i = 0; i < r; i++) res = (res * (uint64_t)(n - i)) / (uint64_t)(i + 1);
    return res;
}

int or_num_ref(int M, int p) { return (int)bincoef(M + p - 1, p); }

int or_auto_p(int M, int N)
{
    int p = 1;
    while ((int64_t)bincoef(M + p - 1, p) <= N) p++;
    return p - 1;
}

/* rank r -> multiset x_1 <= ... <= x_p of {1..M} in lexicographic order;
 * coordinate x-1 gets 1/p per occurrence (accumulated in float). */
static void nunrank(int r, float *pt, int mm, int p)
{
    int x = 1;
    float inc = 1.0f / (float)p;
    for (int i = 1; i <= p; i++) {
        uint64_t y = bincoef(mm - x - i + 1, p - i);
        while (y <= (uint64_t)r) {
            r -= (int)y;
            x++;
            if (x > mm) return;
            y = bincoef(mm - x - i + 1, p - i);
        }
        pt[x - 1] += inc;
    }
}

void or_das_dennis(int M, int p, float *out)
{
    int R = or_num_ref(M, p);
    memset(out, 0, sizeof(float) * (size_t)R * (size_t)M);
    for (int r = 0; r < R; r++) nunrank(r, out + (size_t)r * M, M + p - 1, p);
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon et al., SC'11).  Replaces the reference's XORWOW     */
/* streams (src/main.cu:35): every draw is keyed by (seed, tag, generation,  */
/* individual, position, j), independent of how work is scheduled.          */
/* ------------------------------------------------------------------------ */

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; r++) {
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += PHILOX_W0; k1 += PHILOX_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

uint32_t or_draw(uint64_t seed, uint32_t tag, uint32_t gen, uint32_t idx, uint32_t pos, uint32_t j)
{
    uint32_t ctr[4] = {tag, gen, idx, pos * 8u + (j >> 2)};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    or_philox4x32_10(ctr, key, out);
    return out[j & 3];
}

#define TAG_INIT 1u
#define TAG_OP 2u
#define TAG_MUT 3u
#define TAG_SLMUT 4u
#define TAG_NICHE 5u
#define TAG_MUTP 6u

/* The probability test of codon position pos in a mutation operator: word pos % 4
 * of the Philox block with counter (TAG_MUTP, gen, idx, pos / 4), so one block
 * serves four consecutive positions. */
static uint32_t or_pdraw(uint64_t seed, uint32_t gen, uint32_t idx, uint32_t pos)
{
    uint32_t ctr[4] = {TAG_MUTP, gen, idx, pos >> 2};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t out[4];
    or_philox4x32_10(ctr, key, out);
    return out[pos & 3];
}

static inline uint32_t rng_uint(uint32_t r, uint32_t k) { return (uint32_t)(((uint64_t)r * k) >> 32); }
/* uniform float in (0,1], 24-bit grid */
static inline float rng_u01(uint32_t r) { return (float)((r >> 8) + 1u) * (1.0f / 16777216.0f); }

/* ------------------------------------------------------------------------ */
/* exp(x) for x <= 0 from basic IEEE double operations only (Cody-Waite     */
/* reduction by ln 2, degree-13 Taylor polynomial in Horner form with fma),  */
/* so CPU and GPU produce identical bits.                                   */
/* ------------------------------------------------------------------------ */

double or_det_exp(double x)
{
    if (x < -700.0) return 0.0;
    const double inv_ln2 = 1.4426950408889634;
    const double ln2_hi = 0.6931471803691238;      /* ln 2 with its low 21 bits cleared */
    const double ln2_lo = 1.9082149292705877e-10;  /* ln 2 - ln2_hi */
    double kd = nearbyint(x * inv_ln2);
    double r = fma(-kd, ln2_hi, x);
    r = fma(-kd, ln2_lo, r);
    static const double c[14] = {1.0, 1.0, 0.5, 0.16666666666666666, 0.041666666666666664,
                                 0.008333333333333333, 0.001388888888888889, 0.0001984126984126984,
                                 2.48015873015873e-05, 2.7557319223985893e-06, 2.755731922398589e-07,
                                 2.505210838544172e-08, 2.08767569878681e-09, 1.6059043836821613e-10};
    double p = c[13];
    for (int i = 12; i >= 0; i--) p = fma(p, r, c[i]);
    int k = (int)kd;
    uint64_t bits = (uint64_t)(int64_t)(k + 1023) << 52;
    double scale;
    memcpy(&scale, &bits, sizeof scale);
    return p * scale;
}

/* log w(codon) in 2^-32 fixed point (exact integer sums, order independent) */
void or_log_weight_fixed(const or_codon_table *t, int64_t out[OR_NUM_CODON], uint8_t zero[OR_NUM_CODON])
{
    for (int c = 0; c < OR_NUM_CODON; c++) {
        double w = (double)t->weight[c];
        if (!(w > 0.0)) {
            out[c] = 0;
            zero[c] = 1;
        } else {
            out[c] = (int64_t)llrint(log(w) * 4294967296.0);
            zero[c] = 0;
        }
    }
}

static int64_t cps_fixed(float v) { return (int64_t)llrint((double)v * 4294967296.0); }

/* ------------------------------------------------------------------------ */
/* population generation: include/utils.cuh:1047-1104                       */
/* ------------------------------------------------------------------------ */

void or_gen_solution(const or_problem *pr, int idx, uint8_t *sol)
{
    const or_codon_table *t = pr->tab;
    for (int i = 0; i < pr->m; i++)
        for (int a = 0; a < pr->L; a++) {
            int aa = pr->aa[a];
            int k = t->count[aa];
            int pos;
            if (idx == 0) {
                pos = k - 1; /* HIGHEST_CAI_GEN: last codon of the group */
            } else {
                uint32_t r = or_draw(pr->seed, TAG_INIT, 0, (uint32_t)idx, (uint32_t)(i * pr->L + a), 0);
                pos = (int)rng_uint(r, (uint32_t)k);
            }
            sol[i * pr->L + a] = (uint8_t)(t->start[aa] + pos);
        }
}

/* ------------------------------------------------------------------------ */
/* evaluators                                                               */
/* ------------------------------------------------------------------------ */

static inline int is_stop_nt(const or_codon_table *t, int a, int b, int c)
{
    /* isStopCodon: the last three codons of the table (include/utils.cuh:101-112) */
    for (int s = OR_NUM_CODON - 3; s < OR_NUM_CODON; s++)
        if (t->nt[s][0] == a && t->nt[s][1] == b && t->nt[s][2] == c) return 1;
    return 0;
}

/* hidden stops across the boundary x|y: frames (x1 x2 y0) and (x2 y0 y1)
 * (countRightSideHSC, include/utils.cuh:138-161) */
static inline int hsc_pair(const or_codon_table *t, int x, int y)
{
    return is_stop_nt(t, t->nt[x][1], t->nt[x][2], t->nt[y][0]) +
           is_stop_nt(t, t->nt[x][2], t->nt[y][0], t->nt[y][1]);
}

static inline int compat(int a, int b) { return (a ^ b) == 3; } /* A-U, C-G (isCompatible) */

/* calMaximumSL (include/utils.cuh:712-888) run by one thread over all CDSs.
 * The reference's spinlock picks an arbitrary thread's record on ties; one
 * thread records the LAST cell, in (cds, anti-diagonal t, j) order, whose run
 * count reaches the final maximum -- that is the rule used here. */
static void sl_serial(const uint8_t *nt, int m, int n, int *L_out, int *p_out, int *q_out, int *cds_out)
{
    int l = 0, p = 0, q = 0, cds = 0;
    for (int i = 0; i < m; i++) {
        const uint8_t *s = nt + (size_t)i * n;
        for (int t = 0; t < 2 * n + 1; t++) {
            int diag_len, st_r, st_c;
            if (t < n + 1) {
                diag_len = t + 1;
                st_r = n - diag_len;
                st_c = n;
            } else {
                diag_len = 2 * n + 1 - t;
                st_r = -1;
                st_c = diag_len - 1;
            }
            int tmp = 0;
            for (int j = 1; j < diag_len; j++) {
                int r = st_r + j, c = st_c - j;
                if (compat(s[r], s[c])) {
                    tmp++;
                    if (c > r) {
                        if (c - r > 4 && tmp >= l) {
                            l = tmp;
                            p = r - l + 1;
                            q = c;
                            cds = i;
                        }
                    } else if ((r - tmp + 1) > (c + tmp - 1)) {
                        if (((r - tmp + 1) - (c + tmp - 1)) > 4 && tmp >= l) {
                            l = tmp;
                            p = c;
                            q = r - l + 1;
                            cds = i;
                        }
                    } else {
                        tmp = 0;
                    }
                } else {
                    tmp = 0;
                }
            }
        }
    }
    *L_out = l;
    *p_out = p;
    *q_out = q;
    *cds_out = cds;
}

/* Longest repeated or common substring: the LRCS flavour of the string
 * objective.  The reference has no implementation -- it only names MLRCS among
 * the objectives of its experiment scripts (src/auto_execution_experiments.py:45,
 * 215) -- so the definition is this build's own, written as one thread would
 * run it:
 *   over CDS pairs a <= b in the order (0,0), (0,1), .., (0,m-1), (1,1), (1,2), ..,
 *   the longest run of identical nucleotides s_a[r] == s_b[r + delta] along one
 *   diagonal delta of the CDS-a-against-CDS-b matrix; a < b: every delta in
 *   (-n, n) (a common substring); a == b: delta >= 1 (a substring occurring at two
 *   different starts, overlaps allowed).
 * The record is the first pair reaching the maximum, on it the smallest delta,
 * on that diagonal the smallest start p: (length, p, q = p + delta, a, b).  The
 * objective value is length / n (maximised; stored as is, smaller is better). */
void or_lrcs_pair(const uint8_t *sa, const uint8_t *sb, int n, int self, int32_t *out3)
{
    int best = 0, bd = 0, bp = 0;
    for (int delta = self ? 1 : -(n - 1); delta <= n - 1; delta++) {
        int r_lo = delta < 0 ? -delta : 0, r_hi = delta > 0 ? n - 1 - delta : n - 1;
        int run = 0;
        for (int r = r_lo; r <= r_hi; r++) {
            if (sa[r] == sb[r + delta]) {
                run++;
                if (run > best) {
                    best = run;
                    bd = delta;
                    bp = r - run + 1;
                }
            } else {
                run = 0;
            }
        }
    }
    out3[0] = best;
    out3[1] = bd;
    out3[2] = bp;
}

void or_lrcs(const uint8_t *nt, int m, int n, int32_t *out5)
{
    int best = 0, p = 0, q = 0, ba = 0, bb = 0;
    for (int a = 0; a < m; a++)
        for (int b = a; b < m; b++) {
            int32_t r[3];
            or_lrcs_pair(nt + (size_t)a * n, nt + (size_t)b * n, n, a == b, r);
            if (r[0] > best) {
                best = r[0];
                p = r[2];
                q = r[2] + r[1];
                ba = a;
                bb = b;
            }
        }
    out5[0] = best;
    out5[1] = p;
    out5[2] = q;
    out5[3] = ba;
    out5[4] = bb;
}

int or_sl_serial_one(const uint8_t *nt, int n)
{
    int l, p, q, c;
    sl_serial(nt, 1, n, &l, &p, &q, &c);
    return l;
}

/* The same sweep restricted to anti-diagonals t = offset, offset+stride, ...
 * (a bounded sample of the work, for timing). Returns that sample's max run. */
int or_sl_serial_strided(const uint8_t *s, int n, int offset, int stride)
{
    int l = 0;
    for (int t = offset; t < 2 * n + 1; t += stride) {
        int diag_len, st_r, st_c;
        if (t < n + 1) {
            diag_len = t + 1;
            st_r = n - diag_len;
            st_c = n;
        } else {
            diag_len = 2 * n + 1 - t;
            st_r = -1;
            st_c = diag_len - 1;
        }
        int tmp = 0;
        for (int j = 1; j < diag_len; j++) {
            int r = st_r + j, c = st_c - j;
            if (compat(s[r], s[c])) {
                tmp++;
                if (c > r) {
                    if (c - r > 4 && tmp >= l) l = tmp;
                } else if ((r - tmp + 1) > (c + tmp - 1)) {
                    if (((r - tmp + 1) - (c + tmp - 1)) > 4 && tmp >= l) l = tmp;
                } else {
                    tmp = 0;
                }
            } else {
                tmp = 0;
            }
        }
    }
    return l;
}

/* count CDSs (n nucleotides each) swept in parallel on the sampled anti-diagonals */
void or_sl_sample_batch(const uint8_t *nt, int count, int n, int offset, int stride, int threads, int32_t *out)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int i = 0; i < count; i++) out[i] = or_sl_serial_strided(nt + (size_t)i * n, n, offset, stride);
}

static void expand_nt(const or_problem *pr, const uint8_t *sol, uint8_t *nt)
{
    int n = 3 * pr->L;
    for (int i = 0; i < pr->m; i++)
        for (int a = 0; a < pr->L; a++) {
            const uint8_t *cn = pr->tab->nt[sol[i * pr->L + a]];
            nt[(size_t)i * n + 3 * a + 0] = cn[0];
            nt[(size_t)i * n + 3 * a + 1] = cn[1];
            nt[(size_t)i * n + 3 * a + 2] = cn[2];
        }
}

static void eval_impl(const or_problem *pr, const uint8_t *sol, float *obj, int8_t *objidx, int32_t *pql, int with_sl)
{
    const or_codon_table *t = pr->tab;
    const int L = pr->L, m = pr->m, n = 3 * L;
    const int M = or_num_obj(pr->objset);
    memset(objidx, 0, (size_t)2 * M);
    uint8_t *nt = (uint8_t *)malloc((size_t)m * n);
    expand_nt(pr, sol, nt);

    int s;
    /* calMinimumCAI (include/utils.cuh:271-337): -min_i CAI_i, last i on ties.
     * CAI_i = exp(mean log w) from exact fixed-point sums. */
    if ((s = or_slot_of(pr->objset, OR_K_CAI)) >= 0) {
        int64_t lw[OR_NUM_CODON];
        uint8_t zero[OR_NUM_CODON];
        or_log_weight_fixed(t, lw, zero);
        for (int i = 0; i < m; i++) {
            int64_t S = 0;
            int z = 0;
            for (int a = 0; a < L; a++) {
                int c = sol[i * L + a];
                S += lw[c];
                z |= zero[c];
            }
            double x = ((double)S * (1.0 / 4294967296.0)) / (double)L;
            float cai = z ? 0.0f : (float)or_det_exp(x);
            float v = -cai;
            if (i == 0 || v >= obj[s]) {
                obj[s] = v;
                objidx[2 * s] = (int8_t)i;
            }
        }
    }
    /* calMinimumCBP (include/utils.cuh:339-409): mean CPS over pairs a in [0, L-3] */
    if ((s = or_slot_of(pr->objset, OR_K_CBP)) >= 0) {
        for (int i = 0; i < m; i++) {
            int64_t S = 0;
            for (int a = 0; a < L - 2; a++) {
                int c1 = sol[i * L + a], c2 = sol[i * L + a + 1];
                if (c1 < OR_NUM_SENSE && c2 < OR_NUM_SENSE) S += cps_fixed(t->cps[c1 * OR_NUM_SENSE + c2]);
            }
            double x = ((double)S * (1.0 / 4294967296.0)) / (double)(L - 2);
            float v = -(float)x;
            if (i == 0 || v >= obj[s]) {
                obj[s] = v;
                objidx[2 * s] = (int8_t)i;
            }
        }
    }
    /* calMinimumHSC (include/utils.cuh:411-473): hidden stops / (L-1) */
    if ((s = or_slot_of(pr->objset, OR_K_HSC)) >= 0) {
        for (int i = 0; i < m; i++) {
            int cnt = 0;
            for (int a = 0; a < L - 1; a++) cnt += hsc_pair(t, sol[i * L + a], sol[i * L + a + 1]);
            float v = -((float)cnt / (float)(L - 1));
            if (i == 0 || v >= obj[s]) {
                obj[s] = v;
                objidx[2 * s] = (int8_t)i;
            }
        }
    }
    /* calMinimumHD (include/utils.cuh:475-543): min over i<j of mismatches / n */
    if ((s = or_slot_of(pr->objset, OR_K_HD)) >= 0) {
        int first = 1;
        for (int i = 0; i < m - 1; i++)
            for (int j = i + 1; j < m; j++) {
                int cnt = 0;
                for (int b = 0; b < n; b++) cnt += nt[(size_t)i * n + b] != nt[(size_t)j * n + b];
                float v = -((float)cnt / (float)n);
                if (first || v >= obj[s]) {
                    obj[s] = v;
                    objidx[2 * s] = (int8_t)i;
                    objidx[2 * s + 1] = (int8_t)j;
                    first = 0;
                }
            }
    }
    /* calMaximumGC3 (include/utils.cuh:545-626) or calMaximumGC (:628-710) */
    if ((s = or_slot_of(pr->objset, OR_K_GC)) >= 0) {
        for (int i = 0; i < m; i++) {
            float dev, diff;
            if (pr->gcmode == OR_GC3) {
                int cnt = 0;
                for (int a = 0; a < L; a++) {
                    int b = nt[(size_t)i * n + 3 * a + 2];
                    cnt += (b == 1 || b == 2);
                }
                diff = ((float)cnt / (float)L) - t->ref_gc3;
                dev = fabsf(diff);
            } else {
                int cnt = 0;
                for (int b = 0; b < n; b++) cnt += (nt[(size_t)i * n + b] == 1 || nt[(size_t)i * n + b] == 2);
                float refGC = (float)n * t->ref_gc;
                diff = (float)cnt - refGC;
                dev = fabsf(diff) / refGC;
            }
            if (i == 0 || dev >= obj[s]) {
                obj[s] = dev;
                objidx[2 * s] = (int8_t)i;
                objidx[2 * s + 1] = diff < 0 ? 1 : -1; /* GC_UP / GC_DOWN */
            }
        }
    }
    /* longest repeated/common substring in the string slot (see or_lrcs) */
    if ((s = or_slot_of(pr->objset, OR_K_SL)) >= 0 && with_sl && pr->slkind == OR_SL_LRCS) {
        int32_t r[5];
        or_lrcs(nt, m, n, r);
        obj[s] = (float)r[0] / (float)n;
        objidx[2 * s] = (int8_t)r[3];
        objidx[2 * s + 1] = (int8_t)r[4];
        pql[0] = r[1];
        pql[1] = r[2];
        pql[2] = r[0];
    } else
    /* calMaximumSL (include/utils.cuh:712-888) */
    if ((s = or_slot_of(pr->objset, OR_K_SL)) >= 0 && with_sl) {
        int l, p, q, c;
        sl_serial(nt, m, n, &l, &p, &q, &c);
        int K = (n - 4) / 2;
        obj[s] = (float)l / (float)K;
        objidx[2 * s] = (int8_t)c;
        pql[0] = p;
        pql[1] = q;
        pql[2] = l;
    } else {
        pql[0] = pql[1] = pql[2] = 0;
    }
    free(nt);
}

void or_eval(const or_problem *pr, const uint8_t *sol, float *obj, int8_t *objidx, int32_t *pql)
{
    eval_impl(pr, sol, obj, objidx, pql, 1);
}

/* every objective except the hairpin stem (timing sample helper) */
void or_eval_light(const or_problem *pr, const uint8_t *sol, float *obj, int8_t *objidx, int32_t *pql)
{
    eval_impl(pr, sol, obj, objidx, pql, 0);
}

/* ------------------------------------------------------------------------ */
/* mutation operators: include/mutation.cuh:16-969, dispatch src/main.cu:172-211 */
/* ------------------------------------------------------------------------ */

#define DRAW(pos, j) or_draw(pr->seed, TAG_MUT, gen, (uint32_t)idx, (uint32_t)(pos), (uint32_t)(j))
#define PDRAW(pos) or_pdraw(pr->seed, gen, (uint32_t)idx, (uint32_t)(pos))

/* Fisher-Yates as indexArrayShuffling (include/utils.cuh:203-218), draws 1..k-1 */
static void shuffle_idx(const or_problem *pr, uint32_t gen, int idx, int pos, int k, int *arr)
{
    for (int i = 0; i < k; i++) arr[i] = i;
    int d = 1;
    for (int i = k - 1; i > 0; i--) {
        int j = (int)rng_uint(DRAW(pos, d), (uint32_t)(i + 1));
        d++;
        int tmp = arr[i];
        arr[i] = arr[j];
        arr[j] = tmp;
    }
}

static int gc_of_codon(const or_codon_table *t, int c, int gcmode)
{
    if (gcmode == OR_GC3) return t->nt[c][2] == 1 || t->nt[c][2] == 2;
    int g = 0;
    for (int b = 0; b < 3; b++) g += t->nt[c][b] == 1 || t->nt[c][b] == 2;
    return g;
}

/* does the CDS hold a counted stem of length >= K = (n-4)/2 (the only case in
 * which mutationSL's restore branch runs, include/mutation.cuh:843) */
static int full_hairpin(const or_codon_table *t, const uint8_t *cds_codons, int L)
{
    int n = 3 * L, K = (n - 4) / 2;
    if (K <= 0) return 0;
    uint8_t *s = (uint8_t *)malloc((size_t)n);
    for (int a = 0; a < L; a++)
        for (int b = 0; b < 3; b++) s[3 * a + b] = t->nt[cds_codons[a]][b];
    int found = 0;
    for (int ri = K - 1; ri < n && !found; ri++)
        for (int ci = ri + 5; ci + K - 1 <= n - 1 && !found; ci++) {
            int ok = 1;
            for (int u = 0; u < K && ok; u++) ok = compat(s[ri - u], s[ci + u]);
            found = ok;
        }
    free(s);
    return found;
}

int or_mutate(const or_problem *pr, uint32_t gen, int idx, const uint8_t *parent, const float *pobj,
              const int8_t *pobjidx, const int32_t *ppql, uint8_t *child)
{
    const or_codon_table *t = pr->tab;
    const int L = pr->L, m = pr->m;
    const float pm = pr->pm;
    memcpy(child, parent, (size_t)m * L);
    int op;
    {
        uint32_t r = or_draw(pr->seed, TAG_OP, gen, (uint32_t)idx, 0, 0);
        if (pr->objset == OR_OBJSET_REF6) {
            op = (int)rng_uint(r, 7);
        } else {
            static const int map5[5] = {0, 1, 4, 5, 6};
            op = map5[rng_uint(r, 5)];
        }
    }
    switch (op) {
    case 0: /* mutationRandom (include/mutation.cuh:16-63) */
        for (int pos = 0; pos < m * L; pos++) {
            int aa = pr->aa[pos % L];
            int k = t->count[aa];
            if (rng_u01(PDRAW(pos)) > pm || k == 1) continue;
            int cur = child[pos] - t->start[aa];
            int nw = (int)rng_uint(DRAW(pos, 1), (uint32_t)(k - 1));
            if (nw >= cur) nw++;
            child[pos] = (uint8_t)(t->start[aa] + nw);
        }
        break;
    case 1: { /* mutationCAI SELECT_UPPER_RANDOM (include/mutation.cuh:65-142) */
        int c = pobjidx[2 * or_slot_of(pr->objset, OR_K_CAI)];
        for (int a = 0; a < L; a++) {
            int aa = pr->aa[a];
            int k = t->count[aa];
            if (rng_u01(PDRAW(a)) > pm || k == 1) continue;
            int cur = child[c * L + a] - t->start[aa];
            if (cur == k - 1) continue;
            int nw = cur + 1 + (int)rng_uint(DRAW(a, 1), (uint32_t)(k - 1 - cur));
            child[c * L + a] = (uint8_t)(t->start[aa] + nw);
        }
        break;
    }
    case 2: { /* mutationCBP SELECT_UPPER_RANDOM, prob 2Pm, parity gen%2 (:144-262).
               * Position 0 has no left neighbour (the reference reads before the
               * CDS there); its left term is taken as absent. */
        int c = pobjidx[2 * or_slot_of(pr->objset, OR_K_CBP)];
        float pm2 = pm * 2.0f;
        int parity = (int)(gen & 1u);
        const uint8_t *par = parent + (size_t)c * L;
        for (int a = 0; a < L - 1; a++) {
            if ((a % 2) != parity) continue;
            int aa = pr->aa[a];
            int k = t->count[aa];
            if (rng_u01(PDRAW(a)) > pm2 || k == 1) continue;
            int curg = par[a];
            int cur = curg - t->start[aa];
            int left = a > 0 ? par[a - 1] : -1;
            int right = par[a + 1];
            float curs = 0.0f;
            if (left >= 0 && left < OR_NUM_SENSE && curg < OR_NUM_SENSE) curs = t->cps[left * OR_NUM_SENSE + curg];
            if (right < OR_NUM_SENSE && curg < OR_NUM_SENSE) curs += t->cps[curg * OR_NUM_SENSE + right];
            int up[6], nup = 0;
            for (int j = 0; j < k; j++) {
                if (j == cur) continue;
                int g = t->start[aa] + j;
                float ns = 0.0f;
                if (left >= 0 && left < OR_NUM_SENSE && g < OR_NUM_SENSE) ns += t->cps[left * OR_NUM_SENSE + g];
                if (right < OR_NUM_SENSE && g < OR_NUM_SENSE) ns += t->cps[g * OR_NUM_SENSE + right];
                if (ns > curs) up[nup++] = j;
            }
            if (nup > 0) {
                int pick = up[rng_uint(DRAW(a, 1), (uint32_t)nup)];
                child[c * L + a] = (uint8_t)(t->start[aa] + pick);
            }
        }
        break;
    }
    case 3: { /* mutationHSC SELECT_UPPER_RANDOM, prob 2Pm, parity gen%2 (:264-388).
               * Position 0 counts its right side only. */
        int c = pobjidx[2 * or_slot_of(pr->objset, OR_K_HSC)];
        float pm2 = pm * 2.0f;
        int parity = (int)(gen & 1u);
        const uint8_t *par = parent + (size_t)c * L;
        for (int a = 0; a < L; a++) {
            if ((a % 2) != parity) continue;
            int aa = pr->aa[a];
            int k = t->count[aa];
            if (rng_u01(PDRAW(a)) > pm2 || k == 1) continue;
            int cur = par[a] - t->start[aa];
            int hasl = a > 0, hasr = a < L - 1;
            int curs = (hasl ? hsc_pair(t, par[a - 1], par[a]) : 0) + (hasr ? hsc_pair(t, par[a], par[a + 1]) : 0);
            int up[6], nup = 0;
            for (int j = 0; j < k; j++) {
                if (j == cur) continue;
                int g = t->start[aa] + j;
                int ns = (hasl ? hsc_pair(t, par[a - 1], g) : 0) + (hasr ? hsc_pair(t, g, par[a + 1]) : 0);
                if (ns > curs) up[nup++] = j;
            }
            if (nup > 0) {
                int pick = up[rng_uint(DRAW(a, 1), (uint32_t)nup)];
                child[c * L + a] = (uint8_t)(t->start[aa] + pick);
            }
        }
        break;
    }
    case 4: { /* mutationHD (include/mutation.cuh:390-534) */
        int sl = or_slot_of(pr->objset, OR_K_HD);
        int c1 = pobjidx[2 * sl], c2 = pobjidx[2 * sl + 1];
        for (int a = 0; a < L; a++) {
            int aa = pr->aa[a];
            int k = t->count[aa];
            if (rng_u01(PDRAW(a)) > pm || k == 1) continue;
            int arr[6];
            shuffle_idx(pr, gen, idx, a, k, arr);
            const uint8_t *x = t->nt[parent[c1 * L + a]];
            int cur = parent[c1 * L + a] - t->start[aa];
            int cur_pair = 0;
            for (int b = 0; b < 3; b++) cur_pair += x[b] != t->nt[parent[c2 * L + a]][b];
            int cur_m = 127;
            for (int j = 0; j < m; j++) {
                if (j == c1) continue;
                int d = 0;
                for (int b = 0; b < 3; b++) d += x[b] != t->nt[parent[j * L + a]][b];
                if (d < cur_m) cur_m = d;
            }
            int best_pair = -1, best_m = -1, best = -1;
            for (int u = 0; u < k; u++) {
                int sh = arr[u];
                if (sh == cur) continue;
                const uint8_t *y = t->nt[t->start[aa] + sh];
                int np = 0;
                for (int b = 0; b < 3; b++) np += y[b] != t->nt[parent[c2 * L + a]][b];
                int nm = 127;
                for (int j = 0; j < m; j++) {
                    if (j == c1) continue;
                    int d = 0;
                    for (int b = 0; b < 3; b++) d += y[b] != t->nt[parent[j * L + a]][b];
                    if (d < nm) nm = d;
                }
                if (nm > cur_m && nm > best_m) {
                    best_m = nm;
                    best = sh;
                } else if (best_m == -1 && nm == cur_m && np > cur_pair && np > best_pair) {
                    best_pair = np;
                    best = sh;
                }
            }
            if (best_m != -1 || best_pair != -1) child[c1 * L + a] = (uint8_t)(t->start[aa] + best);
        }
        break;
    }
    case 5: { /* mutationGC3 (:536-653) / mutationGC (:655-773) with direction from objidx */
        int sl = or_slot_of(pr->objset, OR_K_GC);
        int c = pobjidx[2 * sl];
        int dir = pobjidx[2 * sl + 1];
        if (dir != 1 && dir != -1) break;
        float prob;
        if (pr->gcmode == OR_GC3) {
            prob = pobj[sl];
        } else {
            float refGC = (float)(3 * L) * t->ref_gc;
            prob = (pobj[sl] * refGC) / (float)L;
        }
        for (int a = 0; a < L; a++) {
            int aa = pr->aa[a];
            int k = t->count[aa];
            if (rng_u01(PDRAW(a)) > prob || k == 1) continue;
            int arr[6];
            shuffle_idx(pr, gen, idx, a, k, arr);
            int curg = parent[c * L + a];
            int cur = curg - t->start[aa];
            int cgc = gc_of_codon(t, curg, pr->gcmode);
            for (int u = 0; u < k; u++) {
                int sh = arr[u];
                if (sh == cur) continue;
                int ngc = gc_of_codon(t, t->start[aa] + sh, pr->gcmode);
                if ((dir == 1 && ngc > cgc) || (dir == -1 && ngc < cgc)) {
                    child[c * L + a] = (uint8_t)(t->start[aa] + sh);
                    break;
                }
            }
        }
        break;
    }
    case 6: { /* mutationSL (include/mutation.cuh:775-969).  Each attempt mutates one
               * codon of the stem's 5' arm with prob Pm (new index drawn from
               * [0,k-2], bumped by one when equal to the current one), re-scans
               * the CDS and keeps the change when the parent's SL value exceeds
               * (l' / ((n-4)/2)) in integer division; otherwise it is undone.  The
               * reference restores the r-side attempt into the l-side codon and
               * writes an unset buffer when nothing was mutated; here the attempted
               * codon itself is restored. */
        int sl = or_slot_of(pr->objset, OR_K_SL);
        if (pr->slkind == OR_SL_LRCS) {
            /* LRCS flavour (no reference counterpart): walk outward from the middle
             * codon of the repeat's second occurrence (CDS b, nucleotides q .. q+l-1),
             * mutating each codon with prob Pm (draws as above), and stop at the
             * first codon changed */
            int b = pobjidx[2 * sl + 1], q = ppql[1], l = ppql[2];
            if (l <= 0 || q < 0 || b < 0 || b >= pr->m) break;
            int a0 = q / 3, a1 = (q + l - 1) / 3, mid = (a0 + a1) / 2;
            uint8_t *cds = child + (size_t)b * L;
            int attempt = 0;
            for (int u = 0; u <= 2 * (a1 - a0); u++) {
                int a = (u & 1) ? mid - (u + 1) / 2 : mid + u / 2;
                if (a < a0 || a > a1 || a >= L) continue;
                int aa = pr->aa[a];
                int k = t->count[aa];
                uint32_t r0 = or_draw(pr->seed, TAG_SLMUT, gen, (uint32_t)idx, (uint32_t)attempt, 0);
                uint32_t r1 = or_draw(pr->seed, TAG_SLMUT, gen, (uint32_t)idx, (uint32_t)attempt, 1);
                attempt++;
                if (rng_u01(r0) <= pm && k > 1) {
                    int cur = cds[a] - t->start[aa];
                    int nw = (int)rng_uint(r1, (uint32_t)(k - 1));
                    if (nw == cur) nw++;
                    cds[a] = (uint8_t)(t->start[aa] + nw);
                    break;
                }
            }
            break;
        }
        int c = pobjidx[2 * sl];
        float v = pobj[sl];
        int n = 3 * L, K = (n - 4) / 2;
        int P = ppql[0], Ls = ppql[2];
        int l_idx = P / 3;
        int r_idx = (P + Ls - 1) / 3;
        int mid = (r_idx + l_idx) / 2;
        int stem = r_idx - l_idx + 1;
        int half = stem / 2;
        int odd = (stem % 2) == 1;
        int l_st = odd ? mid - 1 : mid, r_st = mid + 1;
        uint8_t *cds = child + (size_t)c * L;
        int attempt = 0;
        int positions[1 + 2 * 4096];
        int npos = 0;
        if (odd) positions[npos++] = mid;
        for (int i = 1; i <= half && npos + 2 <= (int)(sizeof positions / sizeof positions[0]); i++) {
            positions[npos++] = l_st--;
            positions[npos++] = r_st++;
        }
        for (int u = 0; u < npos; u++) {
            int a = positions[u];
            if (a < 0 || a >= L) break;
            int aa = pr->aa[a];
            int k = t->count[aa];
            uint32_t r0 = or_draw(pr->seed, TAG_SLMUT, gen, (uint32_t)idx, (uint32_t)attempt, 0);
            uint32_t r1 = or_draw(pr->seed, TAG_SLMUT, gen, (uint32_t)idx, (uint32_t)attempt, 1);
            attempt++;
            int old = cds[a];
            int mutated = 0;
            if (rng_u01(r0) <= pm && k > 1) {
                int cur = old - t->start[aa];
                int nw = (int)rng_uint(r1, (uint32_t)(k - 1));
                if (nw == cur) nw++;
                cds[a] = (uint8_t)(t->start[aa] + nw);
                mutated = 1;
            }
            int lprime_ge_K = full_hairpin(t, cds, L);
            float thr = (float)(lprime_ge_K ? 1 : 0);
            if (K > 0 && v > thr) break; /* TERMINATION: keep */
            if (mutated) cds[a] = (uint8_t)old;
        }
        break;
    }
    }
    return op;
}

/* ------------------------------------------------------------------------ */
/* selection: include/sorting.cuh:94-1282                                   */
/* ------------------------------------------------------------------------ */

static int dominate(const float *a, const float *b, int M)
{
    /* dominate (include/sorting.cuh:94-130): |a-b| <= 1e-6 counts as equal */
    int eq = 0, differs[OR_MAX_OBJ];
    for (int k = 0; k < M; k++) {
        if (fabsf(a[k] - b[k]) > 1e-6f) differs[k] = 1;
        else { differs[k] = 0; eq++; }
    }
    if (eq == M) return 0;
    for (int k = 0; k < M; k++)
        if (differs[k] && a[k] > b[k]) return 0;
    return 1;
}

/* findMinValue tree order (include/utils.cuh:1173-1213) over a buffer of B
 * entries: position t keeps its entry unless t+i is strictly smaller. */
static int tree_argmin(float *buf, int *ix, int B)
{
    int i = B / 2;
    while (1) {
        for (int t = 0; t < i; t++)
            if (buf[t + i] < buf[t]) {
                buf[t] = buf[t + i];
                ix[t] = ix[t + i];
            }
        if (i == 1) break;
        if ((i % 2) == 1 && buf[i - 1] < buf[0]) {
            buf[0] = buf[i - 1];
            ix[0] = ix[i - 1];
        }
        i /= 2;
    }
    return ix[0];
}

static float asf(const float *x, const float *ideal, const float *w, int M)
{
    /* ASF (include/sorting.cuh:428-449) */
    float mx = -FLT_MAX;
    for (int k = 0; k < M; k++) {
        float tmp = x[k] - ideal[k];
        if ((double)tmp < 0.001) tmp = 0.0f;
        float q = tmp / w[k];
        if (q > mx) mx = q;
    }
    return mx;
}

int or_select(const or_problem *pr, uint32_t gen, const float *obj, float *ext, const float *refpts, int R,
              int32_t *survivors, int32_t *front, or_select_info *info)
{
    const int N = pr->N, N2 = 2 * N;
    const int M = or_num_obj(pr->objset);
    memset(info, 0, sizeof *info);

    /* ---- nonDominatedSorting (include/sorting.cuh:974-1089), fronts listed in
     * ascending solution index (the reference appends with atomicAdd) ---- */
    int *np = (int *)calloc((size_t)N2, sizeof(int));
    int32_t *sorted_all = (int32_t *)malloc(sizeof(int32_t) * (size_t)N2);
    uint8_t *dom = (uint8_t *)malloc((size_t)N2 * N2); /* dom[j*N2+i]: j dominates i */
    for (int j = 0; j < N2; j++)
        for (int i = 0; i < N2; i++) {
            uint8_t d = (i != j) && dominate(obj + (size_t)j * M, obj + (size_t)i * M, M);
            dom[(size_t)j * N2 + i] = d;
            np[i] += d;
        }
    for (int i = 0; i < N2; i++) front[i] = -1;
    int rc = 0, cur_front = 0, f0 = 0;
    for (int i = 0; i < N2; i++)
        if (np[i] == 0) {
            front[i] = 0;
            sorted_all[rc++] = i;
        }
    f0 = rc;
    int front_start = 0, front_size = rc;
    int cut = 0;
    if (rc == N) {
        cut = 1;
    } else if (rc < N) {
        for (int it = 0; it < N2 - 1; it++) {
            cur_front++;
            int prev_start = front_start, prev_end = front_start + front_size;
            front_start = rc;
            for (int i = 0; i < N2; i++) {
                if (front[i] >= 0) continue;
                int dec = 0;
                for (int u = prev_start; u < prev_end; u++) dec += dom[(size_t)sorted_all[u] * N2 + i];
                np[i] -= dec;
                if (np[i] == 0) {
                    front[i] = cur_front;
                    sorted_all[rc++] = i;
                }
            }
            front_size = rc - front_start;
            if (rc >= N) {
                cut = rc == N;
                break;
            }
        }
    }
    int last_size = front_size; /* size of front cur_front */
    info->rank_count = rc;
    info->last_front_size = last_size;
    info->n_fronts = cur_front + 1;
    info->cut = cut;

    /* ---- updateIdealValue / updateWorstValue (:132-426) ---- */
    float ideal[OR_MAX_OBJ], worst[OR_MAX_OBJ], nadir[OR_MAX_OBJ];
    for (int k = 0; k < M; k++) {
        float mn = FLT_MAX, mx = -FLT_MAX;
        for (int i = 0; i < N2; i++) {
            float v = obj[(size_t)i * M + k];
            if (v < mn) mn = v;
            if (v > mx) mx = v;
        }
        ideal[k] = mn;
        worst[k] = mx;
    }

    /* ---- updateNadirValue_HYP (:911-972): findExtremePoints (:601-683) ---- */
    {
        int B = N2 + M;
        float *buf = (float *)malloc(sizeof(float) * (size_t)B);
        int *ix = (int *)malloc(sizeof(int) * (size_t)B);
        for (int i = 0; i < M; i++) {
            float w[OR_MAX_OBJ];
            for (int j = 0; j < M; j++) w[j] = (i == j) ? 1.0f : 1e-6f;
            for (int t = 0; t < B; t++) {
                buf[t] = FLT_MAX;
                ix[t] = -1;
            }
            for (int t = 0; t < f0 + M; t++) {
                if (t < f0) {
                    buf[t] = asf(obj + (size_t)sorted_all[t] * M, ideal, w, M);
                    ix[t] = sorted_all[t];
                } else {
                    buf[t] = asf(ext + (size_t)(t - f0) * M, ideal, w, M);
                    ix[t] = N2 + (t - f0);
                }
            }
            int sel = tree_argmin(buf, ix, B);
            if (sel >= N2) {
                float tmp[OR_MAX_OBJ];
                memcpy(tmp, ext + (size_t)(sel - N2) * M, sizeof(float) * M);
                memcpy(ext + (size_t)i * M, tmp, sizeof(float) * M);
            } else if (sel >= 0) {
                memcpy(ext + (size_t)i * M, obj + (size_t)sel * M, sizeof(float) * M);
            }
        }
        free(buf);
        free(ix);
    }
    /* GaussianElimination (:555-599) on [E | 1], sequential order */
    float AB[OR_MAX_OBJ][OR_MAX_OBJ + 1], x[OR_MAX_OBJ];
    for (int i = 0; i < M; i++) {
        for (int j = 0; j < M; j++) AB[i][j] = ext[i * M + j];
        AB[i][M] = 1.0f;
    }
    for (int c = 0; c < M; c++) {
        if ((double)fabsf(AB[c][c]) <= 1e-6) {
            int r = c;
            while (r < M && !((double)fabsf(AB[r][c]) > 1e-6)) r++;
            if (r < M)
                for (int j = c; j <= M; j++) AB[c][j] += AB[r][j];
        }
        for (int r = c + 1; r < M; r++) {
            float f = AB[r][c] / AB[c][c];
            for (int j = c; j <= M; j++) {
                float prod = f * AB[c][j];
                AB[r][j] -= prod;
            }
        }
    }
    for (int r = M - 1; r >= 0; r--) {
        float s = 0.0f;
        for (int j = r + 1; j < M; j++) {
            float prod = AB[r][j] * x[j];
            s += prod;
        }
        x[r] = (AB[r][M] - s) / AB[r][r];
    }
    int exc = 0;
    float intercept[OR_MAX_OBJ];
    for (int k = 0; k < M; k++) {
        float res = 0.0f;
        for (int i = 0; i < M; i++) {
            float d = ext[k * M + i] - ideal[i];
            float prod = x[i] * d;
            res += prod;
        }
        if (fabsf(res - 1.0f) > 1e-6f || isnan(res) || isinf(res)) exc = 1;
        intercept[k] = 1.0f / x[k];
        if (intercept[k] <= 1e-6f || isnan(intercept[k]) || isinf(intercept[k])) exc = 1;
    }
    if (!exc) {
        for (int k = 0; k < M; k++) nadir[k] = ideal[k] + intercept[k];
    } else {
        /* updateNadirValue_MNDF (:685-884): max over front 0, worst if too close */
        for (int k = 0; k < M; k++) {
            float mx = -FLT_MAX;
            for (int t = 0; t < f0; t++) {
                float v = obj[(size_t)sorted_all[t] * M + k];
                if (v > mx) mx = v;
            }
            nadir[k] = (mx - ideal[k]) > 1e-6f ? mx : worst[k];
        }
    }
    info->hyp_exception = exc;
    memcpy(info->ideal, ideal, sizeof(float) * M);
    memcpy(info->worst, worst, sizeof(float) * M);
    memcpy(info->nadir, nadir, sizeof(float) * M);

    if (cut) {
        memcpy(survivors, sorted_all, sizeof(int32_t) * (size_t)N);
        free(np);
        free(sorted_all);
        free(dom);
        return 0;
    }

    /* ---- referenceBasedSorting (:1091-1282) ---- */
    int count = rc - last_size;
    int *rho = (int *)calloc((size_t)R, sizeof(int));
    int *ncand = (int *)calloc((size_t)R, sizeof(int));
    int *assoc = (int *)malloc(sizeof(int) * (size_t)rc);
    float *dist = (float *)malloc(sizeof(float) * (size_t)N2);
    for (int t = 0; t < rc; t++) {
        int sol = sorted_all[t];
        float f[OR_MAX_OBJ];
        for (int k = 0; k < M; k++) f[k] = (obj[(size_t)sol * M + k] - ideal[k]) / (nadir[k] - ideal[k]);
        float best = FLT_MAX;
        int bj = 0;
        for (int j = 0; j < R; j++) {
            /* perpendicularDistance (include/utils.cuh:1149-1171) */
            const float *w = refpts + (size_t)j * M;
            float num = 0.0f, den = 0.0f;
            for (int k = 0; k < M; k++) {
                float a = w[k] * f[k];
                num += a;
                float b = w[k] * w[k];
                den += b;
            }
            float kk = num / den;
            float d2 = 0.0f;
            for (int k = 0; k < M; k++) {
                float pk = kk * w[k];
                float e = pk - f[k];
                float e2 = e * e;
                d2 += e2;
            }
            float d = sqrtf(d2);
            if (d < best) {
                best = d;
                bj = j;
            }
        }
        dist[sol] = best;
        assoc[t] = bj;
        if (t < count) rho[bj]++;
        else ncand[bj]++;
    }
    /* candidate lists (CSR), each in ascending position order */
    int *off = (int *)malloc(sizeof(int) * (size_t)(R + 1));
    off[0] = 0;
    for (int j = 0; j < R; j++) off[j + 1] = off[j] + ncand[j];
    int *cand = (int *)malloc(sizeof(int) * (size_t)(off[R] > 0 ? off[R] : 1));
    int *fill = (int *)calloc((size_t)R, sizeof(int));
    for (int t = count; t < rc; t++) {
        int j = assoc[t];
        cand[off[j] + fill[j]++] = sorted_all[t];
    }
    memcpy(survivors, sorted_all, sizeof(int32_t) * (size_t)count);
    for (int level = 0; count < N; level++) {
        for (int j = 0; j < R && count < N; j++) {
            if (rho[j] != level || ncand[j] <= 0) continue;
            int *cl = cand + off[j];
            int slot = 0;
            if (level == 0) {
                float bd = dist[cl[0]];
                for (int u = 1; u < ncand[j]; u++)
                    if (dist[cl[u]] < bd) {
                        bd = dist[cl[u]];
                        slot = u;
                    }
            } else {
                uint32_t r = or_draw(pr->seed, TAG_NICHE, gen, (uint32_t)j, (uint32_t)level, 0);
                slot = (int)rng_uint(r, (uint32_t)ncand[j]);
            }
            survivors[count++] = cl[slot];
            rho[j]++;
            ncand[j]--;
            cl[slot] = cl[ncand[j]];
        }
        if (level >= N2 + 2) break; /* cannot happen: candidates run out first */
    }
    free(rho);
    free(ncand);
    free(assoc);
    free(dist);
    free(off);
    free(cand);
    free(fill);
    free(np);
    free(sorted_all);
    free(dom);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* whole runs: src/main.cu:700-787 (ping-pong populations, survivors)         */
/* ------------------------------------------------------------------------ */

struct or_state {
    or_problem pr;
    int M, R;
    float *refpts;
    uint8_t *pop[2];
    float *obj[2];
    int8_t *objidx[2];
    int32_t *pql[2];
    int32_t *surv;
    int32_t *front;
    float ext[OR_MAX_OBJ * OR_MAX_OBJ];
    uint32_t gen;
    int cur;
};

or_state *or_create(const or_problem *pr)
{
    or_state *st = (or_state *)calloc(1, sizeof *st);
    st->pr = *pr;
    st->M = or_num_obj(pr->objset);
    st->R = or_num_ref(st->M, pr->p);
    st->refpts = (float *)malloc(sizeof(float) * (size_t)st->R * st->M);
    or_das_dennis(st->M, pr->p, st->refpts);
    size_t N2 = 2 * (size_t)pr->N, sl = (size_t)pr->m * pr->L;
    for (int b = 0; b < 2; b++) {
        st->pop[b] = (uint8_t *)calloc(N2 * sl, 1);
        st->obj[b] = (float *)calloc(N2 * st->M, sizeof(float));
        st->objidx[b] = (int8_t *)calloc(N2 * 2 * st->M, 1);
        st->pql[b] = (int32_t *)calloc(N2 * 3, sizeof(int32_t));
    }
    st->surv = (int32_t *)calloc((size_t)pr->N, sizeof(int32_t));
    st->front = (int32_t *)calloc(N2, sizeof(int32_t));
    return st;
}

void or_destroy(or_state *st)
{
    if (!st) return;
    free(st->refpts);
    for (int b = 0; b < 2; b++) {
        free(st->pop[b]);
        free(st->obj[b]);
        free(st->objidx[b]);
        free(st->pql[b]);
    }
    free(st->surv);
    free(st->front);
    free(st);
}

static void set_threads(int threads)
{
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

void or_init(or_state *st, int threads)
{
    /* initializationKernel (src/main.cu:26-119) */
    const or_problem *pr = &st->pr;
    size_t sl = (size_t)pr->m * pr->L;
    int M = st->M;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < pr->N; i++) {
        or_gen_solution(pr, i, st->pop[0] + (size_t)i * sl);
        or_eval(pr, st->pop[0] + (size_t)i * sl, st->obj[0] + (size_t)i * M, st->objidx[0] + (size_t)i * 2 * M,
                st->pql[0] + (size_t)i * 3);
    }
    for (int i = 0; i < pr->N; i++) st->surv[i] = i;
    memset(st->ext, 0, sizeof st->ext);
    for (int k = 0; k < M && k < pr->N; k++) memcpy(st->ext + k * M, st->obj[0] + (size_t)k * M, sizeof(float) * M);
    st->gen = 0;
    st->cur = 0;
}

void or_generation(or_state *st, int threads)
{
    const or_problem *pr = &st->pr;
    const int N = pr->N, M = st->M;
    size_t sl = (size_t)pr->m * pr->L;
    int src = st->cur, dst = 1 - st->cur;
    uint32_t gen = st->gen;
    set_threads(threads);
    /* mutationKernel (src/main.cu:121-240) */
#pragma omp parallel for schedule(dynamic, 1)
    for (int idx = 0; idx < N; idx++) {
        int par = st->surv[idx];
        const uint8_t *ps = st->pop[src] + (size_t)par * sl;
        memcpy(st->pop[dst] + (size_t)idx * sl, ps, sl);
        memcpy(st->obj[dst] + (size_t)idx * M, st->obj[src] + (size_t)par * M, sizeof(float) * M);
        memcpy(st->objidx[dst] + (size_t)idx * 2 * M, st->objidx[src] + (size_t)par * 2 * M, (size_t)2 * M);
        memcpy(st->pql[dst] + (size_t)idx * 3, st->pql[src] + (size_t)par * 3, sizeof(int32_t) * 3);
        size_t ch = (size_t)(N + idx);
        or_mutate(pr, gen, idx, ps, st->obj[src] + (size_t)par * M, st->objidx[src] + (size_t)par * 2 * M,
                  st->pql[src] + (size_t)par * 3, st->pop[dst] + ch * sl);
        or_eval(pr, st->pop[dst] + ch * sl, st->obj[dst] + ch * M, st->objidx[dst] + ch * 2 * M, st->pql[dst] + ch * 3);
    }
    /* sortingKernel (src/main.cu:409-454) */
    or_select_info info;
    or_select(pr, gen, st->obj[dst], st->ext, st->refpts, st->R, st->surv, st->front, &info);
    st->gen = gen + 1;
    st->cur = dst;
}

void or_get(const or_state *st, uint8_t *pop, float *obj, int8_t *objidx, int32_t *pql, int32_t *survivors,
            float *extremes, uint32_t *gen)
{
    const or_problem *pr = &st->pr;
    size_t N2 = 2 * (size_t)pr->N, sl = (size_t)pr->m * pr->L;
    int b = st->cur;
    if (pop) memcpy(pop, st->pop[b], N2 * sl);
    if (obj) memcpy(obj, st->obj[b], N2 * st->M * sizeof(float));
    if (objidx) memcpy(objidx, st->objidx[b], N2 * 2 * st->M);
    if (pql) memcpy(pql, st->pql[b], N2 * 3 * sizeof(int32_t));
    if (survivors) memcpy(survivors, st->surv, sizeof(int32_t) * (size_t)pr->N);
    if (extremes) memcpy(extremes, st->ext, sizeof(float) * st->M * st->M);
    if (gen) *gen = st->gen;
}

void or_eval_batch(const or_problem *pr, const uint8_t *sols, int n, float *obj, int8_t *objidx, int32_t *pql,
                   int threads)
{
    int M = or_num_obj(pr->objset);
    size_t sl = (size_t)pr->m * pr->L;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; i++)
        or_eval(pr, sols + (size_t)i * sl, obj + (size_t)i * M, objidx + (size_t)i * 2 * M, pql + (size_t)i * 3);
}

void or_mutate_eval_batch(const or_problem *pr, uint32_t gen, const int32_t *idx, int n, const uint8_t *parents,
                          const float *pobj, const int8_t *pobjidx, const int32_t *ppql, uint8_t *child, float *cobj,
                          int8_t *cobjidx, int32_t *cpql, int32_t *ops, int threads)
{
    int M = or_num_obj(pr->objset);
    size_t sl = (size_t)pr->m * pr->L;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; i++) {
        int op = or_mutate(pr, gen, idx[i], parents + (size_t)i * sl, pobj + (size_t)i * M, pobjidx + (size_t)i * 2 * M,
                           ppql + (size_t)i * 3, child + (size_t)i * sl);
        if (ops) ops[i] = op;
        or_eval(pr, child + (size_t)i * sl, cobj + (size_t)i * M, cobjidx + (size_t)i * 2 * M, cpql + (size_t)i * 3);
    }
}

void or_mutate_eval_light_batch(const or_problem *pr, uint32_t gen, const int32_t *idx, int n, const uint8_t *parents,
                                 const float *pobj, const int8_t *pobjidx, const int32_t *ppql, uint8_t *child,
                                 float *cobj, int8_t *cobjidx, int32_t *cpql, int threads)
{
    int M = or_num_obj(pr->objset);
    size_t sl = (size_t)pr->m * pr->L;
    set_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; i++) {
        or_mutate(pr, gen, idx[i], parents + (size_t)i * sl, pobj + (size_t)i * M, pobjidx + (size_t)i * 2 * M,
                  ppql + (size_t)i * 3, child + (size_t)i * sl);
        or_eval_light(pr, child + (size_t)i * sl, cobj + (size_t)i * M, cobjidx + (size_t)i * 2 * M, cpql + (size_t)i * 3);
    }
}

/* ------------------------------------------------------------------------ */
/* exact hypervolume (minimisation, reference point r): recursive slicing    */
/* over the last objective with non-dominated filtering of each slice         */
/* (the HSO scheme of While et al., IEEE TEC 2006).                           */
/* ------------------------------------------------------------------------ */

static int dominates_or_eq(const double *a, const double *b, int d)
{
    for (int k = 0; k < d; k++)
        if (a[k] > b[k]) return 0;
    return 1;
}

static int nd_filter(double *pts, int n, int d)
{
    /* keep points not weakly dominated by another kept point (duplicates: keep one) */
    int out = 0;
    for (int i = 0; i < n; i++) {
        int dominated = 0;
        for (int j = 0; j < n && !dominated; j++) {
            if (j == i) continue;
            if (dominates_or_eq(pts + (size_t)j * d, pts + (size_t)i * d, d)) {
                int equal = 1;
                for (int k = 0; k < d; k++)
                    if (pts[(size_t)j * d + k] != pts[(size_t)i * d + k]) { equal = 0; break; }
                if (!equal || j < i) dominated = 1;
            }
        }
        if (!dominated) {
            if (out != i) memmove(pts + (size_t)out * d, pts + (size_t)i * d, sizeof(double) * d);
            out++;
        }
    }
    return out;
}

static int cmp_last;
static int cmp_by_last(const void *a, const void *b)
{
    double x = ((const double *)a)[cmp_last], y = ((const double *)b)[cmp_last];
    return (x > y) - (x < y);
}

static double hv_rec(double *pts, int n, int d, const double *ref)
{
    if (n == 0) return 0.0;
    if (d == 1) {
        double mn = pts[0];
        for (int i = 1; i < n; i++) if (pts[i] < mn) mn = pts[i];
        return ref[0] > mn ? ref[0] - mn : 0.0;
    }
    if (d == 2) {
        /* sort by x ascending; area = sum over strips [x_i, x_{i+1}) of (r_y - min y so far) */
        double *q = (double *)malloc(sizeof(double) * 2 * (size_t)n);
        memcpy(q, pts, sizeof(double) * 2 * (size_t)n);
        cmp_last = 0;
        qsort(q, (size_t)n, sizeof(double) * 2, cmp_by_last);
        double vol = 0.0, miny = ref[1];
        for (int i = 0; i < n; i++) {
            double x = q[2 * i];
            if (x >= ref[0]) break;
            if (q[2 * i + 1] < miny) miny = q[2 * i + 1];
            double xn = (i + 1 < n && q[2 * (i + 1)] < ref[0]) ? q[2 * (i + 1)] : ref[0];
            if (miny < ref[1]) vol += (xn - x) * (ref[1] - miny);
        }
        free(q);
        return vol;
    }
    /* slice along the last objective */
    double *q = (double *)malloc(sizeof(double) * (size_t)n * d);
    memcpy(q, pts, sizeof(double) * (size_t)n * d);
    cmp_last = d - 1;
    qsort(q, (size_t)n, sizeof(double) * (size_t)d, cmp_by_last);
    double vol = 0.0;
    double *slice = (double *)malloc(sizeof(double) * (size_t)n * (d - 1));
    for (int i = 0; i < n; i++) {
        double z = q[(size_t)i * d + d - 1];
        if (z >= ref[d - 1]) break;
        double zn = (i + 1 < n && q[(size_t)(i + 1) * d + d - 1] < ref[d - 1]) ? q[(size_t)(i + 1) * d + d - 1] : ref[d - 1];
        if (zn <= z) continue;
        for (int j = 0; j <= i; j++) memcpy(slice + (size_t)j * (d - 1), q + (size_t)j * d, sizeof(double) * (d - 1));
        int ns = nd_filter(slice, i + 1, d - 1);
        vol += (zn - z) * hv_rec(slice, ns, d - 1, ref);
        cmp_last = d - 1;
    }
    free(slice);
    free(q);
    return vol;
}

double or_hypervolume(const double *pts, int n, int d, const double *ref)
{
    double *q = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1) * d);
    int k = 0;
    for (int i = 0; i < n; i++) {
        int inside = 1;
        for (int j = 0; j < d; j++)
            if (!(pts[(size_t)i * d + j] < ref[j])) inside = 0;
        if (inside) memcpy(q + (size_t)(k++) * d, pts + (size_t)i * d, sizeof(double) * d);
    }
    k = nd_filter(q, k, d);
    double v = hv_rec(q, k, d, ref);
    free(q);
    return v;
}

/* ------------------------------------------------------------------------ */
/* synthetic benchmark inputs, restated so that the CPU baseline never loads */
/* the engine library: SplitMix64 draws, amino acids uniform over the 20     */
/* standard letters plus the appended stop (src/main.cu:517 appends 'Z'),    */
/* codon weights Dirichlet(1) per amino acid scaled to max 1 and ordered     */
/* ascending inside each group (the reference treats the last synonymous     */
/* codon as the best one, include/utils.cuh:1090, include/mutation.cuh:105).  */
/* Both must equal the engine's pe_synthetic_protein / pe_dirichlet_table     */
/* draw for draw (a CPU test compares them).                                  */
/* ------------------------------------------------------------------------ */

static uint64_t or_splitmix64(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

void or_synthetic_protein(int L, uint64_t seed, int8_t *aa_out)
{
    uint64_t x = seed;
    for (int i = 0; i < L; i++) aa_out[i] = (int8_t)(((or_splitmix64(&x) >> 32) * 20ull) >> 32);
    aa_out[L] = 20;
}

void or_dirichlet_table(uint64_t seed, or_codon_table *out)
{
    /* standard genetic code grouped by amino acid in index order A C D E F G H I K L M N P Q R S T V W Y stop */
    static const char *groups[21] = {"GCU GCC GCA GCG", "UGU UGC", "GAU GAC", "GAA GAG", "UUU UUC",
                                     "GGU GGC GGA GGG", "CAU CAC", "AUU AUC AUA", "AAA AAG",
                                     "UUA UUG CUU CUC CUA CUG", "AUG", "AAU AAC", "CCU CCC CCA CCG", "CAA CAG",
                                     "CGU CGC CGA CGG AGA AGG", "UCU UCC UCA UCG AGU AGC", "ACU ACC ACA ACG",
                                     "GUU GUC GUA GUG", "UGG", "UAU UAC", "UAA UAG UGA"};
    memset(out, 0, sizeof *out);
    uint64_t x = seed;
    int id = 0;
    for (int a = 0; a < 21; a++) {
        const char *g = groups[a];
        int k = (int)(strlen(g) + 1) / 4;
        uint8_t base[6][3];
        for (int j = 0; j < k; j++)
            for (int b = 0; b < 3; b++) {
                char c = g[4 * j + b];
                base[j][b] = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : 3;
            }
        double gam[6], gmax = 0.0;
        for (int j = 0; j < k; j++) {
            double u = (double)((or_splitmix64(&x) >> 11) + 1) * (1.0 / 9007199254740992.0);
            gam[j] = -log(u);
            if (gam[j] > gmax) gmax = gam[j];
        }
        float w[6];
        int order[6];
        for (int j = 0; j < k; j++) {
            w[j] = (float)(gam[j] / gmax);
            order[j] = j;
        }
        for (int j = 1; j < k; j++) { /* stable insertion sort, ascending weight */
            int o = order[j], t = j;
            while (t > 0 && w[order[t - 1]] > w[o]) {
                order[t] = order[t - 1];
                t--;
            }
            order[t] = o;
        }
        out->start[a] = (int8_t)id;
        out->count[a] = (int8_t)k;
        for (int j = 0; j < k; j++) {
            memcpy(out->nt[id + j], base[order[j]], 3);
            out->weight[id + j] = w[order[j]];
        }
        id += k;
    }
    for (int i = 0; i < OR_NUM_SENSE * OR_NUM_SENSE; i++) {
        double u = (double)(or_splitmix64(&x) >> 11) * (1.0 / 9007199254740992.0);
        out->cps[i] = (float)(0.8 * u - 0.4);
    }
    out->ref_gc3 = 0.3810f;
    out->ref_gc = 0.3977f;
}

/* Load a 2N state (e.g. the CUDA engine's current population) so that the
 * next or_generation starts from it. */
void or_set_state(or_state *st, const uint8_t *pop, const float *obj, const int8_t *objidx, const int32_t *pql,
                  const int32_t *survivors, const float *extremes, uint32_t gen)
{
    const or_problem *pr = &st->pr;
    size_t N2 = 2 * (size_t)pr->N, sl = (size_t)pr->m * pr->L;
    int b = st->cur;
    memcpy(st->pop[b], pop, N2 * sl);
    memcpy(st->obj[b], obj, N2 * st->M * sizeof(float));
    memcpy(st->objidx[b], objidx, N2 * 2 * st->M);
    memcpy(st->pql[b], pql, N2 * 3 * sizeof(int32_t));
    memcpy(st->surv, survivors, sizeof(int32_t) * (size_t)pr->N);
    memcpy(st->ext, extremes, sizeof(float) * st->M * st->M);
    st->gen = gen;
}
