// pe_internal.h -- internal types shared by the engine's translation units.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pe_nsga3.h"

namespace pe {

// objective kinds in the reference's REF6 slot order (include/common.cuh:23-29)
enum Kind { K_CAI = 0, K_CBP = 1, K_HSC = 2, K_HD = 3, K_GC = 4, K_SL = 5 };

constexpr int kMaxObj = 6;
constexpr int kMaxCds = 64;          // objidx stores CDS indices as int8
constexpr int kSlThreadsMax = 256;   // largest stem-scan CTA (sizes 64, 128, 256)
constexpr int kVarThreads = 256;     // variation / light-eval CTA
constexpr int kSelThreads = 1024;    // selection CTA
constexpr int kSlGuardRows = 8;      // zero guard rows around the shifted T copies

// RNG stream tags (Philox counter word 0)
constexpr uint32_t TAG_INIT = 1u, TAG_OP = 2u, TAG_MUT = 3u, TAG_SLMUT = 4u, TAG_NICHE = 5u, TAG_MUTP = 6u;

// Problem shape, passed by value to every kernel.
struct Shape {
    int L;        // amino-acid positions incl. stop
    int Lp;       // codon-id row stride (L rounded up to 16)
    int m;        // CDSs per solution
    int N;        // population
    int M;        // objectives
    int n;        // nucleotides per CDS (3L)
    int W;        // 32-bit words per nucleotide plane
    int Wp;       // plane row stride in uint2 (W + 1 zero guard, rounded to even)
    int K;        // (n-4)/2, the stem normaliser
    int R;        // reference points
    int objset, gcmode;
    float pm;
    uint64_t seed;
    int slot[6];  // slot of each Kind or -1
    int sl_threads;  // stem-scan CTA size (64, 128 or 256; 0 = 128), picked per instance by timing
    int sl_kind;     // string objective: PE_SL_HAIRPIN or PE_SL_LRCS
    int nres;        // string-objective results per solution: m CDSs (hairpin) or m(m+1)/2 CDS pairs (LRCS)
    int wait_limit;  // polls of a bounded device wait: 0 = the default, < 0 = give up at once (tests)
    int naux;        // int32 words of per-CDS sums per solution: AUX_HD(m) + m(m-1)/2
    int sl_method;   // first pass of the string scan: 0 seeded (word table) where the CDS fits, 1 band scan
};

// Per-solution sums of the light objectives (PopBuf.aux), int32 words: per CDS c the
// CAI value bits, the CBP fixed-point sum (low and high halves), the HSC count and
// the GC count; then the HD mismatch count of every CDS pair (i < j, row-major).
#define AUX_CAI(m) 0
#define AUX_CBP_LO(m) (m)
#define AUX_CBP_HI(m) (2 * (m))
#define AUX_HSC(m) (3 * (m))
#define AUX_GC(m) (4 * (m))
#define AUX_HD(m) (5 * (m))

// polls of a bounded device wait before it gives up and reports PE_ERR_TIMEOUT
__host__ __device__ __forceinline__ int wait_polls(int wait_limit)
{
    return wait_limit > 0 ? wait_limit : (wait_limit < 0 ? 0 : (1 << 22));
}

// Device-resident tables derived from pe_codon_table.
struct DevTables {
    uint8_t nt[64][4];       // nucleotide codes
    int64_t lw[64];          // log w in 2^-32 fixed point
    uint8_t wzero[64];       // w == 0
    uint8_t gc3[64];         // third nucleotide is C or G
    uint8_t gcn[64];         // number of C/G nucleotides
    int8_t start[21];
    int8_t count[21];
    int8_t aa_of[64];        // amino acid of each codon id
    uint8_t hsc[64 * 64];    // hidden stops across a codon boundary
    int64_t cpsf[61 * 61];   // CPS in 2^-32 fixed point
    float cps[61 * 61];
    float ref_gc3, ref_gc;
    uint8_t pair_i[kMaxCds * (kMaxCds - 1) / 2];  // CDS pair pi (i < j, row-major) of the instance's m
    uint8_t pair_j[kMaxCds * (kMaxCds - 1) / 2];
};

// One population buffer (2N solutions).
struct PopBuf {
    uint8_t *ids;      // [2N][m][Lp]
    uint2 *planes;     // [2N][m][Wp]  (lo, hi) nucleotide bit planes
    float *obj;        // [2N][M]
    int8_t *objidx;    // [2N][2M]
    int32_t *pql;      // [2N][3]
    // [2N][nres] string-objective scan of each CDS (hairpin: (longest stem, its
    // anti-diagonal)) or CDS pair (LRCS: (longest common run, delta + n)); x = -1 marks
    // one to scan.  A child's unchanged CDSs (pairs of unchanged CDSs) carry their
    // parent's result, so only what its mutation touched is scanned.  nullptr: every
    // one is scanned.
    int2 *cds;
    // [2N][naux] per-CDS (per-pair) sums of the light objectives: a child's unchanged
    // CDSs take their parent's.  nullptr: every CDS is summed.
    int32_t *aux;
};

struct SelectScratch {
    uint32_t *dom;       // [2N][2N/32] bit j of row i: j dominates i
    int32_t *np;         // [column tiles][2N] dominators of each row per tile of the matrix
    int32_t *front;      // [2N]
    int32_t *sorted;     // [2N] fronts 0..last
    int32_t *assoc;      // [2N]
    float *dist;         // [2N]
    int32_t *rho;        // [R]
    int32_t *ncand;      // [R]
    uint32_t *trank;     // [2N + M] place of each extreme-point search position in the reduction-tree order
    int32_t *info;       // [8] rank_count, last_size, n_fronts, cut, hyp_exc, status
    float *finfo;        // [3*M] ideal, worst, nadir
};

// One batch member's share of a queued stem scan (k_sl_queue): its shape and the
// buffers of the generation's children, and the queue of results its variation kernel
// invalidated (items: sol * nres + c, sol in 0 .. N-1 counted from `base`).
constexpr int kMaxBatchJobs = 1024;
struct SlJob {
    Shape s;
    PopBuf buf;
    int base;
    int2 *part;
    int32_t *counter;
    int32_t *status;
    unsigned long long *scanned;
    int32_t *items;  // [N * nres]
    int32_t *count;  // items queued
};

// launchers (pe_eval.cu)
cudaError_t launch_init(const Shape &s, const DevTables *tab, const int8_t *aa, PopBuf dst, int32_t *surv,
                        cudaStream_t st);
cudaError_t launch_light_eval(const Shape &s, const DevTables *tab, const int8_t *aa, PopBuf buf, int base, int count,
                              cudaStream_t st);
cudaError_t launch_mutate(const Shape &s, const DevTables *tab, const int8_t *aa, PopBuf src, PopBuf dst,
                          const int32_t *parent_of, const int32_t *rng_idx, int count, int copy_base, int child_base,
                          const uint32_t *d_gen, int32_t *ops, int32_t *order, cudaStream_t st,
                          int32_t *q_items = nullptr, int32_t *q_count = nullptr, int32_t *q_counter = nullptr);
// preset: the variation kernel preset each child's counter to the results it kept
// (launch_mutate's q_counter); CTAs whose result is carried over then leave at once
cudaError_t launch_sl(const Shape &s, PopBuf buf, int base, int count, int2 *part, int32_t *counter,
                      int32_t *status, cudaStream_t st, unsigned long long *scanned = nullptr, bool preset = false);
size_t sl_smem_bytes(const Shape &s);
// the batch's queued stem scan (k_sl_queue): shared memory of a job at CTA size nt,
// resident CTAs per SM, and the launch of one wave over jobs[0 .. njobs)
size_t sl_queue_smem_bytes(const Shape &s, int nt);
int sl_queue_ctas_per_sm(int nt, int fl, size_t smem);
cudaError_t launch_sl_queue(const SlJob *jobs, int njobs, int32_t *ticket, int nt, int fl, size_t smem, int ctas,
                            cudaStream_t st);
// Raise a kernel's dynamic shared-memory limit to at least `bytes` on the current
// device.  The limit only grows, so launches from different host threads never
// see it lowered between their own setting and their launch.
cudaError_t raise_smem_limit(const void *func, size_t bytes);
size_t var_smem_bytes(const Shape &s);

// records a message for pe_last_error() (pe_api.cu)
void set_error_text(const char *msg);

// launchers (pe_select.cu)
cudaError_t launch_select(const Shape &s, const float *obj, float *ext, const float *refpts, SelectScratch sc,
                          int32_t *surv, uint32_t *d_gen, int bump_gen, cudaStream_t st);
size_t select_smem_bytes(const Shape &s);
// column tiles of the dominance matrix: SelectScratch.np holds 2N x this many counts
int dom_tile_count(int N2);
size_t niche_smem_bytes(const Shape &s);
// place of every position 0 .. B-1 of the extreme-point search in the reference's
// reduction-tree order (0xffffffff: a position the tree leaves out)
void tree_order_ranks(int B, uint32_t *rank);

}  // namespace pe
