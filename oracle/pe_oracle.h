/*
 * pe_oracle.h -- CPU oracle for the NSGA-III codon-design generation loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (CAU-HPCL/Protein_encoding_v2_NSGA-III) used as the checker for the
 * CUDA engine.  Only the tests, the smoke entry and the CPU-baseline leg of the
 * benchmark may load it; the product never calls it.
 *
 * Semantics follow the reference's device code, run as if by a single thread
 * (which removes the reference's races), with the deterministic rules listed at
 * each function.  Every function cites the reference file:line it restates.
 *
 * Parity pin: the evaluators, Das-Dennis points, non-dominated fronts and the
 * ideal/worst/nadir estimates are checked against outputs of the reference's own
 * device functions (compiled from the reference sources by oracle/Makefile into
 * oracle/_ref/ref_harness and run on a B200); those outputs are committed under
 * tests/golden/.
 */
#ifndef PE_ORACLE_H
#define PE_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_MAX_OBJ 6
#define OR_NUM_AMINO 21
#define OR_NUM_CODON 64
#define OR_NUM_SENSE 61

/* objective kinds, in the reference's REF6 slot order (include/common.cuh:23-29) */
enum { OR_K_CAI = 0, OR_K_CBP = 1, OR_K_HSC = 2, OR_K_HD = 3, OR_K_GC = 4, OR_K_SL = 5 };
enum { OR_OBJSET_REF6 = 0, OR_OBJSET_BASE4 = 1 };
enum { OR_GC3 = 0, OR_GCALL = 1 };
/* flavour of the string objective in the SL slot: the reference's hairpin stem, or
 * the longest repeated/common substring (no reference implementation: parity unpinned) */
enum { OR_SL_HAIRPIN = 0, OR_SL_LRCS = 1 };

typedef struct {
    uint8_t nt[OR_NUM_CODON][3];     /* nucleotide codes A=0 C=1 G=2 U=3 */
    float weight[OR_NUM_CODON];      /* relative adaptiveness w(codon) */
    float cps[OR_NUM_SENSE * OR_NUM_SENSE]; /* codon-pair score, sense codons */
    int8_t start[OR_NUM_AMINO];      /* first global codon id of each amino acid */
    int8_t count[OR_NUM_AMINO];      /* number of synonymous codons */
    float ref_gc3;                   /* 0.3810 in the reference (include/info.cuh:7) */
    float ref_gc;                    /* 0.3977 (include/info.cuh:6) */
} or_codon_table;

typedef struct {
    int L;            /* amino-acid positions including the appended stop */
    int m;            /* CDSs per solution */
    int N;            /* population size */
    int objset;       /* OR_OBJSET_REF6 or OR_OBJSET_BASE4 */
    int gcmode;       /* OR_GC3 or OR_GCALL */
    int p;            /* Das-Dennis partitions (>=1) */
    float pm;         /* per-codon mutation probability */
    uint64_t seed;
    const int8_t *aa; /* [L] amino-acid index (0..20, 20 = stop) */
    const or_codon_table *tab;
    int slkind;       /* OR_SL_HAIRPIN or OR_SL_LRCS */
} or_problem;

/* --- helpers shared with tests --- */
int or_num_obj(int objset);
int or_slot_of(int objset, int kind);           /* slot or -1 */
int or_num_ref(int M, int p);
int or_auto_p(int M, int N);
void or_das_dennis(int M, int p, float *out);   /* R*M floats */
void or_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
uint32_t or_draw(uint64_t seed, uint32_t tag, uint32_t gen, uint32_t idx, uint32_t pos, uint32_t j);
double or_det_exp(double x);
void or_log_weight_fixed(const or_codon_table *t, int64_t out[OR_NUM_CODON], uint8_t zero[OR_NUM_CODON]);

/* --- operators --- */
void or_gen_solution(const or_problem *pr, int idx, uint8_t *sol);
void or_eval(const or_problem *pr, const uint8_t *sol, float *obj, int8_t *objidx, int32_t *pql);
int  or_mutate(const or_problem *pr, uint32_t gen, int idx, const uint8_t *parent,
               const float *pobj, const int8_t *pobjidx, const int32_t *ppql, uint8_t *child);
int  or_sl_serial_one(const uint8_t *nt, int n);   /* calOneCDS_SL max l */
/* longest repeated/common substring of m CDSs of n nucleotides: length, starts p (in
 * CDS a) and q (in CDS b), pair (a, b) -- see lrcs_serial */
void or_lrcs(const uint8_t *nt, int m, int n, int32_t *out5);
/* one pair: longest run on the diagonals delta >= 1 (self) or all (a != b); out: length,
 * delta, start p (first pair rule: smallest delta, then smallest p) */
void or_lrcs_pair(const uint8_t *sa, const uint8_t *sb, int n, int self, int32_t *out3);
/* timing-sample helpers (bounded slices of the same work) */
void or_eval_light(const or_problem *pr, const uint8_t *sol, float *obj, int8_t *objidx, int32_t *pql);
int  or_sl_serial_strided(const uint8_t *nt, int n, int offset, int stride);
void or_sl_sample_batch(const uint8_t *nt, int count, int n, int offset, int stride, int threads, int32_t *out);
void or_mutate_eval_light_batch(const or_problem *pr, uint32_t gen, const int32_t *idx, int n, const uint8_t *parents,
                                 const float *pobj, const int8_t *pobjidx, const int32_t *ppql, uint8_t *child,
                                 float *cobj, int8_t *cobjidx, int32_t *cpql, int threads);

typedef struct {
    int32_t rank_count;      /* solutions in fronts 0..last */
    int32_t last_front_size;
    int32_t n_fronts;        /* fronts assigned */
    int32_t cut;             /* fronts fill N exactly */
    int32_t hyp_exception;   /* 1 = MNDF nadir used */
    float ideal[OR_MAX_OBJ], worst[OR_MAX_OBJ], nadir[OR_MAX_OBJ];
} or_select_info;

/* obj: 2N*M; extremes: M*M in/out; sorted_all: 2N (fronts 0..last then unused);
 * survivors: N; front: 2N (front index or -1).  Returns 0. */
int or_select(const or_problem *pr, uint32_t gen, const float *obj, float *extremes,
              const float *refpts, int R, int32_t *survivors, int32_t *front,
              or_select_info *info);

/* --- whole runs --- */
typedef struct or_state or_state;
or_state *or_create(const or_problem *pr);
void or_destroy(or_state *st);
void or_init(or_state *st, int threads);
void or_generation(or_state *st, int threads);
/* current 2N set (after the last generation's variation) */
void or_get(const or_state *st, uint8_t *pop, float *obj, int8_t *objidx, int32_t *pql,
            int32_t *survivors, float *extremes, uint32_t *gen);
/* evaluate a batch of solutions in parallel (cpu baseline helper) */
void or_eval_batch(const or_problem *pr, const uint8_t *sols, int n, float *obj, int8_t *objidx,
                   int32_t *pql, int threads);
void or_mutate_eval_batch(const or_problem *pr, uint32_t gen, const int32_t *idx, int n,
                          const uint8_t *parents, const float *pobj, const int8_t *pobjidx,
                          const int32_t *ppql, uint8_t *child, float *cobj, int8_t *cobjidx,
                          int32_t *cpql, int32_t *ops, int threads);

/* synthetic inputs (same draws as the engine's pe_synthetic_protein / pe_dirichlet_table):
 * aa_out receives L amino indices and the stop (L+1 entries) */
void or_synthetic_protein(int L, uint64_t seed, int8_t *aa_out);
void or_dirichlet_table(uint64_t seed, or_codon_table *out);
/* replace the current 2N set, survivors, extreme points and generation counter */
void or_set_state(or_state *st, const uint8_t *pop, const float *obj, const int8_t *objidx, const int32_t *pql,
                  const int32_t *survivors, const float *extremes, uint32_t gen);

/* Exact hypervolume of points in [0,1]^d w.r.t. reference point r (minimisation). */
double or_hypervolume(const double *pts, int n, int d, const double *ref);

#ifdef __cplusplus
}
#endif
#endif
