/*
 * pe_nsga3.h -- C ABI of the B200 NSGA-III codon-design engine.
 *
 * The reference (CAU-HPCL/Protein_encoding_v2_NSGA-III) has no library API: its
 * hot path sits behind the device-function signatures of include/utils.cuh,
 * include/mutation.cuh and include/sorting.cuh, the kernel argument lists of
 * src/main.cu:26,121,409 and the command line `Protein_NSGA3 <fasta> <N> <G> <m>
 * <Pm>` (src/main.cu:456-489).  Each entry point below names the reference
 * interface it replaces.  Problem data that the reference keeps in __constant__
 * and __device__ globals (include/common.cuh:45-76) lives in a per-instance
 * handle here, so many problems can share one GPU.
 *
 * Conventions: every function returns PE_OK (0) or a pe_status code and never
 * throws; pe_last_error() describes the last failure of the calling thread.
 * Host pointers are owned by the caller; device memory is owned by the
 * instance.  One host thread drives an instance at a time.
 *
 * Layouts (all row-major, host memory):
 *   codon ids   uint8  [n_solutions][m][L]   global codon id 0..63 (table order)
 *   objectives  float  [n_solutions][M]      minimisation form (see PE_OBJ_*)
 *   objidx      int8   [n_solutions][2M]     [2k] CDS index for objective k,
 *                                            [2k+1] second CDS (HD) or GC direction
 *   pql         int32  [n_solutions][3]      hairpin stem p, q, length
 */
#ifndef PE_NSGA3_H
#define PE_NSGA3_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PE_NUM_AMINO 21
#define PE_NUM_CODON 64
#define PE_NUM_SENSE 61
#define PE_MAX_OBJ 6

typedef enum {
    PE_OK = 0,
    PE_ERR_ARG = 1,         /* invalid argument or unsupported size */
    PE_ERR_OOM = 2,         /* device or host allocation failed */
    PE_ERR_CUDA = 3,        /* CUDA runtime error */
    PE_ERR_TIMEOUT = 4,     /* a bounded device wait gave up */
    PE_ERR_STATE = 5,       /* call out of order (e.g. step before init) */
    PE_ERR_IO = 6,          /* file could not be read or parsed */
    PE_ERR_NO_DEVICE = 7    /* no CUDA device available */
} pe_status;

/* Objective sets.  REF6 is the reference's six (include/common.cuh:23-29):
 *   0 -minCAI, 1 -minCBP, 2 -minHSC, 3 -minHD, 4 max GC3 deviation, 5 max hairpin stem.
 * BASE4 keeps 0 -minCAI, 1 -minHD, 2 max GC(3) deviation, 3 max hairpin stem. */
typedef enum { PE_OBJ_REF6 = 0, PE_OBJ_BASE4 = 1 } pe_objective_set;
typedef enum { PE_GC3 = 0, PE_GC_ALL = 1 } pe_gc_mode;
/* String objective in the stem slot.  HAIRPIN is the reference's calMaximumSL
 * (include/utils.cuh:712-888): longest complementary stem / ((3L-4)/2).  LRCS is
 * the longest repeated or common substring, which the reference only names
 * (MLRCS, src/auto_execution_experiments.py:45,215): the longest run of identical
 * nucleotides shared by two CDSs (any offsets) or repeated inside one CDS (two
 * different starts), / 3L; objidx holds its two CDSs and pql (p, q, length) its
 * starts in them. */
typedef enum { PE_SL_HAIRPIN = 0, PE_SL_LRCS = 1 } pe_string_objective;

/* Genetic code and scores (reference: include/info.cuh:6-54). */
typedef struct pe_codon_table {
    uint8_t nt[PE_NUM_CODON][3];             /* A=0 C=1 G=2 U=3 */
    float weight[PE_NUM_CODON];              /* relative adaptiveness, > 0 */
    float cps[PE_NUM_SENSE * PE_NUM_SENSE];  /* codon-pair score (REF6 only) */
    int8_t start[PE_NUM_AMINO];              /* first codon id per amino acid */
    int8_t count[PE_NUM_AMINO];              /* synonymous codons per amino acid */
    float ref_gc3;                           /* reference GC3 fraction */
    float ref_gc;                            /* reference GC fraction */
} pe_codon_table;

/* Run configuration (reference argv, src/main.cu:481-489, plus explicit knobs). */
typedef struct pe_config {
    int32_t n_cds;          /* m >= 2 */
    int32_t pop_size;       /* N >= 1 */
    float mutation_prob;    /* Pm in [0,1] */
    int32_t objectives;     /* pe_objective_set */
    int32_t gc_mode;        /* pe_gc_mode */
    int32_t ref_p;          /* Das-Dennis partitions; 0 = reference rule (src/main.cu:564-576) */
    uint64_t seed;          /* replaces rand() seeding (src/main.cu:469,525) */
    int32_t stream_priority;/* priority of the stream pe_create makes when given none:
                               0 = default, lower = more urgent (clamped to the
                               device's range); no counterpart in the reference */
    int32_t sl_threads;     /* hairpin-scan CTA size: 64, 128 or 256, or 0 to let
                               pe_init_population time the three on the initial
                               population and keep the fastest (results do not
                               depend on it); no counterpart in the reference */
    int32_t sl_kind;        /* pe_string_objective (0 = the reference's hairpin stem) */
} pe_config;

typedef struct pe_info {
    int32_t L;              /* amino-acid positions incl. stop */
    int32_t m, N, M, R, p;
    uint32_t generation;    /* generations completed */
    int32_t initialized;
    uint64_t device_bytes;  /* device memory held by the instance (512 B granules) */
    int32_t sl_threads;     /* hairpin-scan CTA size in use */
} pe_info;

typedef struct pe_select_info {
    int32_t rank_count;     /* solutions in fronts 0..last */
    int32_t last_front_size;
    int32_t n_fronts;
    int32_t cut;            /* fronts filled N exactly (no niching) */
    int32_t hyp_exception;  /* 1: nadir from the MNDF fallback */
    float ideal[PE_MAX_OBJ], worst[PE_MAX_OBJ], nadir[PE_MAX_OBJ];
} pe_select_info;

typedef struct pe_instance pe_instance;

/* --- lifecycle: replaces main()'s allocation + cudaMemcpyToSymbol uploads
 *     (src/main.cu:630-678).  cuda_stream may be NULL (the instance makes one). */
int pe_create(const pe_config *cfg, const int8_t *aa_idx, int32_t aa_len, const pe_codon_table *table,
              void *cuda_stream, pe_instance **out);
int pe_destroy(pe_instance *inst);
int pe_get_info(const pe_instance *inst, pe_info *info);
/* Device bytes pe_create would allocate for this configuration (for admission
 * control by memory footprint; no counterpart in the reference). */
int pe_instance_bytes(const pe_config *cfg, int32_t aa_len, uint64_t *bytes);

/* --- initializationKernel (src/main.cu:26-119): N random solutions (solution 0
 *     = highest-weight codons), evaluated; extreme points seeded.  With
 *     cfg.sl_threads = 0 the first call also picks the hairpin-scan CTA size by
 *     timing (a few extra scans of the initial population). */
int pe_init_population(pe_instance *inst);

/* --- the generation loop (src/main.cu:708-728): mutationKernel + sortingKernel,
 *     `generations` times, on the device (CUDA-graph replay). */
int pe_step(pe_instance *inst, int32_t generations);
int pe_synchronize(pe_instance *inst);

/* Current 2N set (parents then offspring of the last generation) and survivors
 * (src/main.cu:772-787).  Any pointer may be NULL.  Waits for the instance's
 * stream; call it between pe_step calls (the codon ids are packed on the device in
 * the buffer the next generation overwrites). */
int pe_get_population(pe_instance *inst, uint8_t *codon_idx, float *obj, int8_t *objidx, int32_t *pql,
                      int32_t *survivors);
/* Objectives only (2N*M floats): the per-generation progress read. */
int pe_get_objectives(pe_instance *inst, float *obj);
/* The same read queued on the instance's stream behind the generations already
 * queued, without waiting: obj holds the objectives once pe_synchronize returns (or
 * any later wait on the stream), and must stay valid until then.  With page-locked
 * host memory the copy overlaps the next generations; with pageable memory the call
 * returns only after the copy. */
int pe_read_objectives_async(pe_instance *inst, float *obj);

/* --- operator-level entry points (one device function family each) --- */

/* calMinimumCAI/CBP/HSC/HD, calMaximumGC3/GC, calMaximumSL
 * (include/utils.cuh:271-888) on caller-supplied solutions. */
int pe_eval_objectives(pe_instance *inst, const uint8_t *codon_idx, int32_t n_solutions, float *obj,
                       int8_t *objidx, int32_t *pql);

/* mutationKernel's variation step (src/main.cu:172-211, include/mutation.cuh):
 * child i = mutate(parent i) as offspring index idx[i] of `generation`;
 * ops[i] receives the operator (0 random, 1 CAI, 2 CBP, 3 HSC, 4 HD, 5 GC, 6 SL). */
int pe_mutate(pe_instance *inst, uint32_t generation, const int32_t *idx, int32_t n, const uint8_t *parents,
              const float *pobj, const int8_t *pobjidx, const int32_t *ppql, uint8_t *children, int32_t *ops);

/* sortingKernel (src/main.cu:409-454; include/sorting.cuh:94-1282): fronts,
 * ideal/worst/nadir, extreme points (in/out, M*M), niching -> N survivors. */
int pe_select(pe_instance *inst, uint32_t generation, const float *obj, float *extremes, int32_t *survivors,
              int32_t *front, pe_select_info *info);

/* combinationRepetition (include/sorting.cuh:1338): R*M points; out may be NULL
 * to query R. */
int pe_reference_points(int32_t M, int32_t p, float *out, int32_t *R);

/* --- host-side inputs (no device needed) --- */

/* FASTA loader of src/main.cu:491-523 (header line skipped, newlines dropped,
 * trailing stop 'Z' appended).  aa_out receives amino indices 0..20. */
int pe_parse_fasta(const char *path, int8_t *aa_out, int32_t capacity, int32_t *aa_len);
/* L amino acids i.i.d. uniform over the 20 standard letters, then the stop. */
int pe_synthetic_protein(int32_t L, uint64_t seed, int8_t *aa_out);
/* Standard genetic code; per-amino-acid weights Dirichlet(1) scaled to max 1,
 * codons ordered by ascending weight; seeded codon-pair scores. */
int pe_dirichlet_table(uint64_t seed, pe_codon_table *out);
/* Text table: 64 lines "<CODON> <amino letter> <weight>" in id order, optional
 * "gc3 <v>", "gc <v>", then optional 61*61 CPS values. */
int pe_load_codon_table(const char *path, pe_codon_table *out);

/* --- batched design jobs (no counterpart in the reference, which runs one
 *     protein per process, src/main.cu:467).  count initialised instances, each
 *     on its own stream (pe_create with cuda_stream = NULL), advance together:
 *     one CUDA graph launch covers two generations of every instance, with one
 *     concurrent branch per instance, so the device interleaves their kernels.
 *     Results equal stepping each instance alone (same seed, same arithmetic). */
typedef struct pe_batch pe_batch;
int pe_batch_create(pe_instance *const *instances, int32_t count, pe_batch **out);
int pe_batch_step(pe_batch *batch, int32_t generations);
int pe_batch_synchronize(pe_batch *batch);
int pe_batch_destroy(pe_batch *batch);
/* The string-objective scans of a batch generation queued (1) or not (0, the
 * default): queued, every member's variation kernel appends the CDS (pair) results
 * its children's mutations invalidated, and one wave of CTAs per length class (CTA
 * size = the one the class's members tuned at init, longest CDSs first) takes the
 * whole batch's queue by ticket, between a variation phase and a selection phase of
 * all members; not queued, each member's generation is its own branch of the graph
 * with its own scan launch, so one member's selection overlaps another's scan.
 * Results are the same. */
int pe_batch_set_scan_queue(pe_batch *batch, int32_t enable);

/* --- served design jobs (no counterpart in the reference, which designs one
 *     protein per process, src/main.cu:467-901): continuous batching on one GPU.
 *
 * Jobs are submitted at any time and admitted by device footprint
 * (pe_instance_bytes) against memory_budget and by max_active, in arrival order
 * or shortest estimated work first (a job waiting longer than max_wait_s goes
 * first).  Each resident job keeps its population on the device and is driven by
 * its own host thread, `tick` generations per replay, so the kernels of all
 * resident jobs overlap.  A job retires at its generation budget, when the
 * hypervolume of its survivors' normalised objectives (src/main.cu:789-858) has
 * not improved for `stall` generations (checked every hv_every generations), or
 * when cancelled (between two replays).  A job's result is the same as the job
 * run alone.  All calls are thread-safe. */
typedef enum { PE_ORDER_ARRIVAL = 0, PE_ORDER_SHORTEST = 1 } pe_admission_order;
typedef enum { PE_JOB_QUEUED = 0, PE_JOB_RUNNING = 1, PE_JOB_DONE = 2, PE_JOB_FAILED = 3,
               PE_JOB_CANCELLED = 4 } pe_job_state;
typedef enum { PE_REASON_BUDGET = 0, PE_REASON_STALL = 1, PE_REASON_ERROR = 2,
               PE_REASON_CANCELLED = 3 } pe_job_reason;

typedef struct pe_server_config {
    uint64_t memory_budget;  /* device bytes for resident jobs; 0 = 80 % of the free memory */
    int32_t max_active;      /* resident-job cap (0: nothing is admitted) */
    int32_t tick;            /* generations per replay (0 = 10) */
    int32_t hv_every;        /* generations between hypervolume checks (0 = 25) */
    int32_t order;           /* pe_admission_order */
    double max_wait_s;       /* a job queued longer goes first (0 = off) */
    int32_t priorities;      /* 1: stream priority from estimated work (short jobs first) */
} pe_server_config;

typedef struct pe_job_spec {
    pe_config cfg;                 /* the instance (stream_priority is set by the server) */
    const int8_t *aa_idx;          /* protein, copied at submit */
    int32_t aa_len;
    const pe_codon_table *table;   /* copied at submit */
    int32_t generations;           /* generation budget */
    int32_t stall;                 /* retire after this many generations without a
                                      hypervolume gain (0 = never) */
    int32_t keep_codons;           /* 1: keep the survivors' codon ids for pe_job_result */
} pe_job_spec;

typedef struct pe_job_status {
    int32_t state;                 /* pe_job_state */
    int32_t reason;                /* pe_job_reason, -1 while queued or running */
    int32_t generations_run;
    int32_t priority;              /* stream priority it runs (or would run) at */
    double hypervolume;            /* of the final survivors (done jobs), else -1 */
    double submitted_s, started_s, finished_s;  /* server clock; -1 = not yet */
    uint64_t device_bytes;         /* footprint it was admitted with */
    char error[256];               /* failed jobs: the error */
} pe_job_status;

typedef struct pe_server_stats {
    int32_t queued, active, peak_active;
    uint64_t used_bytes, peak_used_bytes, memory_budget;
} pe_server_stats;

typedef struct pe_server pe_server;
int pe_server_create(const pe_server_config *cfg, pe_server **out);
int pe_batch_submit(pe_server *server, const pe_job_spec *spec, int64_t *job_id);
int pe_poll(pe_server *server, int64_t job_id, pe_job_status *status);
/* Results of a done job: survivor_obj [N][M] (minimisation form, the survivors in
 * selection order) and, when submitted with keep_codons, survivor_codons [N][m][L];
 * either may be NULL. */
int pe_job_result(pe_server *server, int64_t job_id, float *survivor_obj, uint8_t *survivor_codons);
/* A queued job is dropped at once; a running one stops after its current replay
 * (nothing of it left in flight) and frees its memory; a finished one is kept. */
int pe_cancel(pe_server *server, int64_t job_id);
int pe_server_clock(pe_server *server, double *seconds);   /* seconds since pe_server_create */
int pe_server_get_stats(pe_server *server, pe_server_stats *stats);
/* Wait until no job is queued or running (timeout_s <= 0: no limit; PE_ERR_TIMEOUT). */
int pe_server_drain(pe_server *server, double timeout_s);
/* Cancels what is queued or running, waits for the running jobs to stop, frees. */
int pe_server_destroy(pe_server *server);

/* --- instrumentation (no counterpart in the reference, which only times the
 *     whole loop with cudaEvents, src/main.cu:702-731) --- */

/* Record CUDA events around the three stages of each generation (variation +
 * light evaluation, hairpin-stem scan, selection); rebuilds the graphs. */
int pe_set_profiling(pe_instance *inst, int32_t enable);
/* Device milliseconds of those stages in the last completed generation
 * (call after pe_synchronize). */
int pe_stage_times(pe_instance *inst, float *ms3);
/* Polls a bounded device wait (the hairpin/LRCS scan's wait for its staged planes)
 * makes before it gives up, sets a status and lets pe_synchronize return
 * PE_ERR_TIMEOUT: 0 = the default (4,194,304), > 0 = that many, < 0 = none (it gives
 * up at once: a test of the timeout path; the kernel still lets its copy land, within
 * a second bound, before it returns).  pe_init_population clears the status and
 * restarts the population.  No counterpart in the reference, whose spin-waits are
 * unbounded (include/utils.cuh:873, include/sorting.cuh:939,949). */
int pe_set_wait_limit(pe_instance *inst, int32_t polls);
/* String-objective scans run since pe_create (no reference counterpart): one per
 * hairpin CDS or LRCS CDS pair.  A child's CDS that its mutation left unchanged
 * (for LRCS: a pair of two such CDSs) keeps its parent's result and is not
 * scanned again.  Waits for the instance's stream. */
int pe_scan_count(pe_instance *inst, uint64_t *count);
/* Counted cells of those scans (no reference counterpart): (n-5)(n-4)/2 per hairpin
 * CDS scan (the anti-diagonal cells with a loop of >= 4), n^2 per LRCS scan of two
 * CDSs and n(n-1)/2 per LRCS scan of one CDS against itself, n = 3L nucleotides.
 * The unit of work of the string-objective kernel's throughput.  Waits for the
 * instance's stream. */
int pe_scan_cells(pe_instance *inst, uint64_t *cells);
/* Scans whose seeded first pass gave up (no reference counterpart).  The string
 * scan first looks up T's 6- or 7-nucleotide words in a table (linear in n for
 * random-like CDSs); on a repetitive CDS, whose table chains grow long, it hands
 * the CDS to the band scan, which visits every counted cell.  Both give the same
 * result.  Waits for the instance's stream. */
int pe_scan_fallbacks(pe_instance *inst, uint64_t *count);
/* First pass of the string scan (no reference counterpart): 0 = seeded, the
 * default (CDSs of up to 12,288 nucleotides; longer ones take the band scan),
 * 1 = the band scan for every CDS.  The result does not depend on it; a test of
 * the band scan, and a way to compare the two.  Rebuilds the instance's graphs. */
int pe_set_scan_method(pe_instance *inst, int32_t method);

/* --- allocation-free hairpin-stem evaluation (no counterpart in the reference).
 *
 * For callers that may not allocate device memory (their host application's
 * memory manager already owns the GPU, or their loop cannot afford
 * cudaMalloc/cudaFree): the longest-stem objective of n solutions already on the
 * device, computed with no allocation.  All pointers are device pointers:
 *   d_nt     uint8 [n][m][3L]  nucleotide codes (A=0 C=1 G=2 U=3)
 *   d_value  float [n]         stem length / ((3L-4)/2)
 *   d_pql    int32 [n][3]      stem p, q, length
 *   d_cds    int8  [n]         CDS holding the stem
 * A solution whose scan did not finish (a bounded device wait gave up) reads
 * NaN, (-1, -1, -1) and -1.  Scratch is one fixed 8 MiB device array; calls
 * needing more (roughly n*m*3L/4 bytes) return PE_ERR_ARG.  The array is taken
 * from the device's memory when this code is first used on that device (CUDA
 * loads device code lazily by default): a call with n_solutions = 0 (pointers
 * may be NULL) does only that set-up, so make it while setting up, before the
 * application's memory manager takes the device's memory and before any stream
 * capture; after it the array stays reserved until the process exits and no call
 * allocates.  Asynchronous on cuda_stream (NULL = default stream).  Every call
 * shares the array, so calls that overlap on the GPU race and give wrong results. */
int pe_hairpin_noalloc(const uint8_t *d_nt, int32_t n_solutions, int32_t m, int32_t L, float *d_value,
                       int32_t *d_pql, int8_t *d_cds, void *cuda_stream);

/* Exact hypervolume of n points (d <= 6) in minimisation form w.r.t. ref. */
int pe_hypervolume(const double *pts, int32_t n, int32_t d, const double *ref, double *out);

const char *pe_last_error(void);
const char *pe_version(void);

#ifdef __cplusplus
}
#endif
#endif
