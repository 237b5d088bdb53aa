// ref_harness.cu -- drives the reference's own device functions on supplied
// inputs so that the CPU oracle can be checked against them.
//
// TEST INFRASTRUCTURE ONLY (built into oracle/_ref/, never shipped).  Compiled
// against the unmodified reference headers (-I<reference>/include); the kernels
// below only sequence calls to the reference's functions the way
// src/main.cu:26-119 and :409-454 do.
//
//   ref_harness <job.bin> <out.bin>
//
// job.bin (little endian): char magic[4]="PEH1", int32 mode, then
//   mode 1 (evaluate): int32 L, m, nsol, custom_table; [custom: char codons[192],
//           float weight[64], int8 start[21], int8 count[21], float cps[3721]];
//           int8 aa[L]; char sol[nsol*m*3L]
//     -> per solution: float obj[6], int8 objidx[12], int32 pql[3], int32 sl_written
//   mode 2 (selection): int32 N, p; float extremes[36]; float obj[2N*6]
//     -> int32 rank_count, cur_front, n_cut, hyp_exc; int32 front_count[2N];
//        int32 sorted[2N]; float ideal[6], worst[6], nadir[6], extremes[36];
//        float dist[2N]; int32 included[R]
//   mode 3 (reference points): int32 M, p -> int32 R; float pts[R*M]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <curand_kernel.h>

#include "common.cuh"
#include "info.cuh"
#include "utils.cuh"
#include "mutation.cuh"
#include "sorting.cuh"

using namespace cooperative_groups;

#define HCHECK(x)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            fprintf(stderr, "CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            exit(2);                                                                       \
        }                                                                                  \
    } while (0)

// ---------------------------------------------------------------- evaluate
__global__ void harness_eval(const char *d_aa, const char *d_sol, int nsol, float *d_obj, char *d_objidx,
                             int *d_pql, int *d_slw)
{
    auto tb = this_thread_block();
    extern __shared__ int smem[];
    int *s_pql = smem;
    int *s_mutex = s_pql + 3;
    float *s_obj_val = (float *)(s_mutex + 1);
    float *s_obj_buffer = s_obj_val + OBJECTIVE_NUM;
    char *s_aa = (char *)(s_obj_buffer + tb.size());
    char *s_sol = s_aa + c_amino_seq_len;
    char *s_objidx = s_sol + c_solution_len;

    for (int i = tb.thread_rank(); i < c_amino_seq_len; i += tb.size()) s_aa[i] = d_aa[i];
    for (int idx = blockIdx.x; idx < nsol; idx += gridDim.x) {
        for (int i = tb.thread_rank(); i < c_solution_len; i += tb.size()) s_sol[i] = d_sol[(size_t)idx * c_solution_len + i];
        if (tb.thread_rank() < 3) s_pql[tb.thread_rank()] = -7;
        if (tb.thread_rank() < OBJECTIVE_NUM) s_obj_val[tb.thread_rank()] = -7.0f;
        if (tb.thread_rank() < OBJECTIVE_NUM * 2) s_objidx[tb.thread_rank()] = 0;
        tb.sync();
        calMinimumCAI(tb, s_sol, s_aa, s_obj_buffer, s_obj_val, s_objidx);
        tb.sync();
        calMinimumCBP(tb, s_sol, s_aa, s_obj_buffer, s_obj_val, s_objidx);
        tb.sync();
        calMinimumHSC(tb, s_sol, s_aa, s_obj_buffer, s_obj_val, s_objidx);
        tb.sync();
        calMinimumHD(tb, s_sol, s_aa, s_obj_buffer, s_obj_val, s_objidx);
        tb.sync();
        calMaximumGC3(tb, s_sol, s_aa, s_obj_buffer, s_obj_val, s_objidx);
        tb.sync();
        calMaximumSL(tb, s_sol, s_aa, s_obj_buffer, s_obj_val, s_objidx, s_pql, s_mutex);
        tb.sync();
        if (tb.thread_rank() < OBJECTIVE_NUM) d_obj[idx * OBJECTIVE_NUM + tb.thread_rank()] = s_obj_val[tb.thread_rank()];
        if (tb.thread_rank() < OBJECTIVE_NUM * 2) d_objidx[idx * OBJECTIVE_NUM * 2 + tb.thread_rank()] = s_objidx[tb.thread_rank()];
        if (tb.thread_rank() < 3) d_pql[idx * 3 + tb.thread_rank()] = s_pql[tb.thread_rank()];
        if (tb.thread_rank() == 0) d_slw[idx] = (s_pql[2] != -7);
        tb.sync();
    }
}

// ---------------------------------------------------------------- selection
__global__ void harness_curand(curandStateXORWOW *st, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) curand_init(12345ull, i, 0, &st[i]);
}

__global__ void harness_select(curandStateXORWOW *random_generator, const float *d_obj_val, int *d_sorted_array,
                               bool *F_set, bool *Sp_set, int *d_np, int *d_rank_count, float *d_buffer,
                               int *index_num, const float *d_reference_points, int *d_included_solution_num,
                               int *d_not_included_solution_num, int *d_solution_index_for_sorting,
                               float *d_dist_of_solution, int *d_flags)
{
    auto g = this_grid();
    auto tb = this_thread_block();
    extern __shared__ int smem[];
    int *s_index_num = smem;
    float *s_buffer = (float *)&s_index_num[tb.size()];
    float *s_normalized_obj_val = (float *)&s_buffer[tb.size()];
    curandStateXORWOW *s_generator = (curandStateXORWOW *)&s_normalized_obj_val[OBJECTIVE_NUM];
    if (tb.thread_rank() == 0) *s_generator = random_generator[g.block_rank()];

    nonDominatedSorting(g, d_obj_val, d_sorted_array, F_set, Sp_set, d_np, d_rank_count);
    g.sync();
    updateIdealValue(g, d_obj_val, d_buffer, index_num);
    g.sync();
    updateWorstValue(g, d_obj_val, d_buffer, index_num);
    g.sync();
    updateNadirValue_HYP(g, d_obj_val, d_buffer, d_sorted_array, d_rank_count, index_num);
    g.sync();
    if (g.thread_rank() == 0) {
        d_flags[0] = rank_count;
        d_flags[1] = cur_front;
        d_flags[2] = N_cut_check ? 1 : 0;
        d_flags[3] = HYP_EXCEPTION ? 1 : 0;
    }
    g.sync();
    if (!N_cut_check)
        referenceBasedSorting(s_generator, g, tb, d_obj_val, d_sorted_array, d_rank_count, d_reference_points,
                              d_included_solution_num, d_not_included_solution_num, d_solution_index_for_sorting,
                              d_dist_of_solution, s_buffer, s_index_num, s_normalized_obj_val);
    g.sync();
}

// ---------------------------------------------------------------- reference points
__global__ void harness_dd(int M, int p, float *d_ref)
{
    auto g = this_grid();
    combinationRepetition(g, M, p, d_ref);
}

template <class T> static void rd(FILE *f, T *p, size_t n)
{
    if (fread(p, sizeof(T), n, f) != n) {
        fprintf(stderr, "short read\n");
        exit(3);
    }
}
template <class T> static void wr(FILE *f, const T *p, size_t n) { fwrite(p, sizeof(T), n, f); }

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s job.bin out.bin\n", argv[0]);
        return 1;
    }
    FILE *f = fopen(argv[1], "rb");
    FILE *o = fopen(argv[2], "wb");
    if (!f || !o) return 1;
    char magic[4];
    rd(f, magic, 4);
    if (memcmp(magic, "PEH1", 4) != 0) return 1;
    int mode;
    rd(f, &mode, 1);
    HCHECK(cudaSetDevice(0));
    cudaDeviceProp prop;
    HCHECK(cudaGetDeviceProperties(&prop, 0));

    if (mode == 1) {
        int aalen, m, nsol, custom;
        rd(f, &aalen, 1);
        rd(f, &m, 1);
        rd(f, &nsol, 1);
        rd(f, &custom, 1);
        char h_codons[TOTAL_CODON_NUM * CODON_SIZE + 1];
        float h_w[TOTAL_CODON_NUM];
        char h_start[21], h_count[21];
        std::vector<float> h_cps((TOTAL_CODON_NUM - STOP_CODON_NUM) * (TOTAL_CODON_NUM - STOP_CODON_NUM));
        memcpy(h_codons, codons, sizeof h_codons);
        memcpy(h_w, codons_weight, sizeof h_w);
        memcpy(h_start, codons_start_idx, 21);
        memcpy(h_count, syn_codons_num, 21);
        memcpy(h_cps.data(), cps, sizeof(float) * h_cps.size());
        if (custom) {
            rd(f, h_codons, TOTAL_CODON_NUM * CODON_SIZE);
            rd(f, h_w, TOTAL_CODON_NUM);
            rd(f, h_start, 21);
            rd(f, h_count, 21);
            rd(f, h_cps.data(), h_cps.size());
        }
        std::vector<char> aa(aalen), sol((size_t)nsol * m * 3 * aalen);
        rd(f, aa.data(), aa.size());
        rd(f, sol.data(), sol.size());
        int cds_len = 3 * aalen, sol_len = cds_len * m;
        char cm = (char)m;
        HCHECK(cudaMemcpyToSymbol(c_ref_GC3_percent, &ref_GC3_percent, sizeof(float)));
        HCHECK(cudaMemcpyToSymbol(c_codons_start_idx, h_start, 21));
        HCHECK(cudaMemcpyToSymbol(c_syn_codons_num, h_count, 21));
        HCHECK(cudaMemcpyToSymbol(c_codons, h_codons, sizeof h_codons));
        HCHECK(cudaMemcpyToSymbol(c_codons_weight, h_w, sizeof h_w));
        HCHECK(cudaMemcpyToSymbol(c_cps, h_cps.data(), sizeof(float) * h_cps.size()));
        HCHECK(cudaMemcpyToSymbol(c_amino_seq_len, &aalen, sizeof(int)));
        HCHECK(cudaMemcpyToSymbol(c_solution_len, &sol_len, sizeof(int)));
        HCHECK(cudaMemcpyToSymbol(c_cds_len, &cds_len, sizeof(int)));
        HCHECK(cudaMemcpyToSymbol(c_cds_num, &cm, sizeof(char)));
        char *d_aa, *d_sol, *d_objidx;
        float *d_obj;
        int *d_pql, *d_slw;
        HCHECK(cudaMalloc(&d_aa, aalen));
        HCHECK(cudaMalloc(&d_sol, sol.size()));
        HCHECK(cudaMalloc(&d_obj, sizeof(float) * 6 * nsol));
        HCHECK(cudaMalloc(&d_objidx, 12 * nsol));
        HCHECK(cudaMalloc(&d_pql, sizeof(int) * 3 * nsol));
        HCHECK(cudaMalloc(&d_slw, sizeof(int) * nsol));
        HCHECK(cudaMemcpy(d_aa, aa.data(), aalen, cudaMemcpyHostToDevice));
        HCHECK(cudaMemcpy(d_sol, sol.data(), sol.size(), cudaMemcpyHostToDevice));
        // padded: the reference reads the amino array past its end inside the block
        size_t smem = sizeof(int) * 4 + sizeof(float) * (OBJECTIVE_NUM + 256) + aalen + sol_len + 12 + 1024;
        if (smem > 48 * 1024) HCHECK(cudaFuncSetAttribute(harness_eval, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        harness_eval<<<nsol < 1024 ? nsol : 1024, 256, smem>>>(d_aa, d_sol, nsol, d_obj, d_objidx, d_pql, d_slw);
        HCHECK(cudaGetLastError());
        HCHECK(cudaDeviceSynchronize());
        std::vector<float> obj(6 * nsol);
        std::vector<char> objidx(12 * nsol);
        std::vector<int> pql(3 * nsol), slw(nsol);
        HCHECK(cudaMemcpy(obj.data(), d_obj, sizeof(float) * obj.size(), cudaMemcpyDeviceToHost));
        HCHECK(cudaMemcpy(objidx.data(), d_objidx, objidx.size(), cudaMemcpyDeviceToHost));
        HCHECK(cudaMemcpy(pql.data(), d_pql, sizeof(int) * pql.size(), cudaMemcpyDeviceToHost));
        HCHECK(cudaMemcpy(slw.data(), d_slw, sizeof(int) * slw.size(), cudaMemcpyDeviceToHost));
        for (int i = 0; i < nsol; i++) {
            wr(o, &obj[6 * i], 6);
            wr(o, &objidx[12 * i], 12);
            wr(o, &pql[3 * i], 3);
            wr(o, &slw[i], 1);
        }
    } else if (mode == 2) {
        int N, p;
        rd(f, &N, 1);
        rd(f, &p, 1);
        float ext[36];
        rd(f, ext, 36);
        int N2 = 2 * N;
        std::vector<float> obj((size_t)N2 * 6);
        rd(f, obj.data(), obj.size());
        int R = (int)combination(OBJECTIVE_NUM + p - 1, p);
        HCHECK(cudaMemcpyToSymbol(c_N, &N, sizeof(int)));
        HCHECK(cudaMemcpyToSymbol(c_ref_points_num, &R, sizeof(int)));
        HCHECK(cudaMemcpyToSymbol(extreme_points, ext, sizeof ext));
        float *d_obj, *d_buffer, *d_ref, *d_dist;
        int *d_sorted, *d_np, *d_rc, *d_index, *d_inc, *d_ninc, *d_sifs, *d_flags;
        bool *d_F, *d_Sp;
        HCHECK(cudaMalloc(&d_obj, sizeof(float) * obj.size()));
        HCHECK(cudaMalloc(&d_buffer, sizeof(float) * (N2 + OBJECTIVE_NUM)));
        HCHECK(cudaMalloc(&d_ref, sizeof(float) * R * OBJECTIVE_NUM));
        HCHECK(cudaMalloc(&d_dist, sizeof(float) * N2));
        HCHECK(cudaMalloc(&d_sorted, sizeof(int) * N2));
        HCHECK(cudaMalloc(&d_np, sizeof(int) * N2));
        HCHECK(cudaMalloc(&d_rc, sizeof(int) * N2));
        HCHECK(cudaMalloc(&d_index, sizeof(int) * (N2 + OBJECTIVE_NUM)));
        HCHECK(cudaMalloc(&d_inc, sizeof(int) * R));
        HCHECK(cudaMalloc(&d_ninc, sizeof(int) * R));
        HCHECK(cudaMalloc(&d_sifs, sizeof(int) * (size_t)R * N2));
        HCHECK(cudaMalloc(&d_flags, sizeof(int) * 4));
        HCHECK(cudaMalloc(&d_F, (size_t)N2 * N2));
        HCHECK(cudaMalloc(&d_Sp, (size_t)N2 * N2));
        HCHECK(cudaMemcpy(d_obj, obj.data(), sizeof(float) * obj.size(), cudaMemcpyHostToDevice));
        HCHECK(cudaMemset(d_ref, 0, sizeof(float) * R * OBJECTIVE_NUM));
        {
            int M = OBJECTIVE_NUM;
            void *args[] = {&M, &p, &d_ref};
            HCHECK(cudaLaunchCooperativeKernel((void *)harness_dd, 1, 256, args, 0));
            HCHECK(cudaDeviceSynchronize());
        }
        HCHECK(cudaMemset(d_F, 0, (size_t)N2 * N2));
        HCHECK(cudaMemset(d_Sp, 0, (size_t)N2 * N2));
        HCHECK(cudaMemset(d_rc, 0, sizeof(int) * N2));
        HCHECK(cudaMemset(d_np, 0, sizeof(int) * N2));
        HCHECK(cudaMemset(d_inc, 0, sizeof(int) * R));
        HCHECK(cudaMemset(d_ninc, 0, sizeof(int) * R));
        HCHECK(cudaMemset(d_sifs, EMPTY, sizeof(int) * (size_t)R * N2));
        HCHECK(cudaMemset(d_dist, EMPTY, sizeof(float) * N2));
        HCHECK(cudaMemset(d_sorted, EMPTY, sizeof(int) * N2));
        int threads = 256, per_sm = 0;
        size_t smem = sizeof(int) * threads + sizeof(float) * (threads + OBJECTIVE_NUM) + sizeof(curandStateXORWOW);
        HCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, harness_select, threads, smem));
        int blocks = prop.multiProcessorCount * per_sm;
        curandStateXORWOW *d_gen;
        HCHECK(cudaMalloc(&d_gen, sizeof(curandStateXORWOW) * blocks));
        harness_curand<<<(blocks + 255) / 256, 256>>>(d_gen, blocks);
        HCHECK(cudaDeviceSynchronize());
        void *args[] = {&d_gen, &d_obj, &d_sorted, &d_F, &d_Sp, &d_np, &d_rc, &d_buffer, &d_index, &d_ref,
                        &d_inc, &d_ninc, &d_sifs, &d_dist, &d_flags};
        HCHECK(cudaLaunchCooperativeKernel((void *)harness_select, blocks, threads, args, smem));
        HCHECK(cudaDeviceSynchronize());
        int flags[4];
        std::vector<int> rc(N2), sorted(N2), inc(R);
        std::vector<float> dist(N2);
        float ideal[6], worst[6], nadir[6], ext2[36];
        HCHECK(cudaMemcpy(flags, d_flags, sizeof flags, cudaMemcpyDeviceToHost));
        HCHECK(cudaMemcpy(rc.data(), d_rc, sizeof(int) * N2, cudaMemcpyDeviceToHost));
        HCHECK(cudaMemcpy(sorted.data(), d_sorted, sizeof(int) * N2, cudaMemcpyDeviceToHost));
        HCHECK(cudaMemcpy(dist.data(), d_dist, sizeof(float) * N2, cudaMemcpyDeviceToHost));
        HCHECK(cudaMemcpy(inc.data(), d_inc, sizeof(int) * R, cudaMemcpyDeviceToHost));
        HCHECK(cudaMemcpyFromSymbol(ideal, estimated_ideal_value, sizeof ideal));
        HCHECK(cudaMemcpyFromSymbol(worst, estimated_worst_value, sizeof worst));
        HCHECK(cudaMemcpyFromSymbol(nadir, estimated_nadir_value, sizeof nadir));
        HCHECK(cudaMemcpyFromSymbol(ext2, extreme_points, sizeof ext2));
        wr(o, flags, 4);
        wr(o, rc.data(), N2);
        wr(o, sorted.data(), N2);
        wr(o, ideal, 6);
        wr(o, worst, 6);
        wr(o, nadir, 6);
        wr(o, ext2, 36);
        wr(o, dist.data(), N2);
        wr(o, inc.data(), R);
    } else if (mode == 3) {
        int M, p;
        rd(f, &M, 1);
        rd(f, &p, 1);
        int R = (int)combination(M + p - 1, p);
        float *d_ref;
        HCHECK(cudaMalloc(&d_ref, sizeof(float) * R * M));
        HCHECK(cudaMemset(d_ref, 0, sizeof(float) * R * M));
        void *args[] = {&M, &p, &d_ref};
        HCHECK(cudaLaunchCooperativeKernel((void *)harness_dd, 1, 256, args, 0));
        HCHECK(cudaDeviceSynchronize());
        std::vector<float> pts((size_t)R * M);
        HCHECK(cudaMemcpy(pts.data(), d_ref, sizeof(float) * pts.size(), cudaMemcpyDeviceToHost));
        wr(o, &R, 1);
        wr(o, pts.data(), pts.size());
    } else {
        return 1;
    }
    fclose(o);
    fclose(f);
    return 0;
}
