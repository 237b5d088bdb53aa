// pe_cli.cpp -- command line with the reference's run surface (src/main.cu:456-901):
//
//   pe_nsga3 <fasta> <N> <G> <m> <Pm> [options]
//
// Same five positional arguments and the same outputs (Result.txt,
// Normalized_value_quality_computation.txt, hypervolume / minimum distance /
// timing lines), computed through the C ABI.  Options:
//   --seed S                  RNG seed (the reference seeds from time())
//   --objectives ref6|base4   objective set (default ref6, as the reference)
//   --gc gc3|gc               GC objective flavour (default gc3)
//   --string hairpin|lrcs     string objective: the reference's hairpin stem (default)
//                             or the longest repeated/common substring
//   --ref-p P                 Das-Dennis partitions (default: reference rule)
//   --codon-table FILE        codon table text file (default: the reference table
//                             shipped in data/ref_codon_table.txt next to lib/)
//   --dirichlet SEED          synthetic Dirichlet(1) codon weights instead
//   --synthetic-protein L:SEED  ignore <fasta>; use a seeded synthetic protein
//   --out DIR                 directory for the output files (default .)
#include <algorithm>
#include <chrono>
#include <ctime>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <dlfcn.h>
#include <limits.h>
#include <unistd.h>

#include "../../include/pe_nsga3.h"

static int die(const char *what)
{
    fprintf(stderr, "%s: %s\n", what, pe_last_error());
    return EXIT_FAILURE;
}

static std::string exe_dir()
{
    char buf[PATH_MAX];
    ssize_t n = readlink("/proc/self/exe", buf, sizeof buf - 1);
    if (n <= 0) return ".";
    buf[n] = 0;
    std::string p(buf);
    size_t k = p.rfind('/');
    return k == std::string::npos ? "." : p.substr(0, k);
}

int main(int argc, char **argv)
{
    if (argc < 6) {
        fprintf(stderr, "usage: %s <fasta> <N> <G> <m> <Pm> [--seed S] [--objectives ref6|base4] [--gc gc3|gc] [--string hairpin|lrcs]\n"
                        "       [--ref-p P] [--codon-table FILE | --dirichlet SEED] [--synthetic-protein L:SEED]"
                        " [--out DIR]\n",
                argv[0]);
        return EXIT_FAILURE;
    }
    int N = atoi(argv[2]), G = atoi(argv[3]), m = atoi(argv[4]);
    float pm = (float)atof(argv[5]);
    // same checks as src/main.cu:482-486
    if (N <= 0 || G < 0 || m <= 1 || pm < 0.f || pm > 1.f) {
        printf("Please check input parameters.\n");
        return EXIT_FAILURE;
    }
    pe_config cfg{};
    cfg.n_cds = m;
    cfg.pop_size = N;
    cfg.mutation_prob = pm;
    cfg.objectives = PE_OBJ_REF6;
    cfg.gc_mode = PE_GC3;
    cfg.ref_p = 0;
    cfg.seed = (uint64_t)time(nullptr);
    std::string table_path = exe_dir() + "/../data/ref_codon_table.txt", outdir = ".";
    long dirichlet = -1;
    int synL = 0;
    unsigned long long synSeed = 0;
    for (int i = 6; i < argc; i++) {
        std::string a = argv[i];
        auto next = [&]() -> const char * {
            if (i + 1 >= argc) {
                fprintf(stderr, "missing value for %s\n", a.c_str());
                exit(EXIT_FAILURE);
            }
            return argv[++i];
        };
        if (a == "--seed") cfg.seed = strtoull(next(), nullptr, 10);
        else if (a == "--objectives") cfg.objectives = std::string(next()) == "base4" ? PE_OBJ_BASE4 : PE_OBJ_REF6;
        else if (a == "--gc") cfg.gc_mode = std::string(next()) == "gc" ? PE_GC_ALL : PE_GC3;
        else if (a == "--string") cfg.sl_kind = std::string(next()) == "lrcs" ? PE_SL_LRCS : PE_SL_HAIRPIN;
        else if (a == "--ref-p") cfg.ref_p = atoi(next());
        else if (a == "--codon-table") table_path = next();
        else if (a == "--dirichlet") dirichlet = atol(next());
        else if (a == "--synthetic-protein") {
            if (sscanf(next(), "%d:%llu", &synL, &synSeed) != 2) {
                fprintf(stderr, "--synthetic-protein wants L:SEED\n");
                return EXIT_FAILURE;
            }
        } else if (a == "--out") outdir = next();
        else {
            fprintf(stderr, "unknown option %s\n", a.c_str());
            return EXIT_FAILURE;
        }
    }

    std::vector<int8_t> aa;
    if (synL > 0) {
        aa.resize(synL + 1);
        if (pe_synthetic_protein(synL, synSeed, aa.data())) return die("synthetic protein");
    } else {
        int32_t len = 0;
        if (pe_parse_fasta(argv[1], nullptr, 0, &len)) return die("FASTA");
        aa.resize(len);
        if (pe_parse_fasta(argv[1], aa.data(), len, &len)) return die("FASTA");
    }
    pe_codon_table tab;
    if (dirichlet >= 0) {
        if (pe_dirichlet_table((uint64_t)dirichlet, &tab)) return die("codon table");
    } else if (pe_load_codon_table(table_path.c_str(), &tab)) {
        return die("codon table");
    }
    const int L = (int)aa.size(), cds_len = 3 * L;

    auto t0 = std::chrono::steady_clock::now();
    pe_instance *inst = nullptr;
    if (pe_create(&cfg, aa.data(), L, &tab, nullptr, &inst)) return die("pe_create");
    pe_info info;
    pe_get_info(inst, &info);
    const int M = info.M;
    printf("Protein length (incl. stop) : %d, CDSs : %d, population : %d, objectives : %d, reference points : %d\n", L,
           m, N, M, info.R);
    auto t1 = std::chrono::steady_clock::now();
    if (pe_init_population(inst) || pe_synchronize(inst)) return die("initialisation");
    auto t2 = std::chrono::steady_clock::now();
    if (pe_step(inst, G) || pe_synchronize(inst)) return die("generation loop");
    auto t3 = std::chrono::steady_clock::now();
    const int N2 = 2 * N;
    std::vector<uint8_t> pop((size_t)N2 * m * L);
    std::vector<float> obj((size_t)N2 * M);
    std::vector<int8_t> objidx((size_t)N2 * 2 * M);
    if (pe_get_population(inst, pop.data(), obj.data(), objidx.data(), nullptr, nullptr)) return die("read back");
    const int nsol = G == 0 ? N : N2;

    // Result.txt (src/main.cu:789-818): maximised objectives back to positive
    static const char *names6[6] = {"mCAI", "mCBP", "mHSC", "mHD", "MGC", "MSL"};
    static const char *names4[4] = {"mCAI", "mHD", "MGC", "MSL"};
    const char **names = M == 6 ? names6 : names4;
    const int nneg = M == 6 ? 4 : 2;
    for (int i = 0; i < nsol; i++)
        for (int k = 0; k < nneg; k++) obj[(size_t)i * M + k] = -obj[(size_t)i * M + k];
    std::string res_path = outdir + "/Result.txt";
    FILE *fp = fopen(res_path.c_str(), "w");
    if (!fp) {
        fprintf(stderr, "cannot write %s\n", res_path.c_str());
        return EXIT_FAILURE;
    }
    for (int i = 0; i < nsol; i++) {
        fprintf(fp, "%d Solutions\n", i + 1);
        for (int j = 0; j < m; j++) {
            fprintf(fp, "%d CDS : ", j + 1);
            for (int a = 0; a < L; a++) {
                const uint8_t *c = tab.nt[pop[((size_t)i * m + j) * L + a]];
                for (int b = 0; b < 3; b++) fputc("ACGU"[c[b]], fp);
            }
            fprintf(fp, "\n");
        }
        fprintf(fp, "\n %d Solution\n", i + 1);
        for (int k = 0; k < M; k++) {
            const int8_t *ix = &objidx[(size_t)i * 2 * M + 2 * k];
            if (!strcmp(names[k], "mHD")) fprintf(fp, "%d %d\t%s : %f\n", ix[0], ix[1], names[k], obj[(size_t)i * M + k]);
            else fprintf(fp, "%d\t%s : %f\n", ix[0], names[k], obj[(size_t)i * M + k]);
        }
    }
    fclose(fp);

    // normalisation with fixed ideal / nadir (src/main.cu:23-24, 820-835; the
    // four-objective constants of src/auto_execution_experiments.py:47-48)
    static const float ideal6[6] = {1.f, 0.2f, 0.4f, 0.5f, 0.f, 0.f}, nadir6[6] = {0.f, -0.15f, 0.f, 0.f, 0.6f, 1.f};
    static const float ideal4[4] = {1.f, 0.4f, 0.f, 0.f}, nadir4[4] = {0.f, 0.f, 0.6f, 1.f};
    const float *ideal = M == 6 ? ideal6 : ideal4, *nadir = M == 6 ? nadir6 : nadir4;
    std::vector<double> norm((size_t)nsol * M);
    double min_dist = 1e300;
    for (int i = 0; i < nsol; i++) {
        double d2 = 0.0;
        for (int k = 0; k < M; k++) {
            float v = (obj[(size_t)i * M + k] - ideal[k]) / (nadir[k] - ideal[k]);
            if (v >= 1.f) v = 0.999999f;
            if (v < 0.f) v = 0.f;
            obj[(size_t)i * M + k] = v;
            norm[(size_t)i * M + k] = v;
            d2 += (double)v * v;
        }
        min_dist = std::min(min_dist, std::sqrt(d2));
    }
    std::string norm_path = outdir + "/Normalized_value_quality_computation.txt";
    fp = fopen(norm_path.c_str(), "w");
    if (!fp) {
        fprintf(stderr, "cannot write %s\n", norm_path.c_str());
        return EXIT_FAILURE;
    }
    for (int i = 0; i < nsol; i++) {
        for (int k = 0; k < M; k++) fprintf(fp, k ? " %f" : "%f", obj[(size_t)i * M + k]);
        fprintf(fp, "\n");
    }
    fclose(fp);
    std::vector<double> ref(M, 1.0);
    double hv = 0.0;
    if (pe_hypervolume(norm.data(), nsol, M, ref.data(), &hv)) return die("hypervolume");
    pe_destroy(inst);

    double ti = std::chrono::duration<double>(t2 - t1).count();
    double tg = std::chrono::duration<double>(t3 - t2).count();
    double tc = std::chrono::duration<double>(t1 - t0).count();
    printf("\n\nHypervolume : %f\n", hv);
    printf("Minimum Distance to Ideal Point : %f\n", min_dist);
    printf("Setup time : %f seconds\n", tc);
    printf("Initialization time : %f seconds\n", ti);
    printf("Generation cycles time : %f seconds\n", tg);
    printf("Generations per second : %f\n", tg > 0 ? G / tg : 0.0);
    printf("Total time : %f seconds\n", ti + tg);
    return EXIT_SUCCESS;
}
