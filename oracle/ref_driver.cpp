// Test-infrastructure driver for the hilbertJoin reference built from its own
// sources (oracle/build_ref.sh). It is the "reference" arm of the parity tests
// and of bench.py's CPU baseline, never part of the shipped engine.
//
// It binds the reference's two library entry points exactly as its CLIs do
// (main.cpp:95 and mainJoin.cpp:111) but skips the outputStatistics +
// reorder_dimensions pre-step (main.cpp:87-88, mainJoin.cpp:97-100): that step
// corrupts rows when d % 8 != 0 and is nondeterministic (drand48 from several
// threads), so the reference is only a valid oracle without it.
//
//   hj_ref self  <pts.bin> n d eps stripes      -> test_ego_loop3_macro  (hilbertjoin/egojoin.cpp:777)
//   hj_ref join  <A.bin> <B.bin> nA nB d eps    -> test_ego_loop3_noself (hilbertjoin/egojoin.cpp:840)
//   hj_ref egosort <pts.bin> n d eps <out.bin>  -> epsilonGridOrdering    (hilbertjoin/egojoin.cpp:159)
//
// Inputs are raw little-endian FP64 row-major files. Buffers get the 64-byte
// alignment and the +16384-byte slack that main.cpp:59 allocates, because the
// reference's loads and its NOSELF padding (hilbertjoin/egojoin.h:419-424) run
// past row n. One JSON line goes to stdout.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <omp.h>

void test_ego_loop3_macro(size_t n, size_t d, double epsilon, double *array, size_t *countresult,
                          int stripes, double *sortTime, double *indextime, double *loadpercent);
void test_ego_loop3_noself(const size_t nA, const size_t nB, const int d, const double epsilon,
                           double *arrayA, double *arrayB, size_t *countresult, const int activedims,
                           double *sortTime, double *indextime, double *loadpercent);
void epsilonGridOrdering(size_t n, size_t d, double epsilon, double *array);

static double *load_rows(const char *path, size_t n, size_t d) {
    size_t bytes = n * d * sizeof(double) + 16384;
    bytes = (bytes + 63) / 64 * 64;
    double *p = (double *)aligned_alloc(64, bytes);
    if (!p) { fprintf(stderr, "alloc failed\n"); exit(2); }
    memset(p, 0, bytes);
    FILE *f = fopen(path, "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(2); }
    size_t got = fread(p, sizeof(double), n * d, f);
    fclose(f);
    if (got != n * d) { fprintf(stderr, "short read %s: %zu of %zu\n", path, got, n * d); exit(2); }
    return p;
}

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int main(int argc, char **argv) {
    if (argc < 2) { fprintf(stderr, "usage: see header\n"); return 2; }
    omp_set_num_threads(NUM_THREADS);
    if (!strcmp(argv[1], "self") && argc == 7) {
        size_t n = strtoull(argv[3], 0, 10), d = strtoull(argv[4], 0, 10);
        double eps = atof(argv[5]);
        int stripes = atoi(argv[6]);
        double *x = load_rows(argv[2], n, d);
        size_t count = 0;
        double st = 0, it = 0, lp = 0;
        double t0 = now_s();
        test_ego_loop3_macro(n, d, eps, x, &count, stripes, &st, &it, &lp);
        double alg = now_s() - t0;
        printf("{\"count\": %zu, \"alg_s\": %.9f, \"sort_s\": %.9f, \"index_s\": %.9f, \"loadpercent\": %.9f, "
               "\"threads\": %d, \"kblock\": %d}\n", count, alg, st, it, lp, NUM_THREADS, KBLOCK);
        free(x);
        return 0;
    }
    if (!strcmp(argv[1], "join") && argc == 8) {
        size_t nA = strtoull(argv[4], 0, 10), nB = strtoull(argv[5], 0, 10);
        int d = atoi(argv[6]);
        double eps = atof(argv[7]);
        double *a = load_rows(argv[2], nA, d);
        double *b = load_rows(argv[3], nB, d);
        size_t count = 0;
        double st = 0, it = 0, lp = 0;
        double t0 = now_s();
        test_ego_loop3_noself(nA, nB, d, eps, a, b, &count, 2, &st, &it, &lp);
        double alg = now_s() - t0;
        printf("{\"count\": %zu, \"alg_s\": %.9f, \"sort_s\": %.9f, \"index_s\": %.9f, \"loadpercent\": %.9f, "
               "\"threads\": %d, \"kblock\": %d}\n", count, alg, st, it, lp, NUM_THREADS, KBLOCK);
        free(a);
        free(b);
        return 0;
    }
    if (!strcmp(argv[1], "egosort") && argc == 7) {
        size_t n = strtoull(argv[3], 0, 10), d = strtoull(argv[4], 0, 10);
        double eps = atof(argv[5]);
        double *x = load_rows(argv[2], n, d);
        epsilonGridOrdering(n, d, eps, x);
        FILE *f = fopen(argv[6], "wb");
        if (!f || fwrite(x, sizeof(double), n * d, f) != n * d) { fprintf(stderr, "write failed\n"); return 2; }
        fclose(f);
        printf("{\"sorted\": %zu}\n", n);
        free(x);
        return 0;
    }
    fprintf(stderr, "bad arguments\n");
    return 2;
}
