// hj_cli.cpp -- the two executables of the reference, on the GPU engine.
//
// Built twice: -DHJ_CLI_SELF gives hilbertSelfJoinCardinality (the reference's
// main.cpp), -DHJ_CLI_JOIN gives hilbertJoinCardinality (mainJoin.cpp). Same
// flags (util/arguments.cpp:24, :100):
//   -n N    points in set A            -m M    points in set B (join)
//   -e EPS  epsilon                    -d D    dimensionality
//   -f FILE set A (.csv or .bin)       -g FILE set B (join; the reference reads
//                                               B from -f instead, mainJoin.cpp:77)
//   -s S    active dimensions, (3^S+1)/2 stripes (0..5; the join ignores it as
//           the reference does, which hard-codes 2)
//   -t T, -k K, -a A   accepted and ignored, as in the reference
// Extensions: -F plain|fp16|tf32|bf16x3|auto (distance form, default plain),
//             -r (count like the reference: first 8*floor(n/8) EGO-sorted points),
//             -R 0|1 (dimension reordering off/on; on by default for the join,
//             which the reference's join driver always reorders,
//             mainJoin.cpp:97-100, off for the self-join, which never does).
// Output: the reference's one-line format (main.cpp:122, mainJoin.cpp:139).
// THREADS reports the GPU's SM count, KBLOCK the early-exit granularity (8
// dims), REORDERTIME the dimension cost and ordering step, WH is 0.
//
// Without -f/-g the sets are uniform [0,1) from the MCG31m1 recurrence
// x <- 1132489760 x mod (2^31 - 1), seeded 15 * seed with seed 1 for A and 2
// for B, first d values discarded -- the structure of the reference's
// random_init_unif (util/dataIo.cpp:4-33), whose MKL stream is not reproduced.
//
// Input files: CSV (',' separated, lines starting with '%' skipped, at most
// 2048 characters per line, missing values 0, as util/dataIo.cpp:113-165), raw
// little-endian FP64 '.bin' (dataIo.cpp:128-138), or raw FP32 '.f32'.
#include <getopt.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "hj.h"

static bool ends_with(const std::string &s, const char *suf) {
    size_t n = strlen(suf);
    return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

static void gen_uniform(std::vector<double> &x, size_t n, size_t d, int seed) {
    const uint64_t m = 2147483647ull;
    uint64_t s = (uint64_t)(15 * seed) % m;
    if (s == 0) s = 1;
    x.resize(n * d);
    for (size_t i = 0; i < d; ++i) s = (1132489760ull * s) % m;  // discarded, as the reference does
    for (size_t i = 0; i < n * d; ++i) {
        s = (1132489760ull * s) % m;
        x[i] = (double)s / (double)m;
    }
}

static bool read_points(const std::string &path, size_t n, size_t d, std::vector<double> &x, std::vector<float> &xf,
                        bool *is_f32) {
    *is_f32 = false;
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) {
        fprintf(stderr, "File '%s' does not exist!\n", path.c_str());
        return false;
    }
    if (ends_with(path, ".bin")) {
        x.assign(n * d, 0.0);
        size_t got = fread(x.data(), sizeof(double), n * d, f);
        fclose(f);
        if (got != n * d) {
            fprintf(stderr, "Binary file '%s' holds %zu values, %zu expected.\n", path.c_str(), got, n * d);
            return false;
        }
        return true;
    }
    if (ends_with(path, ".f32")) {
        xf.assign(n * d, 0.0f);
        size_t got = fread(xf.data(), sizeof(float), n * d, f);
        fclose(f);
        if (got != n * d) {
            fprintf(stderr, "Binary file '%s' holds %zu values, %zu expected.\n", path.c_str(), got, n * d);
            return false;
        }
        *is_f32 = true;
        return true;
    }
    x.assign(n * d, 0.0);
    char line[2049];
    size_t i = 0;
    while (i < n && fgets(line, sizeof line, f)) {
        if (line[0] == '%') continue;
        size_t j = 0;
        char *save = nullptr;
        for (char *tok = strtok_r(line, ",", &save); tok && j < d; tok = strtok_r(nullptr, ",", &save))
            x[i * d + j++] = atof(tok);
        ++i;
    }
    fclose(f);
    if (i < n) {
        fprintf(stderr, "Text file '%s' holds %zu rows, %zu expected.\n", path.c_str(), i, n);
        return false;
    }
    return true;
}

static void usage(const char *prog) {
#ifdef HJ_CLI_JOIN
    fprintf(stderr, "Usage: %s -n N -m M -e EPS -d D [-f fileA] [-g fileB] [-F plain|fp16|tf32|bf16x3|auto] [-r] [-R 0|1]\n",
            prog);
    fprintf(stderr, "Example: %s -n 200000 -m 200000 -e 0.2 -d 20\n", prog);
#else
    fprintf(stderr, "Usage: %s -n N -e EPS -d D [-f file] [-s activedims] [-F plain|fp16|tf32|bf16x3|auto] [-r] [-R 0|1]\n",
            prog);
    fprintf(stderr, "Example: %s -n 200000 -e 0.2 -d 64\n", prog);
#endif
}

int main(int argc, char **argv) {
    size_t n = 200000, m = 200000, d = 64;
    double eps = 0.2;
    std::string fa, fb;
    int actdim = 3;
    int form = HJ_FORM_PLAIN_FP64;
    bool refc = false;
#ifdef HJ_CLI_JOIN
    int reorder = 1;
#else
    int reorder = 0;
#endif
    if (argc < 5) {
        usage(argv[0]);
        return 1;
    }
    int c;
    while ((c = getopt(argc, argv, "n:m:e:d:t:f:g:k:a:s:F:rR:")) != -1) {
        switch (c) {
            case 'n': n = strtoull(optarg, 0, 10); break;
            case 'm': m = strtoull(optarg, 0, 10); break;
            case 'e': eps = atof(optarg); break;
            case 'd': d = strtoull(optarg, 0, 10); break;
            case 'f': fa = optarg; break;
            case 'g': fb = optarg; break;
            case 's': actdim = atoi(optarg); break;
            case 'r': refc = true; break;
            case 'R': reorder = atoi(optarg) != 0; break;
            case 'F':
                if (!strcmp(optarg, "plain")) form = HJ_FORM_PLAIN_FP64;
                else if (!strcmp(optarg, "tf32")) form = HJ_FORM_TC_TF32;
                else if (!strcmp(optarg, "fp16")) form = HJ_FORM_TC_FP16;
                else if (!strcmp(optarg, "bf16x3")) form = HJ_FORM_TC_BF16X3;
                else if (!strcmp(optarg, "auto")) form = HJ_FORM_AUTO;
                else {
                    fprintf(stderr, "unknown form '%s'\n", optarg);
                    return 1;
                }
                break;
            case 't': case 'k': case 'a': break;
            default: usage(argv[0]); return 1;
        }
    }
    if (actdim < 0 || actdim > 5) {
        fprintf(stderr, "parameter active dimensions must be in [0, 5]\n");
        return 1;
    }
    std::vector<double> A, B;
    std::vector<float> Af, Bf;
    bool af32 = false, bf32 = false;
    if (fa.empty()) gen_uniform(A, n, d, 1);
    else if (!read_points(fa, n, d, A, Af, &af32)) return 1;
#ifdef HJ_CLI_JOIN
    if (fb.empty()) gen_uniform(B, m, d, 2);
    else if (!read_points(fb, m, d, B, Bf, &bf32)) return 1;
    if (af32 != bf32) {  // mixed precision files: widen the FP32 one
        if (af32) { A.assign(Af.begin(), Af.end()); af32 = false; }
        if (bf32) { B.assign(Bf.begin(), Bf.end()); bf32 = false; }
    }
#endif
    hj_opts o;
    hj_opts_init(&o);
    o.form = form;
    o.ref_compat = refc ? 1 : 0;
    o.reorder_dims = reorder;
    hj_stats st;
    uint64_t count = 0;
    auto t0 = std::chrono::steady_clock::now();
#ifdef HJ_CLI_JOIN
    o.active_dims = 2;
    int r = af32 ? hj_join_count_f32(Af.data(), n, Bf.data(), m, (uint32_t)d, eps, &o, &count, &st)
                 : hj_join_count(A.data(), n, B.data(), m, (uint32_t)d, eps, &o, &count, &st);
#else
    o.active_dims = actdim;
    int r = af32 ? hj_self_join_count_f32(Af.data(), n, (uint32_t)d, eps, &o, &count, &st)
                 : hj_self_join_count(A.data(), n, (uint32_t)d, eps, &o, &count, &st);
#endif
    double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (r != HJ_OK) {
        fprintf(stderr, "join failed: %s: %s\n", hj_status_str(r), hj_last_error());
        return 2;
    }
    int sms = hj_device_sm_count(-1);
    double sort_s = st.sort_ms / 1e3, index_s = st.index_ms / 1e3, reorder_s = st.reorder_ms / 1e3;
    double jppp = count == 0 ? 0.0 : (double)count / (double)n;
    const int kblock = 8;
    int stripes = st.stripes;
#ifdef HJ_CLI_JOIN
    printf("%zu;%zu;%zu;%f;%d;%2.14f;%d;%d;%f;%f;%f;%f;%f;%ld;%f;%f\n", n, m, d, jppp, sms, eps, stripes, kblock,
           total, total - sort_s - reorder_s, sort_s, index_s, reorder_s, (long)count, st.loadpercent, 0.0);
#else
    printf("%zu;%zu;%f;%d;%2.14f;%d;%d;%f;%f;%f;%f;%f;%zu;%f;%f\n", n, d, jppp, sms, eps, stripes, kblock, total,
           total - sort_s - reorder_s, sort_s, index_s, reorder_s, (size_t)count, st.loadpercent, 0.0);
#endif
    return 0;
}
