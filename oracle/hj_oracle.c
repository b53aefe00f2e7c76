/* hj_oracle.c -- CPU oracle for the epsilon-join cardinality path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that the GPU engine is
 * compared against. Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load it. The engine under hilbertjoin_b200/ never
 * links, loads or calls it, and has no CPU fallback.
 *
 * It restates, in plain C, the algorithm of the hilbertJoin reference
 * (perdacherMartin/hilbertJoin) for the count path:
 *
 *   - cell of a coordinate: floor(x / eps) in FP64, as epsilonGridCompare
 *     does (hilbertjoin/egojoin.cpp:9-17);
 *   - epsilon-grid order (EGO): lexicographic order of the cell vectors, dim 0
 *     most significant (hilbertjoin/egojoin.cpp:159-168). The reference sorts
 *     with an unstable parallel quicksort (egojoin.cpp:594-634); this oracle
 *     sorts stably (ties keep input order), which is the order the GPU engine
 *     produces, so permutations can be compared exactly;
 *   - stripes: per point, contiguous ranges of the EGO order that can hold its
 *     neighbours, one per combination of neighbour cells in the first
 *     `active_dims` dimensions (prepareStripes, egojoin.cpp:270-464, and
 *     prepareStripesNoSelf, egojoin.cpp:1126-1240). Two deliberate fixes: the
 *     upper bound is inclusive (the reference's "first >=" search at
 *     egojoin.cpp:408-412 excludes the cell of x+eps itself), and the
 *     displacement is widened from eps to eps' = eps + 2^-40 (eps + max|x|), so
 *     the ranges provably contain every pair the FP64 test accepts even when
 *     floor(x/eps) jitters at cell borders;
 *   - the pair test: the reference evaluates (eps^2 - |a-b|^2)/2 by norm
 *     expansion and counts a pair when its sign bit is clear
 *     (egojoin.h:329-392, egojoin.cpp:803-813), i.e. |a-b|^2 <= eps^2,
 *     inclusive. This oracle -- and the engine's plain FP64 form -- evaluate
 *     |a-b|^2 by direct difference: acc = fma(a_k - b_k, a_k - b_k, acc) for
 *     k = 0..d-1 in FP64, and count iff acc <= eps*eps (FP64). On continuous
 *     data both agree; on exact ties at eps the direct difference is the
 *     defined semantics of this engine;
 *   - count convention: self-join counts unordered pairs {a,b}, a != b
 *     (the diagonal mask at egojoin.h:383-392); the two-set join counts ordered
 *     pairs (a in A, b in B) (EGO_LOOP_TRAN_NOSELF, egojoin.h:482-553). The
 *     reference only looks at the first 8*floor(n/8) EGO-sorted points of each
 *     set (its loops run over floor(n/8) blocks); `tail_drop` reproduces that.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define HJO_EXPORT __attribute__((visibility("default")))

/* The pair test, shared by every counting routine below. */
static inline double dist2(const double *a, const double *b, uint32_t d) {
    double acc = 0.0;
    for (uint32_t k = 0; k < d; ++k) {
        double df = a[k] - b[k];
        acc = fma(df, df, acc);
    }
    return acc;
}

HJO_EXPORT double hjo_dist2(const double *a, const double *b, uint32_t d) { return dist2(a, b, d); }

HJO_EXPORT double hjo_eps_wide(double eps, double maxabs) {
    return eps + ldexp(eps + maxabs, -40);
}

static void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

/* Brute-force count over all pairs (i in A, j in B), restricted to j > i for a
 * self-join (A == B). Cache-blocked so that it stays compute-bound at a
 * million points: B is cut into chunks of kJC partners, each thread copies one
 * chunk transposed ([d][kJC], about 0.5 MB at d = 64) and streams every A row
 * past it, 4 rows x 8 partners at a time. Each pair keeps the exact sequential
 * FMA order of dist2 (the vector lanes are different pairs), so the count is
 * the pair test's, bit for bit. */
#define kJC 1024
#ifdef __AVX2__
#include <immintrin.h>
#endif

static uint64_t brute_chunk(const double *A, uint64_t ilim, const double *bt, uint64_t j0, uint64_t w, uint32_t d,
                            double T, int self) {
    uint64_t cnt = 0;
    for (uint64_t i = 0; i < ilim; i += 4) {
        const uint64_t nr = ilim - i < 4 ? ilim - i : 4;
        const double *a[4];
        for (int r = 0; r < 4; ++r) a[r] = A + (size_t)(i + ((uint64_t)r < nr ? (uint64_t)r : 0)) * d;
        uint64_t lstart = 0;
        if (self && i + 1 > j0) lstart = (i + 1 - j0) / 8 * 8;
        for (uint64_t lb = lstart; lb < w; lb += 8) {
            double acc[4][8];
#ifdef __AVX2__
            __m256d c00 = _mm256_setzero_pd(), c01 = c00, c10 = c00, c11 = c00, c20 = c00, c21 = c00, c30 = c00,
                    c31 = c00;
            for (uint32_t k = 0; k < d; ++k) {
                const double *b = bt + (size_t)k * kJC + lb;
                const __m256d b0 = _mm256_loadu_pd(b), b1 = _mm256_loadu_pd(b + 4);
                __m256d x = _mm256_set1_pd(a[0][k]), d0 = _mm256_sub_pd(x, b0), d1 = _mm256_sub_pd(x, b1);
                c00 = _mm256_fmadd_pd(d0, d0, c00);
                c01 = _mm256_fmadd_pd(d1, d1, c01);
                x = _mm256_set1_pd(a[1][k]), d0 = _mm256_sub_pd(x, b0), d1 = _mm256_sub_pd(x, b1);
                c10 = _mm256_fmadd_pd(d0, d0, c10);
                c11 = _mm256_fmadd_pd(d1, d1, c11);
                x = _mm256_set1_pd(a[2][k]), d0 = _mm256_sub_pd(x, b0), d1 = _mm256_sub_pd(x, b1);
                c20 = _mm256_fmadd_pd(d0, d0, c20);
                c21 = _mm256_fmadd_pd(d1, d1, c21);
                x = _mm256_set1_pd(a[3][k]), d0 = _mm256_sub_pd(x, b0), d1 = _mm256_sub_pd(x, b1);
                c30 = _mm256_fmadd_pd(d0, d0, c30);
                c31 = _mm256_fmadd_pd(d1, d1, c31);
            }
            _mm256_storeu_pd(acc[0], c00);
            _mm256_storeu_pd(acc[0] + 4, c01);
            _mm256_storeu_pd(acc[1], c10);
            _mm256_storeu_pd(acc[1] + 4, c11);
            _mm256_storeu_pd(acc[2], c20);
            _mm256_storeu_pd(acc[2] + 4, c21);
            _mm256_storeu_pd(acc[3], c30);
            _mm256_storeu_pd(acc[3] + 4, c31);
#else
            for (int r = 0; r < 4; ++r)
                for (int l = 0; l < 8; ++l) acc[r][l] = 0.0;
            for (uint32_t k = 0; k < d; ++k) {
                const double *b = bt + (size_t)k * kJC + lb;
                for (int r = 0; r < 4; ++r)
                    for (int l = 0; l < 8; ++l) {
                        const double df = a[r][k] - b[l];
                        acc[r][l] = fma(df, df, acc[r][l]);
                    }
            }
#endif
            for (uint64_t r = 0; r < nr; ++r)
                for (uint64_t l = 0; l < 8; ++l) {
                    const uint64_t j = j0 + lb + l;
                    if (lb + l < w && (!self || j > i + r) && acc[r][l] <= T) ++cnt;
                }
        }
    }
    return cnt;
}

static uint64_t brute_count(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d, double eps,
                            int self) {
    const double T = eps * eps;
    const uint64_t nch = (nB + kJC - 1) / kJC;
    uint64_t total = 0;
#pragma omp parallel reduction(+ : total)
    {
        double *bt = (double *)malloc(sizeof(double) * (size_t)kJC * d + 64);
#pragma omp for schedule(dynamic, 1)
        for (int64_t c = (int64_t)nch - 1; c >= 0; --c) { /* largest self-join chunks first */
            const uint64_t j0 = (uint64_t)c * kJC, w = nB - j0 < kJC ? nB - j0 : kJC;
            for (uint32_t k = 0; k < d; ++k)
                for (uint64_t l = 0; l < kJC; ++l) bt[(size_t)k * kJC + l] = l < w ? B[(size_t)(j0 + l) * d + k] : 0.0;
            const uint64_t ilim = self ? (j0 + w < nA ? j0 + w : nA) : nA;
            total += brute_chunk(A, ilim, bt, j0, w, d, T, self);
        }
        free(bt);
    }
    return total;
}

HJO_EXPORT uint64_t hjo_self_count_brute(const double *X, uint64_t n, uint32_t d, double eps, int nthreads) {
    set_threads(nthreads);
    return brute_count(X, n, X, n, d, eps, 1);
}

/* Brute-force two-set join: ordered pairs (a in A, b in B). */
HJO_EXPORT uint64_t hjo_join_count_brute(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d,
                                        double eps, int nthreads) {
    set_threads(nthreads);
    return brute_count(A, nA, B, nB, d, eps, 0);
}

/* Per-row neighbour counts (all partners j != i in the same set) for a list of
 * rows: lets a test check a sample of rows at sizes where the full brute force
 * would take too long. */
HJO_EXPORT void hjo_self_row_counts(const double *X, uint64_t n, uint32_t d, double eps, const uint64_t *rows,
                                    uint64_t nrows, uint64_t *out, int nthreads) {
    const double T = eps * eps;
    set_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t r = 0; r < (int64_t)nrows; ++r) {
        uint64_t i = rows[r], cnt = 0;
        for (uint64_t j = 0; j < n; ++j)
            if (j != i && dist2(X + (size_t)i * d, X + (size_t)j * d, d) <= T) ++cnt;
        out[r] = cnt;
    }
}

/* ---------------------------------------------------------------- pair lists */

/* The qualifying pairs themselves, as (i, j) input indices sorted by (i, j):
 * self joins i < j, two-set joins (index in A, index in B). The reference
 * would push join_pair{p1, p2} (hilbertjoin/egojoin.h:32-35) per qualifying
 * pair (hilbertjoin/test_ego_loop3_queue.cpp:19-37); that code is compiled out
 * of its count build, so this restates the pair list from the same pair test.
 * Two passes: per-row counts, then each row's pairs at its prefix offset.
 * Writes out[0 .. 2*total) only if total <= cap; returns total. */
static uint64_t pairs_brute(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d, double eps,
                            int self, uint64_t *out, uint64_t cap, int nthreads) {
    const double T = eps * eps;
    set_threads(nthreads);
    uint64_t *rc = (uint64_t *)calloc((size_t)nA + 1, sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t ii = 0; ii < (int64_t)nA; ++ii) {
        uint64_t i = (uint64_t)ii, cnt = 0;
        for (uint64_t j = self ? i + 1 : 0; j < nB; ++j)
            if (dist2(A + (size_t)i * d, B + (size_t)j * d, d) <= T) ++cnt;
        rc[i] = cnt;
    }
    uint64_t total = 0;
    for (uint64_t i = 0; i < nA; ++i) {
        uint64_t c = rc[i];
        rc[i] = total;
        total += c;
    }
    if (total <= cap && out) {
#pragma omp parallel for schedule(dynamic, 16)
        for (int64_t ii = 0; ii < (int64_t)nA; ++ii) {
            uint64_t i = (uint64_t)ii, o = rc[i];
            for (uint64_t j = self ? i + 1 : 0; j < nB; ++j)
                if (dist2(A + (size_t)i * d, B + (size_t)j * d, d) <= T) {
                    out[2 * o] = i;
                    out[2 * o + 1] = j;
                    ++o;
                }
        }
    }
    free(rc);
    return total;
}

HJO_EXPORT uint64_t hjo_self_pairs_brute(const double *X, uint64_t n, uint32_t d, double eps, uint64_t *out,
                                         uint64_t cap, int nthreads) {
    return pairs_brute(X, n, X, n, d, eps, 1, out, cap, nthreads);
}

HJO_EXPORT uint64_t hjo_join_pairs_brute(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d,
                                         double eps, uint64_t *out, uint64_t cap, int nthreads) {
    return pairs_brute(A, nA, B, nB, d, eps, 0, out, cap, nthreads);
}

/* ---------------------------------------------------------- dimension order */

static int cmp_double(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* Per-dim cost of the Super-EGO dimension reordering, the estimate of the
 * reference's outputStatistics (hilbertjoin/egojoin.cpp:523-592): with h the
 * histogram of the sampled points' cells floor(x/eps) in dim j,
 * cost_j = sum_c h[c](h[c]-1)/2 + sum_c h[c-1] h[c], i.e. the number of
 * unordered sample pairs whose cells are equal or adjacent. The reference
 * samples with drand48 and skips dims with cells beyond +-100000; this
 * restatement uses the engine's deterministic sample (S = min(n, 8192) points,
 * point floor(s n / S) for s = 0..S-1) and costs every dim. */
HJO_EXPORT void hjo_dim_costs(const double *X, uint64_t n, uint32_t d, double eps, uint64_t *costs) {
    const uint64_t S = n < 8192 ? n : 8192;
    double *v = (double *)malloc((S ? S : 1) * sizeof(double));
    for (uint32_t t = 0; t < d; ++t) {
        for (uint64_t s = 0; s < S; ++s) v[s] = floor(X[(s * n / S) * d + t] / eps);
        qsort(v, S, sizeof(double), cmp_double);
        uint64_t cost = 0, q = 0;
        for (uint64_t s = 0; s < S; ++s) {
            if (q < s + 1) q = s + 1;
            while (q < S && v[q] <= v[s] + 1.0) ++q;
            cost += q - s - 1;
        }
        costs[t] = cost;
    }
    free(v);
}

/* ---------------------------------------------------------------- EGO order */

HJO_EXPORT void hjo_cells(const double *X, uint64_t n, uint32_t d, double eps, double *cells) {
    for (uint64_t i = 0; i < n * (uint64_t)d; ++i) cells[i] = floor(X[i] / eps);
}

typedef struct {
    const double *cells;
    uint32_t d;
} ego_ctx;

static int cmp_vec(const double *a, const double *b, uint32_t d) {
    for (uint32_t t = 0; t < d; ++t) {
        if (a[t] < b[t]) return -1;
        if (a[t] > b[t]) return 1;
    }
    return 0;
}

/* Stable merge sort of indices by cell vector. */
static void merge_sort_idx(uint64_t *idx, uint64_t *tmp, uint64_t n, const ego_ctx *c) {
    for (uint64_t w = 1; w < n; w *= 2) {
        for (uint64_t lo = 0; lo < n; lo += 2 * w) {
            uint64_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
            uint64_t i = lo, j = mid, o = lo;
            while (i < mid && j < hi) {
                if (cmp_vec(c->cells + idx[j] * c->d, c->cells + idx[i] * c->d, c->d) < 0)
                    tmp[o++] = idx[j++];
                else
                    tmp[o++] = idx[i++];
            }
            while (i < mid) tmp[o++] = idx[i++];
            while (j < hi) tmp[o++] = idx[j++];
        }
        memcpy(idx, tmp, n * sizeof(uint64_t));
    }
}

/* perm[r] = input index of the point at EGO rank r (stable). */
HJO_EXPORT void hjo_ego_order(const double *X, uint64_t n, uint32_t d, double eps, uint64_t *perm) {
    double *cells = (double *)malloc(sizeof(double) * n * d + 8);
    hjo_cells(X, n, d, eps, cells);
    uint64_t *tmp = (uint64_t *)malloc(sizeof(uint64_t) * n + 8);
    for (uint64_t i = 0; i < n; ++i) perm[i] = i;
    ego_ctx c = {cells, d};
    merge_sort_idx(perm, tmp, n, &c);
    free(tmp);
    free(cells);
}

/* --------------------------------------------------------------- stripes */

/* First rank r in [0,n) whose cell vector is >= q (strict=0) or > q (strict=1). */
static uint64_t search(const double *sc, uint64_t n, uint32_t d, const double *q, int strict) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = lo + (hi - lo) / 2;
        int c = cmp_vec(sc + mid * d, q, d);
        if (c < 0 || (strict && c == 0))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

/* Neighbour-cell bounds of one point: lo_t = cell(x_t - eps'), hi_t = cell(x_t + eps'). */
static void point_bounds(const double *x, uint32_t d, double eps, double epsw, double *lo, double *hi) {
    for (uint32_t t = 0; t < d; ++t) {
        lo[t] = floor((x[t] - epsw) / eps);
        hi[t] = floor((x[t] + epsw) / eps);
    }
}

/* Counts via EGO order + stripes + the FP64 pair test. B is sorted once; for
 * every point a of A, each combination of neighbour cells over the first
 * k = active_dims dimensions gives one range [first >= (v, lo_k..), first >
 * (v, hi_k..)) of B's EGO order (the stripe of that combination). The ranges
 * of one point are disjoint because their first k cells differ. For a
 * self-join only partners at a later EGO rank are taken. Returns the count and
 * the number of candidate pairs tested (the work the stripes leave). */
static uint64_t ego_count(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d, double eps,
                          int active_dims, int self, uint64_t tail_drop, uint64_t *candidates) {
    const double T = eps * eps;
    double maxabs = 0.0;
    for (uint64_t i = 0; i < nA * (uint64_t)d; ++i) maxabs = fmax(maxabs, fabs(A[i]));
    for (uint64_t i = 0; i < nB * (uint64_t)d; ++i) maxabs = fmax(maxabs, fabs(B[i]));
    const double epsw = hjo_eps_wide(eps, maxabs);

    uint64_t *pb = (uint64_t *)malloc(sizeof(uint64_t) * nB + 8);
    hjo_ego_order(B, nB, d, eps, pb);
    double *sb = (double *)malloc(sizeof(double) * nB * d + 8); /* sorted B rows */
    double *sc = (double *)malloc(sizeof(double) * nB * d + 8); /* sorted B cells */
    for (uint64_t r = 0; r < nB; ++r) {
        memcpy(sb + r * d, B + pb[r] * d, sizeof(double) * d);
        for (uint32_t t = 0; t < d; ++t) sc[r * d + t] = floor(sb[r * d + t] / eps);
    }
    uint64_t *pa = pb;
    const double *sa = sb;
    double *sa_own = 0;
    uint64_t *pa_own = 0;
    if (!self) {
        pa_own = (uint64_t *)malloc(sizeof(uint64_t) * nA + 8);
        hjo_ego_order(A, nA, d, eps, pa_own);
        sa_own = (double *)malloc(sizeof(double) * nA * d + 8);
        for (uint64_t r = 0; r < nA; ++r) memcpy(sa_own + r * d, A + pa_own[r] * d, sizeof(double) * d);
        pa = pa_own;
        sa = sa_own;
    }
    uint64_t na_eff = nA, nb_eff = nB;
    if (tail_drop) {
        na_eff = nA / 8 * 8;
        nb_eff = nB / 8 * 8;
    }
    uint32_t k = (uint32_t)active_dims < d ? (uint32_t)active_dims : d;
    uint64_t total = 0, cand = 0;
#pragma omp parallel reduction(+ : total, cand)
    {
        double *lo = (double *)malloc(sizeof(double) * d), *hi = (double *)malloc(sizeof(double) * d);
        double *ql = (double *)malloc(sizeof(double) * d), *qh = (double *)malloc(sizeof(double) * d);
#pragma omp for schedule(dynamic, 64)
        for (int64_t ii = 0; ii < (int64_t)na_eff; ++ii) {
            const double *a = sa + (uint64_t)ii * d;
            point_bounds(a, d, eps, epsw, lo, hi);
            /* A combination only splits dims whose neighbour set is <= 3 cells wide
             * (always, unless floor(x/eps) jitters); the first wider dim and all
             * later ones stay ranges. */
            uint32_t ke = 0;
            while (ke < k && hi[ke] - lo[ke] <= 2.0) ++ke;
            uint64_t ncomb = 1;
            for (uint32_t t = 0; t < ke; ++t) ncomb *= (uint64_t)(hi[t] - lo[t] + 1.0);
            for (uint64_t c = 0; c < ncomb; ++c) {
                uint64_t rem = c;
                for (int t = (int)ke - 1; t >= 0; --t) {
                    uint64_t w = (uint64_t)(hi[t] - lo[t] + 1.0);
                    ql[t] = qh[t] = lo[t] + (double)(rem % w);
                    rem /= w;
                }
                for (uint32_t t = ke; t < d; ++t) {
                    ql[t] = lo[t];
                    qh[t] = hi[t];
                }
                uint64_t r0 = search(sc, nb_eff, d, ql, 0), r1 = search(sc, nb_eff, d, qh, 1);
                if (self && r0 < (uint64_t)ii + 1) r0 = (uint64_t)ii + 1;
                for (uint64_t r = r0; r < r1; ++r) {
                    ++cand;
                    if (dist2(a, sb + r * d, d) <= T) ++total;
                }
            }
        }
        free(lo);
        free(hi);
        free(ql);
        free(qh);
    }
    if (candidates) *candidates = cand;
    free(pb);
    free(sb);
    free(sc);
    free(pa_own);
    free(sa_own);
    (void)pa;
    return total;
}

HJO_EXPORT uint64_t hjo_self_count_ego(const double *X, uint64_t n, uint32_t d, double eps, int active_dims,
                                      int tail_drop, int nthreads, uint64_t *candidates) {
    set_threads(nthreads);
    return ego_count(X, n, X, n, d, eps, active_dims, 1, (uint64_t)tail_drop, candidates);
}

HJO_EXPORT uint64_t hjo_join_count_ego(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d,
                                      double eps, int active_dims, int tail_drop, int nthreads,
                                      uint64_t *candidates) {
    set_threads(nthreads);
    return ego_count(A, nA, B, nB, d, eps, active_dims, 0, (uint64_t)tail_drop, candidates);
}
