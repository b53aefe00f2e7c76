/* Stand-in for the two MKL VSL calls the reference's data generator makes
 * (util/dataIo.cpp:4-33). The reference links MKL only to generate its default
 * uniform data; the join path never touches it. This header implements the
 * MCG31m1 generator from its public definition (x <- 1132489760*x mod 2^31-1,
 * u = x / (2^31-1)) so the reference's sources compile unmodified. It is used by
 * oracle/build_ref.sh only; the driver always feeds data from files, so the
 * generated stream being different from MKL's does not matter. */
#ifndef HJ_SHIM_MKL_VSL_H
#define HJ_SHIM_MKL_VSL_H
#include <stdint.h>
#include <stdlib.h>

#define VSL_BRNG_MCG31 1
#define VSL_ERROR_OK 0
#define VSL_STATUS_OK 0
#define VSL_RNG_METHOD_UNIFORM_STD 0

typedef struct hj_shim_vsl_stream { uint64_t x; } *VSLStreamStatePtr;

static inline int vslNewStream(VSLStreamStatePtr *s, int brng, unsigned int seed) {
    (void)brng;
    *s = (VSLStreamStatePtr)malloc(sizeof(struct hj_shim_vsl_stream));
    if (!*s) return -1;
    uint64_t x = seed % 2147483647ull;
    (*s)->x = x ? x : 1;
    return VSL_STATUS_OK;
}

static inline int vdRngUniform(int method, VSLStreamStatePtr s, int n, double *r, double a, double b) {
    (void)method;
    const uint64_t m = 2147483647ull;
    for (int i = 0; i < n; ++i) {
        s->x = (1132489760ull * s->x) % m;
        r[i] = a + (b - a) * ((double)s->x / (double)m);
    }
    return VSL_STATUS_OK;
}
#endif
