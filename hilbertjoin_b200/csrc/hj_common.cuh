// hj_common.cuh -- shared device helpers of the B200 epsilon-join engine:
// bounded mbarrier waits, 1D bulk copies and 2D TMA tile loads (inline PTX for
// sm_100a), error words, and small integer utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#ifndef HJ_DEVICE_INLINE
#define HJ_DEVICE_INLINE __device__ __forceinline__
#endif

namespace hj {

// Error bits a kernel can raise in its device error word. A kernel that raises
// one returns early; the host maps the word to an hj_status.
enum : uint32_t {
    kErrTimeout = 1u,      // a bounded wait on an mbarrier gave up
    kErrBandOverflow = 2u, // band queue full (host regrows and reruns)
    kErrBounds = 4u,       // an index check failed (debug builds)
};

// Upper bound of one device-side wait, in nanoseconds of %globaltimer. Every
// legitimate wait in this engine lasts at most a few tile times (microseconds);
// the bound only exists so that a logic error ends in an error status instead
// of a hung GPU.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s

HJ_DEVICE_INLINE uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

HJ_DEVICE_INLINE uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

HJ_DEVICE_INLINE void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

HJ_DEVICE_INLINE void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

HJ_DEVICE_INLINE void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

HJ_DEVICE_INLINE void mbar_arrive(uint64_t *bar) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
        : "memory");
}

HJ_DEVICE_INLINE void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

HJ_DEVICE_INLINE bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits until the phase with the given parity has completed. Returns false
// (and raises kErrTimeout in *err, with `site` in bits 8..15 to tell which
// wait gave up) if that takes longer than kWaitLimitNs or if another thread
// already raised an error.
HJ_DEVICE_INLINE bool mbar_wait(uint64_t *bar, uint32_t parity, volatile uint32_t *err, uint32_t site = 0) {
    if (mbar_try_wait(bar, parity)) return true;
    uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0) {
            if (*err != 0) return false;
            if (globaltimer_ns() - t0 > kWaitLimitNs) {
                atomicOr((uint32_t *)err, kErrTimeout | ((site & 0xffu) << 8));
                return false;
            }
        }
    }
}

// 1D bulk copy global -> shared, completion counted on `bar` (complete_tx).
// Both addresses 16-byte aligned, bytes a multiple of 16.
HJ_DEVICE_INLINE void bulk_g2s(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// 2D tiled TMA load (no multicast): box at coordinates (x = innermost, y).
HJ_DEVICE_INLINE void tma_load_2d(void *smem_dst, const void *tmap, int32_t x, int32_t y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(smem_dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

HJ_DEVICE_INLINE void prefetch_tmap(const void *tmap) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(tmap) : "memory");
}

HJ_DEVICE_INLINE uint32_t lane_id() { return threadIdx.x & 31u; }

HJ_DEVICE_INLINE unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// floor(x / eps) with x / eps the IEEE (correctly rounded) FP64 quotient --
// the cell of the pair test's convention -- without a division in the common
// case. With inv = fl(1 / eps), q = fl(x * inv) differs from x / eps by at
// most |x / eps| (2u + u^2) and from fl(x / eps) by at most 3.01 u |q|
// (u = 2^-53), so every value within 2^-50 |q| of q has the same floor as
// fl(x / eps) whenever q - 2^-50 |q| and q + 2^-50 |q| do (the margin also
// covers the rounding of those two bounds). Only near a cell border, where
// they differ, is the quotient computed by division.
__device__ __forceinline__ double cell_of(double x, double eps, double inv) {
    const double q = x * inv;
    const double m = fabs(q) * 8.881784197001252e-16;  // 2^-50
    const double lo = floor(q - m);
    if (lo == floor(q + m)) return lo;
    return floor(x / eps);
}

}  // namespace hj

// Host-side helpers ---------------------------------------------------------
__host__ __device__ static inline uint64_t hj_ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }
__host__ __device__ static inline uint64_t hj_umin(uint64_t a, uint64_t b) { return a < b ? a : b; }
