// hj_noalloc.cu -- EGO sort of device-resident points without any allocation.
//
// Some callers cannot call cudaMalloc while they run: an application whose own
// memory pool owns the whole device and forbids libraries from allocating, or
// a loop on a latency-critical stream that must not pay the implicit device
// synchronisation and possible failure of cudaMalloc/cudaFree in the middle of
// its work. For them, hj_ego_sort_device_noalloc keeps every temporary (cell
// statistics, packing tables, packed keys, the second permutation buffer and
// the radix histograms) in one fixed array inside the library: the caller
// passes only the input points and the output permutation. The array is a
// file-scope __device__ object of kScratchBytes, so every GPU that loads this
// library holds it until the process exits.
//
// Host code cannot use the array's name as a device address, so on the first
// call on each device (with that device current) the entry point looks the
// address up once with cudaGetSymbolAddress and keeps it. That first call
// should therefore come before any stream capture. Every call shares the
// array and it keeps the last call's contents: what must start at zero is
// cleared by the call itself, and calls that overlap on the GPU (different
// streams or threads) race on it; calls on one stream run in order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/hj.h"
#include "hj_common.cuh"
#include "hj_internal.h"

namespace hj {
namespace {

constexpr size_t kScratchBytes = 32ull << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_addr[kMaxDevices] = {};

int scratch_address(int dev, unsigned char **out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return engine_fail(HJ_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                                cudaGetErrorString(e));
        }
        g_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_addr[dev];
    return HJ_OK;
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

int bits_of(unsigned long long v) {
    int b = 0;
    while (b < 64 && (v >> b) != 0) ++b;
    return b;
}

}  // namespace
}  // namespace hj

using namespace hj;

extern "C" int hj_ego_sort_device_noalloc(const void *pts, int dtype_bytes, uint64_t n, uint32_t d, double eps,
                                          uint32_t *perm, void *stream) {
    engine_clear_error();
    if (!perm || (n && !pts)) return engine_fail(HJ_ERR_INVALID_ARG, "null pointer");
    if (dtype_bytes != 4 && dtype_bytes != 8) return engine_fail(HJ_ERR_INVALID_ARG, "dtype_bytes must be 4 or 8");
    if (d == 0 || d > kMaxDim) return engine_fail(HJ_ERR_INVALID_ARG, "d out of range");
    if (n >= (1ull << 31)) return engine_fail(HJ_ERR_INVALID_ARG, "n must be below 2^31");
    if (!(eps > 0.0) || !std::isfinite(eps)) return engine_fail(HJ_ERR_INVALID_ARG, "eps must be finite and > 0");
    if (n == 0) return HJ_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // scratch layout: stats | maxabs, bad | off | bits | word | shift | keys [W][n] | radix sort scratch
    const size_t o_stats = 0;
    const size_t o_small = align256(o_stats + (size_t)d * sizeof(DimStats));
    const size_t o_off = align256(o_small + 16);
    const size_t o_bits = align256(o_off + (size_t)d * 8);
    const size_t o_word = align256(o_bits + (size_t)d * 4);
    const size_t o_shift = align256(o_word + (size_t)d * 4);
    const size_t o_keys = align256(o_shift + (size_t)d * 4);
    const size_t rs_bytes = radix_scratch_bytes(n);
    // at least one key word: reject before touching the device when even that does not fit
    if (o_keys + align256(n * 4) + rs_bytes > kScratchBytes)
        return engine_fail(HJ_ERR_INVALID_ARG, "n too large for the fixed 32 MiB scratch array");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return engine_fail(HJ_ERR_NO_DEVICE, "no usable CUDA device");
    }
    unsigned char *base = nullptr;
    if (int r = scratch_address(dev, &base)) return r;
    DimStats *ds = reinterpret_cast<DimStats *>(base + o_stats);
    unsigned long long *d_maxabs = reinterpret_cast<unsigned long long *>(base + o_small);
    uint32_t *d_bad = reinterpret_cast<uint32_t *>(base + o_small + 8);

    // 1. cell statistics (the init kernel clears what the call accumulates into)
    launch_dim_stats_init(ds, d, d_maxabs, d_bad, st);
    launch_dim_stats(pts, dtype_bytes, n, d, eps, ds, d_maxabs, d_bad, st);
    DimStats hds[kMaxDim];
    uint32_t hbad = 0;
    cudaMemcpyAsync(hds, ds, d * sizeof(DimStats), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&hbad, d_bad, 4, cudaMemcpyDeviceToHost, st);
    if (cudaError_t e = cudaStreamSynchronize(st)) {
        cudaGetLastError();
        return engine_fail(HJ_ERR_CUDA, std::string("cell statistics: ") + cudaGetErrorString(e));
    }
    if (hbad & 1u) return engine_fail(HJ_ERR_INVALID_ARG, "input holds a non-finite coordinate");
    if (hbad) return engine_fail(HJ_ERR_INVALID_ARG, "a cell index floor(x/eps) exceeds 2^62");

    // 2. packed key layout (same rule as the allocating path)
    long long off[kMaxDim];
    uint32_t bits[kMaxDim], word[kMaxDim], shift[kMaxDim];
    long long range[kMaxDim];
    uint32_t w = 0, left = 32;
    for (uint32_t t = 0; t < d; ++t) {
        long long lo = hds[t].cmin, hi = hds[t].cmax;
        if (lo > hi) lo = hi = 0;
        range[t] = hi - lo;
        if (range[t] < 0 || range[t] > (1ll << 30))
            return engine_fail(HJ_ERR_INVALID_ARG, "a dimension spans more than 2^30 cells");
        const uint32_t b = (uint32_t)bits_of((unsigned long long)range[t] + 4);
        if (b > left) {
            ++w;
            left = 32;
        }
        off[t] = lo - 2;
        bits[t] = b;
        word[t] = w;
        shift[t] = left - b;
        left -= b;
    }
    const uint32_t W = w + 1;
    const size_t o_rs = align256(o_keys + (size_t)W * n * 4);
    if (o_rs + rs_bytes > kScratchBytes)
        return engine_fail(HJ_ERR_INVALID_ARG, "packed keys of this input exceed the fixed 32 MiB scratch array");
    GridDev gd;
    gd.off = reinterpret_cast<long long *>(base + o_off);
    gd.bits = reinterpret_cast<uint32_t *>(base + o_bits);
    gd.word = reinterpret_cast<uint32_t *>(base + o_word);
    gd.shift = reinterpret_cast<uint32_t *>(base + o_shift);
    cudaMemcpyAsync(gd.off, off, d * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(gd.bits, bits, d * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(gd.word, word, d * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(gd.shift, shift, d * 4, cudaMemcpyHostToDevice, st);
    uint32_t *keys = reinterpret_cast<uint32_t *>(base + o_keys);
    void *rs = base + o_rs;
    launch_pack_keys(pts, dtype_bytes, n, d, eps, gd, W, keys, st);

    // 3. stable LSD passes over the digit windows that can vary (the same
    //    rule as the allocating path), into the caller's buffer
    static thread_local std::pair<uint32_t, uint32_t> passes[4 * kMaxDim];
    uint32_t np = 0;
    for (int ww = (int)W - 1; ww >= 0; --ww)
        for (uint32_t lowbit = 0; lowbit < 32; lowbit += 8) {
            bool active = false;
            for (uint32_t t = 0; t < d && !active; ++t) {
                if ((int)word[t] != ww || range[t] == 0) continue;
                const uint32_t vb = (uint32_t)bits_of((unsigned long long)range[t] + 2);
                const uint32_t f0 = shift[t], f1 = shift[t] + (vb < bits[t] ? vb : bits[t]);
                if (f0 < lowbit + 8 && f1 > lowbit) active = true;
            }
            if (active) passes[np++] = {(uint32_t)ww, lowbit};
        }
    radix_sort_perm(keys, n, passes, np, perm, rs, st, nullptr);
    if (cudaError_t e = cudaGetLastError()) return engine_fail(HJ_ERR_CUDA, cudaGetErrorString(e));
    return HJ_OK;
}
