// hj_prep.cu -- epsilon-grid-order (EGO) stage of the join: per-dimension cell
// statistics, packed cell keys, a stable LSD radix sort of the permutation, and
// the gather of every sorted layout the distance kernels read.
//
// Replaces the reference's epsilonGridOrdering + omp_qsort
// (hilbertjoin/egojoin.cpp:159-168, :594-634), an unstable in-place quicksort
// of whole d-double rows that compares floor(x/eps) dimension by dimension
// (epsilonGridCompare, egojoin.cpp:9-17). Here the comparison is done once per
// point, when its cell vector is packed into 32-bit key words whose unsigned
// order is the lexicographic cell order; the sort then only moves 4-byte
// indices, and every data layout is written once, by the gather.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <map>
#include <mutex>

#include "hj_common.cuh"
#include "hj_internal.h"

namespace hj {

template <typename T>
__device__ __forceinline__ double load_coord(const void *x, uint64_t i) {
    return (double)static_cast<const T *>(x)[i];
}

__device__ __forceinline__ double coord(const void *x, int dtype_bytes, uint64_t i) {
    return dtype_bytes == 8 ? static_cast<const double *>(x)[i] : (double)static_cast<const float *>(x)[i];
}

// ------------------------------------------------------------ dim stats

__global__ void k_dim_stats_init(DimStats *s, uint32_t d, unsigned long long *maxabs, uint32_t *bad) {
    for (uint32_t t = threadIdx.x + blockIdx.x * blockDim.x; t < d; t += blockDim.x * gridDim.x) {
        s[t].cmin = LLONG_MAX;
        s[t].cmax = LLONG_MIN;
        s[t].xmin = ~0ull;
        s[t].xmax = 0ull;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *maxabs = 0ull;
        *bad = 0u;
    }
}

// Cells beyond +-2^62 cannot be represented; such inputs are rejected.
constexpr double kCellLimit = 4.611686018427388e18;

// Thread k handles dim t = k % d of rows k / d, k / d + R, ... (R = threads /
// d): consecutive threads read consecutive coordinates of a row (coalesced),
// and every thread keeps its dim's minima and maxima in registers; one
// shared-memory atomic per thread and statistic at the end.
__global__ void k_dim_stats(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, DimStats *s,
                            unsigned long long *maxabs_bits, uint32_t *bad) {
    extern __shared__ long long sh[];  // [4][d]
    long long *smin = sh, *smax = sh + d;
    unsigned long long *sxmin = reinterpret_cast<unsigned long long *>(sh + 2 * d), *sxmax = sxmin + d;
    for (uint32_t t = threadIdx.x; t < d; t += blockDim.x) {
        smin[t] = LLONG_MAX;
        smax[t] = LLONG_MIN;
        sxmin[t] = ~0ull;
        sxmax[t] = 0ull;
    }
    __syncthreads();
    const uint64_t threads = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t rows_per_step = threads / d;  // >= 1 (the launch ensures threads >= d)
    const uint32_t t = (uint32_t)(k % d);
    long long cmin = LLONG_MAX, cmax = LLONG_MIN;
    unsigned long long xmin = ~0ull, xmax = 0ull;
    double amax = 0.0;
    uint32_t lbad = 0;
    if (k < rows_per_step * d) {
        for (uint64_t r = k / d; r < n; r += rows_per_step) {
            const double v = coord(x, dtype_bytes, r * d + t);
            if (!isfinite(v)) {
                lbad |= 1u;
                continue;
            }
            const double c = floor(v / eps);
            if (!(fabs(c) < kCellLimit)) {
                lbad |= 2u;
                continue;
            }
            amax = fmax(amax, fabs(v));
            const long long ci = (long long)c;
            cmin = min(cmin, ci);
            cmax = max(cmax, ci);
            const unsigned long long ov = ordered_from_double(v);
            xmin = min(xmin, ov);
            xmax = max(xmax, ov);
        }
    }
    if (cmin != LLONG_MAX) {
        atomicMin(&smin[t], cmin);
        atomicMax(&smax[t], cmax);
        atomicMin(&sxmin[t], xmin);
        atomicMax(&sxmax[t], xmax);
    }
    __syncthreads();
    for (uint32_t u = threadIdx.x; u < d; u += blockDim.x) {
        if (smin[u] != LLONG_MAX) {
            atomicMin(&s[u].cmin, smin[u]);
            atomicMax(&s[u].cmax, smax[u]);
            atomicMin(&s[u].xmin, sxmin[u]);
            atomicMax(&s[u].xmax, sxmax[u]);
        }
    }
    // non-negative doubles order like their bit patterns
    if (amax > 0.0) atomicMax(maxabs_bits, (unsigned long long)__double_as_longlong(amax));
    if (lbad) atomicOr(bad, lbad);
}

void launch_dim_stats_init(DimStats *dstats, uint32_t d, unsigned long long *d_maxabs_bits, uint32_t *d_bad,
                           cudaStream_t st) {
    k_dim_stats_init<<<(d + 255) / 256, 256, 0, st>>>(dstats, d, d_maxabs_bits, d_bad);
}

void launch_dim_stats(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, DimStats *dstats,
                      unsigned long long *d_maxabs_bits, uint32_t *d_bad, cudaStream_t st) {
    uint64_t total = n * d;
    int blocks = (int)std::min<uint64_t>(hj_ceil_div(total, 256 * 8), 148 * 8);
    if (blocks < 1) blocks = 1;
    if ((uint64_t)blocks * 256 < d) blocks = (int)hj_ceil_div(d, 256);  // every dim gets a thread
    k_dim_stats<<<blocks, 256, 4 * d * sizeof(long long), st>>>(x, dtype_bytes, n, d, eps, dstats, d_maxabs_bits,
                                                                 d_bad);
}

// ------------------------------------------------------------ key packing

// One thread per point: digit of every dim, OR-ed into the running key word
// (fields in key order, so words never decrease). Consecutive threads read
// rows d coordinates apart; the rows of a block stay in L1 across the loop,
// which measured faster than a warp per row with per-word reductions.
__global__ void k_pack_keys(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, GridDev g,
                            uint32_t W, uint32_t *keys_wm) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t cur_word = 0, acc = 0;
    for (uint32_t pos = 0; pos < d; ++pos) {
        const uint32_t t = grid_dim_at(g, pos);
        uint32_t w = g.word[t];
        if (w != cur_word) {
            keys_wm[(uint64_t)cur_word * n + i] = acc;
            for (uint32_t z = cur_word + 1; z < w; ++z) keys_wm[(uint64_t)z * n + i] = 0u;
            cur_word = w;
            acc = 0;
        }
        double c = floor(coord(x, dtype_bytes, i * d + t) / eps);
        long long dig = (long long)c - g.off[t];
        acc |= (uint32_t)dig << g.shift[t];
    }
    keys_wm[(uint64_t)cur_word * n + i] = acc;
    for (uint32_t z = cur_word + 1; z < W; ++z) keys_wm[(uint64_t)z * n + i] = 0u;
}

// One warp per point: |x - center|^2 over lanes (coalesced), warp sum.
__global__ void k_norm_key(const void *x, int dtype_bytes, uint64_t n, uint32_t d,
                           const double *__restrict__ center, double scale, uint32_t *key_out) {
    const uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (i >= n) return;
    double s = 0.0;
    for (uint32_t k = lane; k < d; k += 32) {
        const double v = coord(x, dtype_bytes, i * d + k) - center[k];
        s = fma(v, v, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const double q = floor(s * scale);
        key_out[i] = q < 65535.0 ? (uint32_t)q : 65535u;
    }
}

void launch_norm_key(const void *x, int dtype_bytes, uint64_t n, uint32_t d, const double *center, double scale,
                     uint32_t *key_out, cudaStream_t st) {
    if (n == 0) return;
    k_norm_key<<<(unsigned)hj_ceil_div(n, 8), 256, 0, st>>>(x, dtype_bytes, n, d, center, scale, key_out);
}

// Dimension cost (the selectivity estimate of the reference's
// outputStatistics, hilbertjoin/egojoin.cpp:523-592): the sample's cell
// indices of one dim are sorted in shared memory (bitonic), and every sample
// position s counts the positions q > s with cell[q] <= cell[s] + 1 by a
// binary search -- together the pairs in equal cells, sum h(h-1)/2, plus the
// pairs in adjacent cells, sum h[c-1] h[c].
__global__ void __launch_bounds__(1024) k_dim_cost(const void *x, int dtype_bytes, uint64_t n, uint32_t d,
                                                   double eps, const DimStats *__restrict__ ds,
                                                   unsigned long long *cost) {
    __shared__ uint32_t v[kCostSample];
    __shared__ unsigned long long total;
    const uint32_t t = blockIdx.x, tid = threadIdx.x;
    const uint32_t S = (uint32_t)(n < kCostSample ? n : kCostSample);
    const long long cmin = ds[t].cmin;
    if (tid == 0) total = 0;
    for (uint32_t s = tid; s < kCostSample; s += blockDim.x) {
        uint32_t c = 0xffffffffu;  // padding sorts last
        if (s < S) {
            const uint64_t i = (uint64_t)s * n / S;
            long long q = (long long)floor(coord(x, dtype_bytes, i * d + t) / eps) - cmin;
            q = q < 0 ? 0 : (q > 0x7fffffffll ? 0x7fffffffll : q);
            c = (uint32_t)q;
        }
        v[s] = c;
    }
    __syncthreads();
    for (uint32_t k = 2; k <= kCostSample; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = tid; i < kCostSample; i += blockDim.x) {
                const uint32_t p = i ^ j;
                if (p > i) {
                    const uint32_t a = v[i], b = v[p];
                    if ((a > b) == ((i & k) == 0)) {
                        v[i] = b;
                        v[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    unsigned long long mine = 0;
    for (uint32_t s = tid; s < S; s += blockDim.x) {
        const uint32_t lim = v[s] + 1;  // cells are below 2^31: no wrap
        uint32_t lo = s + 1, hi = S;    // first q in (s, S) with v[q] > lim
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (v[mid] <= lim)
                lo = mid + 1;
            else
                hi = mid;
        }
        mine += lo - s - 1;
    }
    mine = warp_sum_u64(mine);
    if ((tid & 31u) == 0 && mine) atomicAdd(&total, mine);
    __syncthreads();
    if (tid == 0) cost[t] = total;
}

void launch_dim_cost(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, const DimStats *ds,
                     unsigned long long *cost, cudaStream_t st) {
    k_dim_cost<<<d, 1024, 0, st>>>(x, dtype_bytes, n, d, eps, ds, cost);
}

void launch_pack_keys(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, const GridDev &g,
                      uint32_t W, uint32_t *keys_wm, cudaStream_t st) {
    if (n == 0) return;
    k_pack_keys<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(x, dtype_bytes, n, d, eps, g, W, keys_wm);
}

// ------------------------------------------------------------ radix sort
//
// Stable LSD radix sort of a permutation. Each pass orders by one 8-bit window
// of one key word, read through the current permutation. Three kernels per
// pass: per-tile digit histograms, one exclusive scan over (digit, tile), and a
// stable scatter that ranks equal digits in index order (warp match + per-warp
// prefix), so ties keep their previous order and the sort is stable overall.

constexpr int kRsThreads = 256;
constexpr int kRsTile = 4096;  // items per block
constexpr int kRsWarps = kRsThreads / 32;

size_t radix_hist_entries(uint64_t n) { return 256 * (size_t)hj_ceil_div(n, kRsTile); }

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint32_t *__restrict__ keyw,
                                                       const uint32_t *__restrict__ perm_in, uint64_t n,
                                                       uint32_t shift, uint32_t *__restrict__ hist,
                                                       uint32_t nblocks) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    uint64_t base = (uint64_t)blockIdx.x * kRsTile;
    uint64_t end = base + kRsTile < n ? base + kRsTile : n;
    for (uint64_t i = base + threadIdx.x; i < end; i += kRsThreads) {
        uint32_t src = perm_in ? perm_in[i] : (uint32_t)i;
        atomicAdd(&h[(keyw[src] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of `count` u32 entries in place, one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan_u32(uint32_t *a, uint64_t count, unsigned long long *total_out) {
    __shared__ unsigned long long part[1024];
    const uint64_t per = hj_ceil_div(count, 1024);
    const uint64_t b = threadIdx.x * per, e = b + per < count ? b + per : count;
    unsigned long long s = 0;
    for (uint64_t i = b; i < e; ++i) s += a[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        unsigned long long v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0ull;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    unsigned long long run = threadIdx.x ? part[threadIdx.x - 1] : 0ull;
    for (uint64_t i = b; i < e; ++i) {
        uint32_t v = a[i];
        a[i] = (uint32_t)run;
        run += v;
    }
    if (total_out && threadIdx.x == 1023) *total_out = part[1023];
}

__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint32_t *__restrict__ keyw,
                                                          const uint32_t *__restrict__ perm_in, uint64_t n,
                                                          uint32_t shift, const uint32_t *__restrict__ hist,
                                                          uint32_t nblocks, uint32_t *__restrict__ perm_out) {
    __shared__ uint32_t s_base[256];
    __shared__ uint32_t s_wcnt[kRsWarps][256];
    const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u;
    s_base[t] = hist[(size_t)t * nblocks + blockIdx.x];
    const uint32_t lt_mask = (1u << lane) - 1u;
    const uint64_t base = (uint64_t)blockIdx.x * kRsTile;
    for (int r = 0; r < kRsTile / kRsThreads; ++r) {
        uint64_t i = base + (uint64_t)r * kRsThreads + t;
        bool valid = i < n;
        uint32_t src = 0, dig = 256u;
        if (valid) {
            src = perm_in ? perm_in[i] : (uint32_t)i;
            dig = (keyw[src] >> shift) & 255u;
        }
#pragma unroll
        for (int w = 0; w < kRsWarps; ++w) s_wcnt[w][t] = 0;
        __syncthreads();
        uint32_t peers = __match_any_sync(0xffffffffu, dig);
        uint32_t rank = __popc(peers & lt_mask);
        if (valid && rank == 0) s_wcnt[warp][dig] = __popc(peers);
        __syncthreads();
        {
            uint32_t run = s_base[t];
#pragma unroll
            for (int w = 0; w < kRsWarps; ++w) {
                uint32_t c = s_wcnt[w][t];
                s_wcnt[w][t] = run;
                run += c;
            }
            s_base[t] = run;
        }
        __syncthreads();
        if (valid) perm_out[s_wcnt[warp][dig] + rank] = src;
        __syncthreads();
    }
}

void ensure_max_dynamic_smem(const void *func, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, int> done;  // (function, device) -> bytes set
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    int &cur = done[{func, dev}];
    if (bytes > cur) {
        // never above what fits next to the kernel's static shared memory
        int optin = 0;
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, func) == cudaSuccess && optin > 0) {
            const int room = optin - (int)fa.sharedSizeBytes;
            if (bytes > room) bytes = room;
        }
        cudaGetLastError();
        if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess)
            cur = bytes;
        cudaGetLastError();
    }
}

void launch_scan_u32(uint32_t *a, uint64_t count, unsigned long long *total, cudaStream_t st) {
    k_scan_u32<<<1, 1024, 0, st>>>(a, count, total);
}

__global__ void k_iota(uint32_t *p, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = (uint32_t)i;
}

void radix_sort_perm(const uint32_t *keys_wm, uint64_t n, const std::vector<std::pair<uint32_t, uint32_t>> &passes,
                     uint32_t *perm_out, uint32_t *perm_tmp, uint32_t *hist, cudaStream_t st, int *launches) {
    if (n == 0) return;
    const uint32_t nb = (uint32_t)hj_ceil_div(n, kRsTile);
    if (passes.empty()) {
        k_iota<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(perm_out, n);
        if (launches) *launches += 1;
        return;
    }
    // ping-pong so that the last pass writes perm_out
    const size_t np = passes.size();
    uint32_t *bufs[2] = {perm_out, perm_tmp};
    const uint32_t *src = nullptr;
    for (size_t p = 0; p < np; ++p) {
        uint32_t *dst = bufs[(np - 1 - p) & 1];
        const uint32_t *kw = keys_wm + (size_t)passes[p].first * n;
        const uint32_t shift = passes[p].second;
        k_rs_hist<<<nb, kRsThreads, 0, st>>>(kw, src, n, shift, hist, nb);
        k_scan_u32<<<1, 1024, 0, st>>>(hist, (uint64_t)nb * 256, nullptr);
        k_rs_scatter<<<nb, kRsThreads, 0, st>>>(kw, src, n, shift, hist, nb, dst);
        if (launches) *launches += 3;
        src = dst;
    }
}

// One radix pass (histogram, scan, stable scatter) and a plain iota, for
// callers that drive the passes themselves (hj_noalloc.cu).
void radix_sort_pass(const uint32_t *keyw, uint64_t n, uint32_t shift, const uint32_t *perm_in,
                     uint32_t *perm_out, uint32_t *hist, cudaStream_t st) {
    const uint32_t nb = (uint32_t)hj_ceil_div(n, kRsTile);
    k_rs_hist<<<nb, kRsThreads, 0, st>>>(keyw, perm_in, n, shift, hist, nb);
    k_scan_u32<<<1, 1024, 0, st>>>(hist, (uint64_t)nb * 256, nullptr);
    k_rs_scatter<<<nb, kRsThreads, 0, st>>>(keyw, perm_in, n, shift, hist, nb, perm_out);
}

void launch_iota(uint32_t *p, uint64_t n, cudaStream_t st) {
    if (n) k_iota<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(p, n);
}

// ------------------------------------------------------------ gather

// Sorted keys row-major [n][W] (for binary searches) and sorted rows.
// One warp per sorted rank: the key words and the row of input index perm[r]
// (lanes over words and coordinates: coalesced reads and writes).
__global__ void k_gather_keys_rows(const void *x, int dtype_bytes, uint64_t n, uint32_t d,
                                   const uint32_t *__restrict__ perm, const uint32_t *__restrict__ keys_wm,
                                   uint32_t W, uint32_t *__restrict__ keys_rm, void *rows_out) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (r >= n) return;
    const uint32_t src = perm[r];
    if (keys_rm)
        for (uint32_t w = lane; w < W; w += 32) keys_rm[r * W + w] = keys_wm[(uint64_t)w * n + src];
    if (rows_out) {
        if (dtype_bytes == 8) {
            const double *xs = static_cast<const double *>(x) + (uint64_t)src * d;
            double *o = static_cast<double *>(rows_out) + r * d;
            for (uint32_t k = lane; k < d; k += 32) o[k] = xs[k];
        } else {
            const float *xs = static_cast<const float *>(x) + (uint64_t)src * d;
            float *o = static_cast<float *>(rows_out) + r * d;
            for (uint32_t k = lane; k < d; k += 32) o[k] = xs[k];
        }
    }
}

// Plain layout [tile][d][64]: element (rank r, dim k) at ((r/64)*d + k)*64 + r%64.
// One thread per output element, so the writes are coalesced.
__global__ void k_gather_plain(const void *x, int dtype_bytes, uint64_t n, uint32_t d,
                               const uint32_t *__restrict__ perm, double *__restrict__ out, uint64_t n_tiles) {
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t total = n_tiles * d * 64;
    if (e >= total) return;
    uint32_t lane = (uint32_t)(e & 63u);
    uint64_t q = e >> 6;
    uint32_t k = (uint32_t)(q % d);
    uint64_t tile = q / d;
    uint64_t r = tile * 64 + lane;
    double v = 0.0;
    if (r < n) v = coord(x, dtype_bytes, (uint64_t)perm[r] * d + k);
    out[e] = v;
}

__device__ __forceinline__ float to_tf32_rn(float v) {
    uint32_t u;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(v));
    return __uint_as_float(u);
}

// Tensor-core layouts, one thread per (row, k) element of the padded matrix:
// TF32 rows [npad][kp32], BF16 hi/lo rows [npad][kp16]. The operands are the
// coordinates minus `center` (per dim): distances are shift invariant, and the
// smaller norms narrow the error band of the norm expansion.
// FP16 (f16 != nullptr): (x - center) * scale rounded once from FP64 to FP16
// (round to nearest even); scale is a power of two, so the scaling is exact.
__global__ void k_gather_tc(const void *x, int dtype_bytes, uint64_t n, uint32_t d,
                            const uint32_t *__restrict__ perm, const double *__restrict__ center, uint64_t npad,
                            uint32_t kp, float *tf32, uint16_t *bf_hi, uint16_t *bf_lo, uint16_t *f16,
                            double scale) {
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= npad * kp) return;
    uint64_t r = e / kp;
    uint32_t k = (uint32_t)(e % kp);
    if (f16) {
        double w = 0.0;
        if (r < n && k < d) w = (coord(x, dtype_bytes, (uint64_t)perm[r] * d + k) - center[k]) * scale;
        f16[e] = __half_as_ushort(__double2half(w));
        return;
    }
    float v = 0.0f;
    if (r < n && k < d) v = (float)(coord(x, dtype_bytes, (uint64_t)perm[r] * d + k) - center[k]);
    if (tf32) tf32[e] = to_tf32_rn(v);
    if (bf_hi) {
        __nv_bfloat16 h = __float2bfloat16_rn(v);
        float rem = v - __bfloat162float(h);  // exact: h holds the leading bits of v
        __nv_bfloat16 l = __float2bfloat16_rn(rem);
        bf_hi[e] = __bfloat16_as_ushort(h);
        bf_lo[e] = __bfloat16_as_ushort(l);
    }
}

// |x - center|^2 per sorted row in FP64 (input precision widened exactly),
// stored as FP32; padding rows get kPadNorm so that they never pass a threshold.
__global__ void k_norms(const void *x, int dtype_bytes, uint64_t n, uint32_t d, const uint32_t *__restrict__ perm,
                        const double *__restrict__ center, uint64_t npad, double scale2, float *norms) {
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (r >= npad) return;
    if (r >= n) {
        if (lane == 0) norms[r] = kPadNorm;
        return;
    }
    const uint64_t src = perm[r];
    double s = 0.0;
    for (uint32_t k = lane; k < d; k += 32) {
        const double v = coord(x, dtype_bytes, src * d + k) - center[k];
        s = fma(v, v, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) norms[r] = (float)(s * scale2);
}

// Per-tile maximum norm over real rows (padding rows excluded).
__global__ void k_tile_max(const float *__restrict__ v, uint64_t npad, int tile, float *out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t * tile >= npad) return;
    float m = 0.0f;
    for (int i = 0; i < tile; ++i) {
        float x = v[t * tile + i];
        if (x < 1e29f) m = fmaxf(m, x);
    }
    out[t] = m;
}

// Per-group minimum norm (padding rows hold kPadNorm and never lower it).
__global__ void k_group_min(const float *__restrict__ v, uint64_t npad, int group, float *out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t * group >= npad) return;
    float m = 3.0e38f;
    for (int i = 0; i < group; ++i) m = fminf(m, v[t * group + i]);
    out[t] = m;
}

void launch_gather(const void *x, int dtype_bytes, uint64_t n, uint32_t d, const uint32_t *perm,
                   const uint32_t *keys_wm, uint32_t W, const SortedSet &o, uint32_t flags, cudaStream_t st,
                   int *launches) {
    int L = 0;
    if (n == 0) return;
    if (flags & (kGatherKeys | kGatherRows)) {
        k_gather_keys_rows<<<(unsigned)hj_ceil_div(n, 8), 256, 0, st>>>(  // a warp per rank
            x, dtype_bytes, n, d, perm, keys_wm, W, (flags & kGatherKeys) ? o.keys : nullptr,
            (flags & kGatherRows) ? const_cast<void *>(o.rows) : nullptr);
        ++L;
    }
    if (flags & kGatherPlain) {
        uint64_t total = o.n_tiles64 * d * 64;
        k_gather_plain<<<(unsigned)hj_ceil_div(total, 256), 256, 0, st>>>(x, dtype_bytes, n, d, perm, o.tiles64,
                                                                         o.n_tiles64);
        ++L;
    }
    if (flags & kGatherTf32) {
        uint64_t total = o.npad_tc * o.kpad_tf32;
        k_gather_tc<<<(unsigned)hj_ceil_div(total, 256), 256, 0, st>>>(x, dtype_bytes, n, d, perm, o.center,
                                                                      o.npad_tc, o.kpad_tf32, o.tf32, nullptr,
                                                                      nullptr, nullptr, 1.0);
        ++L;
    }
    if (flags & kGatherBf16) {
        uint64_t total = o.npad_tc * o.kpad_bf16;
        k_gather_tc<<<(unsigned)hj_ceil_div(total, 256), 256, 0, st>>>(x, dtype_bytes, n, d, perm, o.center,
                                                                      o.npad_tc, o.kpad_bf16, nullptr, o.bf_hi,
                                                                      o.bf_lo, nullptr, 1.0);
        ++L;
    }
    if (flags & kGatherF16) {
        uint64_t total = o.npad_tc * o.kpad_bf16;
        k_gather_tc<<<(unsigned)hj_ceil_div(total, 256), 256, 0, st>>>(x, dtype_bytes, n, d, perm, o.center,
                                                                      o.npad_tc, o.kpad_bf16, nullptr, nullptr,
                                                                      nullptr, o.bf_hi, o.op_scale);
        ++L;
    }
    if (flags & kGatherNorms) {
        k_norms<<<(unsigned)hj_ceil_div(o.npad_tc, 8), 256, 0, st>>>(x, dtype_bytes, n, d, perm, o.center,
                                                                      o.npad_tc, o.op_scale * o.op_scale,
                                                                      o.norms);
        k_tile_max<<<(unsigned)hj_ceil_div(o.npad_tc / kTcTileA, 256), 256, 0, st>>>(o.norms, o.npad_tc, kTcTileA,
                                                                                    o.tile_maxnorm_a);
        k_tile_max<<<(unsigned)hj_ceil_div(o.npad_tc / kTcTileB, 256), 256, 0, st>>>(o.norms, o.npad_tc, kTcTileB,
                                                                                    o.tile_maxnorm_b);
        k_group_min<<<(unsigned)hj_ceil_div(o.npad_tc / 32, 256), 256, 0, st>>>(o.norms, o.npad_tc, 32,
                                                                              o.group_minnorm);
        L += 4;
    }
    if (launches) *launches += L;
}

void launch_norm_summaries(const float *norms, uint64_t npad, float *tmax128, float *tmax256, float *gmin32,
                           cudaStream_t st) {
    if (npad == 0) return;
    k_tile_max<<<(unsigned)hj_ceil_div(npad / 128, 256), 256, 0, st>>>(norms, npad, 128, tmax128);
    k_tile_max<<<(unsigned)hj_ceil_div(npad / 256, 256), 256, 0, st>>>(norms, npad, 256, tmax256);
    k_group_min<<<(unsigned)hj_ceil_div(npad / 32, 256), 256, 0, st>>>(norms, npad, 32, gmin32);
}

}  // namespace hj
