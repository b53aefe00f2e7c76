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
#include <type_traits>

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


// Per-dim coordinate range, maximum |x| and the non-finite check, reading the
// rows as one flat array of n*d coordinates with 128-bit loads (V = 4 FP32 or
// 2 FP64 coordinates per load; V = 1 when the array is not 16-byte aligned).
// The grid is sized so that threads * V is a multiple of d: thread k then sees
// the same V dims (k*V + j) % d at every step and keeps their minima and
// maxima in registers. The cells need no division per coordinate: floor(x/eps)
// is monotone in x (IEEE division by a positive eps rounds monotonically), so
// a dim's smallest and largest cells are those of its smallest and largest
// coordinate; k_dim_stats_cells computes them once per dim.
// Per-dim minima and maxima of the block's threads are combined in three
// steps without contention: lanes of a warp whose elements fall in the same
// dims (lanes P apart, P = d / gcd(d, V)) by shuffles; the warps' results in
// per-warp shared arrays (warps = 1 when they would not fit: one array); the
// arrays per dim, then one global atomic per dim and block. The largest |x|
// and the non-finite flag are reduced over the block before their single
// global atomic.
constexpr uint32_t kStatsWarpArraysMaxDim = 384;  // 8 warps x 2 x d x 8 bytes <= 48 KB
__host__ __device__ inline uint32_t gcd_u32(uint32_t a, uint32_t b) {
    while (b) {
        const uint32_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}
template <typename T, int V>
__global__ void __launch_bounds__(256) k_dim_stats(const T *__restrict__ x, uint64_t total, uint32_t d,
                                                   DimStats *s, unsigned long long *maxabs_bits, uint32_t *bad) {
    extern __shared__ unsigned long long shx[];  // [arrays][2][d]
    __shared__ T red_amax[8];
    __shared__ uint32_t red_bad[8];
    const uint32_t arrays = d <= kStatsWarpArraysMaxDim ? (blockDim.x >> 5) : 1u;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    unsigned long long *sxmin = shx + (size_t)(arrays > 1 ? warp : 0) * 2 * d, *sxmax = sxmin + d;
    for (uint32_t t = threadIdx.x; t < arrays * 2 * d; t += blockDim.x) shx[t] = (t / d) % 2 == 0 ? ~0ull : 0ull;
    __syncthreads();
    const uint64_t threads = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    // running minima and maxima in the input type (non-finite values skipped),
    // turned into the order-preserving encoding once at the end; four loads
    // in flight per thread (the steps k*V + i*threads*V, i = 0..3, hit the same
    // dims because threads * V is a multiple of d)
    T xmin[V], xmax[V];
#pragma unroll
    for (int j = 0; j < V; ++j) xmin[j] = T(INFINITY), xmax[j] = T(-INFINITY);
    T amax = T(0);
    uint32_t lbad = 0;
    using Vec = typename std::conditional<V == 4, float4, typename std::conditional<V == 2, double2, T>::type>::type;
    auto take = [&](const T (&v)[V]) {
#pragma unroll
        for (int j = 0; j < V; ++j) {
            const T w = v[j];
            if (isfinite(w)) {
                amax = fmax(amax, fabs(w));
                xmin[j] = fmin(xmin[j], w);
                xmax[j] = fmax(xmax[j], w);
            } else {
                lbad |= 1u;
            }
        }
    };
    const uint64_t stride = threads * V;
    uint64_t e = k * V;
    for (; e + 3 * stride + V <= total; e += 4 * stride) {
        Vec q[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) q[i] = __ldg(reinterpret_cast<const Vec *>(x + e + i * stride));
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            T v[V];
            memcpy(v, &q[i], sizeof(v));
            take(v);
        }
    }
    for (; e < total; e += stride) {
        T v[V];
        if (e + V <= total) {
            const Vec q = __ldg(reinterpret_cast<const Vec *>(x + e));
            memcpy(v, &q, sizeof(v));
            take(v);
        } else {
#pragma unroll
            for (int j = 0; j < V; ++j) {
                if (e + j >= total) continue;
                const T w = x[e + j];
                if (isfinite(w)) {
                    amax = fmax(amax, fabs(w));
                    xmin[j] = fmin(xmin[j], w);
                    xmax[j] = fmax(xmax[j], w);
                } else {
                    lbad |= 1u;
                }
            }
        }
    }
    // lanes P apart hold the same dims (k * V + j mod d depends on k mod P);
    // min / max are idempotent, so overlapping shuffle windows are harmless
    const uint32_t P = d / gcd_u32(d, (uint32_t)V);
    for (uint32_t off = P; off < 32; off <<= 1) {
#pragma unroll
        for (int j = 0; j < V; ++j) {
            xmin[j] = fmin(xmin[j], __shfl_down_sync(0xffffffffu, xmin[j], off));
            xmax[j] = fmax(xmax[j], __shfl_down_sync(0xffffffffu, xmax[j], off));
        }
    }
    if (lane < P) {
#pragma unroll
        for (int j = 0; j < V; ++j) {
            if (!(xmin[j] <= xmax[j])) continue;  // no finite value in these dims
            const uint32_t t = (uint32_t)((k * V + j) % d);
            atomicMin(&sxmin[t], ordered_from_double((double)xmin[j]));
            atomicMax(&sxmax[t], ordered_from_double((double)xmax[j]));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        lbad |= __shfl_xor_sync(0xffffffffu, lbad, o);
    }
    if (lane == 0) {
        red_amax[warp] = amax;
        red_bad[warp] = lbad;
    }
    __syncthreads();
    for (uint32_t u = threadIdx.x; u < d; u += blockDim.x) {
        unsigned long long mn = ~0ull, mx = 0ull;
        for (uint32_t w = 0; w < arrays; ++w) {
            mn = min(mn, shx[(size_t)w * 2 * d + u]);
            mx = max(mx, shx[(size_t)w * 2 * d + d + u]);
        }
        if (mn != ~0ull) {
            atomicMin(&s[u].xmin, mn);
            atomicMax(&s[u].xmax, mx);
        }
    }
    if (threadIdx.x == 0) {
        T am = T(0);
        uint32_t b = 0;
        for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) {
            am = fmax(am, red_amax[w]);
            b |= red_bad[w];
        }
        // non-negative doubles order like their bit patterns
        if (am > T(0)) atomicMax(maxabs_bits, (unsigned long long)__double_as_longlong((double)am));
        if (b) atomicOr(bad, b);
    }
}

// Cells beyond +-2^62 cannot be represented; such inputs are rejected.
constexpr double kCellLimit = 4.611686018427388e18;

// Per dim: the cells of its smallest and largest coordinate.
__global__ void k_dim_stats_cells(DimStats *s, uint32_t d, double eps, uint32_t *bad) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d || s[t].xmin == ~0ull) return;
    const double lo = floor(double_from_ordered(s[t].xmin) / eps), hi = floor(double_from_ordered(s[t].xmax) / eps);
    if (!(fabs(lo) < kCellLimit) || !(fabs(hi) < kCellLimit)) {
        atomicOr(bad, 2u);
        return;
    }
    s[t].cmin = (long long)lo;
    s[t].cmax = (long long)hi;
}

void launch_dim_stats_init(DimStats *dstats, uint32_t d, unsigned long long *d_maxabs_bits, uint32_t *d_bad,
                           cudaStream_t st) {
    k_dim_stats_init<<<(d + 255) / 256, 256, 0, st>>>(dstats, d, d_maxabs_bits, d_bad);
}

static uint64_t gcd_u64(uint64_t a, uint64_t b) {
    while (b) {
        const uint64_t r = a % b;
        a = b;
        b = r;
    }
    return a;
}

template <typename T, int V>
static void dim_stats_launch(const T *x, uint64_t n, uint32_t d, DimStats *dstats, unsigned long long *maxabs,
                             uint32_t *bad, cudaStream_t st) {
    const uint64_t total = n * d;
    // threads * V must be a multiple of d: blocks a multiple of L
    const uint64_t dv = d / gcd_u64(d, V);
    const uint64_t L = dv / gcd_u64(dv, 256);
    uint64_t want = std::min<uint64_t>(hj_ceil_div(total, 256 * V * 16), 148 * 4);
    if (want < 1) want = 1;
    const uint64_t blocks = hj_ceil_div(want, L) * L;
    const uint32_t arrays = d <= kStatsWarpArraysMaxDim ? 8u : 1u;
    k_dim_stats<T, V><<<(unsigned)blocks, 256, arrays * 2 * d * sizeof(unsigned long long), st>>>(x, total, d, dstats,
                                                                                                  maxabs, bad);
}

void launch_dim_stats(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, DimStats *dstats,
                      unsigned long long *d_maxabs_bits, uint32_t *d_bad, cudaStream_t st) {
    const bool vec = ((uintptr_t)x & 15u) == 0;
    if (n) {
        if (dtype_bytes == 8) {
            if (vec)
                dim_stats_launch<double, 2>(static_cast<const double *>(x), n, d, dstats, d_maxabs_bits, d_bad, st);
            else
                dim_stats_launch<double, 1>(static_cast<const double *>(x), n, d, dstats, d_maxabs_bits, d_bad, st);
        } else {
            if (vec)
                dim_stats_launch<float, 4>(static_cast<const float *>(x), n, d, dstats, d_maxabs_bits, d_bad, st);
            else
                dim_stats_launch<float, 1>(static_cast<const float *>(x), n, d, dstats, d_maxabs_bits, d_bad, st);
        }
    }
    k_dim_stats_cells<<<(d + 255) / 256, 256, 0, st>>>(dstats, d, eps, d_bad);
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

// Packing with the rows staged in shared memory: a block of kPkRows threads
// packs kPkRows consecutive points, whose rows form one contiguous range of
// kPkRows * d coordinates. The block loads it with 128-bit loads (coalesced)
// into a [d][kPkRows] layout, so that thread t then reads its own row with
// consecutive threads on consecutive banks. The quantised norm key of the
// tensor-core forms comes out of the same pass (norm_key != null): the rows
// are read from memory once for both. Rows of up to 512 bytes (d <= 128 FP32,
// d <= 64 FP64) take this path.
constexpr int kPkRows = 128;
constexpr uint32_t kPkMaxRowBytes = 512;
// Per key position: the dim, its word and shift (word << 8 | shift), the cell
// offset; staged in shared memory once per block so that the packing loop
// reads one broadcast 16-byte entry per position.
struct PkPos {
    long long off;
    uint32_t dim, word_shift;
};

template <typename T>
__global__ void __launch_bounds__(kPkRows) k_pack_keys_staged(const T *__restrict__ x, uint64_t n, uint32_t d,
                                                              double eps, double inv_eps, GridDev g, uint32_t W,
                                                              uint32_t *__restrict__ keys_wm,
                                                              const double *__restrict__ center, double nscale,
                                                              uint32_t *__restrict__ norm_key, bool vec) {
    extern __shared__ __align__(16) unsigned char pk_smem[];
    T *cols = reinterpret_cast<T *>(pk_smem);  // [d][kPkRows]
    PkPos *prm = reinterpret_cast<PkPos *>(pk_smem + (size_t)d * kPkRows * sizeof(T));  // [d] (16-byte aligned)
    double *cen = reinterpret_cast<double *>(prm + d);                                 // [d]
    for (uint32_t pos = threadIdx.x; pos < d; pos += kPkRows) {
        const uint32_t dim = grid_dim_at(g, pos);
        prm[pos] = PkPos{g.off[dim], dim, (g.word[dim] << 8) | g.shift[dim]};
        if (norm_key) cen[pos] = center[pos];
    }
    const uint64_t r0 = (uint64_t)blockIdx.x * kPkRows;
    const uint32_t m = (uint32_t)(n - r0 < (uint64_t)kPkRows ? n - r0 : kPkRows);
    const uint32_t ne = m * d;
    const T *src = x + r0 * d;
    const float inv_d = 1.0f / (float)d;
    // element e of the block's range -> (row e / d, col e % d); e < 2^17, so
    // the FP32 quotient is off by at most one and one correction step fixes it
    auto put = [&](uint32_t e, T v) {
        uint32_t r = (uint32_t)((float)e * inv_d);
        int c = (int)e - (int)(r * d);
        if (c < 0) c += (int)d, --r;
        if (c >= (int)d) c -= (int)d, ++r;
        cols[(uint32_t)c * kPkRows + r] = v;
    };
    constexpr uint32_t V = 16 / sizeof(T);
    if (vec) {
        const uint32_t nv = ne / V;
        const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
        for (uint32_t u = threadIdx.x; u < nv; u += kPkRows) {
            const uint4 q = __ldg(s4 + u);
            T v[V];
            memcpy(v, &q, 16);
#pragma unroll
            for (uint32_t j = 0; j < V; ++j) put(u * V + j, v[j]);
        }
        for (uint32_t e = nv * V + threadIdx.x; e < ne; e += kPkRows) put(e, __ldg(src + e));
    } else {
        for (uint32_t e = threadIdx.x; e < ne; e += kPkRows) put(e, __ldg(src + e));
    }
    __syncthreads();
    const uint32_t t = threadIdx.x;
    if (t >= m) return;
    const uint64_t i = r0 + t;
    uint32_t cur_word = 0, acc = 0;
    for (uint32_t pos = 0; pos < d; ++pos) {
        const PkPos pp = prm[pos];
        const uint32_t w = pp.word_shift >> 8;
        if (w != cur_word) {
            keys_wm[(uint64_t)cur_word * n + i] = acc;
            for (uint32_t z = cur_word + 1; z < w; ++z) keys_wm[(uint64_t)z * n + i] = 0u;
            cur_word = w;
            acc = 0;
        }
        const double c = cell_of((double)cols[pp.dim * kPkRows + t], eps, inv_eps);
        const long long dig = (long long)c - pp.off;
        acc |= (uint32_t)dig << (pp.word_shift & 255u);
    }
    keys_wm[(uint64_t)cur_word * n + i] = acc;
    for (uint32_t z = cur_word + 1; z < W; ++z) keys_wm[(uint64_t)z * n + i] = 0u;
    if (norm_key) {
        double sum = 0.0;
        for (uint32_t k = 0; k < d; ++k) {
            const double v = (double)cols[k * kPkRows + t] - cen[k];
            sum = fma(v, v, sum);
        }
        const double q = floor(sum * nscale);
        norm_key[i] = q < 65535.0 ? (uint32_t)q : 65535u;
    }
}

void launch_pack_keys(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, const GridDev &g,
                      uint32_t W, uint32_t *keys_wm, cudaStream_t st, const double *center, double norm_scale,
                      uint32_t *norm_key) {
    if (n == 0) return;
    const bool vec = ((uintptr_t)x & 15u) == 0;
    if ((uint64_t)d * dtype_bytes <= kPkMaxRowBytes) {
        const unsigned blocks = (unsigned)hj_ceil_div(n, kPkRows);
        // rows (<= 64 KB; a multiple of 16 bytes), then the positions and the centre
        const size_t smem = (size_t)kPkRows * d * dtype_bytes + (size_t)d * (sizeof(PkPos) + 8);
        const int smem_max = (int)(64 * 1024 + (kPkMaxRowBytes / 4) * (sizeof(PkPos) + 8));
        if (dtype_bytes == 8) {
            ensure_max_dynamic_smem((const void *)k_pack_keys_staged<double>, smem_max);
            k_pack_keys_staged<double><<<blocks, kPkRows, smem, st>>>(static_cast<const double *>(x), n, d, eps,
                                                                      1.0 / eps, g,
                                                                      W, keys_wm, center, norm_scale, norm_key, vec);
        } else {
            ensure_max_dynamic_smem((const void *)k_pack_keys_staged<float>, smem_max);
            k_pack_keys_staged<float><<<blocks, kPkRows, smem, st>>>(static_cast<const float *>(x), n, d, eps,
                                                                     1.0 / eps, g, W,
                                                                     keys_wm, center, norm_scale, norm_key, vec);
        }
        return;
    }
    k_pack_keys<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(x, dtype_bytes, n, d, eps, g, W, keys_wm);
    if (norm_key) launch_norm_key(x, dtype_bytes, n, d, center, norm_scale, norm_key, st);
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

// ------------------------------------------------------------ radix sort
//
// Stable LSD radix sort of a permutation by 8-bit windows of word-major keys.
// Every pass moves (key, index) pairs: the index (the permutation) and the
// current key word in the current order, so that a pass reads both with
// coalesced 128-bit loads. Per pass:
//   k_rs_count      per 2048-item tile, the 256 digit counts;
//   k_rs_scan_rows  one block per digit: exclusive scan of that digit's tile
//                   counts, and the digit's total;
//   k_rs_scatter    per tile, a stable local sort by digit in shared memory
//                   (warp match + per-warp running counts, warps in order),
//                   then coalesced stores of each digit's run at its global
//                   offset (digit base + the tile's prefix within the digit).
// The next pass's key word travels with the pair: the current word when the
// next pass reads the same word, else the next word gathered once by index
// (4-byte reads from an array that stays in L2 at the engine's sizes).

constexpr int kRsThreads = 256;
constexpr int kRsIpt = 8;                       // items per thread
constexpr int kRsTile = kRsThreads * kRsIpt;    // 2048 items per tile
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsWarpItems = kRsTile / kRsWarps;  // 256 consecutive items per warp

static uint64_t rs_round4(uint64_t n) { return hj_ceil_div(n, 4) * 4; }

size_t radix_scratch_bytes(uint64_t n) {
    // index and key ping-pong buffers (16-byte aligned), tile counts, digit totals
    return (3 * rs_round4(n) + 256 * hj_ceil_div(std::max<uint64_t>(n, 1), kRsTile) + 256) * 4;
}

// Tile items [base, base + kRsTile) of a u32 array into s[0 .. kRsTile): 128-bit
// loads when the array is 16-byte aligned, 32-bit loads otherwise; items past
// n are not loaded.
__device__ __forceinline__ void rs_load_tile(const uint32_t *__restrict__ a, uint64_t base, uint64_t n, bool vec,
                                             uint32_t *s) {
    const uint32_t t = threadIdx.x;
    if (vec && base + kRsTile <= n) {
        const uint4 *a4 = reinterpret_cast<const uint4 *>(a + base);
#pragma unroll
        for (int k = 0; k < kRsIpt / 4; ++k) {
            const uint4 v = __ldg(a4 + t + k * kRsThreads);
            reinterpret_cast<uint4 *>(s)[t + k * kRsThreads] = v;
        }
    } else {
        for (uint32_t i = t; i < kRsTile; i += kRsThreads)
            if (base + i < n) s[i] = __ldg(a + base + i);
    }
}

__global__ void __launch_bounds__(kRsThreads) k_rs_count(const uint32_t *__restrict__ key, uint64_t n, uint32_t shift,
                                                        uint32_t nb, bool vec, uint32_t *__restrict__ counts) {
    __shared__ uint32_t h[256];
    __shared__ __align__(16) uint32_t s_key[kRsTile];
    const uint32_t t = threadIdx.x, lane = t & 31u;
    h[t] = 0;
    const uint64_t base = (uint64_t)blockIdx.x * kRsTile;
    rs_load_tile(key, base, n, vec, s_key);
    __syncthreads();
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll 4
    for (int k = 0; k < kRsIpt; ++k) {
        const uint32_t i = t + k * kRsThreads;
        const uint32_t dg = base + i < n ? (s_key[i] >> shift) & 255u : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, dg);
        if (dg < 256u && (peers & lt) == 0) atomicAdd(&h[dg], (uint32_t)__popc(peers));
    }
    __syncthreads();
    counts[(size_t)t * nb + blockIdx.x] = h[t];
}

// Exclusive scan of 1024 values held one per thread; returns the thread's
// exclusive prefix, *total gets the sum (all threads).
__device__ __forceinline__ unsigned long long rs_block_scan1024(unsigned long long v, unsigned long long *sh,
                                                                unsigned long long *total) {
    const uint32_t t = threadIdx.x, lane = t & 31u, w = t >> 5;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned long long s = sh[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= (uint32_t)o) s += y;
        }
        sh[lane] = s;  // inclusive over warps
    }
    __syncthreads();
    const unsigned long long before = (w ? sh[w - 1] : 0ull) + x - v;
    *total = sh[31];
    __syncthreads();
    return before;
}

// One block (1024 threads) per digit: counts[dg][0 .. nb) becomes its
// exclusive scan; totals[dg] = the digit's count over all tiles.
__global__ void __launch_bounds__(1024) k_rs_scan_rows(uint32_t *__restrict__ counts, uint32_t nb,
                                                      uint32_t *__restrict__ totals) {
    __shared__ unsigned long long sh[32];
    uint32_t *row = counts + (size_t)blockIdx.x * nb;
    const uint32_t per = (nb + 1023) / 1024;
    const uint32_t b = threadIdx.x * per, e = min(b + per, nb);
    unsigned long long s = 0;
    for (uint32_t i = b; i < e; ++i) s += row[i];
    unsigned long long total;
    unsigned long long run = rs_block_scan1024(s, sh, &total);
    for (uint32_t i = b; i < e; ++i) {
        const uint32_t v = row[i];
        row[i] = (uint32_t)run;
        run += v;
    }
    if (threadIdx.x == 0) totals[blockIdx.x] = (uint32_t)total;
}

// val_in null: the identity (first pass). key_out null: no next pass.
// next_word non-null: key_out receives next_word[index] (the next pass reads
// another word), else the current key. Dynamic shared memory: two tiles of
// (key, index), the loaded one and the locally sorted one (64 KB).
constexpr int kRsScatterSmem = 4 * kRsTile * 4;

__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint32_t *__restrict__ key_in,
                                                          const uint32_t *__restrict__ val_in, uint64_t n,
                                                          uint32_t shift, uint32_t nb, bool vec_key,
                                                          const uint32_t *__restrict__ counts,
                                                          const uint32_t *__restrict__ totals,
                                                          uint32_t *__restrict__ val_out, uint32_t *__restrict__ key_out,
                                                          const uint32_t *__restrict__ next_word) {
    extern __shared__ __align__(16) uint32_t rs_smem[];
    uint32_t *s_key = rs_smem, *s_val = rs_smem + kRsTile;              // loaded tile
    uint32_t *o_key = rs_smem + 2 * kRsTile, *o_val = rs_smem + 3 * kRsTile;  // sorted tile
    __shared__ uint32_t s_cnt[kRsWarps][256];
    __shared__ uint32_t s_dstart[256], s_gbase[256];
    __shared__ unsigned long long sh[16];
    const uint32_t t = threadIdx.x, warp = t >> 5, lane = t & 31u;
    const uint64_t base = (uint64_t)blockIdx.x * kRsTile;
    const uint32_t m = (uint32_t)(n - base < (uint64_t)kRsTile ? n - base : kRsTile);  // items in this tile
    rs_load_tile(key_in, base, n, vec_key, s_key);
    if (val_in) {
        rs_load_tile(val_in, base, n, ((uintptr_t)val_in & 15u) == 0, s_val);
    } else {
        for (uint32_t i = t; i < m; i += kRsThreads) s_val[i] = (uint32_t)(base + i);
    }
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) s_cnt[w][t] = 0;
    __syncthreads();
    // 1. ranks within each warp's kRsWarpItems items, in item order (stable): warp-local
    //    rank of item j of this lane, 0xffff for items past the tile's end
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t r_reg[kRsIpt / 2];
#pragma unroll
    for (int j = 0; j < kRsIpt; ++j) {
        const uint32_t i = warp * kRsWarpItems + j * 32 + lane;
        const bool ok = i < m;
        const uint32_t dg = ok ? (s_key[i] >> shift) & 255u : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, dg);
        const uint32_t before = dg < 256u ? s_cnt[warp][dg] : 0u;
        __syncwarp();
        if (dg < 256u && (peers & lt) == 0) s_cnt[warp][dg] = before + __popc(peers);
        __syncwarp();
        const uint32_t r = ok ? before + __popc(peers & lt) : 0xffffu;  // < kRsWarpItems for real items
        if (j & 1)
            r_reg[j >> 1] |= r << 16;
        else
            r_reg[j >> 1] = r;
    }
    __syncthreads();
    // 2. per digit (thread t = digit t): warp offsets in warp order, the tile's
    //    local digit starts, and the digit's global base for this tile
    {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kRsWarps; ++w) {
            const uint32_t c = s_cnt[w][t];
            s_cnt[w][t] = run;
            run += c;
        }
        // exclusive scans over the 256 digits of the tile's digit counts (x0)
        // and of the digits' totals over all tiles (x1)
        const unsigned long long x0 = run, x1 = totals[t];
        unsigned long long a = x0, b = x1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long ya = __shfl_up_sync(0xffffffffu, a, o);
            const unsigned long long yb = __shfl_up_sync(0xffffffffu, b, o);
            if (lane >= (uint32_t)o) a += ya, b += yb;
        }
        if (lane == 31) sh[warp] = a, sh[8 + warp] = b;
        __syncthreads();
        unsigned long long pa = 0, pb = 0;
        for (uint32_t w = 0; w < warp; ++w) pa += sh[w], pb += sh[8 + w];
        s_dstart[t] = (uint32_t)(pa + a - x0);
        s_gbase[t] = (uint32_t)(pb + b - x1) + counts[(size_t)t * nb + blockIdx.x];
    }
    __syncthreads();
    // 3. the tile sorted by digit into the second buffer
#pragma unroll
    for (int j = 0; j < kRsIpt; ++j) {
        const uint32_t r = (r_reg[j >> 1] >> ((j & 1) * 16)) & 0xffffu;
        if (r == 0xffffu) continue;
        const uint32_t i = warp * kRsWarpItems + j * 32 + lane;
        const uint32_t key = s_key[i];
        const uint32_t dg = (key >> shift) & 255u;
        const uint32_t pos = s_dstart[dg] + s_cnt[warp][dg] + r;
        o_key[pos] = key;
        o_val[pos] = s_val[i];
    }
    __syncthreads();
    // 4. each digit's run to its global offset: consecutive positions of a run
    //    go to consecutive addresses
    for (uint32_t p = t; p < m; p += kRsThreads) {
        const uint32_t key = o_key[p], val = o_val[p];
        const uint32_t dg = (key >> shift) & 255u;
        const uint32_t g = s_gbase[dg] + (p - s_dstart[dg]);
        val_out[g] = val;
        if (key_out) key_out[g] = next_word ? __ldg(next_word + val) : key;
    }
}

__global__ void k_iota(uint32_t *p, uint64_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = (uint32_t)i;
}

void radix_sort_perm(const uint32_t *keys_wm, uint64_t n, const std::pair<uint32_t, uint32_t> *passes, size_t np,
                     uint32_t *perm_out, void *scratch, cudaStream_t st, int *launches) {
    if (n == 0) return;
    if (np == 0) {
        k_iota<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(perm_out, n);
        if (launches) *launches += 1;
        return;
    }
    const uint64_t nn = rs_round4(n);
    uint32_t *vtmp = static_cast<uint32_t *>(scratch);
    uint32_t *kb[2] = {vtmp + nn, vtmp + 2 * nn};
    const uint32_t nb = (uint32_t)hj_ceil_div(n, kRsTile);
    uint32_t *counts = vtmp + 3 * nn;
    uint32_t *totals = counts + (size_t)256 * nb;
    ensure_max_dynamic_smem((const void *)k_rs_scatter, kRsScatterSmem);
    const uint32_t *val_in = nullptr;
    for (size_t p = 0; p < np; ++p) {
        const uint32_t shift = passes[p].second;
        // pass 0 reads its word of the input keys (identity order); later
        // passes read the key that the previous pass carried
        const uint32_t *key_in = p == 0 ? keys_wm + (size_t)passes[0].first * n : kb[p & 1];
        const bool vec_key = ((uintptr_t)key_in & 15u) == 0;
        uint32_t *val_out = ((np - 1 - p) & 1) ? vtmp : perm_out;
        uint32_t *key_out = p + 1 < np ? kb[(p + 1) & 1] : nullptr;
        const uint32_t *next_word = nullptr;
        if (key_out && passes[p + 1].first != passes[p].first) next_word = keys_wm + (size_t)passes[p + 1].first * n;
        k_rs_count<<<nb, kRsThreads, 0, st>>>(key_in, n, shift, nb, vec_key, counts);
        k_rs_scan_rows<<<256, 1024, 0, st>>>(counts, nb, totals);
        k_rs_scatter<<<nb, kRsThreads, kRsScatterSmem, st>>>(key_in, val_in, n, shift, nb, vec_key, counts, totals,
                                                             val_out, key_out, next_word);
        if (launches) *launches += 3;
        val_in = val_out;
    }
}

void radix_sort_perm(const uint32_t *keys_wm, uint64_t n, const std::vector<std::pair<uint32_t, uint32_t>> &passes,
                     uint32_t *perm_out, void *scratch, cudaStream_t st, int *launches) {
    radix_sort_perm(keys_wm, n, passes.data(), passes.size(), perm_out, scratch, st, launches);
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

// Multi-block exclusive scan (u32 values, u32 results as the single-block scan's,
// u64 total): per 2048-entry tile a local scan in shared memory and its sum;
// the tile sums scanned by one block; the tile offsets added.
constexpr uint32_t kScanTile = 2048;

__global__ void __launch_bounds__(256) k_scan_tiles(uint32_t *a, uint64_t count, unsigned long long *tile_sums) {
    __shared__ uint32_t sv[kScanTile];
    __shared__ unsigned long long wsum[8];
    const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    for (uint32_t j = threadIdx.x; j < kScanTile; j += 256) sv[j] = base + j < count ? a[base + j] : 0u;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t vals[8];
    unsigned long long run = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        vals[k] = sv[8 * threadIdx.x + k];
        run += vals[k];
    }
    unsigned long long incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    unsigned long long woff = 0, tot = 0;
    for (uint32_t w = 0; w < 8; ++w) {
        if (w < warp) woff += wsum[w];
        tot += wsum[w];
    }
    unsigned long long e = woff + incl - run;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        sv[8 * threadIdx.x + k] = (uint32_t)e;
        e += vals[k];
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < kScanTile; j += 256)
        if (base + j < count) a[base + j] = sv[j];
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// Exclusive scan of n u64 tile sums in place (one block), total into *total.
__global__ void __launch_bounds__(1024) k_scan_u64_one(unsigned long long *v, uint64_t n,
                                                       unsigned long long *total_out) {
    __shared__ unsigned long long part[1024];
    const uint64_t per = hj_ceil_div(n, 1024);
    const uint64_t b = threadIdx.x * per, e = b + per < n ? b + per : n;
    unsigned long long s = 0;
    for (uint64_t i = b; i < e; ++i) s += v[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        unsigned long long x = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0ull;
        __syncthreads();
        part[threadIdx.x] += x;
        __syncthreads();
    }
    unsigned long long run = threadIdx.x ? part[threadIdx.x - 1] : 0ull;
    for (uint64_t i = b; i < e; ++i) {
        const unsigned long long x = v[i];
        v[i] = run;
        run += x;
    }
    if (total_out && threadIdx.x == 1023) *total_out = part[1023];
}

__global__ void k_scan_add(uint32_t *a, uint64_t count, const unsigned long long *tile_off) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) a[i] += (uint32_t)tile_off[i / kScanTile];
}

size_t scan_scratch_bytes(uint64_t count) { return hj_ceil_div(count, kScanTile) * sizeof(unsigned long long); }

void launch_scan_u32(uint32_t *a, uint64_t count, unsigned long long *total, cudaStream_t st,
                     unsigned long long *sums) {
    const uint64_t tiles = hj_ceil_div(count, kScanTile);
    if (tiles <= 1 || !sums) {  // small, or no scratch: the single-block scan
        k_scan_u32<<<1, 1024, 0, st>>>(a, count, total);
        return;
    }
    k_scan_tiles<<<(unsigned)tiles, 256, 0, st>>>(a, count, sums);
    k_scan_u64_one<<<1, 1024, 0, st>>>(sums, tiles, total);
    k_scan_add<<<(unsigned)hj_ceil_div(count, 256), 256, 0, st>>>(a, count, sums);
}

void launch_iota(uint32_t *p, uint64_t n, cudaStream_t st) {
    if (n) k_iota<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(p, n);
}

// ------------------------------------------------------------ fused gathers
//
// One pass over the sorted ranks writes every layout a form reads, so each
// input row is read from memory once. A group of 8 threads handles one sorted
// rank; thread j of the group covers the 8-coordinate chunks j, j + 8, ... of
// the padded width, reading the row's coordinates with 128-bit loads when
// rows are 16-byte aligned (d * dtype_bytes a multiple of 16) and writing the
// chunk of each layout with 128-bit stores.

constexpr int kGrpRows = 32;  // ranks per 256-thread block

template <typename T>
__device__ __forceinline__ void load_chunk8(const T *row, uint32_t k0, uint32_t d, bool vec, double (&v)[8]) {
    if (vec && k0 + 8 <= d) {
        if (sizeof(T) == 4) {
            const float4 a = __ldg(reinterpret_cast<const float4 *>(row + k0));
            const float4 b = __ldg(reinterpret_cast<const float4 *>(row + k0 + 4));
            v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double2 a = __ldg(reinterpret_cast<const double2 *>(row + k0) + q);
                v[2 * q] = a.x, v[2 * q + 1] = a.y;
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = k0 + q < d ? (double)__ldg(row + k0 + q) : 0.0;
    }
}

template <typename T>
__device__ __forceinline__ void store_row_chunk(T *row, uint32_t k0, uint32_t d, bool vec, const double (&v)[8]) {
    if (vec && k0 + 8 <= d) {
        if (sizeof(T) == 4) {
            reinterpret_cast<float4 *>(row + k0)[0] = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
            reinterpret_cast<float4 *>(row + k0)[1] = make_float4((float)v[4], (float)v[5], (float)v[6], (float)v[7]);
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) reinterpret_cast<double2 *>(row + k0)[q] = make_double2(v[2 * q], v[2 * q + 1]);
        }
    } else {
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (k0 + q < d) row[k0 + q] = (T)v[q];
    }
}


__device__ __forceinline__ float to_tf32_rn(float v) {
    uint32_t u;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(v));
    return __uint_as_float(u);
}

// Tensor-core forms: sorted keys (row-major [n][W]), sorted rows (input
// precision), the operand matrix ([npad][kp]: TF32, BF16 hi/lo, or FP16) of
// the centred coordinates, and the FP64 centred norm of every rank (FP32,
// padding ranks kPadNorm). FP16 operands are (x - center) * scale rounded once
// from FP64 (scale a power of two: exact); TF32 and BF16 from the FP32 value
// of x - center, BF16 as hi + lo with lo the BF16 of the exact remainder.
template <typename T, int OP>  // OP: 0 TF32, 1 BF16 hi/lo, 2 FP16
__global__ void __launch_bounds__(256) k_gather_tc_fused(const T *__restrict__ x, uint64_t n, uint32_t d,
                                                         const uint32_t *__restrict__ perm,
                                                         const uint32_t *__restrict__ keys_wm, uint32_t W,
                                                         const double *__restrict__ center, uint64_t npad, uint32_t kp,
                                                         double scale, double scale2, bool vec,
                                                         uint32_t *__restrict__ keys_rm, T *__restrict__ rows_out,
                                                         void *__restrict__ op_hi, uint16_t *__restrict__ op_lo,
                                                         float *__restrict__ norms) {
    const uint64_t r = (uint64_t)blockIdx.x * kGrpRows + (threadIdx.x >> 3);
    const uint32_t j = threadIdx.x & 7u;
    const bool in = r < npad;  // npad is a multiple of kGrpRows: always true at the engine's launches
    const bool real = r < n;
    const uint32_t src = real ? perm[r] : 0u;
    const T *row = x + (uint64_t)src * d;
    double part = 0.0;
    for (uint32_t k0 = 8 * j; in && k0 < kp; k0 += 64) {
        double v[8];
        if (real) {
            load_chunk8(row, k0, d, vec, v);
            if (rows_out && k0 < d) store_row_chunk(rows_out + r * d, k0, d, vec, v);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const double c = k0 + q < d ? v[q] - center[k0 + q] : 0.0;
                part = fma(c, c, part);
                v[q] = c;
            }
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = 0.0;
        }
        if (OP == 2) {
            uint32_t h[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                h[q] = (uint32_t)__half_as_ushort(__double2half(v[2 * q] * scale)) |
                       ((uint32_t)__half_as_ushort(__double2half(v[2 * q + 1] * scale)) << 16);
            reinterpret_cast<uint4 *>(static_cast<uint16_t *>(op_hi) + r * kp + k0)[0] = make_uint4(h[0], h[1], h[2], h[3]);
        } else if (OP == 0) {
            float f[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) f[q] = to_tf32_rn((float)v[q]);
            float4 *o = reinterpret_cast<float4 *>(static_cast<float *>(op_hi) + r * kp + k0);
            o[0] = make_float4(f[0], f[1], f[2], f[3]);
            o[1] = make_float4(f[4], f[5], f[6], f[7]);
        } else {
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                uint32_t hh[2], ll[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const float f = (float)v[2 * q + e];
                    const __nv_bfloat16 b = __float2bfloat16_rn(f);
                    const float rem = f - __bfloat162float(b);  // exact: b holds the leading bits of f
                    hh[e] = __bfloat16_as_ushort(b);
                    ll[e] = __bfloat16_as_ushort(__float2bfloat16_rn(rem));
                }
                hi[q] = hh[0] | (hh[1] << 16);
                lo[q] = ll[0] | (ll[1] << 16);
            }
            reinterpret_cast<uint4 *>(static_cast<uint16_t *>(op_hi) + r * kp + k0)[0] = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            reinterpret_cast<uint4 *>(op_lo + r * kp + k0)[0] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        }
    }
    // norm of the rank: sum over the group's 8 lanes
    part += __shfl_xor_sync(0xffffffffu, part, 4);
    part += __shfl_xor_sync(0xffffffffu, part, 2);
    part += __shfl_xor_sync(0xffffffffu, part, 1);
    if (in && j == 0) norms[r] = real ? (float)(part * scale2) : kPadNorm;
    if (real && keys_rm)
        for (uint32_t w = j; w < W; w += 8) keys_rm[r * W + w] = keys_wm[(uint64_t)w * n + src];
}

// Plain form and row-only gathers: sorted keys and sorted rows, a group of 8
// threads per rank as above (no padding ranks).
template <typename T>
__global__ void __launch_bounds__(256) k_gather_rows_fused(const T *__restrict__ x, uint64_t n, uint32_t d,
                                                           const uint32_t *__restrict__ perm,
                                                           const uint32_t *__restrict__ keys_wm, uint32_t W, bool vec,
                                                           uint32_t *__restrict__ keys_rm, T *__restrict__ rows_out) {
    const uint64_t r = (uint64_t)blockIdx.x * kGrpRows + (threadIdx.x >> 3);
    const uint32_t j = threadIdx.x & 7u;
    if (r >= n) return;
    const uint32_t src = perm[r];
    if (rows_out) {
        const T *row = x + (uint64_t)src * d;
        for (uint32_t k0 = 8 * j; k0 < d; k0 += 64) {
            double v[8];
            load_chunk8(row, k0, d, vec, v);
            store_row_chunk(rows_out + r * d, k0, d, vec, v);
        }
    }
    if (keys_rm)
        for (uint32_t w = j; w < W; w += 8) keys_rm[r * W + w] = keys_wm[(uint64_t)w * n + src];
}

// Plain layout [tile][d][64]: element (rank r, dim k) at ((r/64)*d + k)*64 + r%64.
// One block per 64-rank tile; thread (k4 = t / 64, lane = t % 64) writes dims
// k4, k4 + 4, ... of rank lane: each store instruction writes 64 consecutive
// doubles, and the tile's rows are re-read from L1.
template <typename T>
__global__ void __launch_bounds__(256) k_gather_plain_tiles(const T *__restrict__ x, uint64_t n, uint32_t d,
                                                            const uint32_t *__restrict__ perm,
                                                            double *__restrict__ out) {
    const uint64_t tile = blockIdx.x;
    const uint32_t lane = threadIdx.x & 63u, k4 = threadIdx.x >> 6;
    const uint64_t r = tile * 64 + lane;
    const T *row = r < n ? x + (uint64_t)perm[r] * d : nullptr;
    double *o = out + tile * d * 64 + lane;
    for (uint32_t k = k4; k < d; k += 4) o[(uint64_t)k * 64] = row ? (double)__ldg(row + k) : 0.0;
}

// ------------------------------------------------------------ norm summaries

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

// ------------------------------------------------------------ per-block centring

// One CUDA block per 128-rank block of a sorted set (kBcBlock threads). The
// block's rows are read once (contiguous in the sorted layout), shifted and
// scaled ((x - center) * scale in FP64, the largest coordinate below 2^10),
// and kept in shared memory; per dim the midpoint of the block's range,
// rounded to FP16, is the centre c; every rank's residual h = fl16(x - c)
// (round to nearest, once), q = |h|^2 + 2 h.c from the FP16 values in FP64,
// and |h|; then the operand rows (four blocks of dp columns, zero padded)
//     [h | h | c m1 m2 m3 | h -2^15 -2^4 -2^-7]
// are written as 16-byte chunks, consecutive threads on consecutive chunks,
// with q / 2 = 2^15 m1 + 2^4 m2 + 2^-7 m3 + r: m1 = fl16(q / 2^16), m2 and m3
// the FP16 of the exact remainders, |r| <= 2^-33 |q| + 2^-32. Bounds: with
// |x - center| * scale < 2^10 per coordinate, |h_t| < 2^10 (1 + 2^-11) and
// |q| < 3 2^20 d <= 3 2^26, so every piece is below 2^12 in magnitude.
// Ranks past n (up to npad) are padding: zero rows, q = kPadNorm, |h| = 0.
// Operand element of the block-centred rows: FP16 bits, or a TF32 value in an
// FP32 container (rounded to nearest through FP32; the error stays within the
// 2^-11 relative radius the bound allows, with its 1.001 margin).
template <int OP> struct BcElem;
template <> struct BcElem<2> {  // FP16
    using E = uint16_t;
    __device__ static E round(double v, double *back) {
        const __half h = __double2half(v);
        *back = (double)__half2float(h);
        return __half_as_ushort(h);
    }
};
template <> struct BcElem<0> {  // TF32
    using E = uint32_t;
    __device__ static E round(double v, double *back) {
        const float f = to_tf32_rn((float)v);
        *back = (double)f;
        return __float_as_uint(f);
    }
};
template <> struct BcElem<1> {  // BF16 hi + lo (BF16x3): hi in the low 16 bits, lo in the high 16 bits;
    using E = uint32_t;         // the stored value hi + lo is within 2^-17 |v| of v
    __device__ static E round(double v, double *back) {
        const __nv_bfloat16 hi = __double2bfloat16(v);
        const double h = (double)__bfloat162float(hi);
        const __nv_bfloat16 lo = __double2bfloat16(v - h);  // v - h exact in FP64
        *back = h + (double)__bfloat162float(lo);
        return (uint32_t)__bfloat16_as_ushort(hi) | ((uint32_t)__bfloat16_as_ushort(lo) << 16);
    }
};

// Shared memory of k_bc_prepare for dimension d and element size eb: the rows
// in FP64 with an odd row stride (fewer bank conflicts when a thread walks its
// own row), the centre, per-part minima and maxima, and the operand bits of the
// residuals, the centre and the pieces of q / 2.
struct BcSmem {
    uint32_t xstride, hstride, parts;
    size_t o_x, o_c, o_min, o_max, o_h, o_ch, o_m, bytes;
};
__host__ __device__ inline BcSmem bc_smem_plan(uint32_t d, uint32_t eb) {
    BcSmem p;
    p.xstride = d | 1u;
    p.hstride = d;
    p.parts = kBcBlock / d < 8 ? kBcBlock / d : 8;
    if (p.parts < 1) p.parts = 1;
    p.o_x = 0;
    p.o_c = p.o_x + (size_t)kBcBlock * p.xstride * 8;
    p.o_min = p.o_c + (size_t)d * 8;
    p.o_max = p.o_min + (size_t)p.parts * d * 8;
    p.o_h = p.o_max + (size_t)p.parts * d * 8;
    p.o_ch = p.o_h + ((size_t)kBcBlock * p.hstride * eb + 7) / 8 * 8;
    p.o_m = p.o_ch + ((size_t)d * eb + 7) / 8 * 8;
    p.bytes = p.o_m + (size_t)kBcBlock * 4 * eb;
    return p;
}

template <typename T, int OP>
__global__ void __launch_bounds__(kBcBlock) k_bc_prepare(const T *__restrict__ rows, uint64_t n, uint32_t d,
                                                         const double *__restrict__ center, double scale,
                                                         uint32_t dp, bool vec, void *__restrict__ op_out,
                                                         void *__restrict__ op_lo, float *__restrict__ norms,
                                                         float *__restrict__ xn, float4 *__restrict__ blk,
                                                         float *__restrict__ cent) {
    using El = BcElem<OP>;
    using E = typename El::E;
    constexpr bool kSplit = OP == 1;                          // BF16 hi / lo into two row buffers
    constexpr uint32_t kEpc = kSplit ? 8u : 16 / sizeof(E);  // elements per 16-byte chunk (of each buffer)
    extern __shared__ __align__(16) unsigned char bc_raw[];
    const BcSmem P = bc_smem_plan(d, sizeof(E));
    double *xs = reinterpret_cast<double *>(bc_raw + P.o_x);    // [kBcBlock][xstride]
    double *cs = reinterpret_cast<double *>(bc_raw + P.o_c);    // [d]
    double *pmin = reinterpret_cast<double *>(bc_raw + P.o_min);  // [parts][d]
    double *pmax = reinterpret_cast<double *>(bc_raw + P.o_max);
    E *hs = reinterpret_cast<E *>(bc_raw + P.o_h);    // [kBcBlock][d] operand bits of h
    E *chs = reinterpret_cast<E *>(bc_raw + P.o_ch);  // [d] operand bits of c
    E *ms = reinterpret_cast<E *>(bc_raw + P.o_m);    // [kBcBlock][4] operand bits of m1 m2 m3
    __shared__ float red_x[kBcBlock / 32], red_p[kBcBlock / 32];
    const uint64_t r0 = (uint64_t)blockIdx.x * kBcBlock;
    const uint32_t nr = r0 >= n ? 0u : (n - r0 < kBcBlock ? (uint32_t)(n - r0) : kBcBlock);
    const T *src = rows + r0 * d;
    const uint32_t ne = nr * d;
    // 1. the block's rows (one contiguous range), shifted and scaled in FP64;
    // element e -> (e / d, e % d) by an FP32 quotient (e < 2^14: off by at most
    // one, corrected)
    const float inv_d = 1.0f / (float)d;
    auto put = [&](uint32_t e, T v) {
        uint32_t r = (uint32_t)((float)e * inv_d);
        int t = (int)e - (int)(r * d);
        if (t < 0) t += (int)d, --r;
        if (t >= (int)d) t -= (int)d, ++r;
        xs[r * P.xstride + (uint32_t)t] = ((double)v - center[t]) * scale;
    };
    constexpr uint32_t V = 16 / sizeof(T);
    using Vec = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    uint32_t e0 = 0;
    if (vec) {
        const uint32_t nv = ne / V;
        const Vec *s4 = reinterpret_cast<const Vec *>(src);
        for (uint32_t u = threadIdx.x; u < nv; u += kBcBlock) {
            const Vec q = __ldg(s4 + u);
            T v[V];
            memcpy(v, &q, 16);
#pragma unroll
            for (uint32_t j = 0; j < V; ++j) put(u * V + j, v[j]);
        }
        e0 = nv * V;
    }
    for (uint32_t e = e0 + threadIdx.x; e < ne; e += kBcBlock) put(e, __ldg(src + e));
    __syncthreads();
    // 2. per dim the range of the block, `parts` threads per dim
    if (threadIdx.x < P.parts * d) {
        const uint32_t t = threadIdx.x % d, part = threadIdx.x / d;
        double lo = INFINITY, hi = -INFINITY;
        for (uint32_t r = part; r < nr; r += P.parts) {
            const double v = xs[r * P.xstride + t];
            lo = fmin(lo, v);
            hi = fmax(hi, v);
        }
        pmin[part * d + t] = lo;
        pmax[part * d + t] = hi;
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < d; t += kBcBlock) {
        double lo = INFINITY, hi = -INFINITY;
        for (uint32_t part = 0; part < P.parts; ++part) {
            lo = fmin(lo, pmin[part * d + t]);
            hi = fmax(hi, pmax[part * d + t]);
        }
        double c;
        chs[t] = El::round(nr ? 0.5 * lo + 0.5 * hi : 0.0, &c);
        cs[t] = c;
    }
    __syncthreads();
    // 3. per rank: residual (rounded once), q = |h|^2 + 2 h.c, |h|, pieces of q / 2
    const uint32_t r = threadIdx.x;
    float my_x = 0.f, my_p = 0.f;
    E mb0 = 0, mb1 = 0, mb2 = 0;
    if (r < nr) {
        double hh = 0.0, hc = 0.0;
        for (uint32_t t = 0; t < d; ++t) {
            double h;
            hs[r * P.hstride + t] = El::round(xs[r * P.xstride + t] - cs[t], &h);
            hh = fma(h, h, hh);
            hc = fma(h, cs[t], hc);
        }
        const double q = fma(2.0, hc, hh);
        norms[r0 + r] = (float)q;
        my_p = fabsf((float)q) * (1.0f + 2.4e-7f);
        my_x = (float)sqrt(hh) * (1.0f + 2.4e-7f);
        if (xn) xn[r0 + r] = my_x;
        // q / 2 in three pieces: FP16 at scales 2^15, 2^4, 2^-7 (the A side's
        // constants); TF32 and BF16 hi + lo at scale 1
        const double s1 = OP == 2 ? 0x1p15 : 1.0, s2 = OP == 2 ? 0x1p4 : 1.0, s3 = OP == 2 ? 0x1p-7 : 1.0;
        double b1, b2, b3;
        const double v1 = 0.5 * q;
        mb0 = El::round(v1 / s1, &b1);
        const double v2 = v1 - b1 * s1;
        mb1 = El::round(v2 / s2, &b2);
        const double v3 = v2 - b2 * s2;
        mb2 = El::round(v3 / s3, &b3);
        (void)b3;
    } else {
        norms[r0 + r] = kPadNorm;
        if (xn) xn[r0 + r] = 0.f;
    }
    ms[4 * r] = mb0;
    ms[4 * r + 1] = mb1;
    ms[4 * r + 2] = mb2;
    __syncthreads();
    // 4. the rows [h | h | c m | h a] as 16-byte chunks, consecutive threads on
    // consecutive chunks (operand bits copied, no conversion)
    double unused;
    const E ab0 = El::round(OP == 2 ? -0x1p15 : -1.0, &unused), ab1 = El::round(OP == 2 ? -0x1p4 : -1.0, &unused),
            ab2 = El::round(OP == 2 ? -0x1p-7 : -1.0, &unused);
    // chunk e = (row rr, chunk q of the row), q = (block b, chunk within it);
    // the indices advance by kBcBlock chunks per step without divisions
    const uint32_t cpb = dp / kEpc, cpr = 4 * cpb;  // 16-byte chunks per block, per row (4 dp elements)
    const uint32_t step_r = kBcBlock / cpr, step_q = kBcBlock - step_r * cpr;
    uint32_t rr = threadIdx.x / cpr, q = threadIdx.x - rr * cpr;
    for (uint32_t e = threadIdx.x; e < kBcBlock * cpr; e += kBcBlock) {
        const uint32_t b = (q >= cpb) + (q >= 2 * cpb) + (q >= 3 * cpb), t0 = kEpc * (q - b * cpb);
        uint32_t w[4] = {0u, 0u, 0u, 0u}, wl[4] = {0u, 0u, 0u, 0u};
        if (rr < nr) {
#pragma unroll
            for (uint32_t z = 0; z < kEpc; ++z) {
                const uint32_t t = t0 + z;
                uint32_t bits = 0;
                if (t < d)
                    bits = b == 2 ? chs[t] : hs[rr * P.hstride + t];
                else if (t < d + 3)
                    bits = b == 2 ? ms[4 * rr + (t - d)] : (b == 3 ? (t == d ? ab0 : (t == d + 1 ? ab1 : ab2)) : 0u);
                if (kSplit) {
                    w[z >> 1] |= (bits & 0xffffu) << (16 * (z & 1));
                    wl[z >> 1] |= (bits >> 16) << (16 * (z & 1));
                } else if (sizeof(E) == 2) {
                    w[z >> 1] |= bits << (16 * (z & 1));
                } else {
                    w[z] = bits;
                }
            }
        }
        reinterpret_cast<uint4 *>(op_out)[(r0 + rr) * cpr + q] = make_uint4(w[0], w[1], w[2], w[3]);
        if (kSplit) reinterpret_cast<uint4 *>(op_lo)[(r0 + rr) * cpr + q] = make_uint4(wl[0], wl[1], wl[2], wl[3]);
        rr += step_r;
        q += step_q;
        if (q >= cpr) q -= cpr, ++rr;
    }
    // block summaries: max |h|, |c|, max |q| (all rounded up)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        my_x = fmaxf(my_x, __shfl_xor_sync(0xffffffffu, my_x, o));
        my_p = fmaxf(my_p, __shfl_xor_sync(0xffffffffu, my_p, o));
    }
    if ((threadIdx.x & 31u) == 0) {
        red_x[threadIdx.x >> 5] = my_x;
        red_p[threadIdx.x >> 5] = my_p;
    }
    for (uint32_t t = threadIdx.x; t < kBcCentStride; t += kBcBlock)
        cent[(uint64_t)blockIdx.x * kBcCentStride + t] = t < d ? (float)cs[t] : 0.f;
    __syncthreads();
    if (threadIdx.x == 0) {
        float mx = 0.f, mp = 0.f;
        for (int w = 0; w < (int)(kBcBlock / 32); ++w) {
            mx = fmaxf(mx, red_x[w]);
            mp = fmaxf(mp, red_p[w]);
        }
        double cc = 0.0;
        for (uint32_t t = 0; t < d; ++t) cc = fma(cs[t], cs[t], cc);
        blk[blockIdx.x] = make_float4(mx, (float)sqrt(cc) * (1.0f + 2.4e-7f), mp, 0.f);
    }
}

void launch_bc_prepare(const SortedSet &s, const double *center, double scale, void *op, void *op_lo, float *norms,
                       float *xn, float4 *blk, float *cent, cudaStream_t st, int *launches) {
    if (s.npad_tc == 0) return;
    const unsigned blocks = (unsigned)(s.npad_tc / kBcBlock);
    const uint32_t eb = s.bc_form == HJ_FORM_TC_FP16 ? 2u : 4u;  // shared-memory element (BF16: hi and lo)
    const size_t smem = bc_smem_plan(s.d, eb).bytes;
    // the block's rows start at r0 d coordinates: 16-byte loads when that and the base allow
    const bool vec = ((uintptr_t)s.rows & 15u) == 0 && ((uint64_t)kBcBlock * s.d * s.dtype_bytes) % 16 == 0;
    const int smem_max = (int)bc_smem_plan(kBcMaxDim, 4).bytes;
#define HJ_BC_PREP(T, OPV)                                                                                        \
    do {                                                                                                          \
        ensure_max_dynamic_smem((const void *)k_bc_prepare<T, OPV>, smem_max);                                    \
        k_bc_prepare<T, OPV><<<blocks, kBcBlock, smem, st>>>(static_cast<const T *>(s.rows), s.n, s.d, center,    \
                                                             scale, s.bc_dp, vec, op, op_lo, norms, xn, blk,      \
                                                             cent);                                               \
    } while (0)
    if (s.bc_form == HJ_FORM_TC_TF32) {
        if (s.dtype_bytes == 8) HJ_BC_PREP(double, 0); else HJ_BC_PREP(float, 0);
    } else if (s.bc_form == HJ_FORM_TC_BF16X3) {
        if (s.dtype_bytes == 8) HJ_BC_PREP(double, 1); else HJ_BC_PREP(float, 1);
    } else {
        if (s.dtype_bytes == 8) HJ_BC_PREP(double, 2); else HJ_BC_PREP(float, 2);
    }
#undef HJ_BC_PREP
    if (launches) *launches += 1;
}

void launch_gather(const void *x, int dtype_bytes, uint64_t n, uint32_t d, const uint32_t *perm,
                   const uint32_t *keys_wm, uint32_t W, const SortedSet &o, uint32_t flags, cudaStream_t st,
                   int *launches) {
    int L = 0;
    if (n == 0) return;
    const bool vec = ((uintptr_t)x & 15u) == 0 && ((uint64_t)d * dtype_bytes) % 16 == 0;
    uint32_t *keys_rm = (flags & kGatherKeys) ? o.keys : nullptr;
    void *rows_out = (flags & kGatherRows) ? const_cast<void *>(o.rows) : nullptr;
    const int op = (flags & kGatherTf32) ? 0 : (flags & kGatherBf16) ? 1 : (flags & kGatherF16) ? 2 : -1;
    if (op >= 0) {
        // every tensor-core layout in one pass (operands, norms, keys, rows)
        const uint32_t kp = op == 0 ? o.kpad_tf32 : o.kpad_bf16;
        void *hi = op == 0 ? (void *)o.tf32 : (void *)o.bf_hi;
        const double scale = op == 2 ? o.op_scale : 1.0;
        const double scale2 = op == 2 ? o.op_scale * o.op_scale : 1.0;
        const unsigned blocks = (unsigned)hj_ceil_div(o.npad_tc, kGrpRows);
#define HJ_GATHER_TC(T, OPV)                                                                                        \
    k_gather_tc_fused<T, OPV><<<blocks, 256, 0, st>>>(static_cast<const T *>(x), n, d, perm, keys_wm, W, o.center,   \
                                                      o.npad_tc, kp, scale, scale2, vec, keys_rm,                    \
                                                      static_cast<T *>(rows_out), hi, o.bf_lo, o.norms)
        if (dtype_bytes == 8) {
            if (op == 0) HJ_GATHER_TC(double, 0); else if (op == 1) HJ_GATHER_TC(double, 1); else HJ_GATHER_TC(double, 2);
        } else {
            if (op == 0) HJ_GATHER_TC(float, 0); else if (op == 1) HJ_GATHER_TC(float, 1); else HJ_GATHER_TC(float, 2);
        }
#undef HJ_GATHER_TC
        launch_norm_summaries(o.norms, o.npad_tc, o.tile_maxnorm_a, o.tile_maxnorm_b, o.group_minnorm, st);
        L += 4;
    } else if (keys_rm || rows_out) {
        const unsigned blocks = (unsigned)hj_ceil_div(n, kGrpRows);
        if (dtype_bytes == 8)
            k_gather_rows_fused<double><<<blocks, 256, 0, st>>>(static_cast<const double *>(x), n, d, perm, keys_wm, W,
                                                                vec, keys_rm, static_cast<double *>(rows_out));
        else
            k_gather_rows_fused<float><<<blocks, 256, 0, st>>>(static_cast<const float *>(x), n, d, perm, keys_wm, W,
                                                               vec, keys_rm, static_cast<float *>(rows_out));
        ++L;
    }
    if (flags & kGatherPlain) {
        if (dtype_bytes == 8)
            k_gather_plain_tiles<double><<<(unsigned)o.n_tiles64, 256, 0, st>>>(static_cast<const double *>(x), n, d,
                                                                                perm, o.tiles64);
        else
            k_gather_plain_tiles<float><<<(unsigned)o.n_tiles64, 256, 0, st>>>(static_cast<const float *>(x), n, d,
                                                                               perm, o.tiles64);
        ++L;
    }
    if (launches) *launches += L;
}

void launch_norm_summaries(const float *norms, uint64_t npad, float *tmax_a, float *tmax_b, float *gmin32,
                           cudaStream_t st) {
    if (npad == 0) return;
    k_tile_max<<<(unsigned)hj_ceil_div(npad / kTcTileA, 256), 256, 0, st>>>(norms, npad, kTcTileA, tmax_a);
    k_tile_max<<<(unsigned)hj_ceil_div(npad / kTcTileB, 256), 256, 0, st>>>(norms, npad, kTcTileB, tmax_b);
    k_group_min<<<(unsigned)hj_ceil_div(npad / 32, 256), 256, 0, st>>>(norms, npad, 32, gmin32);
}

}  // namespace hj
