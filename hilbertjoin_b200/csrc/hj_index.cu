// hj_index.cu -- stripe bounds and the block-pair work list.
//
// Replaces the reference's prepareStripes / prepareStripesNoSelf
// (hilbertjoin/egojoin.cpp:270-464, :1126-1240), which binary-search, per point
// and per stripe, the EGO position of the point displaced by a per-stripe
// offset, aggregate the bounds to 8-point blocks and build min/max segment
// trees, and the Hilbert loop FGF_HILBERT_FOR (hilbertjoin/hilloop.h:9-82) that
// walks the (i-block, j-block) grid and prunes with those trees.
//
// Here the work is organised per A tile (the point tile of the distance
// kernel). Every neighbour b of a point a has cell(b)_t in
// [lo_t(a), hi_t(a)] = [cell(a_t - eps'), cell(a_t + eps')] for every dim t,
// with eps' = eps + 2^-40 (eps + max|x|) slightly wider than eps so that the
// bound also holds for the FP64 pair test and for floor(x/eps) jitter at cell
// borders. A stripe fixes the cells of the first k = active_dims dims to one
// combination v in the neighbour range and spans
//   [first key >= (v, lo_k, .., lo_{d-1}),  first key > (v, hi_k, .., hi_{d-1}))
// of B's EGO order (the reference's upper search uses ">=", which can miss the
// cell of x + eps itself; this one is inclusive). Because adding the same
// offset to every vector preserves lexicographic order, the union of a
// stripe's ranges over all points of an A tile is obtained from two points
// only: the lexicographic minimum of the lo vectors and the maximum of the
// (lo_<k, hi_>=k) vectors. So each A tile costs 2 * 3^k binary searches, not
// 2 * 3^k per point. The ranges are rounded out to B tiles, merged into runs,
// split into work items of at most `chunk` B tiles, and the items sorted by the
// Hilbert index of (A tile, B chunk), so that the items that run at the same
// time on the GPU's SMs share their B tiles in L2 -- the role the Hilbert
// traversal plays for the CPU caches in the reference.
#include "hj_common.cuh"
#include "hj_internal.h"

namespace hj {

struct BoundsArgs {
    const void *rows;  // A sorted rows
    int dtype_bytes;
    uint64_t na;       // A rows considered
    uint32_t d;
    double eps, epsw, inv;  // inv = fl(1 / eps) (cell_of)
    GridDev g;
    uint32_t W;
    int k;             // active dims requested
    const uint32_t *bkeys;  // B sorted keys [nb][W]
    uint64_t nb;
    int tile_a, tile_b;
    int self;
    uint2 *runs;       // [n_tiles][kMaxCombos]
    uint32_t *nruns;   // [n_tiles]
    unsigned long long *cand;  // candidate pairs (tile granularity)
    uint32_t *lokeys, *hikeys;  // per A row [na][W]: packed digits of cell_lo / cell_hi (k_bound_keys)
};

__device__ __forceinline__ double crd(const BoundsArgs &a, uint64_t r, uint32_t t) {
    return a.dtype_bytes == 8 ? static_cast<const double *>(a.rows)[r * a.d + t]
                              : (double)static_cast<const float *>(a.rows)[r * a.d + t];
}

__device__ __forceinline__ uint32_t digit_of(const BoundsArgs &a, double cell, uint32_t t) {
    long long v = (long long)cell - a.g.off[t];
    long long mx = (1ll << a.g.bits[t]) - 1;
    v = v < 0 ? 0 : (v > mx ? mx : v);
    return (uint32_t)v;
}

// floor((x -+ epsw) / eps) with the quotient rounded as FP64 division does
// (cell_of: a multiply, and the division only next to a cell border)
__device__ __forceinline__ double cell_lo(const BoundsArgs &a, double x) { return cell_of(x - a.epsw, a.eps, a.inv); }
__device__ __forceinline__ double cell_hi(const BoundsArgs &a, double x) { return cell_of(x + a.epsw, a.eps, a.inv); }

// Per A row, the clamped digits of its cell_lo and cell_hi vectors packed like
// the sort keys (fields in key order from the most significant bit of word 0):
// unsigned word-by-word order of these keys is the lexicographic order of the
// digit vectors. One thread per row, written row-major [na][W].
__global__ void k_bound_keys(BoundsArgs a) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.na) return;
    uint32_t *lo = a.lokeys + r * a.W, *hi = a.hikeys + r * a.W;
    uint32_t cur = 0, al = 0, ah = 0;
    for (uint32_t pos = 0; pos < a.d; ++pos) {
        const uint32_t t = grid_dim_at(a.g, pos), w = a.g.word[t];
        if (w != cur) {
            lo[cur] = al;
            hi[cur] = ah;
            for (uint32_t z = cur + 1; z < w; ++z) lo[z] = hi[z] = 0u;
            cur = w;
            al = ah = 0;
        }
        const double x = crd(a, r, t);
        al |= digit_of(a, cell_lo(a, x), t) << a.g.shift[t];
        ah |= digit_of(a, cell_hi(a, x), t) << a.g.shift[t];
    }
    lo[cur] = al;
    hi[cur] = ah;
    for (uint32_t z = cur + 1; z < a.W; ++z) lo[z] = hi[z] = 0u;
}

// Word w of row p's upper key: lo digits at key positions < kt, hi digits from
// kt on; `mw` / `mbits` describe the boundary (positions < kt fill the words
// before mw and the bits of word mw above mbits).
__device__ __forceinline__ uint32_t up_word(const BoundsArgs &a, uint64_t p, uint32_t w, uint32_t mw, uint32_t mbits) {
    const uint32_t m = w < mw ? 0xffffffffu : (w > mw || mbits >= 32 ? 0u : ~((1u << mbits) - 1u));
    return (__ldg(a.lokeys + p * a.W + w) & m) | (__ldg(a.hikeys + p * a.W + w) & ~m);
}
// -1, 0, 1: lexicographic comparison of the lo digit vectors of rows p and q.
__device__ int cmp_lo(const BoundsArgs &a, uint64_t p, uint64_t q) {
    for (uint32_t w = 0; w < a.W; ++w) {
        const uint32_t kp = __ldg(a.lokeys + p * a.W + w), kq = __ldg(a.lokeys + q * a.W + w);
        if (kp != kq) return kp < kq ? -1 : 1;
    }
    return 0;
}
// Same for the upper vectors (lo digits at key positions < kt, hi digits from kt on).
__device__ int cmp_up(const BoundsArgs &a, uint64_t p, uint64_t q, uint32_t mw, uint32_t mbits) {
    for (uint32_t w = 0; w < a.W; ++w) {
        const uint32_t kp = up_word(a, p, w, mw, mbits), kq = up_word(a, q, w, mw, mbits);
        if (kp != kq) return kp < kq ? -1 : 1;
    }
    return 0;
}

// First index in [0, n) whose key is >= q (strict = 0) or > q (strict = 1).
// The query is the base words `base` with its first `np` words replaced by `pw`.
__device__ uint64_t key_search(const uint32_t *__restrict__ keys, uint64_t n, uint32_t W, const uint32_t *base,
                               const uint32_t *pw, int np, int strict) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        uint64_t mid = lo + ((hi - lo) >> 1);
        const uint32_t *kr = keys + mid * W;
        int c = 0;
        for (uint32_t w = 0; w < W; ++w) {
            uint32_t kw = __ldg(kr + w);
            uint32_t qw = (int)w < np ? pw[w] : base[w];
            if (kw != qw) {
                c = kw < qw ? -1 : 1;
                break;
            }
        }
        if (c < 0 || (strict && c == 0))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

constexpr int kBoundsWarps = 4;

// One warp per A tile. Dynamic smem: per warp 2*W key words + kMaxCombos
// intervals.
__global__ void __launch_bounds__(kBoundsWarps * 32) k_tile_bounds(BoundsArgs a, uint64_t n_tiles) {
    extern __shared__ uint32_t sm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t tile = (uint64_t)blockIdx.x * kBoundsWarps + warp;
    uint32_t *qlo = sm + (size_t)warp * (2 * a.W + 2 * kMaxCombos);
    uint32_t *qhi = qlo + a.W;
    uint2 *iv = reinterpret_cast<uint2 *>(qhi + a.W);
    if (tile >= n_tiles) return;
    const uint64_t p0 = tile * a.tile_a;
    const uint64_t p1 = hj_umin(p0 + a.tile_a, a.na);
    if (p0 >= p1) {
        if (lane == 0) a.nruns[tile] = 0;
        return;
    }
    // 1. effective active dims: dims whose neighbour range is at most 3 cells wide
    int kt = a.k;
    for (uint64_t p = p0 + lane; p < p1; p += 32) {
        int ke = 0;
        while (ke < kt) {
            double x = crd(a, p, grid_dim_at(a.g, ke));
            if (cell_hi(a, x) - cell_lo(a, x) > 2.0) break;
            ++ke;
        }
        kt = ke;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) kt = min(kt, __shfl_xor_sync(0xffffffffu, kt, o));
    // the upper key's boundary: the field of key position kt (hi from there on)
    uint32_t mw = 0xffffffffu, mbits = 0;  // kt >= d: every position takes its lo digit
    if ((uint32_t)kt < a.d) {
        const uint32_t t = grid_dim_at(a.g, (uint32_t)kt);
        mw = a.g.word[t];
        mbits = a.g.shift[t] + a.g.bits[t];
    }
    // 2. lexicographic min of lo vectors, max of upper vectors (packed keys)
    uint64_t pmin = p0 + hj_umin(lane, p1 - p0 - 1), pmax = pmin;
    for (uint64_t p = p0 + lane + 32; p < p1; p += 32) {
        if (cmp_lo(a, p, pmin) < 0) pmin = p;
        if (cmp_up(a, p, pmax, mw, mbits) > 0) pmax = p;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        uint64_t qmin = __shfl_xor_sync(0xffffffffu, pmin, o);
        uint64_t qmax = __shfl_xor_sync(0xffffffffu, pmax, o);
        int c1 = cmp_lo(a, qmin, pmin);
        if (c1 < 0 || (c1 == 0 && qmin < pmin)) pmin = qmin;
        int c2 = cmp_up(a, qmax, pmax, mw, mbits);
        if (c2 > 0 || (c2 == 0 && qmax < pmax)) pmax = qmax;
    }
    // 3. packed base queries: the lo key of pmin and the upper key of pmax
    for (uint32_t w = lane; w < a.W; w += 32) {
        qlo[w] = __ldg(a.lokeys + pmin * a.W + w);
        qhi[w] = up_word(a, pmax, w, mw, mbits);
    }
    __syncwarp();
    // 4. one pair of searches per combination of the first kt dims
    int ncomb = 1;
    for (int t = 0; t < kt; ++t) ncomb *= 3;
    const int np = kt > 0 ? (int)a.g.word[grid_dim_at(a.g, kt - 1)] + 1 : 0;  // words holding active dims
    for (int c = lane; c < ncomb; c += 32) {
        uint32_t pl[kMaxActiveDims], ph[kMaxActiveDims];
        for (int w = 0; w < np; ++w) {
            pl[w] = qlo[w];
            ph[w] = qhi[w];
        }
        int rem = c;
        for (int pos = kt - 1; pos >= 0; --pos) {
            const uint32_t t = grid_dim_at(a.g, (uint32_t)pos);
            uint32_t delta = (uint32_t)(rem % 3);
            rem /= 3;
            uint32_t w = a.g.word[t], sh = a.g.shift[t];
            uint32_t mask = ((1u << a.g.bits[t]) - 1u);
            uint32_t fmax = mask;
            uint32_t vl = min(((pl[w] >> sh) & mask) + delta, fmax);
            uint32_t vh = min(((ph[w] >> sh) & mask) + delta, fmax);
            pl[w] = (pl[w] & ~(mask << sh)) | (vl << sh);
            ph[w] = (ph[w] & ~(mask << sh)) | (vh << sh);
        }
        uint64_t lower = key_search(a.bkeys, a.nb, a.W, qlo, pl, np, 0);
        uint64_t upper = key_search(a.bkeys, a.nb, a.W, qhi, ph, np, 1);
        if (a.self && lower < p0) lower = p0;
        uint2 v = make_uint2(1u, 0u);  // empty
        if (lower < upper) v = make_uint2((uint32_t)(lower / a.tile_b), (uint32_t)hj_ceil_div(upper, a.tile_b));
        iv[c] = v;
    }
    __syncwarp();
    // 5. merge the intervals into disjoint runs (lane 0)
    if (lane == 0) {
        int m = 0;
        for (int c = 0; c < ncomb; ++c)
            if (iv[c].x < iv[c].y) iv[m++] = iv[c];
        for (int i = 1; i < m; ++i) {  // insertion sort by start
            uint2 v = iv[i];
            int j = i - 1;
            while (j >= 0 && iv[j].x > v.x) {
                iv[j + 1] = iv[j];
                --j;
            }
            iv[j + 1] = v;
        }
        int r = 0;
        unsigned long long cols = 0;
        uint2 *out = a.runs + tile * kMaxCombos;
        for (int i = 0; i < m; ++i) {
            if (r > 0 && iv[i].x <= out[r - 1].y) {
                out[r - 1].y = max(out[r - 1].y, iv[i].y);
            } else {
                out[r++] = iv[i];
            }
        }
        for (int i = 0; i < r; ++i) {
            uint64_t b0 = (uint64_t)out[i].x * a.tile_b, b1 = hj_umin((uint64_t)out[i].y * a.tile_b, a.nb);
            cols += b1 > b0 ? b1 - b0 : 0;
        }
        a.nruns[tile] = (uint32_t)r;
        atomicAdd(a.cand, cols * (p1 - p0));
    }
}

__global__ void k_item_counts(const uint2 *__restrict__ runs, const uint32_t *__restrict__ nruns, uint64_t n_tiles,
                              uint32_t chunk, uint32_t *counts, unsigned long long *tile_pairs) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tiles) return;
    uint32_t c = 0;
    unsigned long long tp = 0;
    for (uint32_t i = 0; i < nruns[t]; ++i) {
        uint2 r = runs[t * kMaxCombos + i];
        c += (uint32_t)hj_ceil_div(r.y - r.x, chunk);
        tp += r.y - r.x;
    }
    counts[t] = c;
    if (tp) atomicAdd(tile_pairs, tp);
}

// Hilbert index of (x, y) on a side-`side` grid (side a power of two); the
// classic iterative conversion (rotate the quadrant, accumulate s*s*quadrant).
__device__ __forceinline__ unsigned long long hilbert_index(unsigned long long side, unsigned long long x,
                                                            unsigned long long y) {
    unsigned long long dd = 0;
    for (unsigned long long s = side >> 1; s > 0; s >>= 1) {
        unsigned long long rx = (x & s) ? 1 : 0, ry = (y & s) ? 1 : 0;
        dd += s * s * ((3 * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = side - 1 - x;
                y = side - 1 - y;
            }
            unsigned long long tmp = x;
            x = y;
            y = tmp;
        }
    }
    return dd;
}

__global__ void k_item_write(const uint2 *__restrict__ runs, const uint32_t *__restrict__ nruns,
                             const uint32_t *__restrict__ offsets, uint64_t n_tiles, uint32_t chunk,
                             unsigned long long side, uint32_t key_words, WorkItem *items, uint32_t *keys_wm,
                             uint64_t n_items) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tiles) return;
    uint64_t o = offsets[t];
    for (uint32_t i = 0; i < nruns[t]; ++i) {
        uint2 r = runs[t * kMaxCombos + i];
        for (uint32_t b = r.x; b < r.y; b += chunk) {
            WorkItem it;
            it.a = (uint32_t)t;
            it.b0 = b;
            it.b1 = min(b + chunk, r.y);
            it.pad = 0;
            items[o] = it;
            unsigned long long h = hilbert_index(side, t, b / chunk);
            if (key_words == 1) {
                keys_wm[o] = (uint32_t)h;
            } else {
                keys_wm[o] = (uint32_t)(h >> 32);          // word 0: most significant
                keys_wm[n_items + o] = (uint32_t)h;        // word 1
            }
            ++o;
        }
    }
}

__global__ void k_permute_items(const WorkItem *__restrict__ in, const uint32_t *__restrict__ perm, uint64_t n,
                                WorkItem *out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[perm[i]];
}

// Scratch slots requested through the caller's allocator.
enum { kSlotRuns = kSlotIndexFirst, kSlotNruns, kSlotCounts, kSlotItemsTmp, kSlotItems, kSlotItemKeys, kSlotItemPerm,
       kSlotItemPermTmp, kSlotItemHist, kSlotIdxStats, kSlotSplitFlags, kSlotSplitTc, kSlotSplitFp, kSlotSplitStats,
       kSlotShardLoad, kSlotShardCut, kSlotBoundKeysLo, kSlotBoundKeysHi, kSlotScanTiles, kSlotIndexEnd };
static_assert(kSlotIndexEnd <= kSlotIndexFirst + 32, "index-stage slots");

__global__ void k_item_loads(const WorkItem *__restrict__ items, uint64_t n, uint32_t *load) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) load[i] = items[i].b1 - items[i].b0;
}

// cut[0], cut[1]: first items whose exclusive load prefix reaches lo and hi.
__global__ void k_shard_cut(const uint32_t *__restrict__ prefix, uint64_t n, unsigned long long lo,
                            unsigned long long hi, unsigned long long *cut) {
    for (int c = 0; c < 2; ++c) {
        const unsigned long long target = c ? hi : lo;
        uint64_t a = 0, b = n;
        while (a < b) {
            uint64_t m = (a + b) >> 1;
            if ((unsigned long long)prefix[m] < target) a = m + 1; else b = m;
        }
        cut[c] = a;
    }
}

int shard_items(const IndexResult &in, int k, int K, void *(*alloc)(void *ctx, int slot, size_t bytes), void *actx,
                cudaStream_t st, IndexResult *out) {
    *out = in;
    if (K <= 1 || in.n_items == 0) return 0;
    const uint64_t n = in.n_items;
    uint32_t *load = (uint32_t *)alloc(actx, kSlotShardLoad, (n + 1) * sizeof(uint32_t));
    unsigned long long *cut = (unsigned long long *)alloc(actx, kSlotShardCut, 4 * sizeof(unsigned long long));
    if (!load || !cut) return 2;
    k_item_loads<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(in.items, n, load);
    launch_scan_u32(load, n, cut + 2, st,
                    (unsigned long long *)alloc(actx, kSlotScanTiles, scan_scratch_bytes(n)));
    unsigned long long total = 0;
    cudaMemcpyAsync(&total, cut + 2, 8, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return 3;
    const unsigned long long lo = total * (unsigned long long)k / (unsigned long long)K;
    const unsigned long long hi = total * (unsigned long long)(k + 1) / (unsigned long long)K;
    k_shard_cut<<<1, 1, 0, st>>>(load, n, lo, hi, cut);
    unsigned long long hc[2];
    cudaMemcpyAsync(hc, cut, 16, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return 3;
    const uint64_t a = hc[0], b = k + 1 == K ? n : hc[1];
    out->items = in.items + a;
    out->n_items = b > a ? b - a : 0;
    return 0;
}

__global__ void k_item_precision_flags(const WorkItem *__restrict__ items, uint64_t n, const float *__restrict__ tmax_a,
                                       const float *__restrict__ tmax_b, double c_rel, double c_abs, double limit,
                                       uint32_t *flags, unsigned long long *tile_pairs_fp) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const WorkItem w = items[i];
    float mb = 0.f;
    for (uint32_t b = w.b0; b < w.b1; ++b) mb = fmaxf(mb, tmax_b[b]);
    const double tau = c_rel * ((double)tmax_a[w.a] + (double)mb) + c_abs;
    const bool tc = tau <= limit;
    flags[i] = tc ? 1u : 0u;
    if (!tc) atomicAdd(tile_pairs_fp, (unsigned long long)(w.b1 - w.b0));
}

// Per-block-centred operands: the item's bound from its A block's summary and
// the largest of its B blocks' (two per 256-rank B tile), at D = 0 (the D term
// only grows with the block distance, where every pair is far outside).
__global__ void k_item_precision_flags_bc(const WorkItem *__restrict__ items, uint64_t n,
                                          const float4 *__restrict__ blk_a, const float4 *__restrict__ blk_b,
                                          BcConsts k, double limit, uint32_t *flags,
                                          unsigned long long *tile_pairs_fp) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const WorkItem w = items[i];
    const float4 a = blk_a[w.a];
    float xb = 0.f, cb = 0.f, qb = 0.f;
    for (uint32_t b = 2 * w.b0; b < 2 * w.b1; ++b) {
        const float4 v = blk_b[b];
        xb = fmaxf(xb, v.x);
        cb = fmaxf(cb, v.y);
        qb = fmaxf(qb, v.z);
    }
    const float tau = bc_tau(a.x, a.y, a.z, xb, cb, qb, 0.f, k, nullptr);
    const bool tc = (double)tau <= limit;
    flags[i] = tc ? 1u : 0u;
    if (!tc) atomicAdd(tile_pairs_fp, (unsigned long long)(w.b1 - w.b0));
}

// flags[] holds the exclusive prefix count of tensor-core items.
__global__ void k_item_split(const WorkItem *__restrict__ items, uint64_t n, const uint32_t *__restrict__ flags_scan,
                             unsigned long long n_tc, WorkItem *tc_out, WorkItem *fp_out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t before = flags_scan[i];
    const uint32_t next = i + 1 < n ? flags_scan[i + 1] : (uint32_t)n_tc;
    const WorkItem w = items[i];
    constexpr uint32_t r = kTcTileA / kPlainTile, c = kTcTileB / kPlainTile;
    if (next != before) {
        tc_out[before] = w;
    } else {
        const uint64_t k = (uint64_t)r * (i - before);
        for (uint32_t h = 0; h < r; ++h) {
            WorkItem p;
            p.a = w.a * r + h;
            p.b0 = w.b0 * c;
            p.b1 = w.b1 * c;
            p.pad = 0;
            fp_out[k + h] = p;
        }
    }
}

int split_items_by_precision(const IndexResult &in, const SortedSet &A, const SortedSet &B, double c_rel,
                             double c_abs, double limit, const BcConsts *bc,
                             void *(*alloc)(void *ctx, int slot, size_t bytes), void *actx, cudaStream_t st,
                             IndexResult *tc_out, IndexResult *fp_out) {
    *tc_out = in;
    *fp_out = IndexResult();
    if (in.n_items == 0) return 0;
    const uint64_t n = in.n_items;
    uint32_t *flags = (uint32_t *)alloc(actx, kSlotSplitFlags, (n + 1) * sizeof(uint32_t));
    unsigned long long *stats = (unsigned long long *)alloc(actx, kSlotSplitStats, 2 * sizeof(unsigned long long));
    if (!flags || !stats) return 2;
    cudaMemsetAsync(stats, 0, 2 * sizeof(unsigned long long), st);
    if (bc)
        k_item_precision_flags_bc<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(in.items, n, A.bc_blk, B.bc_blk, *bc,
                                                                                limit, flags, stats + 1);
    else
        k_item_precision_flags<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(in.items, n, A.tile_maxnorm_a,
                                                                             B.tile_maxnorm_b, c_rel, c_abs, limit,
                                                                             flags, stats + 1);
    launch_scan_u32(flags, n, stats, st,
                    (unsigned long long *)alloc(actx, kSlotScanTiles, scan_scratch_bytes(n)));
    unsigned long long h[2];
    cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return 3;
    const uint64_t n_tc = h[0], n_fp = n - n_tc;
    if (n_fp == 0) return 0;
    WorkItem *tc = (WorkItem *)alloc(actx, kSlotSplitTc, (n_tc + 1) * sizeof(WorkItem));
    constexpr uint32_t rows_per_tc = kTcTileA / kPlainTile;  // FP64 items per routed tensor-core item
    WorkItem *fp = (WorkItem *)alloc(actx, kSlotSplitFp, rows_per_tc * n_fp * sizeof(WorkItem));
    if (!tc || !fp) return 2;
    k_item_split<<<(unsigned)hj_ceil_div(n, 256), 256, 0, st>>>(in.items, n, flags, n_tc, tc, fp);
    tc_out->items = tc;
    tc_out->n_items = n_tc;
    tc_out->tile_pairs = in.tile_pairs - h[1];
    fp_out->items = fp;
    fp_out->n_items = rows_per_tc * n_fp;
    fp_out->tile_pairs = h[1] * (kTcTileA / kPlainTile) * (kTcTileB / kPlainTile);
    return 0;
}

int build_index(const SortedSet &A, const SortedSet &B, const Grid &grid, const GridDev &gdev, bool self,
                uint64_t na_eff, uint64_t nb_eff, int tile_a, int tile_b, int active_dims, uint32_t chunk,
                void *(*alloc)(void *ctx, int slot, size_t bytes), void *actx, cudaStream_t st, IndexResult *out,
                int *launches, std::string *err) {
    *out = IndexResult();
    const uint64_t n_tiles = hj_ceil_div(na_eff, tile_a);
    if (n_tiles == 0 || nb_eff == 0) return 0;
    int k = active_dims < 0 ? 0 : (active_dims > kMaxActiveDims ? kMaxActiveDims : active_dims);
    if ((uint32_t)k > grid.d) k = (int)grid.d;
    uint2 *runs = (uint2 *)alloc(actx, kSlotRuns, n_tiles * kMaxCombos * sizeof(uint2));
    uint32_t *nruns = (uint32_t *)alloc(actx, kSlotNruns, n_tiles * sizeof(uint32_t));
    uint32_t *counts = (uint32_t *)alloc(actx, kSlotCounts, (n_tiles + 1) * sizeof(uint32_t));
    unsigned long long *stats = (unsigned long long *)alloc(actx, kSlotIdxStats, 4 * sizeof(unsigned long long));
    uint32_t *lokeys = (uint32_t *)alloc(actx, kSlotBoundKeysLo, na_eff * grid.W * sizeof(uint32_t));
    uint32_t *hikeys = (uint32_t *)alloc(actx, kSlotBoundKeysHi, na_eff * grid.W * sizeof(uint32_t));
    if (!runs || !nruns || !counts || !stats || !lokeys || !hikeys) {
        *err = "out of device memory (index scratch)";
        return 2;
    }
    cudaMemsetAsync(stats, 0, 4 * sizeof(unsigned long long), st);
    BoundsArgs ba;
    ba.rows = A.rows;
    ba.dtype_bytes = A.dtype_bytes;
    ba.na = na_eff;
    ba.d = grid.d;
    ba.eps = grid.eps;
    ba.epsw = grid.eps_wide;
    ba.inv = 1.0 / grid.eps;
    ba.g = gdev;
    ba.W = grid.W;
    ba.k = k;
    ba.bkeys = B.keys;
    ba.nb = nb_eff;
    ba.tile_a = tile_a;
    ba.tile_b = tile_b;
    ba.self = self ? 1 : 0;
    ba.runs = runs;
    ba.nruns = nruns;
    ba.cand = stats;
    ba.lokeys = lokeys;
    ba.hikeys = hikeys;
    k_bound_keys<<<(unsigned)hj_ceil_div(na_eff, 256), 256, 0, st>>>(ba);
    size_t smem = (size_t)kBoundsWarps * (2 * grid.W + 2 * kMaxCombos) * sizeof(uint32_t);
    if (smem > 48 * 1024) ensure_max_dynamic_smem((const void *)k_tile_bounds, (int)smem);
    k_tile_bounds<<<(unsigned)hj_ceil_div(n_tiles, kBoundsWarps), kBoundsWarps * 32, smem, st>>>(ba, n_tiles);
    k_item_counts<<<(unsigned)hj_ceil_div(n_tiles, 256), 256, 0, st>>>(runs, nruns, n_tiles, chunk, counts,
                                                                     stats + 1);
    launch_scan_u32(counts, n_tiles, stats + 2, st,
                    (unsigned long long *)alloc(actx, kSlotScanTiles, scan_scratch_bytes(n_tiles)));
    unsigned long long hstats[4];
    cudaMemcpyAsync(hstats, stats, sizeof(hstats), cudaMemcpyDeviceToHost, st);
    if (launches) *launches += 4;
    cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        *err = std::string("index stage: ") + cudaGetErrorString(e);
        return 3;
    }
    const uint64_t n_items = hstats[2];
    out->candidate_pairs = hstats[0];
    out->tile_pairs = hstats[1];
    out->n_items = n_items;
    if (n_items == 0) return 0;
    if (n_items >= (1ull << 31)) {
        *err = "work list too large";
        return 1;
    }
    unsigned long long side = 1;
    const uint64_t n_chunks_b = hj_ceil_div(hj_ceil_div(B.n, tile_b), chunk) + 1;
    while (side < n_tiles || side < n_chunks_b) side <<= 1;
    int hbits = 0;
    while ((1ull << hbits) < side * side) ++hbits;
    const uint32_t key_words = hbits > 32 ? 2 : 1;
    WorkItem *tmp = (WorkItem *)alloc(actx, kSlotItemsTmp, n_items * sizeof(WorkItem));
    WorkItem *items = (WorkItem *)alloc(actx, kSlotItems, n_items * sizeof(WorkItem));
    uint32_t *keys = (uint32_t *)alloc(actx, kSlotItemKeys, n_items * key_words * sizeof(uint32_t));
    uint32_t *perm = (uint32_t *)alloc(actx, kSlotItemPerm, n_items * sizeof(uint32_t));
    void *rs = alloc(actx, kSlotItemHist, radix_scratch_bytes(n_items));
    if (!tmp || !items || !keys || !perm || !rs) {
        *err = "out of device memory (work list)";
        return 2;
    }
    k_item_write<<<(unsigned)hj_ceil_div(n_tiles, 256), 256, 0, st>>>(runs, nruns, counts, n_tiles, chunk, side,
                                                                     key_words, tmp, keys, n_items);
    std::vector<std::pair<uint32_t, uint32_t>> passes;
    if (key_words == 1) {
        for (int b = 0; b < hbits; b += 8) passes.push_back({0u, (uint32_t)b});
    } else {
        for (int b = 0; b < 32; b += 8) passes.push_back({1u, (uint32_t)b});
        for (int b = 0; b < hbits - 32; b += 8) passes.push_back({0u, (uint32_t)b});
    }
    radix_sort_perm(keys, n_items, passes, perm, rs, st, launches);
    k_permute_items<<<(unsigned)hj_ceil_div(n_items, 256), 256, 0, st>>>(tmp, perm, n_items, items);
    if (launches) *launches += 2;
    out->items = items;
    return 0;
}

}  // namespace hj
