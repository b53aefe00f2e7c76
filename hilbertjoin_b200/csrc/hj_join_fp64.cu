// hj_join_fp64.cu -- the plain FP64 distance kernel (HJ_FORM_PLAIN_FP64).
//
// Replaces the reference's 8x8 block-pair kernel EGO_LOOP_TRAN /
// EGO_LOOP_TRAN_NOSELF (hilbertjoin/egojoin.h:311-392, :482-553) and its
// count (egojoin.cpp:803-813, :871-881): 64 pairs per visit by norm expansion
// on AVX-512 FMAs, early exit every KBLOCK dims once all 64 exceed eps^2,
// counted by sign bit, summed per thread (egojoin.cpp:466-474).
//
// Here a persistent CTA of 256 threads takes work items (an A tile of 64 EGO
// ranks against a run of B tiles of 64 ranks) in Hilbert order. The A tile is
// staged once per item and the B tiles are double-buffered, each by one 1D
// bulk copy (cp.async.bulk, the non-tensor TMA) of its [d][64] FP64 block into
// shared memory (above d = 128 by 64-dim chunks, which keeps d <= 256 within
// 192 KB), completion tracked by mbarriers. Each thread owns a 4 x 4
// block of pairs and evaluates the pair test exactly as the oracle defines it:
// acc = fma(a_k - b_k, a_k - b_k, acc) in IEEE FP64, k = 0..d-1 in order,
// count iff acc <= eps*eps. The partial sums never decrease, so a warp whose
// 512 pairs all exceed eps^2 after some dims stops early (checked every 8
// dims) without changing any decision. Counts are reduced by warp shuffles and
// one 64-bit atomic per warp.
//
// The same kernel materialises the pairs (hj_self_join_pairs / hj_join_pairs)
// in two more modes: kModeItemCounts adds each warp's count of an item into
// item_cnt[item] (one 32-bit atomic per warp and item), and after an exclusive
// scan of those counts kModeEmit writes every qualifying pair as (input index
// of the A point, input index of the B point) at item_cnt[item] (now the
// item's cursor), reserving each warp's block of slots per B tile with one
// atomic and placing the lanes by a warp prefix sum.
#include "hj_common.cuh"
#include "hj_internal.h"

namespace hj {

struct PlainArgs {
    const double *A, *B;  // [tile][d][64]
    uint32_t d;
    double T;
    const WorkItem *items;
    uint64_t n_items;
    uint64_t na, nb;
    int self;
    unsigned long long *count;
    uint32_t *err;
    // pair modes
    uint32_t *item_cnt;                 // per item: count (kModeItemCounts) / cursor (kModeEmit)
    const uint32_t *perm_a, *perm_b;    // EGO rank -> input index
    uint32_t *out_i, *out_j;            // emitted pairs
};

enum PlainMode { kModeCount = 0, kModeItemCounts = 1, kModeEmit = 2 };

constexpr int kPlainThreads = 256;
constexpr int kPlainWarps = kPlainThreads / 32;

// Dims per B stage: the whole tile up to d = 128; above, 64-dim chunks, so that
// the A tile (d <= 256: at most 128 KB) and two B stages fit one CTA's smem.
__host__ __device__ constexpr uint32_t plain_chunk_dims(uint32_t d) { return d <= 128 ? d : 64; }
constexpr uint32_t kPlainMaxDims = 256;

__host__ __device__ constexpr size_t plain_smem_bytes(uint32_t d) {
    return ((size_t)d + 2 * plain_chunk_dims(d)) * kPlainTile * sizeof(double);
}

// Waits for a bulk copy to land regardless of the error word, bounded in time:
// used only to drain copies still in flight before the CTA exits.
__device__ __forceinline__ void drain_wait(uint64_t *bar, uint32_t parity) {
    uint64_t t0 = globaltimer_ns();
    while (!mbar_try_wait(bar, parity)) {
        if (globaltimer_ns() - t0 > kWaitLimitNs) break;
    }
}

// One dimension of a thread's 4 x 4 pair block: acc[i][j] += (a_i - b_j)^2,
// rounded as the pair test defines it (one FP64 subtract, one FMA).
__device__ __forceinline__ void fma_dim(const double *pa, const double *pb, double (&acc)[4][4]) {
    const double2 a01 = *reinterpret_cast<const double2 *>(pa);
    const double2 a23 = *reinterpret_cast<const double2 *>(pa + 2);
    const double2 b01 = *reinterpret_cast<const double2 *>(pb);
    const double2 b23 = *reinterpret_cast<const double2 *>(pb + 2);
    const double av[4] = {a01.x, a01.y, a23.x, a23.y};
    const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double df = __dsub_rn(av[i], bv[j]);
            acc[i][j] = __fma_rn(df, df, acc[i][j]);
        }
}

template <int MODE>
__global__ void __launch_bounds__(kPlainThreads, 2) k_join_fp64(PlainArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar_a, bar_full[2], bar_empty[2];
    const uint32_t d = a.d;
    const uint32_t kc = plain_chunk_dims(d);  // dims per B stage
    const uint32_t tile_elems = d * kPlainTile;
    double *sA = reinterpret_cast<double *>(smem_raw);
    double *sB[2] = {sA + tile_elems, sA + tile_elems + kc * kPlainTile};
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const uint32_t ty = tid >> 4, tx = tid & 15u;
    volatile uint32_t *err = a.err;

    if (tid == 0) {
        mbar_init(&bar_a, 1);
        mbar_init(&bar_full[0], 1);
        mbar_init(&bar_full[1], 1);
        mbar_init(&bar_empty[0], kPlainWarps);
        mbar_init(&bar_empty[1], kPlainWarps);
        fence_barrier_init();
    }
    __syncthreads();

    // Producer state (thread 0): the next (B tile, dim chunk) to load in this
    // CTA's sequence; the chunk at dim k0 of a tile is the contiguous [kc][64]
    // block at row k0 of the tile's [d][64] layout.
    uint64_t p_item = blockIdx.x;
    uint32_t p_bt = 0, p_end = 0, p_k0 = 0;
    uint32_t issued = 0;
    if (tid == 0 && p_item < a.n_items) {
        WorkItem w = a.items[p_item];
        p_bt = w.b0;
        p_end = w.b1;
    }
    auto issue_next = [&](uint32_t consumed) {
        // loads `consumed` and `consumed + 1` in flight; load j reuses the stage
        // of load j - 2, so it waits until all warps have released that one
        while (p_item < a.n_items && issued < consumed + 2) {
            const uint32_t s = issued & 1u, u = issued >> 1;
            if (u >= 1) mbar_wait(&bar_empty[s], (u - 1) & 1u, err);
            const uint32_t bytes = (d - p_k0 < kc ? d - p_k0 : kc) * kPlainTile * 8u;
            mbar_arrive_expect_tx(&bar_full[s], bytes);
            bulk_g2s(sB[s], a.B + (uint64_t)p_bt * tile_elems + p_k0 * kPlainTile, bytes, &bar_full[s]);
            ++issued;
            if ((p_k0 += kc) < d) continue;
            p_k0 = 0;
            if (++p_bt >= p_end) {
                p_item += gridDim.x;
                if (p_item < a.n_items) {
                    WorkItem w = a.items[p_item];
                    p_bt = w.b0;
                    p_end = w.b1;
                }
            }
        }
    };
    if (tid == 0) issue_next(0);

    unsigned long long cnt = 0;
    uint32_t consumed = 0, a_phase = 0;
    const double T = a.T;
    for (uint64_t it = blockIdx.x; it < a.n_items; it += gridDim.x) {
        const WorkItem w = a.items[it];
        __syncthreads();  // all warps are done with the previous A tile
        if (tid == 0) {
            mbar_arrive_expect_tx(&bar_a, tile_elems * 8u);
            bulk_g2s(sA, a.A + (uint64_t)w.a * tile_elems, tile_elems * 8u, &bar_a);
        }
        mbar_wait(&bar_a, a_phase, err);
        a_phase ^= 1u;
        const uint64_t ia0 = (uint64_t)w.a * kPlainTile + ty * 4;
        for (uint32_t bt = w.b0; bt < w.b1; ++bt) {
            double acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
            bool live = true;  // some pair of this warp may still qualify
            for (uint32_t c0 = 0; c0 < d; c0 += kc) {
                const uint32_t s = consumed & 1u;
                if (tid == 0) issue_next(consumed);
                mbar_wait(&bar_full[s], (consumed >> 1) & 1u, err);
                const uint32_t c1 = c0 + kc < d ? c0 + kc : d;
                const double *pa = sA + ty * 4;
                const double *pb = sB[s] + tx * 4;
                for (uint32_t k = c0; live && k < c1;) {
                    const uint32_t kend = k + 8 <= c1 ? k + 8 : c1;
                    const double *pak = pa + k * kPlainTile, *pbk = pb + (k - c0) * kPlainTile;
                    if (kend - k == 8) {
#pragma unroll
                        for (int kk = 0; kk < 8; ++kk) fma_dim(pak + kk * kPlainTile, pbk + kk * kPlainTile, acc);
                    } else {
                        for (uint32_t kk = 0; kk < kend - k; ++kk) fma_dim(pak + kk * kPlainTile, pbk + kk * kPlainTile, acc);
                    }
                    k = kend;
                    if (k < d) {
                        bool any = false;
#pragma unroll
                        for (int i = 0; i < 4; ++i)
#pragma unroll
                            for (int j = 0; j < 4; ++j) any |= acc[i][j] <= T;
                        live = __any_sync(0xffffffffu, any);
                    }
                }
                // a warp that stopped early still waits for and releases every
                // chunk of this tile, so the stage sequence stays in step
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar_empty[s]);
                ++consumed;
            }
            const uint64_t jb0 = (uint64_t)bt * kPlainTile + tx * 4;
            uint32_t hits = 0;  // bit 4i+j: pair (i, j) of this thread's block qualifies
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const uint64_t pi = ia0 + i, pj = jb0 + j;
                    const bool valid = pi < a.na && pj < a.nb && (!a.self || pj > pi);
                    hits |= (valid && acc[i][j] <= T) ? 1u << (4 * i + j) : 0u;
                }
            const uint32_t nh = __popc(hits);
            if (MODE != kModeEmit) {
                cnt += nh;
            } else if (__any_sync(0xffffffffu, nh != 0)) {
                uint32_t incl = nh;  // inclusive warp prefix sum of the hit counts
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= (uint32_t)o) incl += v;
                }
                const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(a.item_cnt + it, total);
                base = __shfl_sync(0xffffffffu, base, 0) + incl - nh;
                while (hits) {
                    const int b = __ffs(hits) - 1;
                    hits &= hits - 1;
                    const uint32_t ri = (uint32_t)(ia0 + (b >> 2)), rj = (uint32_t)(jb0 + (b & 3));
                    uint32_t gi = a.perm_a[ri], gj = a.perm_b[rj];
                    if (a.self && gi > gj) {
                        const uint32_t t = gi;
                        gi = gj;
                        gj = t;
                    }
                    a.out_i[base] = gi;
                    a.out_j[base] = gj;
                    ++base;
                }
            }
        }
        if (MODE == kModeItemCounts) {
            const unsigned long long wc = warp_sum_u64(cnt);
            if (lane == 0 && wc) atomicAdd(a.item_cnt + it, (uint32_t)wc);
            cnt = 0;
        }
    }
    if (MODE == kModeCount) {
        cnt = warp_sum_u64(cnt);
        if (lane == 0 && cnt) atomicAdd(a.count, cnt);
    }
    // Every issued copy has been consumed unless a wait gave up; then drain.
    if (tid == 0 && *err != 0) {
        for (uint32_t j = consumed; j < issued; ++j) drain_wait(&bar_full[j & 1u], (j >> 1) & 1u);
    }
}

template <int MODE>
static void launch_plain(const PlainArgs &a, uint64_t n_items, int num_sms, cudaStream_t st) {
    const size_t smem = plain_smem_bytes(a.d);
    // the largest this kernel ever needs (d = 128 and d = 256 both take 192 KB), set once
    static_assert(plain_smem_bytes(128) == plain_smem_bytes(kPlainMaxDims), "plain smem maximum");
    ensure_max_dynamic_smem((const void *)k_join_fp64<MODE>, (int)plain_smem_bytes(kPlainMaxDims));
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_join_fp64<MODE>, kPlainThreads, smem);
    if (per_sm < 1) per_sm = 1;
    uint64_t grid = (uint64_t)per_sm * num_sms;
    if (grid > n_items) grid = n_items;
    k_join_fp64<MODE><<<(unsigned)grid, kPlainThreads, smem, st>>>(a);
}

static PlainArgs plain_args(const SortedSet &A, const SortedSet &B, bool self, uint64_t na_eff, uint64_t nb_eff,
                            double T, const IndexResult &idx, uint32_t *d_err) {
    PlainArgs a;
    memset(&a, 0, sizeof(a));
    a.A = A.tiles64;
    a.B = B.tiles64;
    a.d = A.d;
    a.T = T;
    a.items = idx.items;
    a.n_items = idx.n_items;
    a.na = na_eff;
    a.nb = nb_eff;
    a.self = self ? 1 : 0;
    a.err = d_err;
    return a;
}

void launch_join_fp64(const SortedSet &A, const SortedSet &B, bool self, uint64_t na_eff, uint64_t nb_eff,
                      double T, const IndexResult &idx, unsigned long long *d_count, uint32_t *d_err, int num_sms,
                      cudaStream_t st) {
    if (idx.n_items == 0) return;
    PlainArgs a = plain_args(A, B, self, na_eff, nb_eff, T, idx, d_err);
    a.count = d_count;
    launch_plain<kModeCount>(a, idx.n_items, num_sms, st);
}

void launch_pairs_fp64(const SortedSet &A, const SortedSet &B, bool self, uint64_t na_eff, uint64_t nb_eff,
                       double T, const IndexResult &idx, uint32_t *item_cnt, uint32_t *out_i, uint32_t *out_j,
                       uint32_t *d_err, int num_sms, cudaStream_t st) {
    if (idx.n_items == 0) return;
    PlainArgs a = plain_args(A, B, self, na_eff, nb_eff, T, idx, d_err);
    a.item_cnt = item_cnt;
    a.perm_a = A.perm;
    a.perm_b = B.perm;
    a.out_i = out_i;
    a.out_j = out_j;
    if (out_i)
        launch_plain<kModeEmit>(a, idx.n_items, num_sms, st);
    else
        launch_plain<kModeItemCounts>(a, idx.n_items, num_sms, st);
}

}  // namespace hj
