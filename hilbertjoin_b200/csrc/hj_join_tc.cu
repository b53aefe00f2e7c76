// hj_join_tc.cu -- tensor-core forms (HJ_FORM_TC_TF32, HJ_FORM_TC_BF16X3, HJ_FORM_TC_FP16).
//
// Replaces the same block-pair kernel as hj_join_fp64.cu (the reference's
// EGO_LOOP_TRAN[_NOSELF], hilbertjoin/egojoin.h:311-392, :482-553), but with
// the norm expansion the reference itself uses,
//     |a - b|^2 = |a|^2 + |b|^2 - 2 a.b      (egojoin.h:182-195, :329-381),
// and the a.b tile on the 5th-generation tensor cores:
//
//   * one persistent CTA per SM, 6 warps, warp-specialised:
//       warp 0   TMA producer: the A tile (128 EGO ranks x K) once per work
//                item into one of two A buffers, then the B tiles (256 ranks)
//                one 128-byte K atom (32 KB) at a time into a ring of stages;
//       warp 1   MMA issuer (one thread): tcgen05.mma, M=128, N=256, operands
//                from shared memory (128-byte swizzled, K-major), accumulator
//                in tensor memory, two accumulators in flight (512 columns);
//       warps 2-9 epilogue: tcgen05.ld of the accumulator rows (TMEM lane
//                quadrant = warp % 4, two warps per quadrant on 128 columns
//                each), dist^2 estimate, classification, count;
//   * TF32: operands rounded to TF32 on the device (round to nearest), one
//     MMA per K step; BF16X3: a = a_hi + a_lo in BF16, a.b =
//     a_hi.b_hi + a_lo.b_hi + a_hi.b_lo (three MMAs per K step); FP16: the
//     operands scaled by a power of two into FP16's range and rounded once
//     (the precision of TF32 at twice its MMA rate), one MMA per K step, the
//     norms, eps^2 and the bound in the same scaled units;
//   * exact count: with s = |a|^2 + |b|^2 - 2 v (v the tensor-core dot product),
//     every error of v, of the FP32 norms and of the FP32 epilogue is bounded
//     by c_rel * (|a|^2 + |b|^2) + c_abs (tc_band_constants). A pair with
//     s + bound <= eps^2 is certainly inside, one with s - bound > eps^2 is
//     certainly outside, and every other pair (the band) is queued and
//     re-evaluated by k_recheck with the FP64 pair test. So the count equals
//     the plain FP64 form's, bit for bit.
//   * fast path: per row and 32-column half the epilogue takes the minimum of
//     |b|^2 - 2 v; only if that can still reach eps^2 + bound (rare: neighbours
//     are a small fraction of the candidates) does the warp classify the half,
//     branch-free against per-tile bounds, and queue the band pairs.
//
// Every mbarrier wait is bounded in time (hj_common.cuh); on a timeout the
// kernel raises kErrTimeout (with the number of the wait that gave up in bits
// 8..15 of the error word), every role stops at its next wait, the copies and
// MMAs already issued are drained, the tensor memory is freed and the kernel
// returns. hj_debug_set_wait_gate makes the epilogue's first wait one that
// nothing ends, so that tests run this path.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <type_traits>

#include "../../include/hj.h"
#include "hj_common.cuh"
#include "hj_internal.h"

namespace hj {

// Epilogue warps: kEpiWarps / 4 per TMEM lane quadrant, each on kEpiCols of the
// 256 accumulator columns, in two chunks of kChunkCols (one TMEM load each).
constexpr int kEpiWarps = 8;
constexpr int kEpiCols = 4 * kTcTileB / kEpiWarps;
// 8 warps: two 64-column chunks each; 16 warps: one 64-column chunk each
constexpr int kChunkCols = 64;
constexpr int kChunkGroups = kChunkCols / 32;  // 32-column groups per chunk
constexpr int kEpiChunks = kEpiCols / kChunkCols;
constexpr int kEpiVec = kEpiCols / 32;  // norms per lane, group minima per warp
// Block centring, where tiles in which near pairs are common make up much of
// the work: the lanes classify their own rows against a 32-column group (the
// dense path) instead of the warp walking row by row, and band slots are
// reserved by each epilogue warp in chunks (one atomic per chunk); slots a
// warp leaves unused are marked with ia = kBandHole. With one global centre
// (near pairs rare) both measured slower, the row walk with one atomic per
// band pair stays.
constexpr uint32_t kBandChunk = 256;
constexpr uint32_t kBandHole = 0xffffffffu;
// 16 epilogue warps (4 per quadrant) were measured slower: at 18 warps the
// register cap is 96 (spills) and the static shared memory no longer fits next
// to the 225 KB operand plan.
static_assert(kEpiWarps == 8, "the shared-memory plan and register budget assume 8 epilogue warps");
constexpr int kTcThreads = 64 + 32 * kEpiWarps;
constexpr uint32_t kAtomBytes = 128;                  // bytes of K per row per swizzle atom
constexpr uint32_t kAStageBytes = kTcTileA * kAtomBytes;  // 16 KB per A atom
constexpr uint32_t kBStageBytes = kTcTileB * kAtomBytes;  // 32 KB per B atom
constexpr uint32_t kTmemCols = 512;

struct BandEntry {
    uint32_t ia, jb;  // EGO ranks in A and B
    float s_hat;      // tensor-core estimate of dist^2
    uint32_t pad;
};

struct TcArgs {
    uint32_t ka;        // K atoms per operand buffer, the largest of the jobs' (TF32: kpad/32; BF16, FP16: kpad16/64)
                        // (each job multiplies only its own ksteps)
    uint32_t a_bufs;    // 1 or 2 A buffers
    uint32_t nst;       // B ring stages
    const WorkItem *items;
    uint64_t n_items;
    const float *norm_a, *norm_b;   // FP32 |x|^2 per EGO rank (padding: kPadNorm)
    const float *tmax_b;            // per 256-rank B tile: max |x|^2
    const float *gmin_b;            // per 32-rank B group: min |x|^2
    const TcJob *jobs;              // per job: counted rows, thresholds, count (item.pad = job)
    uint64_t na, nb;                // job 0's counted ranks (debug output only)
    BandEntry *band;
    uint64_t band_cap;
    unsigned long long *band_total;  // slots reserved (chunks of kBandChunk per warp)
    unsigned long long *band_holes;  // reserved slots left unused (marked kBandHole); may be null
    uint32_t *err;
    float *dbg;                     // optional: s_hat for every pair, input order [na][nb] (tests)
    const uint32_t *perm_a, *perm_b;  // EGO rank -> input index (for dbg)
    uint32_t a_xoff;                // first column of the A operand in its rows (block centring: dp)
    uint64_t gate_ns;               // test hook: > 0 makes the epilogue wait this long on a barrier
                                    // that nothing arrives on, then raise kErrTimeout
    // per-block centring (BC kernels): norm_a is then q of the A rows (norm_b and
    // gmin_b unused: the accumulator holds w = v - q_j / 2); |h| of the A rows,
    // block summaries and centres of both sets
    const float *xn_a;
    const float4 *blk_a, *blk_b;
    const float *cent_a, *cent_b;
    BcConsts bc;
};

// ---------------------------------------------------------------- PTX helpers

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

template <int FORM>
__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    if constexpr (FORM == HJ_FORM_TC_TF32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
            : "memory");
    }
}

// 64 consecutive accumulator columns of this thread's TMEM lane (two x32
// loads, one wait).
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
    uint32_t r[64];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
            "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(r[32 * h + 0]), "=r"(r[32 * h + 1]), "=r"(r[32 * h + 2]), "=r"(r[32 * h + 3]),
              "=r"(r[32 * h + 4]), "=r"(r[32 * h + 5]), "=r"(r[32 * h + 6]), "=r"(r[32 * h + 7]),
              "=r"(r[32 * h + 8]), "=r"(r[32 * h + 9]), "=r"(r[32 * h + 10]), "=r"(r[32 * h + 11]),
              "=r"(r[32 * h + 12]), "=r"(r[32 * h + 13]), "=r"(r[32 * h + 14]), "=r"(r[32 * h + 15]),
              "=r"(r[32 * h + 16]), "=r"(r[32 * h + 17]), "=r"(r[32 * h + 18]), "=r"(r[32 * h + 19]),
              "=r"(r[32 * h + 20]), "=r"(r[32 * h + 21]), "=r"(r[32 * h + 22]), "=r"(r[32 * h + 23]),
              "=r"(r[32 * h + 24]), "=r"(r[32 * h + 25]), "=r"(r[32 * h + 26]), "=r"(r[32 * h + 27]),
              "=r"(r[32 * h + 28]), "=r"(r[32 * h + 29]), "=r"(r[32 * h + 30]), "=r"(r[32 * h + 31])
            : "r"(taddr + 32 * h));
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// max(a, b, c) in one instruction (three-input max.f32, sm_100).
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Shared-memory matrix descriptor: K-major operand in 128-byte swizzle atoms
// (8 rows x 128 B, atoms stacked along M/N every 1024 B).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: D = F32, A/B K-major, M = 128, N = 256.
template <int FORM>
__device__ __forceinline__ constexpr uint32_t instr_desc() {
    constexpr uint32_t ab = FORM == HJ_FORM_TC_TF32 ? 2u : (FORM == HJ_FORM_TC_BF16X3 ? 1u : 0u);  // TF32, BF16, F16
    return (1u << 4) | (ab << 7) | (ab << 10) | ((uint32_t)(kTcTileB >> 3) << 17) | ((uint32_t)(kTcTileA >> 4) << 24);
}

// Waits for a phase regardless of the error word, until `deadline`
// (%globaltimer): the drain of copies and MMAs already issued.
__device__ __forceinline__ void drain_until(uint64_t *bar, uint32_t parity, uint64_t deadline) {
    while (!mbar_try_wait(bar, parity)) {
        if (globaltimer_ns() > deadline) break;
    }
}

// ---------------------------------------------------------------- the kernel

template <int FORM, bool BC>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_join_tc(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_a2,
              const __grid_constant__ CUtensorMap tm_b, const __grid_constant__ CUtensorMap tm_b2, TcArgs p) {
    // A atoms per buffer: TF32 ka; BF16 2*ka (hi atoms, then lo atoms). B atoms
    // per tile, in ring order: TF32 q = 0..ka-1; BF16 (hi q, lo q) for each q.
    constexpr bool kBf = FORM == HJ_FORM_TC_BF16X3;
    constexpr int32_t kAtomElems = FORM == HJ_FORM_TC_TF32 ? 32 : 64;  // K elements per 128-byte atom
    const uint32_t a_atoms = kBf ? 2 * p.ka : p.ka;
    const uint32_t a_buf_bytes = a_atoms * kAStageBytes;

    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t bar_afull[2], bar_aempty[2], bar_accfull[2], bar_accempty[2], bar_drain, bar_gate;
    __shared__ __align__(8) uint64_t bar_bfull[8], bar_bempty[8];
    __shared__ uint32_t tmem_base_sh;
    __shared__ __align__(16) float epi_row[kEpiWarps][32];

    const uint32_t smem_base = (smem_u32(smem_raw) + 1023u) & ~1023u;
    const uint32_t a_base = smem_base;
    const uint32_t b_base = smem_base + p.a_bufs * a_buf_bytes;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    volatile uint32_t *err = p.err;

    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(&bar_afull[i], 1);
            mbar_init(&bar_aempty[i], 1);
            mbar_init(&bar_accfull[i], 1);
            mbar_init(&bar_accempty[i], kEpiWarps);
        }
        for (uint32_t i = 0; i < p.nst; ++i) {
            mbar_init(&bar_bfull[i], 1);
            mbar_init(&bar_bempty[i], 1);
        }
        mbar_init(&bar_drain, 1);
        mbar_init(&bar_gate, 1);
        fence_barrier_init();
    }
    if (warp == 0) {
        tmem_alloc(&tmem_base_sh, kTmemCols);
        if (lane == 0) {
            prefetch_tmap(&tm_a);
            prefetch_tmap(&tm_b);
            if (kBf) {
                prefetch_tmap(&tm_a2);
                prefetch_tmap(&tm_b2);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t a_cnt = 0, b_cnt = 0;
            bool ok = true;
            for (uint64_t it = blockIdx.x; ok && it < p.n_items; it += gridDim.x) {
                const WorkItem w = p.items[it];
                const uint32_t ka = p.jobs[w.pad].ka;  // this job's K atoms (<= p.ka)
                const uint32_t ja_atoms = kBf ? 2 * ka : ka;
                const uint32_t abuf = a_cnt % p.a_bufs, au = a_cnt / p.a_bufs;
                if (au >= 1 && !mbar_wait(&bar_aempty[abuf], (au - 1) & 1u, err, 1)) break;
                mbar_arrive_expect_tx(&bar_afull[abuf], ja_atoms * kAStageBytes);
                const uint32_t adst = a_base + abuf * a_buf_bytes;
                for (uint32_t q = 0; q < ja_atoms; ++q) {
                    const bool lo = kBf && q >= ka;
                    const uint32_t kq = kBf ? (lo ? q - ka : q) : q;
                    tma_load_2d(smem_raw + (adst + q * kAStageBytes - smem_u32(smem_raw)), lo ? &tm_a2 : &tm_a,
                                (int32_t)(kq * kAtomElems + p.a_xoff), (int32_t)(w.a * kTcTileA), &bar_afull[abuf]);
                }
                ++a_cnt;
                for (uint32_t bt = w.b0; ok && bt < w.b1; ++bt) {
                    for (uint32_t q = 0; q < ja_atoms; ++q) {
                        const uint32_t s = b_cnt % p.nst, u = b_cnt / p.nst;
                        if (u >= 1 && !mbar_wait(&bar_bempty[s], (u - 1) & 1u, err, 2)) {
                            ok = false;
                            break;
                        }
                        mbar_arrive_expect_tx(&bar_bfull[s], kBStageBytes);
                        const bool lo = kBf && (q & 1u);
                        const uint32_t kq = kBf ? (q >> 1) : q;
                        tma_load_2d(smem_raw + (b_base + s * kBStageBytes - smem_u32(smem_raw)), lo ? &tm_b2 : &tm_b,
                                    (int32_t)(kq * kAtomElems), (int32_t)(bt * kTcTileB), &bar_bfull[s]);
                        ++b_cnt;
                    }
                }
            }
            // Drain: on the normal path every copy has been consumed; after an
            // error (the loops stop at the first failed wait) every copy issued
            // has landed before the CTA leaves (its full barrier's phase).
            if (*err) {
                const uint64_t deadline = globaltimer_ns() + kWaitLimitNs;
                for (uint32_t k = 0; k < p.nst && k < b_cnt; ++k) {
                    const uint32_t j = b_cnt - 1 - k;
                    drain_until(&bar_bfull[j % p.nst], (j / p.nst) & 1u, deadline);
                }
                for (uint32_t k = 0; k < p.a_bufs && k < a_cnt; ++k) {
                    const uint32_t j = a_cnt - 1 - k;
                    drain_until(&bar_afull[j % p.a_bufs], (j / p.a_bufs) & 1u, deadline);
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            constexpr uint32_t idesc = instr_desc<FORM>();
            uint32_t a_cnt = 0, b_cnt = 0, t_cnt = 0;
            bool issued_any = false, ok = true;
            for (uint64_t it = blockIdx.x; ok && it < p.n_items; it += gridDim.x) {
                const WorkItem w = p.items[it];
                const uint32_t ka = p.jobs[w.pad].ka, ksteps = p.jobs[w.pad].ksteps;
                const uint32_t jb_atoms = kBf ? 2 * ka : ka;
                const uint32_t abuf = a_cnt % p.a_bufs, au = a_cnt / p.a_bufs;
                if (!mbar_wait(&bar_afull[abuf], au & 1u, err, 3)) break;
                tc_fence_after();
                const uint32_t abase = a_base + abuf * a_buf_bytes;
                for (uint32_t bt = w.b0; ok && bt < w.b1; ++bt) {
                    const uint32_t acc = t_cnt & 1u, tu = t_cnt >> 1;
                    if (tu >= 1 && !mbar_wait(&bar_accempty[acc], (tu - 1) & 1u, err, 4)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t dcol = tmem + acc * kTcTileB;
                    uint32_t accumulate = 0;
                    for (uint32_t q = 0; q < jb_atoms; ++q) {
                        const uint32_t s = b_cnt % p.nst;
                        if (!mbar_wait(&bar_bfull[s], (b_cnt / p.nst) & 1u, err, 5)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t bsm = b_base + s * kBStageBytes;
                        if constexpr (!kBf) {
                            const uint32_t asm_ = abase + q * kAStageBytes;
                            // 4 K steps per atom, fewer in the last (zero columns not multiplied)
                            const uint32_t kk_end = ksteps - 4 * q < 4 ? ksteps - 4 * q : 4;
                            if (kk_end == 4) {
#pragma unroll
                                for (uint32_t kk = 0; kk < 4; ++kk) {
                                    mma_issue<FORM>(dcol, sw128_desc(asm_ + kk * 32), sw128_desc(bsm + kk * 32), idesc,
                                                    accumulate);
                                    accumulate = 1;
                                }
                            } else {
#pragma unroll
                                for (uint32_t kk = 0; kk < 3; ++kk) {
                                    if (kk < kk_end) {
                                        mma_issue<FORM>(dcol, sw128_desc(asm_ + kk * 32), sw128_desc(bsm + kk * 32),
                                                        idesc, accumulate);
                                        accumulate = 1;
                                    }
                                }
                            }
                        } else {
                            const uint32_t kq = q >> 1;
                            const uint32_t kk_end = ksteps - 4 * kq < 4 ? ksteps - 4 * kq : 4;
                            const uint32_t a_hi = abase + kq * kAStageBytes;
                            const uint32_t a_lo = abase + (ka + kq) * kAStageBytes;
                            if ((q & 1u) == 0) {  // B_hi atom: A_hi.B_hi + A_lo.B_hi
#pragma unroll
                                for (uint32_t kk = 0; kk < 4; ++kk) {
                                    if (kk >= kk_end) break;
                                    mma_issue<FORM>(dcol, sw128_desc(a_hi + kk * 32), sw128_desc(bsm + kk * 32),
                                                    idesc, accumulate);
                                    accumulate = 1;
                                    mma_issue<FORM>(dcol, sw128_desc(a_lo + kk * 32), sw128_desc(bsm + kk * 32),
                                                    idesc, 1);
                                }
                            } else {  // B_lo atom: A_hi.B_lo
#pragma unroll
                                for (uint32_t kk = 0; kk < 4; ++kk)
                                    if (kk < kk_end)
                                        mma_issue<FORM>(dcol, sw128_desc(a_hi + kk * 32), sw128_desc(bsm + kk * 32),
                                                        idesc, 1);
                            }
                        }
                        mma_commit(&bar_bempty[s]);  // stage free once these MMAs have read it
                        ++b_cnt;
                        issued_any = true;
                    }
                    if (!ok) break;
                    mma_commit(&bar_accfull[acc]);
                    ++t_cnt;
                }
                mma_commit(&bar_aempty[abuf]);
                ++a_cnt;
            }
            // all MMAs complete before the tensor memory is released
            if (issued_any) {
                mma_commit(&bar_drain);
                drain_until(&bar_drain, 0, globaltimer_ns() + kWaitLimitNs);
            }
        }
    } else {
        // ------------------------------------------------ epilogue
        const uint32_t quad = warp & 3u;
        const uint32_t half = (warp - 2) >> 2;  // columns [kEpiCols half, kEpiCols (half + 1))
        const uint32_t lane_base = (quad * 32u) << 16;
        float *srow = epi_row[warp - 2];
        unsigned long long cnt = 0;
        uint32_t t_cnt = 0;
        bool run = true;
        if (p.gate_ns) {  // test hook: a wait that nothing ends
            const uint64_t t0 = globaltimer_ns();
            while (!mbar_try_wait(&bar_gate, 0)) {
                if (globaltimer_ns() - t0 > p.gate_ns) {
                    atomicOr((uint32_t *)err, kErrTimeout | (9u << 8));
                    break;
                }
            }
            run = false;
        }
        // All classification is in FP32 with eps^2 rounded outward (T_lo, T_hi)
        // and the bound rounded up; the FP32 rounding of the epilogue itself is
        // part of c_rel. A pair is inside if s + tau <= T_lo, outside if
        // s - tau > T_hi, and in the band otherwise.
        // Walk over (item, B tile). Per item: this lane's row (A rank), its norm
        // and the classification thresholds, taken against the largest B-tile
        // norm of the item (a band at least as wide as any tile's: still
        // exact). Per tile only the group minima are needed on the fast path;
        // they are loaded one tile ahead so that their latency overlaps the
        // current tile. B norms and column bounds are read on the slow path.
        const uint64_t stride = gridDim.x;
        uint64_t it = run ? blockIdx.x : p.n_items;
        WorkItem w = it < p.n_items ? p.items[it] : WorkItem{0, 0, 0, 0};
        WorkItem wn = it + stride < p.n_items ? p.items[it + stride] : WorkItem{0, 0, 0, 0};
        uint32_t bt = w.b0;
        // per-block centring: the row's p, |h| and |p|, its block's |c| and centre
        // coordinates (lane, lane + 32), the job's eps^2 bounds; per tile the B
        // block's summary and centre, prefetched one tile ahead with the minima
        float p_row = 0.f, xa = 0.f, pa = 0.f, cna = 0.f, t_lo = 0.f, t_hi = 0.f;
        float ca[2] = {0.f, 0.f}, pf_cb[2] = {0.f, 0.f};
        float4 pf_blk = make_float4(0.f, 0.f, 0.f, 0.f);
        float pf_gmin[kEpiVec];
        auto prefetch = [&](uint32_t b) {
            const uint64_t g = (uint64_t)b * kTcTileB + half * kEpiCols;
            if constexpr (!BC) {
                const float4 m = __ldg(reinterpret_cast<const float4 *>(p.gmin_b + g / 32));
                pf_gmin[0] = m.x, pf_gmin[1] = m.y, pf_gmin[2] = m.z, pf_gmin[3] = m.w;
            } else {
                const uint64_t blkb = g / kBcBlock;
                pf_blk = __ldg(p.blk_b + blkb);
                pf_cb[0] = __ldg(p.cent_b + blkb * kBcCentStride + lane);
                pf_cb[1] = __ldg(p.cent_b + blkb * kBcCentStride + 32 + lane);
            }
        };
#pragma unroll
        for (int q = 0; q < kEpiVec; ++q) pf_gmin[q] = 0.f;
        if (it < p.n_items) prefetch(bt);
        // per-item row state, and the job whose count the warp is accumulating
        uint64_t gi = 0, b_end = 0;
        bool row_ok = false, self = false;
        float na = kPadNorm, thr_out = -3.0e38f, thr_in = -3.0e38f, s_unscale = 1.f;
        uint32_t job = 0xffffffffu;
        auto flush = [&]() {
            const unsigned long long wc = warp_sum_u64(cnt);
            if (lane == 0 && wc) atomicAdd(p.jobs[job].count, wc);
            cnt = 0;
        };
        // the warp's current chunk of band slots [bslot, bend) (warp-uniform);
        // slot of the entry of rank `rank` among `c` <= 32 new entries
        unsigned long long bslot = 0, bend = 0;
        // the unused rest of the warp's chunk: marked for the recheck to skip
        auto band_holes = [&]() {
            for (unsigned long long k = bslot + lane; k < bend; k += 32)
                if (k < p.band_cap) {
                    BandEntry e;
                    e.ia = kBandHole;
                    e.jb = 0;
                    e.s_hat = 0.f;
                    e.pad = 0;
                    p.band[k] = e;
                }
            if (lane == 0 && bend > bslot && p.band_holes) atomicAdd(p.band_holes, bend - bslot);
            bslot = bend;
        };
        // c new slots (warp-uniform c): the rest of the warp's chunk first, then a
        // new chunk of max(kBandChunk, the remainder); the slot of rank r is
        // r < rem ? k0 + r : nb + (r - rem)
        struct BandSlots {
            unsigned long long k0, nb;
            uint32_t rem;
            __device__ unsigned long long at(uint32_t r) const { return r < rem ? k0 + r : nb + (r - rem); }
        };
        auto band_reserve = [&](uint32_t c) -> BandSlots {
            BandSlots b{bslot, 0, (uint32_t)(bend - bslot)};
            if (c <= b.rem) {
                bslot += c;
                return b;
            }
            const uint32_t need = c - b.rem, size = need > kBandChunk ? need : kBandChunk;
            unsigned long long nb = 0;
            if (lane == 0) nb = atomicAdd(p.band_total, (unsigned long long)size);
            b.nb = __shfl_sync(0xffffffffu, nb, 0);
            bslot = b.nb + need;
            bend = b.nb + size;
            return b;
        };
        auto item_rows = [&](const WorkItem &ww) {
            if (ww.pad != job) {
                if (job != 0xffffffffu) flush();
                job = ww.pad;
            }
            const TcJob &J = p.jobs[job];
            const float T_lo = J.T_lo, T_hi = J.T_hi, crel = J.c_rel_f, cabs = J.c_abs_f;
            b_end = J.b_end;
            self = J.self != 0;
            s_unscale = J.s_unscale;
            gi = (uint64_t)ww.a * kTcTileA + quad * 32 + lane;
            row_ok = gi >= J.a_row0 && gi < J.a_end;
            if constexpr (BC) {
                // thresholds per tile (they depend on the B block): see the tile loop
                p_row = row_ok ? __ldg(p.norm_a + gi) : 0.f;
                xa = row_ok ? __ldg(p.xn_a + gi) : 0.f;
                pa = fabsf(p_row);
                const uint64_t blka = (uint64_t)ww.a * kTcTileA / kBcBlock;
                cna = __ldg(&p.blk_a[blka].y);
                ca[0] = __ldg(p.cent_a + blka * kBcCentStride + lane);
                ca[1] = __ldg(p.cent_a + blka * kBcCentStride + 32 + lane);
                t_lo = T_lo;
                t_hi = T_hi;
                na = p_row;
                thr_out = thr_in = -3.0e38f;
                (void)crel;
                (void)cabs;
                return;
            }
            na = row_ok ? __ldg(p.norm_a + gi) : kPadNorm;
            float tmaxb = 0.f;
            for (uint32_t b = ww.b0 + lane; b < ww.b1; b += 32) tmaxb = fmaxf(tmaxb, __ldg(p.tmax_b + b));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) tmaxb = fmaxf(tmaxb, __shfl_xor_sync(0xffffffffu, tmaxb, o));
            // With tau_max = c_rel (|a|^2 + max |b|^2) + c_abs >= tau of every pair
            // of the item, and t_j = |b_j|^2 - 2 v_j, s_j = |a|^2 + t_j:
            //   t_j <= thr_in  => s_j + tau <= eps^2  (certainly inside),
            //   t_j >  thr_out => s_j - tau >  eps^2  (certainly outside),
            // anything between is a band pair. Both thresholds carry margins
            // for their own FP32 rounding (rounded inward / outward).
            const float tau_max = fmaf(crel, na + tmaxb, cabs) * 1.001f;
            const float marg = 8.0f * 5.9604645e-8f * (fabsf(T_hi) + fabsf(na) + tmaxb + tau_max);
            thr_out = (T_hi + tau_max) - na + marg;
            thr_in = (T_lo - tau_max) - na - marg;
            if (!row_ok) thr_out = thr_in = -3.0e38f;
        };
        if (it < p.n_items) item_rows(w);
        while (it < p.n_items) {
            float gmin[kEpiVec];
#pragma unroll
            for (int q = 0; q < kEpiVec; ++q) gmin[q] = pf_gmin[q];
            if constexpr (BC) {
                // this tile's B block: D = |c_A - c_B|^2 (FP32, lanes over the
                // dims), the band half-width of the lane's row against the block,
                // and the thresholds on t = -2 w (s = q_row + D + t; |w| <= S)
                float D = 0.f;
#pragma unroll
                for (int m = 0; m < 2; ++m) {
                    const float df = ca[m] - pf_cb[m];
                    D = fmaf(df, df, D);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) D += __shfl_xor_sync(0xffffffffu, D, o);
                float S;
                const float tau = bc_tau(xa, cna, pa, pf_blk.x, pf_blk.y, pf_blk.z, D, p.bc, &S);
                const float marg = 8.0f * 5.9604645e-8f * (fabsf(t_hi) + pa + pf_blk.z + D + tau + 2.0f * S);
                na = p_row + D;
                thr_out = row_ok ? (t_hi + tau) - p_row - D + marg : -3.0e38f;
                thr_in = row_ok ? (t_lo - tau) - p_row - D - marg : -3.0e38f;
            }
            const uint32_t cur_bt = bt;
            // the item's rows stay for its last tile; the next item's are set after it
            const bool last_tile = bt + 1 >= w.b1;
            if (!last_tile) {
                ++bt;
            } else {
                it += stride;
                w = wn;
                bt = w.b0;
                wn = it + stride < p.n_items ? p.items[it + stride] : WorkItem{0, 0, 0, 0};
            }
            if (it < p.n_items) prefetch(bt);
            {
                const uint32_t acc = t_cnt & 1u;
                const uint64_t gj0 = (uint64_t)cur_bt * kTcTileB + half * kEpiCols;
                if (!mbar_wait(&bar_accfull[acc], (t_cnt >> 1) & 1u, err, 6)) break;
                tc_fence_after();
#pragma unroll
                for (uint32_t c = 0; c < kEpiChunks; ++c) {
                    float v[kChunkCols];
                    const uint32_t taddr = tmem + lane_base + acc * kTcTileB + half * kEpiCols + c * kChunkCols;
                    tmem_ld64(taddr, v);
                    if (c + 1 == kEpiChunks) {
                        // the last chunk is in registers (its slow path too works from
                        // them): the accumulator goes back to the MMA warp before the
                        // chunk is classified
                        tc_fence_before();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&bar_accempty[acc]);
                    }
                    // max_j v_j per 32-column group: with the group's minimum norm,
                    // min_j (|b_j|^2 - 2 v_j) >= gmin - 2 max_j v_j
                    float mg[kChunkGroups];
#pragma unroll
                    for (int g = 0; g < kChunkGroups; ++g) {
                        // 16 three-input maxima in a tree of depth 4 (10 + 4 + 1, then one
                        // two-input max) for the group's 32 values
                        const float *vg = v + 32 * g;
                        float t[10];
#pragma unroll
                        for (int i = 0; i < 10; ++i) t[i] = fmax3(vg[3 * i], vg[3 * i + 1], vg[3 * i + 2]);
                        const float u0 = fmax3(t[0], t[1], t[2]), u1 = fmax3(t[3], t[4], t[5]);
                        const float u2 = fmax3(t[6], t[7], t[8]), u3 = fmax3(t[9], vg[30], vg[31]);
                        mg[g] = fmaf(-2.0f, fmaxf(fmax3(u0, u1, u2), u3), gmin[c * kChunkGroups + g]);
                    }
#pragma unroll
                    for (int h2 = 0; h2 < kChunkGroups; ++h2) {
                        // Rare: a 32-column half of some rows of the warp may hold a
                        // pair that is not certainly outside. For each such row the
                        // owning lane publishes its 32 values through shared memory
                        // and the whole warp classifies the 32 columns at once (lane
                        // = column), branch-free; band pairs are queued.
                        const bool need = mg[h2] <= thr_out || (p.dbg != nullptr && row_ok);
                        uint32_t rows = __ballot_sync(0xffffffffu, need);
                        if (!rows) continue;
                        const int cb = (int)(c * kChunkCols + h2 * 32);
                        // the column's |b|^2 (block centring: 0, q_j / 2 is in the accumulator)
                        const float nbl = BC ? 0.f : __ldg(p.norm_b + gj0 + cb + lane);
                        // columns that may be counted at all: gj < nb, and gj > gi for a self-join
                        int jlo = 0, jhi = kEpiCols;
                        {
                            const int64_t lim = (int64_t)b_end - (int64_t)gj0;
                            jhi = lim < kEpiCols ? (lim < 0 ? 0 : (int)lim) : kEpiCols;
                            if (self) {
                                const int64_t first = (int64_t)gi + 1 - (int64_t)gj0;
                                jlo = first > 0 ? (first > kEpiCols ? kEpiCols : (int)first) : 0;
                            }
                        }
                        if constexpr (BC) {
                            if (p.dbg == nullptr) {
                                // Dense path: every lane classifies its own row against the
                                // group's 32 columns (the column norm is in the accumulator);
                                // band entries straight from the lane's registers: ranks by a
                                // warp prefix sum, slots from one warp-wide reservation
                                // t = -2 w, so t <= thr  <=>  w >= -thr / 2 (exact scaling);
                                // the columns the row may count form one mask per group
                                const float *vg = v + h2 * 32;
                                const float w_in = -0.5f * thr_in, w_out = -0.5f * thr_out;
                                const int lo = jlo - cb > 0 ? jlo - cb : 0, hi = jhi - cb < 32 ? jhi - cb : 32;
                                const uint32_t colmask =
                                    (need && row_ok && lo < hi)
                                        ? ((hi >= 32 ? 0xffffffffu : (1u << hi) - 1u) & ~((1u << lo) - 1u))
                                        : 0u;
                                uint32_t g_in = 0, g_out = 0;
#pragma unroll
                                for (int j = 0; j < 32; ++j) {
                                    g_in |= vg[j] >= w_in ? (1u << j) : 0u;
                                    g_out |= vg[j] >= w_out ? (1u << j) : 0u;
                                }
                                g_in &= colmask;
                                uint32_t bbits = g_out & colmask & ~g_in;
                                cnt += __popc(g_in);
                                const uint32_t nbits = __popc(bbits);
                                uint32_t incl = nbits;
#pragma unroll
                                for (int o = 1; o < 32; o <<= 1) {
                                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                                    if (lane >= (uint32_t)o) incl += y;
                                }
                                const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
                                if (total) {
                                    // the estimate is not kept here (reading it back by column
                                    // index would take the values out of registers): NaN, which
                                    // the recheck's error statistic skips
                                    const BandSlots sl = band_reserve(total);
                                    uint32_t rank = incl - nbits;
                                    while (bbits) {
                                        const int j = __ffs(bbits) - 1;
                                        bbits &= bbits - 1;
                                        const unsigned long long k = sl.at(rank++);
                                        if (k < p.band_cap) {
                                            BandEntry e;
                                            e.ia = (uint32_t)gi;
                                            e.jb = (uint32_t)(gj0 + cb + j);
                                            e.s_hat = __int_as_float(0x7fc00000);
                                            e.pad = job;
                                            p.band[k] = e;
                                        }
                                    }
                                }
                                continue;
                            }
                        }
                        while (rows) {
                            const int L = __ffs(rows) - 1;
                            rows &= rows - 1;
                            if (lane == (uint32_t)L) {
#pragma unroll
                                for (int q = 0; q < 8; ++q)
                                    reinterpret_cast<float4 *>(srow)[q] =
                                        make_float4(v[h2 * 32 + 4 * q], v[h2 * 32 + 4 * q + 1], v[h2 * 32 + 4 * q + 2],
                                                    v[h2 * 32 + 4 * q + 3]);
                            }
                            __syncwarp();
                            const float naL = __shfl_sync(0xffffffffu, na, L);
                            const float tinL = __shfl_sync(0xffffffffu, thr_in, L);
                            const float toutL = __shfl_sync(0xffffffffu, thr_out, L);
                            const int jloL = __shfl_sync(0xffffffffu, jlo, L);
                            const int jhiL = __shfl_sync(0xffffffffu, jhi, L);
                            const uint64_t giL = gi - (uint64_t)lane + (uint64_t)L;
                            const float t = fmaf(-2.0f, srow[lane], nbl);
                            const int col = cb + (int)lane;
                            const bool rokL = __shfl_sync(0xffffffffu, row_ok, L);
                            const bool ok = (unsigned)(col - jloL) < (unsigned)(jhiL - jloL) && rokL;
                            cnt += (ok && t <= tinL) ? 1ull : 0ull;
                            if (p.dbg != nullptr && giL < p.na && gj0 + col < p.nb)
                                p.dbg[(uint64_t)p.perm_a[giL] * p.nb + p.perm_b[gj0 + col]] = (naL + t) * s_unscale;
                            // band pairs of the row: one reservation for the warp
                            const bool isb = ok && t > tinL && t <= toutL;
                            unsigned long long k = 0;
                            if constexpr (BC) {
                                const uint32_t bm = __ballot_sync(0xffffffffu, isb);
                                if (bm) k = band_reserve(__popc(bm)).at(__popc(bm & ((1u << lane) - 1u)));
                            } else if (isb) {  // band pair: rare with one centre
                                k = atomicAdd(p.band_total, 1ull);
                            }
                            if (isb && k < p.band_cap) {
                                BandEntry e;
                                e.ia = (uint32_t)giL;
                                e.jb = (uint32_t)(gj0 + col);
                                e.s_hat = (naL + t) * s_unscale;
                                e.pad = job;
                                p.band[k] = e;
                            }
                            __syncwarp();
                        }
                    }
                }
                ++t_cnt;
            }
            if (last_tile && it < p.n_items) item_rows(w);
        }
        if (job != 0xffffffffu) flush();
        if constexpr (BC) band_holes();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, kTmemCols);

}

// ---------------------------------------------------------------- recheck

// FP64 pair test (the oracle's) on every band pair, against the pair's job
// (BandEntry.pad); also the largest |s_hat - dist2| seen, as FP32 bits in
// max_err_bits.
// 16-byte loads of both rows where the rows allow it (every job's d * sizeof(TIn)
// a multiple of 16: `vec`); the FP64 sum runs over the dims in order either way.
template <typename TIn>
__device__ __forceinline__ double pair_dist2(const TIn *a, const TIn *b, uint32_t d, bool vec) {
    double acc = 0.0;
    if (vec) {
        constexpr uint32_t V = 16 / sizeof(TIn);
        using Vec = typename std::conditional<sizeof(TIn) == 4, float4, double2>::type;
        const Vec *av = reinterpret_cast<const Vec *>(a), *bv = reinterpret_cast<const Vec *>(b);
        for (uint32_t k = 0; k < d / V; ++k) {
            const Vec x = __ldg(av + k), y = __ldg(bv + k);
            TIn xs[V], ys[V];
            memcpy(xs, &x, 16);
            memcpy(ys, &y, 16);
#pragma unroll
            for (uint32_t j = 0; j < V; ++j) {
                const double df = __dsub_rn((double)xs[j], (double)ys[j]);
                acc = __fma_rn(df, df, acc);
            }
        }
        return acc;
    }
    for (uint32_t k = 0; k < d; ++k) {
        const double df = __dsub_rn((double)a[k], (double)b[k]);
        acc = __fma_rn(df, df, acc);
    }
    return acc;
}

template <typename TIn>
__global__ void k_recheck(const TcJob *__restrict__ jobs, const BandEntry *__restrict__ band,
                          const unsigned long long *band_total, uint64_t cap, unsigned int *max_err_bits, bool vec) {
    const uint64_t n = min((unsigned long long)cap, *band_total);
    const uint32_t lane = threadIdx.x & 31u;
    float emax = 0.f;
    // counts accumulate per thread while its entries stay in one job (a launch of
    // one join: always), flushed when the job changes and once at the end
    unsigned long long c_acc = 0;
    uint32_t cur = 0xffffffffu;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const BandEntry e = band[i];
        if (e.ia == kBandHole) continue;  // a slot reserved and left unused
        const TcJob &J = jobs[e.pad];
        const TIn *a = static_cast<const TIn *>(J.rows_a) + (uint64_t)(e.ia - J.a_row0) * J.d;
        const TIn *b = static_cast<const TIn *>(J.rows_b) + (uint64_t)(e.jb - J.b_row0) * J.d;
        const double acc = pair_dist2(a, b, J.d, vec);
        if (e.pad != cur) {
            if (c_acc) atomicAdd(jobs[cur].count, c_acc);
            cur = e.pad;
            c_acc = 0;
        }
        c_acc += acc <= J.T ? 1ull : 0ull;
        emax = fmaxf(emax, (float)fabs((double)e.s_hat - acc));  // NaN estimates (not kept) are skipped
    }
    // one atomic per warp when the warp's lanes end in the same job (the usual case)
    const uint32_t j0 = __shfl_sync(0xffffffffu, cur, 0);
    if (__all_sync(0xffffffffu, cur == j0 || c_acc == 0)) {
        const unsigned long long c = warp_sum_u64(c_acc);
        if (lane == 0 && c) atomicAdd(jobs[j0].count, c);
    } else if (c_acc) {
        atomicAdd(jobs[cur].count, c_acc);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) emax = fmaxf(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    if (lane == 0) atomicMax(max_err_bits, __float_as_uint(emax));
}

// ---------------------------------------------------------------- host side

// Error bound of the tensor-core estimate s = |a|^2 + |b|^2 - 2 v against the
// FP64 pair test, |s - dist2| <= c_rel (|a|^2 + |b|^2) + c_abs, built from:
//   operand rounding (TF32: 2 * 2^-11 relative per product; BF16 split:
//   a = a_hi + a_lo + r with |r| <= 2^-16 |a|, dropped a_lo b_lo and r terms
//   <= 3.1 * 2^-16 |a_k b_k|), FP32 rounding of FP64 inputs (2 * 2^-24),
//   tensor-core FP32 accumulation budgeted at 2^-22 of S = sum |a_k b_k| per
//   product term (K terms TF32, 3K BF16). The budget follows the model that
//   Fasi, Higham, Mikaitis and Pranesh (Numerical behavior of NVIDIA tensor
//   cores, PeerJ Computer Science 7:e330, 2021) measured for earlier tensor
//   cores: each hardware step adds k products (exact) to the accumulator after
//   aligning all k + 1 terms to the largest exponent and truncating them to
//   FP32's 24 bits, then truncates the sum to FP32. Each truncation loses less
//   than 2^-23 of the largest term, which is at most S, so a step loses less
//   than (k + 2) 2^-23 S and the K / k steps less than K (1 + 2/k) 2^-23 S,
//   within K 2^-22 S for every k >= 2. tests/test_gpu_tc.py checks the whole
//   bound on adversarial cancellation at K = 256 (running sums far above the
//   result) for every form. |a.b| <= sum |a_k b_k| <=
//   (|a|^2 + |b|^2) / 2 (Cauchy-Schwarz, AM-GM) -- the dot error enters s
//   twice; FP32 norms (2^-24 each) and the FP32 epilogue (three roundings of
//   values up to 2 (|a|^2 + |b|^2), 6 * 2^-24, budgeted 10 * 2^-24); the FP64
//   direct difference's own rounding (d * 2^-50).
// A margin factor 1.25 covers the bookkeeping in between. c_abs covers
// subnormal operands (TF32/BF16 keep the FP32 exponent range; values below
// 2^-100 times the largest coordinate are the only ones that can lose
// relative accuracy) and is negligible for data of ordinary scale.
//
// FP16 (in units scaled by op_scale^2, where the largest centred coordinate
// is below 2^15): operands rounded once from FP64, 2^-11 relative each, so
// products as TF32's; FP16 subnormals (|v| < 2^-14) carry an absolute error up
// to 2^-25 instead, at most 2 * 2^-25 * 2^15 per product term, d terms, twice
// in s: c_abs = 1.25 * d * 2^-8.
void tc_band_constants(int form, uint32_t d, double maxabs, double *c_rel, double *c_abs) {
    const double u24 = std::ldexp(1.0, -24), acc = std::ldexp(1.0, -22);
    const double kpad = (double)tc_kterms(form, d);  // product terms summed (zero columns are not multiplied)
    double dot;
    if (form == HJ_FORM_TC_TF32 || form == HJ_FORM_TC_FP16) {
        const double u = std::ldexp(1.0, -11);
        dot = 2 * u + u * u + 2 * u24 + kpad * acc;
    } else {
        dot = 3.1 * std::ldexp(1.0, -16) + 2 * u24 + 3 * kpad * acc;
    }
    *c_rel = 1.25 * (dot + 12 * u24 + (double)d * std::ldexp(1.0, -50));
    if (form == HJ_FORM_TC_FP16)
        *c_abs = 1.25 * (double)d * std::ldexp(1.0, -8);
    else
        *c_abs = 1e-30 + 4.0 * (double)d * std::ldexp(std::fmax(maxabs, 1e-30), -100) * std::fmax(maxabs, 1.0);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn(std::string *err) {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        else
            cudaGetLastError();
    });
    if (!fn) *err = "cuTensorMapEncodeTiled unavailable";
    return fn;
}

// 2D map over a row-major [rows][kp] matrix, box = one 128-byte K atom x box_rows.
static bool make_map(CUtensorMap *m, const void *base, CUtensorMapDataType type, uint64_t rows, uint32_t kp,
                     uint32_t box_rows, std::string *err) {
    EncodeTiledFn fn = encode_fn(err);
    if (!fn) return false;
    const uint32_t esz = type == CU_TENSOR_MAP_DATA_TYPE_FLOAT32 ? 4 : 2;
    cuuint64_t gdim[2] = {kp, rows};
    cuuint64_t gstride[1] = {(cuuint64_t)kp * esz};
    cuuint32_t box[2] = {kAtomBytes / esz, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, type, 2,
                    const_cast<void *>(base), gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        *err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return false;
    }
    return true;
}

struct TcLayout {
    uint32_t ka, a_bufs, nst;
    size_t smem;
};

static TcLayout tc_layout(int form, uint32_t d) {
    TcLayout L;
    L.ka = form == HJ_FORM_TC_TF32 ? (d + 31) / 32 : (d + 63) / 64;
    const uint32_t a_atoms = form == HJ_FORM_TC_BF16X3 ? 2 * L.ka : L.ka;
    const size_t a_bytes = (size_t)a_atoms * kAStageBytes;
    const size_t budget = 224 * 1024;  // + 1 KB alignment + ~1.3 KB static smem <= 227 KB per block
    L.a_bufs = 2 * a_bytes + 3 * kBStageBytes <= budget ? 2 : 1;
    size_t left = budget - L.a_bufs * a_bytes;
    L.nst = (uint32_t)(left / kBStageBytes);
    if (L.nst > 8) L.nst = 8;
    L.smem = L.a_bufs * a_bytes + (size_t)L.nst * kBStageBytes + 1024;  // <= 225 KB
    return L;
}

uint32_t tc_atoms(int form, uint32_t kcols) { return tc_layout(form, kcols).ka; }
uint32_t tc_ksteps(int form, uint32_t kcols) {
    const uint32_t k = form == HJ_FORM_TC_TF32 ? 8u : 16u;
    return (kcols + k - 1) / k;
}
uint32_t tc_kterms(int form, uint32_t kcols) { return tc_ksteps(form, kcols) * (form == HJ_FORM_TC_TF32 ? 8u : 16u); }

// Per-block centring constants (operand units, FP16 form):
//   kp21: the accumulation model above, K = 3d + 3 rounded up to the MMA's 16
//     (the product terms summed) of magnitude sum <= S per dot, the dot
//     entering s twice: 2 K 2^-22;
//   rho_u: |fl16(h) - h| <= 2^-11 |h| per coordinate (normal range), with
//     |h| <= |fl16(h)| (1 + 2^-10): 1.001 * 2^-11 per unit of the stored |h|;
//   rho_c: subnormal FP16 (|h| < 2^-14) is off by at most 2^-25 per
//     coordinate, and the FP64 shift (x - center) * scale by 2^-52 of 2^15:
//     sqrt(d) (2^-25 + 2^-37), doubled;
//   u_norm: q rounded once from FP64 to FP32 (2^-24 relative), doubled, and
//     the split of q / 2 into FP16 pieces (2^-34 relative);
//   u_d: D in FP32, two FMAs per lane and a five-step sum of the lanes, with
//     the differences of FP16 values exact or rounded once: 16 * 2^-24;
//   theta_t: the FP64 pair test sums d squares of exact differences with FMAs,
//     relative error below (d + 2) 2^-53 of dist2 ~ eps^2: 2 (d + 2) 2^-53 T.
BcConsts bc_constants(int form, uint32_t d, double T, double op_scale) {
    // BF16x3: three MMAs per K step. A BF16 value has 8 significant bits, so
    // |lo| <= 2^-8 |v| and the dropped lo.lo products stay below 2^-16 S
    // (1.001 covers S being taken over the stored hi + lo), doubled for s.
    const double s2 = op_scale * op_scale,
                 kpad = (double)tc_kterms(form, bc_cols(d, form)) * (form == HJ_FORM_TC_BF16X3 ? 3.0 : 1.0);
    auto up = [](double v) {
        const float f = (float)v;
        return (double)f >= v ? f : std::nextafter(f, INFINITY);
    };
    BcConsts k;
    k.kp21 = up(2.0 * kpad * std::ldexp(1.0, -22) +
                (form == HJ_FORM_TC_BF16X3 ? 2.0 * 1.001 * std::ldexp(1.0, -16) : 0.0));
    k.eps = up(std::sqrt(T * s2) * (1.0 + 1e-12));
    // FP16 / TF32 round once to 11 significant bits; the BF16 hi + lo pair keeps v
    // to 2^-17 (hi to 2^-8 |v|, and lo to half a unit of the last of its 8 bits)
    k.rho_u = up(1.001 * std::ldexp(1.0, form == HJ_FORM_TC_BF16X3 ? -17 : -11));
    // the subnormal spacing of the operand type (half of it per rounding: FP16
    // 2^-25, BF16 2^-134, TF32 2^-150, taken as 2^-140) and the FP64 shift of
    // coordinates below 2^10 (2^-52 of 2^10, generously 2^-37)
    const double sub = form == HJ_FORM_TC_FP16     ? std::ldexp(1.0, -25)
                       : form == HJ_FORM_TC_BF16X3 ? std::ldexp(1.0, -134)
                                                   : std::ldexp(1.0, -140);
    const double floor_abs = sub + std::ldexp(1.0, -37);
    k.rho_c = up(2.0 * std::sqrt((double)d) * floor_abs);
    k.u_norm = up(std::ldexp(1.0, -23) + std::ldexp(1.0, -33));
    k.u_d = up(16.0 * std::ldexp(1.0, -24));
    // + the absolute floor of the q / 2 split (2^-32 in w, 2^-31 in s, twice in tau)
    k.theta_t = up(2.0 * (d + 2.0) * std::ldexp(1.0, -53) * T * s2 + std::ldexp(1.0, -29));
    return k;
}

static float *g_dbg_out = nullptr;  // set by tests through hj_debug_tc_estimates
static uint64_t g_gate_ns = 0;      // set by tests through hj_debug_set_wait_gate

void fill_tc_job(TcJob *j, int form, uint32_t d, double T, double op_scale, double maxabs, uint64_t a_row0,
                 uint64_t na_eff, uint64_t b_row0, uint64_t nb_eff, bool self, unsigned long long *count,
                 const void *rows_a, const void *rows_b, double *c_rel_out, double *c_abs_out) {
    double c_rel = 0, c_abs = 0;
    tc_band_constants(form, d, maxabs, &c_rel, &c_abs);
    const double s2 = op_scale * op_scale;  // FP16: the units of the norms; 1 otherwise
    const double T_tc = T * s2;
    memset(j, 0, sizeof(*j));
    j->a_row0 = a_row0;
    j->a_end = a_row0 + na_eff;
    j->b_row0 = b_row0;
    j->b_end = b_row0 + nb_eff;
    j->T = T;
    j->count = count;
    j->rows_a = rows_a;
    j->rows_b = rows_b;
    const float t = (float)T_tc;  // outward rounding of eps^2 and upward rounding of the bound
    j->T_lo = (double)t <= T_tc ? t : std::nextafter(t, -INFINITY);
    j->T_hi = (double)t >= T_tc ? t : std::nextafter(t, INFINITY);
    const float cr = (float)c_rel, ca = (float)c_abs;
    j->c_rel_f = (double)cr >= c_rel ? cr : std::nextafter(cr, INFINITY);
    j->c_abs_f = (double)ca >= c_abs ? ca : std::nextafter(ca, INFINITY);
    j->s_unscale = (float)(1.0 / s2);  // a power of two: exact
    j->self = self ? 1u : 0u;
    j->ka = tc_layout(form, d).ka;
    j->ksteps = tc_ksteps(form, d);
    j->d = d;
    if (c_rel_out) *c_rel_out = c_rel;
    if (c_abs_out) *c_abs_out = c_abs;
}

int launch_join_tc(const SortedSet &A, const SortedSet &B, int form, const TcJob *d_jobs, uint64_t na0, uint64_t nb0,
                   const IndexResult &idx, uint2 *band, uint64_t band_cap, unsigned long long *d_band_total,
                   uint32_t *d_err, int num_sms, cudaStream_t st, std::string *err, const BcConsts *bc,
                   unsigned long long *d_band_holes) {
    if (idx.n_items == 0) return 0;
    if (bc && (A.d > kBcMaxDim || !A.bc_op || !B.bc_op || A.bc_dp != B.bc_dp || A.bc_form != form ||
               B.bc_form != form || (form == HJ_FORM_TC_BF16X3 && (!A.bc_op_lo || !B.bc_op_lo)))) {
        *err = "per-block centring needs d <= 64 and the centred layouts of the form";
        return 1;
    }
    const TcLayout L = tc_layout(form, bc ? bc_cols(A.d, form) : A.d);
    if (L.nst < 2) {
        *err = "dimension too large for the tensor-core kernel";
        return 1;
    }
    CUtensorMap ma, ma2, mb, mb2;
    if (bc) {
        // rows of 4 dp columns; A reads the window from column dp (the producer's
        // x offset), B from column 0; past the row end the copy fills zeros
        const CUtensorMapDataType ty = form == HJ_FORM_TC_TF32    ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                       : form == HJ_FORM_TC_BF16X3 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                                   : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
        if (!make_map(&ma, A.bc_op, ty, A.npad_tc, 4 * A.bc_dp, kTcTileA, err)) return 1;
        if (!make_map(&mb, B.bc_op, ty, B.npad_tc, 4 * B.bc_dp, kTcTileB, err)) return 1;
        ma2 = ma;
        mb2 = mb;
        if (form == HJ_FORM_TC_BF16X3) {
            if (!make_map(&ma2, A.bc_op_lo, ty, A.npad_tc, 4 * A.bc_dp, kTcTileA, err)) return 1;
            if (!make_map(&mb2, B.bc_op_lo, ty, B.npad_tc, 4 * B.bc_dp, kTcTileB, err)) return 1;
        }
    } else if (form == HJ_FORM_TC_TF32) {
        if (!make_map(&ma, A.tf32, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, A.npad_tc, A.kpad_tf32, kTcTileA, err)) return 1;
        if (!make_map(&mb, B.tf32, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, B.npad_tc, B.kpad_tf32, kTcTileB, err)) return 1;
        ma2 = ma;
        mb2 = mb;
    } else if (form == HJ_FORM_TC_FP16) {
        if (!make_map(&ma, A.bf_hi, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, A.npad_tc, A.kpad_bf16, kTcTileA, err)) return 1;
        if (!make_map(&mb, B.bf_hi, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, B.npad_tc, B.kpad_bf16, kTcTileB, err)) return 1;
        ma2 = ma;
        mb2 = mb;
    } else {
        const CUtensorMapDataType t = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
        if (!make_map(&ma, A.bf_hi, t, A.npad_tc, A.kpad_bf16, kTcTileA, err)) return 1;
        if (!make_map(&ma2, A.bf_lo, t, A.npad_tc, A.kpad_bf16, kTcTileA, err)) return 1;
        if (!make_map(&mb, B.bf_hi, t, B.npad_tc, B.kpad_bf16, kTcTileB, err)) return 1;
        if (!make_map(&mb2, B.bf_lo, t, B.npad_tc, B.kpad_bf16, kTcTileB, err)) return 1;
    }
    TcArgs a;
    memset(&a, 0, sizeof(a));
    a.ka = L.ka;
    a.a_bufs = L.a_bufs;
    a.nst = L.nst;
    a.items = idx.items;
    a.n_items = idx.n_items;
    a.norm_a = A.norms;
    a.norm_b = B.norms;
    a.tmax_b = B.tile_maxnorm_b;
    a.gmin_b = B.group_minnorm;
    a.jobs = d_jobs;
    a.na = na0;
    a.nb = nb0;
    a.band = reinterpret_cast<BandEntry *>(band);
    a.band_cap = band_cap;
    a.band_total = d_band_total;
    a.band_holes = d_band_holes;
    a.err = d_err;
    a.dbg = g_dbg_out;
    a.perm_a = A.perm;
    a.perm_b = B.perm;
    a.gate_ns = g_gate_ns;
    if (bc) {
        a.norm_a = A.bc_norms;
        a.norm_b = nullptr;  // q_j / 2 is folded into the accumulator
        a.gmin_b = nullptr;
        a.tmax_b = nullptr;
        a.xn_a = A.bc_xn;
        a.blk_a = A.bc_blk;
        a.blk_b = B.bc_blk;
        a.cent_a = A.bc_cent;
        a.cent_b = B.bc_cent;
        a.bc = *bc;
        a.a_xoff = A.bc_dp;
    }
    uint64_t grid = (uint64_t)num_sms;
    if (grid > idx.n_items) grid = idx.n_items;
    if (bc && form == HJ_FORM_TC_TF32) {
        ensure_max_dynamic_smem((const void *)k_join_tc<HJ_FORM_TC_TF32, true>, 225 * 1024);
        k_join_tc<HJ_FORM_TC_TF32, true><<<(unsigned)grid, kTcThreads, L.smem, st>>>(ma, ma2, mb, mb2, a);
    } else if (bc && form == HJ_FORM_TC_BF16X3) {
        ensure_max_dynamic_smem((const void *)k_join_tc<HJ_FORM_TC_BF16X3, true>, 225 * 1024);
        k_join_tc<HJ_FORM_TC_BF16X3, true><<<(unsigned)grid, kTcThreads, L.smem, st>>>(ma, ma2, mb, mb2, a);
    } else if (bc) {
        ensure_max_dynamic_smem((const void *)k_join_tc<HJ_FORM_TC_FP16, true>, 225 * 1024);
        k_join_tc<HJ_FORM_TC_FP16, true><<<(unsigned)grid, kTcThreads, L.smem, st>>>(ma, ma2, mb, mb2, a);
    } else if (form == HJ_FORM_TC_TF32) {
        ensure_max_dynamic_smem((const void *)k_join_tc<HJ_FORM_TC_TF32, false>, 225 * 1024);
        k_join_tc<HJ_FORM_TC_TF32, false><<<(unsigned)grid, kTcThreads, L.smem, st>>>(ma, ma2, mb, mb2, a);
    } else if (form == HJ_FORM_TC_FP16) {
        ensure_max_dynamic_smem((const void *)k_join_tc<HJ_FORM_TC_FP16, false>, 225 * 1024);
        k_join_tc<HJ_FORM_TC_FP16, false><<<(unsigned)grid, kTcThreads, L.smem, st>>>(ma, ma2, mb, mb2, a);
    } else {
        ensure_max_dynamic_smem((const void *)k_join_tc<HJ_FORM_TC_BF16X3, false>, 225 * 1024);
        k_join_tc<HJ_FORM_TC_BF16X3, false><<<(unsigned)grid, kTcThreads, L.smem, st>>>(ma, ma2, mb, mb2, a);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        *err = std::string("tensor-core kernel launch: ") + cudaGetErrorString(e);
        return 1;
    }
    return 0;
}

void launch_recheck(const TcJob *d_jobs, int dtype_bytes, const uint2 *band, const unsigned long long *d_band_total,
                    uint64_t band_cap, unsigned int *d_max_err_bits, cudaStream_t st, bool vec_rows) {
    const BandEntry *b = reinterpret_cast<const BandEntry *>(band);
    if (dtype_bytes == 8)
        k_recheck<double><<<1184, 256, 0, st>>>(d_jobs, b, d_band_total, band_cap, d_max_err_bits, vec_rows);
    else
        k_recheck<float><<<1184, 256, 0, st>>>(d_jobs, b, d_band_total, band_cap, d_max_err_bits, vec_rows);
}

void set_tc_debug_output(float *dbg) { g_dbg_out = dbg; }

void set_tc_wait_gate(uint64_t ns) { g_gate_ns = ns; }

}  // namespace hj
