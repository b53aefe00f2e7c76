// hj_engine.cu -- host side of the engine: per-thread device contexts, the
// join pipeline (grid -> keys -> sort -> gather -> index -> distance kernels ->
// count), and the C ABI of include/hj.h.
//
// The pipeline is the reference's test_ego_loop3_macro / test_ego_loop3_noself
// (hilbertjoin/egojoin.cpp:777-838, :840-907) and its macros
// EGO_PARALLEL_TRAN / EGO_PARALLEL_TRAN_NOSELF (hilbertjoin/egojoin.h:164-222,
// :395-479) re-planned for one GPU: every stage is a device kernel on one
// stream, the host only plans the key layout (after one small read-back of the
// per-dimension cell ranges) and sizes the work list (one more read-back).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hj.h"
#include "hj_common.cuh"
#include "hj_internal.h"

namespace hj {

thread_local std::string tl_error;

static int fail(int code, const std::string &msg) {
    tl_error = msg;
    return code;
}

// ------------------------------------------------------------------ context

struct Ctx {
    int device = -1;
    cudaStream_t stream = nullptr;
    int num_sms = 0;
    std::vector<std::pair<void *, size_t>> slots;
    cudaEvent_t ev[8] = {};
    unsigned long long *d_small = nullptr;  // [16] counters
    unsigned long long *h_small = nullptr;  // pinned [16]
    TcJob *h_job = nullptr;                 // pinned: the job table of a single join
    TcJob *d_job = nullptr;
    bool ok = false;
};

static thread_local std::map<int, Ctx *> tl_ctx;

static void *slot_alloc_impl(Ctx *c, cudaStream_t st, int slot, size_t bytes) {
    if ((size_t)slot >= c->slots.size()) c->slots.resize(slot + 1, {nullptr, 0});
    auto &s = c->slots[slot];
    if (bytes == 0) bytes = 16;
    if (s.second >= bytes) return s.first;
    if (s.first) {
        cudaStreamSynchronize(st);
        cudaFree(s.first);
        s.first = nullptr;
        s.second = 0;
    }
    size_t cap = bytes + bytes / 8;
    cap = (cap + 255) / 256 * 256;
    void *p = nullptr;
    if (cudaMalloc(&p, cap) != cudaSuccess) {
        cudaGetLastError();
        if (cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        cap = bytes;
    }
    s.first = p;
    s.second = cap;
    return p;
}

struct AllocCtx {
    Ctx *c;
    cudaStream_t st;
};
static void *slot_alloc_cb(void *ctx, int slot, size_t bytes) {
    AllocCtx *a = static_cast<AllocCtx *>(ctx);
    return slot_alloc_impl(a->c, a->st, slot, bytes);
}

static int get_ctx(int device, Ctx **out) {
    int dev = device;
    if (dev < 0) {
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            return fail(HJ_ERR_NO_DEVICE, "no CUDA device");
        }
    }
    auto it = tl_ctx.find(dev);
    if (it != tl_ctx.end() && it->second->ok) {
        cudaSetDevice(dev);
        *out = it->second;
        return HJ_OK;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || dev >= ndev) {
        cudaGetLastError();
        return fail(HJ_ERR_NO_DEVICE, "no CUDA device");
    }
    cudaSetDevice(dev);
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, dev);
    if (prop.major < 10) return fail(HJ_ERR_NO_DEVICE, "device is not sm_100 class (compute capability 10.x)");
    Ctx *c = new Ctx();
    c->device = dev;
    c->num_sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return fail(HJ_ERR_CUDA, "cudaStreamCreate failed");
    }
    for (auto &e : c->ev) cudaEventCreate(&e);
    cudaMalloc(&c->d_small, 16 * sizeof(unsigned long long));
    cudaMallocHost(&c->h_small, 16 * sizeof(unsigned long long));
    cudaMallocHost(&c->h_job, sizeof(TcJob));
    cudaMalloc(&c->d_job, sizeof(TcJob));
    if (!c->d_small || !c->h_small || !c->h_job || !c->d_job) return fail(HJ_ERR_OOM, "context allocation failed");
    c->ok = true;
    tl_ctx[dev] = c;
    *out = c;
    return HJ_OK;
}

// Slot ids. The index stage's slots (hj_index.cu) start at kSlotIndexFirst;
// the two ranges must not meet, or a buffer of one stage is freed while the
// other still reads it.
enum {
    kSlotInA = 1, kSlotInB, kSlotDimStats, kSlotGridOff, kSlotGridBits, kSlotGridWord, kSlotGridShift,
    kSlotKeysWmA, kSlotKeysWmB, kSlotPermA, kSlotPermB, kSlotPermTmp, kSlotHist,
    kSlotRowsA, kSlotRowsB, kSlotKeysA, kSlotKeysB, kSlotTilesA, kSlotTilesB,
    kSlotTf32A, kSlotTf32B, kSlotHiA, kSlotLoA, kSlotHiB, kSlotLoB, kSlotNormA, kSlotNormB,
    kSlotTmaxAA, kSlotTmaxAB, kSlotTmaxBA, kSlotTmaxBB, kSlotBand, kSlotCenter, kSlotGminA, kSlotGminB,
    kSlotItemCnt, kSlotPairKeys, kSlotPairPerm, kSlotPairTmp, kSlotPairHist, kSlotPairOut, kSlotDimCost,
    kSlotGridOrd, kSlotBcOpA, kSlotBcOpB, kSlotBcNormA, kSlotBcNormB, kSlotBcXnA, kSlotBcXnB, kSlotBcBlkA,
    kSlotBcBlkB, kSlotBcCentA, kSlotBcCentB, kSlotScanTiles, kSlotBcOpLoA, kSlotBcOpLoB,
    kSlotEngineEnd
};
static_assert(kSlotEngineEnd <= kSlotIndexFirst, "engine slots overlap the index stage's");

static int bitwidth(unsigned long long v) {
    int b = 0;
    while (b < 64 && (v >> b) != 0) ++b;
    return b;
}

// Plans the packed key layout from the per-dim cell ranges. `ord` (empty =
// identity) lists the dims from the most significant key field down.
static int plan_grid(const std::vector<DimStats> &ds, uint32_t d, double eps, double maxabs,
                     const std::vector<uint32_t> &ord, Grid *g) {
    g->d = d;
    g->ord = ord;
    if (g->ord.empty())
        for (uint32_t t = 0; t < d; ++t) g->ord.push_back(t);
    g->eps = eps;
    g->maxabs = maxabs;
    g->eps_wide = eps + std::ldexp(eps + maxabs, -40);
    g->off.resize(d);
    g->bits.resize(d);
    g->word.resize(d);
    g->shift.resize(d);
    g->range.resize(d);
    uint32_t w = 0, left = 32;
    for (uint32_t pos = 0; pos < d; ++pos) {
        const uint32_t t = g->ord[pos];
        long long lo = ds[t].cmin, hi = ds[t].cmax;
        if (lo > hi) lo = hi = 0;  // empty set
        long long range = hi - lo;
        if (range < 0 || range > (1ll << 30)) return fail(HJ_ERR_INVALID_ARG,
                                                           "eps too small for the coordinate range: more than 2^30 "
                                                           "cells in one dimension");
        uint32_t b = (uint32_t)bitwidth((unsigned long long)range + 4);
        if (b > left) {
            ++w;
            left = 32;
        }
        g->off[t] = lo - 2;
        g->bits[t] = b;
        g->word[t] = w;
        g->shift[t] = left - b;
        g->range[t] = range;
        left -= b;
    }
    g->W = w + 1;
    // radix windows that can vary: word W-1 first (least significant), low bits first
    g->passes.clear();
    for (int ww = (int)g->W - 1; ww >= 0; --ww) {
        for (uint32_t lowbit = 0; lowbit < 32; lowbit += 8) {
            bool active = false;
            for (uint32_t t = 0; t < d && !active; ++t) {
                if ((int)g->word[t] != ww || g->range[t] == 0) continue;
                uint32_t vb = (uint32_t)bitwidth((unsigned long long)g->range[t] + 2);
                uint32_t f0 = g->shift[t], f1 = g->shift[t] + std::min(vb, g->bits[t]);
                if (f0 < lowbit + 8 && f1 > lowbit) active = true;
            }
            if (active) g->passes.push_back({(uint32_t)ww, lowbit});
        }
    }
    return HJ_OK;
}

struct JoinIn {
    const void *a;  // device
    const void *b;  // device (== a for self)
    uint64_t na, nb;
    int dtype_bytes;
    uint32_t d;
    double eps;
    bool self;
};

static int form_is_tc(int f) { return f == HJ_FORM_TC_TF32 || f == HJ_FORM_TC_BF16X3 || f == HJ_FORM_TC_FP16; }

static int check_cuda(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(HJ_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return HJ_OK;
}

static float ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        return 0.f;
    }
    return ms;
}

// Sorts one set and gathers the layouts the chosen form needs.
static int prepare_set(Ctx *c, cudaStream_t st, const void *x, uint64_t n, int dtype_bytes, const Grid &g,
                       const GridDev &gd, const double *center, double norm_scale, double op_scale, int form,
                       bool is_b, SortedSet *out, int *launches) {
    SortedSet s;
    s.n = n;
    s.d = g.d;
    s.dtype_bytes = dtype_bytes;
    s.src = x;
    s.center = center;
    s.op_scale = form == HJ_FORM_TC_FP16 ? op_scale : 1.0;
    const uint32_t W = g.W;
    const bool norm_order = form_is_tc(form);
    uint32_t *keys_wm = (uint32_t *)slot_alloc_impl(c, st, is_b ? kSlotKeysWmB : kSlotKeysWmA,
                                                    n * (W + (norm_order ? 1 : 0)) * 4);
    uint32_t *perm = (uint32_t *)slot_alloc_impl(c, st, is_b ? kSlotPermB : kSlotPermA, n * 4);
    void *rs = slot_alloc_impl(c, st, kSlotHist, radix_scratch_bytes(n));
    s.keys = (uint32_t *)slot_alloc_impl(c, st, is_b ? kSlotKeysB : kSlotKeysA, n * W * 4);
    s.rows = slot_alloc_impl(c, st, is_b ? kSlotRowsB : kSlotRowsA, n * g.d * dtype_bytes);
    if (!keys_wm || !perm || !rs || !s.keys || !s.rows) return fail(HJ_ERR_OOM, "out of device memory");
    s.perm = perm;
    uint32_t flags = kGatherKeys | kGatherRows;
    if (form == HJ_FORM_PLAIN_FP64) {
        s.n_tiles64 = hj_ceil_div(n, kPlainTile);
        s.tiles64 = (double *)slot_alloc_impl(c, st, is_b ? kSlotTilesB : kSlotTilesA,
                                              s.n_tiles64 * g.d * kPlainTile * 8);
        if (!s.tiles64) return fail(HJ_ERR_OOM, "out of device memory");
        flags |= kGatherPlain;
    } else {
        s.npad_tc = hj_ceil_div(std::max<uint64_t>(n, 1), kTcTileB) * kTcTileB;
        s.kpad_tf32 = (uint32_t)hj_ceil_div(g.d, 32) * 32;
        s.kpad_bf16 = (uint32_t)hj_ceil_div(g.d, 64) * 64;
        if (form == HJ_FORM_TC_TF32) {
            s.tf32 = (float *)slot_alloc_impl(c, st, is_b ? kSlotTf32B : kSlotTf32A, s.npad_tc * s.kpad_tf32 * 4);
            if (!s.tf32) return fail(HJ_ERR_OOM, "out of device memory");
            flags |= kGatherTf32;
        } else if (form == HJ_FORM_TC_FP16) {
            s.bf_hi = (uint16_t *)slot_alloc_impl(c, st, is_b ? kSlotHiB : kSlotHiA, s.npad_tc * s.kpad_bf16 * 2);
            if (!s.bf_hi) return fail(HJ_ERR_OOM, "out of device memory");
            flags |= kGatherF16;
        } else {
            s.bf_hi = (uint16_t *)slot_alloc_impl(c, st, is_b ? kSlotHiB : kSlotHiA, s.npad_tc * s.kpad_bf16 * 2);
            s.bf_lo = (uint16_t *)slot_alloc_impl(c, st, is_b ? kSlotLoB : kSlotLoA, s.npad_tc * s.kpad_bf16 * 2);
            if (!s.bf_hi || !s.bf_lo) return fail(HJ_ERR_OOM, "out of device memory");
            flags |= kGatherBf16;
        }
        s.norms = (float *)slot_alloc_impl(c, st, is_b ? kSlotNormB : kSlotNormA, s.npad_tc * 4);
        s.tile_maxnorm_a = (float *)slot_alloc_impl(c, st, is_b ? kSlotTmaxBA : kSlotTmaxAA,
                                                    (s.npad_tc / kTcTileA) * 4);
        s.tile_maxnorm_b = (float *)slot_alloc_impl(c, st, is_b ? kSlotTmaxBB : kSlotTmaxAB,
                                                    (s.npad_tc / kTcTileB) * 4);
        s.group_minnorm = (float *)slot_alloc_impl(c, st, is_b ? kSlotGminB : kSlotGminA, (s.npad_tc / 32) * 4);
        if (!s.norms || !s.tile_maxnorm_a || !s.tile_maxnorm_b || !s.group_minnorm)
            return fail(HJ_ERR_OOM, "out of device memory");
        flags |= kGatherNorms;
    }
    // the tensor-core forms' least significant key: the quantised norm (ties
    // within a cell by norm), packed in the same pass
    launch_pack_keys(x, dtype_bytes, n, g.d, g.eps, gd, W, keys_wm, st, center, norm_scale,
                     norm_order ? keys_wm + (size_t)W * n : nullptr);
    *launches += 1;
    if (norm_order) {
        std::vector<std::pair<uint32_t, uint32_t>> passes = {{W, 0u}, {W, 8u}};
        passes.insert(passes.end(), g.passes.begin(), g.passes.end());
        radix_sort_perm(keys_wm, n, passes, perm, rs, st, launches);
        *launches += 1;
    } else {
        radix_sort_perm(keys_wm, n, g.passes, perm, rs, st, launches);
    }
    launch_gather(x, dtype_bytes, n, g.d, perm, keys_wm, W, s, flags, st, launches);
    *out = s;
    return check_cuda("sort stage");
}

// The plain FP64 tile layout of a set prepared for a tensor-core form, for the
// work items routed to the FP64 kernel (padded to the 256-rank B tiles).
static int ensure_plain_tiles(Ctx *c, cudaStream_t st, SortedSet *s, bool is_b, int *launches) {
    if (s->tiles64) return HJ_OK;
    s->n_tiles64 = s->npad_tc / kPlainTile;
    s->tiles64 = (double *)slot_alloc_impl(c, st, is_b ? kSlotTilesB : kSlotTilesA,
                                           s->n_tiles64 * s->d * kPlainTile * 8);
    if (!s->tiles64) return fail(HJ_ERR_OOM, "out of device memory");
    launch_gather(s->src, s->dtype_bytes, s->n, s->d, s->perm, nullptr, 0, *s, kGatherPlain, st, launches);
    return check_cuda("plain layout");
}

// Per-block-centred operands of a sorted set (HJ_CENTRING_BLOCK; FP16, TF32 or
// BF16 hi + lo): the operand rows whose windows serve as A and as B, q and |h|
// per rank, block summaries and centres. scale = the FP16 form's operand scale
// times 2^-kBcScaleShift (the largest coordinate below 2^10, every form).
static int prepare_block_centring(Ctx *c, cudaStream_t st, SortedSet *s, bool is_b, const double *center,
                                  double scale, int form, int *launches) {
    const uint64_t npad = s->npad_tc, nblk = npad / kBcBlock;
    s->bc_form = form;
    s->bc_dp = bc_dp(s->d, form);
    s->bc_op = slot_alloc_impl(c, st, is_b ? kSlotBcOpB : kSlotBcOpA, npad * 4 * s->bc_dp * bc_elem_bytes(form));
    s->bc_op_lo = form == HJ_FORM_TC_BF16X3
                      ? slot_alloc_impl(c, st, is_b ? kSlotBcOpLoB : kSlotBcOpLoA, npad * 4 * s->bc_dp * 2)
                      : nullptr;
    s->bc_norms = (float *)slot_alloc_impl(c, st, is_b ? kSlotBcNormB : kSlotBcNormA, npad * 4);
    s->bc_xn = (float *)slot_alloc_impl(c, st, is_b ? kSlotBcXnB : kSlotBcXnA, npad * 4);
    s->bc_blk = (float4 *)slot_alloc_impl(c, st, is_b ? kSlotBcBlkB : kSlotBcBlkA, nblk * sizeof(float4));
    s->bc_cent = (float *)slot_alloc_impl(c, st, is_b ? kSlotBcCentB : kSlotBcCentA, nblk * kBcCentStride * 4);
    if (!s->bc_op || (form == HJ_FORM_TC_BF16X3 && !s->bc_op_lo) || !s->bc_norms || !s->bc_xn || !s->bc_blk ||
        !s->bc_cent)
        return fail(HJ_ERR_OOM, "out of device memory (block-centred operands)");
    launch_bc_prepare(*s, center, scale, s->bc_op, s->bc_op_lo, s->bc_norms, s->bc_xn, s->bc_blk, s->bc_cent, st,
                      launches);
    return check_cuda("block-centred operands");
}

// Key order by ascending dimension cost (ties by dim index) from set A's
// sample; see hj_dim_order. Synchronises once on `st`.
static int dim_order_by_cost(Ctx *c, cudaStream_t st, const void *x, int dtype_bytes, uint64_t n, uint32_t d,
                             double eps, const DimStats *ds, std::vector<uint32_t> *ord,
                             std::vector<unsigned long long> *costs) {
    unsigned long long *dcost = (unsigned long long *)slot_alloc_impl(c, st, kSlotDimCost, d * 8);
    if (!dcost) return fail(HJ_ERR_OOM, "out of device memory");
    launch_dim_cost(x, dtype_bytes, n, d, eps, ds, dcost, st);
    costs->assign(d, 0);
    cudaMemcpyAsync(costs->data(), dcost, d * 8, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("dimension cost");
    if (int r = check_cuda("dimension cost")) return r;
    ord->resize(d);
    for (uint32_t t = 0; t < d; ++t) (*ord)[t] = t;
    std::stable_sort(ord->begin(), ord->end(),
                     [&](uint32_t a, uint32_t b) { return (*costs)[a] < (*costs)[b]; });
    return HJ_OK;
}

// Everything before the distance kernels: cell statistics, key layout, EGO
// sort and layouts of both sets, stripe index and work list (and the shard).
struct Prepared {
    int form = HJ_FORM_PLAIN_FP64;
    int active_dims = 0;
    double maxabs = 0;
    Grid g;
    GridDev gd;
    SortedSet A, B;
    IndexResult idx;
    uint64_t na_eff = 0, nb_eff = 0;
    int launches = 0;
    double reorder_ms = 0;
    double op_scale = 1.0;  // FP16 form: operand scale 2^s
    std::vector<double> center_host;
};

static int prepare_join(Ctx *c, cudaStream_t st, const JoinIn &in, const hj_opts *opts, int form_override,
                        Prepared *P) {
    int form = form_override >= 0 ? form_override : (opts ? opts->form : HJ_FORM_PLAIN_FP64);
    if (form < HJ_FORM_PLAIN_FP64 || form > HJ_FORM_TC_FP16) return fail(HJ_ERR_INVALID_ARG, "unknown form");
    if (opts && opts->item_chunk > 4096) return fail(HJ_ERR_INVALID_ARG, "item_chunk must be at most 4096");
    if (opts && (opts->tc_centring < HJ_CENTRING_AUTO || opts->tc_centring > HJ_CENTRING_BLOCK))
        return fail(HJ_ERR_INVALID_ARG, "unknown tc_centring");
    int active_dims = opts ? opts->active_dims : -1;
    const bool ref_compat = opts && opts->ref_compat;
    if (active_dims < 0) active_dims = in.self ? 3 : 2;
    if (active_dims > kMaxActiveDims) active_dims = kMaxActiveDims;
    int launches = 0;

    const uint32_t d = in.d;
    // 1. per-dim cell ranges (union of both sets), read back to plan the keys
    DimStats *ds = (DimStats *)slot_alloc_impl(c, st, kSlotDimStats, d * sizeof(DimStats));
    if (!ds) return fail(HJ_ERR_OOM, "out of device memory");
    unsigned long long *d_maxabs = c->d_small + 0;
    uint32_t *d_bad = reinterpret_cast<uint32_t *>(c->d_small + 1);
    launch_dim_stats_init(ds, d, d_maxabs, d_bad, st);
    launch_dim_stats(in.a, in.dtype_bytes, in.na, d, in.eps, ds, d_maxabs, d_bad, st);
    launches += 2;
    if (!in.self) {
        launch_dim_stats(in.b, in.dtype_bytes, in.nb, d, in.eps, ds, d_maxabs, d_bad, st);
        ++launches;
    }
    std::vector<DimStats> hds(d);
    cudaMemcpyAsync(hds.data(), ds, d * sizeof(DimStats), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(c->h_small, c->d_small, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("cell statistics");
    if (int r = check_cuda("cell statistics")) return r;
    const uint32_t bad = (uint32_t)c->h_small[1];
    if (bad & 1u) return fail(HJ_ERR_INVALID_ARG, "input holds a non-finite coordinate");
    if (bad & 2u) return fail(HJ_ERR_INVALID_ARG, "a cell index floor(x/eps) exceeds 2^62");
    double maxabs;
    {
        unsigned long long bits = c->h_small[0];
        std::memcpy(&maxabs, &bits, 8);
    }
    if (form == HJ_FORM_AUTO) {
        // small joins: the tensor-core form's extra stages (layouts, precision
        // split, band) cost more than they save below about na * nb * d = 2e10
        // (measured on B200: d = 16, n = 20k is the crossover)
        const double work = (double)in.na * (double)(in.self ? in.na : in.nb) * (double)d;
        const bool small = work <= 2e10 && d <= 128;
        form = (d <= 256 && maxabs < 1e18 && !small) ? HJ_FORM_TC_FP16 : HJ_FORM_PLAIN_FP64;
    }
    if (form_is_tc(form) && d > 256) return fail(HJ_ERR_UNSUPPORTED, "tensor-core forms support d <= 256");
    if (form_is_tc(form) && !(maxabs < 1e18)) return fail(HJ_ERR_UNSUPPORTED, "tensor-core forms need |x| < 1e18");
    if (form == HJ_FORM_PLAIN_FP64 && d > 256) return fail(HJ_ERR_UNSUPPORTED, "plain FP64 form supports d <= 256");
    std::vector<uint32_t> ord;
    if (opts && opts->reorder_dims && d > 1) {
        auto t0 = std::chrono::steady_clock::now();
        std::vector<unsigned long long> costs;
        if (int r = dim_order_by_cost(c, st, in.a, in.dtype_bytes, in.na, d, in.eps, ds, &ord, &costs)) return r;
        ++launches;
        P->reorder_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    Grid &g = P->g;
    if (int r = plan_grid(hds, d, in.eps, maxabs, ord, &g)) return r;
    GridDev &gd = P->gd;
    if (!ord.empty()) {
        gd.ord = (uint32_t *)slot_alloc_impl(c, st, kSlotGridOrd, d * 4);
        if (!gd.ord) return fail(HJ_ERR_OOM, "out of device memory");
        cudaMemcpyAsync(gd.ord, g.ord.data(), d * 4, cudaMemcpyHostToDevice, st);
    }
    gd.off = (long long *)slot_alloc_impl(c, st, kSlotGridOff, d * 8);
    gd.bits = (uint32_t *)slot_alloc_impl(c, st, kSlotGridBits, d * 4);
    gd.word = (uint32_t *)slot_alloc_impl(c, st, kSlotGridWord, d * 4);
    gd.shift = (uint32_t *)slot_alloc_impl(c, st, kSlotGridShift, d * 4);
    if (!gd.off || !gd.bits || !gd.word || !gd.shift) return fail(HJ_ERR_OOM, "out of device memory");
    cudaMemcpyAsync(gd.off, g.off.data(), d * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(gd.bits, g.bits.data(), d * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(gd.word, g.word.data(), d * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(gd.shift, g.shift.data(), d * 4, cudaMemcpyHostToDevice, st);

    // per-dim midpoint of the coordinate range: the shift of the tensor-core operands
    double *center = (double *)slot_alloc_impl(c, st, kSlotCenter, d * 8);
    if (!center) return fail(HJ_ERR_OOM, "out of device memory");
    double norm_scale = 0.0;
    {
        std::vector<double> hc(d);
        double nmax = 0.0;
        for (uint32_t t = 0; t < d; ++t) {
            if (hds[t].cmin > hds[t].cmax) {
                hc[t] = 0.0;
                continue;
            }
            const double lo = double_from_ordered(hds[t].xmin), hi = double_from_ordered(hds[t].xmax);
            hc[t] = 0.5 * lo + 0.5 * hi;
            const double r = std::fmax(hi - hc[t], hc[t] - lo);
            nmax += r * r;
        }
        norm_scale = nmax > 0 ? 65535.0 / (nmax * 1.001) : 0.0;
        // FP16 operand scale: 2^s with the largest centred |coordinate| in [2^14, 2^15)
        double rmax = 0.0;
        for (uint32_t t = 0; t < d; ++t) {
            if (hds[t].cmin > hds[t].cmax) continue;
            const double lo = double_from_ordered(hds[t].xmin), hi = double_from_ordered(hds[t].xmax);
            rmax = std::fmax(rmax, std::fmax(hi - hc[t], hc[t] - lo));
        }
        P->op_scale = rmax > 0 ? std::ldexp(1.0, 14 - std::ilogb(rmax)) : 1.0;
        P->center_host = hc;  // outlives the asynchronous copy (the join synchronises later)
        cudaMemcpyAsync(center, P->center_host.data(), d * 8, cudaMemcpyHostToDevice, st);
    }

    // 2. EGO sort + layouts
    SortedSet &A = P->A, &B = P->B;
    if (int r = prepare_set(c, st, in.a, in.na, in.dtype_bytes, g, gd, center, norm_scale, P->op_scale, form,
                            false, &A, &launches))
        return r;
    if (in.self) {
        B = A;
    } else if (int r = prepare_set(c, st, in.b, in.nb, in.dtype_bytes, g, gd, center, norm_scale, P->op_scale,
                                   form, true, &B, &launches)) {
        return r;
    }
    cudaEventRecord(c->ev[2], st);

    // 3. index
    uint64_t na_eff = in.na, nb_eff = in.nb;
    if (ref_compat) {
        na_eff = na_eff / 8 * 8;
        nb_eff = nb_eff / 8 * 8;
    }
    const bool tc = form_is_tc(form);
    const int tile_a = tc ? kTcTileA : kPlainTile, tile_b = tc ? kTcTileB : kPlainTile;
    // B tiles per work item: 32 x 256 rows (tensor-core forms), 16 x 64 rows (plain), unless set
    const uint32_t chunk = (opts && opts->item_chunk > 0) ? (uint32_t)opts->item_chunk : (tc ? 32u : 16u);
    IndexResult &idx = P->idx;
    AllocCtx actx{c, st};
    std::string err;
    int r = build_index(A, B, g, gd, in.self, na_eff, nb_eff, tile_a, tile_b, active_dims, chunk, slot_alloc_cb,
                        &actx, st, &idx, &launches, &err);
    if (r == 2) return fail(HJ_ERR_OOM, err);
    if (r == 3) return fail(HJ_ERR_CUDA, err);
    if (r) return fail(HJ_ERR_INVALID_ARG, err);
    if (opts && opts->shard_count > 1) {
        if (opts->shard_index < 0 || opts->shard_index >= opts->shard_count)
            return fail(HJ_ERR_INVALID_ARG, "shard_index out of range");
        IndexResult sh;
        int sr = shard_items(idx, opts->shard_index, opts->shard_count, slot_alloc_cb, &actx, st, &sh);
        if (sr == 2) return fail(HJ_ERR_OOM, "out of device memory (shard)");
        if (sr) return check_cuda("shard selection");
        launches += 3;
        idx = sh;
    }
    cudaEventRecord(c->ev[3], st);
    P->form = form;
    P->active_dims = active_dims;
    P->maxabs = maxabs;
    P->na_eff = na_eff;
    P->nb_eff = nb_eff;
    P->launches = launches;
    return HJ_OK;
}

static int run_join(Ctx *c, const JoinIn &in, const hj_opts *opts, uint64_t *count, hj_stats *stats,
                    cudaEvent_t ev_h2d_start) {
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;
    auto t_wall0 = std::chrono::steady_clock::now();
    cudaEventRecord(c->ev[1], st);  // after H2D
    Prepared P;
    if (int r = prepare_join(c, st, in, opts, -1, &P)) return r;
    int form = P.form;
    const int active_dims = P.active_dims;
    const double maxabs = P.maxabs;
    const uint32_t d = in.d;
    SortedSet &A = P.A, &B = P.B;
    IndexResult &idx = P.idx;
    const uint64_t na_eff = P.na_eff, nb_eff = P.nb_eff;
    int launches = P.launches;
    const bool tc = form_is_tc(form);
    AllocCtx actx{c, st};

    // 4. distance kernels. d_small: [2] count of the tensor-core kernel and the
    // recheck, [3] error word, [4] band pairs, [5] max band error bits,
    // [6] count of the FP64 kernel.
    unsigned long long *d_count = c->d_small + 2;
    uint32_t *d_err = reinterpret_cast<uint32_t *>(c->d_small + 3);
    unsigned long long *d_band = c->d_small + 4;
    unsigned long long *d_count_fp = c->d_small + 6;
    unsigned long long *d_band_holes = c->d_small + 7;  // band slots reserved but left unused
    cudaMemsetAsync(c->d_small + 2, 0, 5 * sizeof(unsigned long long), st);
    uint64_t band_total = 0, band_holes = 0, fp_items = 0;
    double c_rel = 0, c_abs = 0;
    bool bc = false;  // per-block-centred operands (tensor-core forms)
    BcConsts bck{};
    const double T = in.eps * in.eps;
    cudaEventRecord(c->ev[6], st);
    if (!tc) {
        launch_join_fp64(A, B, in.self, na_eff, nb_eff, T, idx, d_count_fp, d_err, c->num_sms, st);
        ++launches;
        cudaEventRecord(c->ev[4], st);
        cudaEventRecord(c->ev[5], st);
    } else {
        // Operand centring: one global centre, or a centre per 128-rank block
        // (d <= 64) when asked for, or when the global centre would send more
        // than an eighth of the block pairs to the FP64 kernel.
        const int centring = opts ? opts->tc_centring : HJ_CENTRING_AUTO;
        const bool bc_ok = d <= kBcMaxDim;  // every tensor-core form
        // block-centred operands of both forms: the largest coordinate below 2^10
        const double bc_scale = std::ldexp(P.op_scale, -kBcScaleShift);
        auto enable_bc = [&]() -> int {
            if (int r = prepare_block_centring(c, st, &A, false, A.center, bc_scale, form, &launches)) return r;
            if (in.self) {
                B.bc_op = A.bc_op, B.bc_op_lo = A.bc_op_lo, B.bc_dp = A.bc_dp, B.bc_form = A.bc_form;
                B.bc_norms = A.bc_norms;
                B.bc_xn = A.bc_xn, B.bc_blk = A.bc_blk, B.bc_cent = A.bc_cent;
            } else if (int r = prepare_block_centring(c, st, &B, true, B.center, bc_scale, form, &launches)) {
                return r;
            }
            bc = true;
            bck = bc_constants(form, d, T, bc_scale);
            return HJ_OK;
        };
        // the job in the units of the operands in use (block centring: its own
        // scale and 3d + 3 columns)
        auto fill_job = [&]() {
            fill_tc_job(c->h_job, form, d, T, bc ? bc_scale : A.op_scale, maxabs, 0, na_eff, 0, nb_eff, in.self,
                        d_count, A.rows, B.rows, &c_rel, &c_abs);
            if (bc) {
                c->h_job->ka = tc_atoms(form, bc_cols(d, form));
                c->h_job->ksteps = tc_ksteps(form, bc_cols(d, form));
            }
            cudaMemcpyAsync(c->d_job, c->h_job, sizeof(TcJob), cudaMemcpyHostToDevice, st);
        };
        if (centring == HJ_CENTRING_BLOCK) {
            if (!bc_ok) return fail(HJ_ERR_UNSUPPORTED, "per-block centring needs d <= 64");
            if (int r = enable_bc()) return r;
        }
        // the FP16 form works in scaled units: norms, eps^2 and the bound times op_scale^2
        // one-entry job table: counted ranks, thresholds and bound in the operand units
        fill_job();
        const double T_tc = T * A.op_scale * A.op_scale;
        // Items whose error band would exceed half of eps^2 (eps^2 tiny against
        // the squared norms: the cancellation limit of the norm expansion) run
        // on the FP64 kernel instead.
        IndexResult idx_tc, idx_fp;
        // Routing limits: half of eps^2 for one global centre (wider bands hold
        // billions of pairs there); with block centres the band of a tile is
        // bounded by its residuals, and tiles up to 4 eps^2 (wide clusters,
        // blocks that straddle two clusters) cost less as band pairs than on the
        // FP64 kernel.
        auto route_limit = [&](int attempt) {
            return attempt > 0 ? -1.0 : bc ? 4.0 * T * bc_scale * bc_scale : 0.5 * T_tc;
        };
        for (int attempt = 0;; ++attempt) {
            int sr = split_items_by_precision(idx, A, B, c_rel, c_abs, route_limit(attempt), bc ? &bck : nullptr,
                                              slot_alloc_cb, &actx, st, &idx_tc, &idx_fp);
            if (sr == 2) return fail(HJ_ERR_OOM, "out of device memory (work list split)");
            if (sr) return check_cuda("work list split");
            launches += 2;
            if (attempt == 0 && !bc && bc_ok && centring == HJ_CENTRING_AUTO &&
                idx_fp.tile_pairs * 8 > idx.tile_pairs) {
                // the split synchronised the stream: the job's first copy is done
                if (int r = enable_bc()) return r;
                fill_job();
                sr = split_items_by_precision(idx, A, B, c_rel, c_abs, route_limit(attempt), &bck, slot_alloc_cb,
                                              &actx, st, &idx_tc, &idx_fp);
                if (sr == 2) return fail(HJ_ERR_OOM, "out of device memory (work list split)");
                if (sr) return check_cuda("work list split");
                launches += 2;
            }
            fp_items = idx_fp.n_items;
            cudaMemsetAsync(c->d_small + 2, 0, 5 * sizeof(unsigned long long), st);
            if (attempt == 0 && idx_tc.n_items == 0 && idx_fp.n_items && !(opts && opts->shard_count > 1)) {
                // Every item is routed to FP64: the plain form's own work list
                // (64 x 64 tiles, stripes per 64-rank tile) holds fewer candidate
                // pairs than the tensor-core one, so it replaces it.
                const uint32_t chunk = (opts && opts->item_chunk > 0) ? (uint32_t)opts->item_chunk : 16u;
                std::string ierr;
                int ir = build_index(A, B, P.g, P.gd, in.self, na_eff, nb_eff, kPlainTile, kPlainTile, active_dims,
                                     chunk, slot_alloc_cb, &actx, st, &idx, &launches, &ierr);
                if (ir == 2) return fail(HJ_ERR_OOM, ierr);
                if (ir) return fail(HJ_ERR_CUDA, ierr);
                idx_fp = idx;
            }
            if (idx_fp.n_items) {
                if (int rr = ensure_plain_tiles(c, st, &A, false, &launches)) return rr;
                if (in.self)
                    B.tiles64 = A.tiles64, B.n_tiles64 = A.n_tiles64;
                else if (int rr = ensure_plain_tiles(c, st, &B, true, &launches))
                    return rr;
                launch_join_fp64(A, B, in.self, na_eff, nb_eff, T, idx_fp, d_count_fp, d_err, c->num_sms, st);
                ++launches;
            }
            if (idx_tc.n_items == 0) {
                cudaEventRecord(c->ev[4], st);
                cudaEventRecord(c->ev[5], st);
                break;
            }
            const uint64_t cand_tc = idx_tc.tile_pairs * (uint64_t)kTcTileA * kTcTileB;
            // first band queue: 1/4096 of the candidates (1/512 with block
            // centres, whose wider tiles stay on the tensor cores; 1/256 for
            // BF16x3, whose bound adds three products per K step)
            const uint64_t div = !bc ? 4096 : (form == HJ_FORM_TC_BF16X3 ? 256 : 512);
            uint64_t cap = std::max<uint64_t>(1ull << 20, cand_tc / div);
            const uint64_t cap_limit = std::max<uint64_t>(1ull << 27, cand_tc / 64);
            bool done = false, fallback = false;
            for (int grow = 0; grow < 4; ++grow) {
                uint2 *band = (uint2 *)slot_alloc_impl(c, st, kSlotBand, cap * kBandEntryBytes);
                if (!band) return fail(HJ_ERR_OOM, "out of device memory (band queue)");
                cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), st);
                cudaMemsetAsync(d_band, 0, 2 * sizeof(unsigned long long), st);
                cudaMemsetAsync(d_band_holes, 0, sizeof(unsigned long long), st);
                std::string terr;
                cudaEventRecord(c->ev[6], st);
                if (launch_join_tc(A, B, form, c->d_job, na_eff, nb_eff, idx_tc, band, cap, d_band, d_err,
                                   c->num_sms, st, &terr, bc ? &bck : nullptr, d_band_holes))
                    return fail(HJ_ERR_CUDA, terr);
                ++launches;
                cudaEventRecord(c->ev[4], st);
                cudaMemcpyAsync(c->h_small + 4, d_band, 8, cudaMemcpyDeviceToHost, st);
                cudaMemcpyAsync(c->h_small + 7, d_band_holes, 8, cudaMemcpyDeviceToHost, st);
                if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("tensor-core join");
                band_total = c->h_small[4];
                band_holes = c->h_small[7];
                if (band_total <= cap) {
                    // sorted rows: slot buffers (256-byte aligned) of n rows of d coordinates
                    const bool vec_rows = ((uint64_t)d * A.dtype_bytes) % 16 == 0 &&
                                          ((uintptr_t)A.rows & 15u) == 0 && ((uintptr_t)B.rows & 15u) == 0;
                    launch_recheck(c->d_job, A.dtype_bytes, band, d_band, cap,
                                   reinterpret_cast<unsigned int *>(c->d_small + 5), st, vec_rows);
                    ++launches;
                    cudaEventRecord(c->ev[5], st);
                    done = true;
                    break;
                }
                if (band_total > cap_limit) {  // band too wide to be worth rechecking
                    fallback = true;
                    break;
                }
                cap = band_total + band_total / 4 + 1024;
            }
            if (done) break;
            if (!fallback || attempt >= 1) return fail(HJ_ERR_BAND_OVERFLOW, "band queue overflow");
        }
    }
    cudaMemcpyAsync(c->h_small + 2, c->d_small + 2, 5 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("distance kernel");
    if (int rr = check_cuda("distance kernel")) return rr;
    const uint32_t kerr = (uint32_t)c->h_small[3];
    if (kerr & kErrTimeout) {
        char msg[96];
        snprintf(msg, sizeof msg, "a bounded device-side wait timed out (error word 0x%x)", kerr);
        return fail(HJ_ERR_TIMEOUT, msg);
    }
    if (kerr) return fail(HJ_ERR_CUDA, "device error word set");
    *count = c->h_small[2] + c->h_small[6];
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        if (ev_h2d_start) stats->h2d_ms = ev_ms(ev_h2d_start, c->ev[1]);
        stats->sort_ms = ev_ms(c->ev[1], c->ev[2]);
        stats->index_ms = ev_ms(c->ev[2], c->ev[3]);
        stats->join_ms = ev_ms(c->ev[3], c->ev[4]);
        stats->kernel_ms = ev_ms(c->ev[6], c->ev[4]);
        stats->recheck_ms = ev_ms(c->ev[4], c->ev[5]);
        stats->total_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_wall0).count() +
            stats->h2d_ms;
        double all = in.self ? (double)na_eff * (double)(na_eff > 0 ? na_eff - 1 : 0) / 2.0
                             : (double)na_eff * (double)nb_eff;
        stats->candidate_pairs = idx.candidate_pairs;
        stats->tile_pairs = idx.tile_pairs;
        stats->work_items = idx.n_items;
        stats->loadpercent = all > 0 ? 100.0 * (double)idx.candidate_pairs / all : 0.0;
        const uint64_t band_pairs = band_total - std::min(band_total, band_holes);
        stats->band_pairs = band_pairs;
        stats->band_fraction = idx.candidate_pairs ? (double)band_pairs / (double)idx.candidate_pairs : 0.0;
        stats->band_halfwidth_rel = c_rel;
        {
            uint32_t eb = (uint32_t)c->h_small[5];
            float ef;
            std::memcpy(&ef, &eb, 4);
            stats->max_abs_err_band = tc ? (double)ef : 0.0;
        }
        stats->form_used = form;
        stats->tc_centring = tc ? (bc ? HJ_CENTRING_BLOCK : HJ_CENTRING_GLOBAL) : 0;
        stats->fp64_items = fp_items;
        stats->reorder_ms = P.reorder_ms;
        int s = active_dims;
        int p3 = 1;
        for (int i = 0; i < s; ++i) p3 *= 3;
        stats->stripes = in.self ? (p3 + 1) / 2 : p3;
        stats->kernel_launches = launches;
    }
    return HJ_OK;
}

// ------------------------------------------------------------ pair output

__global__ void k_pairs_gather(const uint32_t *__restrict__ pi, const uint32_t *__restrict__ pj,
                               const uint32_t *__restrict__ perm, uint64_t n, unsigned long long *__restrict__ out) {
    const uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t s = perm[r];
    out[2 * r] = pi[s];
    out[2 * r + 1] = pj[s];
}

// Pair materialisation: the join on the plain FP64 kernel run twice, once
// counting the pairs of every work item, once writing them at the exclusive
// scan of those counts, then a stable radix sort by (i, j) so that the output
// is the same on every run. Nothing is written to `pairs` unless all of them
// fit; *n_pairs is always the exact total.
static int run_pairs(Ctx *c, const JoinIn &in, const hj_opts *opts, uint64_t *pairs, uint64_t capacity,
                     uint64_t *n_pairs, hj_stats *stats, cudaEvent_t ev_h2d_start) {
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;
    auto t_wall0 = std::chrono::steady_clock::now();
    cudaEventRecord(c->ev[1], st);
    Prepared P;
    if (int r = prepare_join(c, st, in, opts, HJ_FORM_PLAIN_FP64, &P)) return r;
    SortedSet &A = P.A, &B = P.B;
    IndexResult &idx = P.idx;
    int launches = P.launches;
    const double T = in.eps * in.eps;
    uint32_t *d_err = reinterpret_cast<uint32_t *>(c->d_small + 3);
    cudaMemsetAsync(c->d_small + 2, 0, 5 * sizeof(unsigned long long), st);
    const uint64_t n_items = idx.n_items;
    uint32_t *item_cnt = (uint32_t *)slot_alloc_impl(c, st, kSlotItemCnt, (n_items + 1) * 4);
    if (!item_cnt) return fail(HJ_ERR_OOM, "out of device memory");
    cudaMemsetAsync(item_cnt, 0, (n_items + 1) * 4, st);
    cudaEventRecord(c->ev[6], st);
    launch_pairs_fp64(A, B, in.self, P.na_eff, P.nb_eff, T, idx, item_cnt, nullptr, nullptr, d_err, c->num_sms, st);
    launch_scan_u32(item_cnt, n_items, c->d_small + 2, st,
                    (unsigned long long *)slot_alloc_impl(c, st, kSlotScanTiles, scan_scratch_bytes(n_items)));
    launches += 2;
    cudaMemcpyAsync(c->h_small + 2, c->d_small + 2, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("pair count");
    if (int rr = check_cuda("pair count")) return rr;
    if ((uint32_t)c->h_small[3] & kErrTimeout) return fail(HJ_ERR_TIMEOUT, "a bounded device-side wait timed out");
    if ((uint32_t)c->h_small[3]) return fail(HJ_ERR_CUDA, "device error word set");
    const uint64_t total = c->h_small[2];
    *n_pairs = total;
    if (total > capacity)
        return fail(HJ_ERR_CAPACITY, "the pairs do not fit into the caller's buffer; *n_pairs holds their number");
    if (total >= (1ull << 32)) return fail(HJ_ERR_UNSUPPORTED, "more than 2^32 - 1 pairs");
    if (total) {
        // keys word-major: word 0 = i (most significant), word 1 = j
        uint32_t *keys = (uint32_t *)slot_alloc_impl(c, st, kSlotPairKeys, total * 8);
        uint32_t *perm = (uint32_t *)slot_alloc_impl(c, st, kSlotPairPerm, total * 4);
        void *rs = slot_alloc_impl(c, st, kSlotPairHist, radix_scratch_bytes(total));
        unsigned long long *out = (unsigned long long *)slot_alloc_impl(c, st, kSlotPairOut, total * 16);
        if (!keys || !perm || !rs || !out) return fail(HJ_ERR_OOM, "out of device memory (pairs)");
        launch_pairs_fp64(A, B, in.self, P.na_eff, P.nb_eff, T, idx, item_cnt, keys, keys + total, d_err,
                          c->num_sms, st);
        ++launches;
        std::vector<std::pair<uint32_t, uint32_t>> passes;
        const int bj = bitwidth(in.nb ? in.nb - 1 : 0), bi = bitwidth(in.na ? in.na - 1 : 0);
        for (int b = 0; b < bj; b += 8) passes.push_back({1u, (uint32_t)b});
        for (int b = 0; b < bi; b += 8) passes.push_back({0u, (uint32_t)b});
        radix_sort_perm(keys, total, passes, perm, rs, st, &launches);
        k_pairs_gather<<<(unsigned)hj_ceil_div(total, 256), 256, 0, st>>>(keys, keys + total, perm, total, out);
        ++launches;
        cudaEventRecord(c->ev[4], st);
        cudaMemcpyAsync(pairs, out, total * 16, cudaMemcpyDeviceToHost, st);
    } else {
        cudaEventRecord(c->ev[4], st);
    }
    cudaMemcpyAsync(c->h_small + 3, c->d_small + 3, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("pair output");
    if (int rr = check_cuda("pair output")) return rr;
    if ((uint32_t)c->h_small[3] & kErrTimeout) return fail(HJ_ERR_TIMEOUT, "a bounded device-side wait timed out");
    if ((uint32_t)c->h_small[3]) return fail(HJ_ERR_CUDA, "device error word set");
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        if (ev_h2d_start) stats->h2d_ms = ev_ms(ev_h2d_start, c->ev[1]);
        stats->sort_ms = ev_ms(c->ev[1], c->ev[2]);
        stats->index_ms = ev_ms(c->ev[2], c->ev[3]);
        stats->join_ms = ev_ms(c->ev[3], c->ev[4]);
        stats->kernel_ms = ev_ms(c->ev[6], c->ev[4]);
        stats->total_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_wall0).count() +
            stats->h2d_ms;
        const double all = in.self ? (double)P.na_eff * (double)(P.na_eff > 0 ? P.na_eff - 1 : 0) / 2.0
                                   : (double)P.na_eff * (double)P.nb_eff;
        stats->candidate_pairs = idx.candidate_pairs;
        stats->tile_pairs = idx.tile_pairs;
        stats->work_items = idx.n_items;
        stats->loadpercent = all > 0 ? 100.0 * (double)idx.candidate_pairs / all : 0.0;
        stats->form_used = HJ_FORM_PLAIN_FP64;
        stats->reorder_ms = P.reorder_ms;
        int p3 = 1;
        for (int i = 0; i < P.active_dims; ++i) p3 *= 3;
        stats->stripes = in.self ? (p3 + 1) / 2 : p3;
        stats->kernel_launches = launches;
    }
    return HJ_OK;
}

static int validate(uint64_t na, uint64_t nb, uint32_t d, double eps) {
    if (d == 0 || d > kMaxDim) return fail(HJ_ERR_INVALID_ARG, "d must be in [1, 1024]");
    if (na >= (1ull << 31) || nb >= (1ull << 31)) return fail(HJ_ERR_INVALID_ARG, "n must be below 2^31");
    if (!(eps > 0.0) || !std::isfinite(eps)) return fail(HJ_ERR_INVALID_ARG, "eps must be positive and finite");
    return HJ_OK;
}

static int join_host(const void *a, uint64_t na, const void *b, uint64_t nb, int dtype_bytes, uint32_t d, double eps,
                     bool self, const hj_opts *opts, uint64_t *count, hj_stats *stats) {
    tl_error.clear();
    if (!count || (na && !a) || (!self && nb && !b)) return fail(HJ_ERR_INVALID_ARG, "null pointer");
    if (int r = validate(na, nb, d, eps)) return r;
    Ctx *c;
    if (int r = get_ctx(opts ? opts->device : -1, &c)) return r;
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;
    *count = 0;
    if (na == 0 || (!self && nb == 0)) {
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return HJ_OK;
    }
    cudaEventRecord(c->ev[0], st);
    void *da = slot_alloc_impl(c, st, kSlotInA, na * d * dtype_bytes);
    void *db = self ? da : slot_alloc_impl(c, st, kSlotInB, nb * d * dtype_bytes);
    if (!da || !db) return fail(HJ_ERR_OOM, "out of device memory");
    cudaMemcpyAsync(da, a, na * d * dtype_bytes, cudaMemcpyHostToDevice, st);
    if (!self) cudaMemcpyAsync(db, b, nb * d * dtype_bytes, cudaMemcpyHostToDevice, st);
    if (int r = check_cuda("host to device copy")) return r;
    JoinIn in{da, db, na, self ? na : nb, dtype_bytes, d, eps, self};
    return run_join(c, in, opts, count, stats, c->ev[0]);
}

static int join_device(const void *a, uint64_t na, const void *b, uint64_t nb, int dtype_bytes, uint32_t d,
                       double eps, bool self, const hj_opts *opts, uint64_t *count, hj_stats *stats) {
    tl_error.clear();
    if (!count || (na && !a) || (!self && nb && !b)) return fail(HJ_ERR_INVALID_ARG, "null pointer");
    if (dtype_bytes != 4 && dtype_bytes != 8) return fail(HJ_ERR_INVALID_ARG, "dtype_bytes must be 4 or 8");
    if (int r = validate(na, nb, d, eps)) return r;
    Ctx *c;
    if (int r = get_ctx(opts ? opts->device : -1, &c)) return r;
    *count = 0;
    if (na == 0 || (!self && nb == 0)) {
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return HJ_OK;
    }
    JoinIn in{a, self ? a : b, na, self ? na : nb, dtype_bytes, d, eps, self};
    return run_join(c, in, opts, count, stats, nullptr);
}

static int pairs_host(const void *a, uint64_t na, const void *b, uint64_t nb, int dtype_bytes, uint32_t d,
                      double eps, bool self, const hj_opts *opts, uint64_t *pairs, uint64_t capacity,
                      uint64_t *n_pairs, hj_stats *stats) {
    tl_error.clear();
    if (!n_pairs || (capacity && !pairs) || (na && !a) || (!self && nb && !b))
        return fail(HJ_ERR_INVALID_ARG, "null pointer");
    if (int r = validate(na, nb, d, eps)) return r;
    if (d > 256) return fail(HJ_ERR_UNSUPPORTED, "pair output supports d <= 256 (plain FP64 form)");
    Ctx *c;
    if (int r = get_ctx(opts ? opts->device : -1, &c)) return r;
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;
    *n_pairs = 0;
    if (na == 0 || (!self && nb == 0)) {
        if (stats) std::memset(stats, 0, sizeof(*stats));
        return HJ_OK;
    }
    cudaEventRecord(c->ev[0], st);
    void *da = slot_alloc_impl(c, st, kSlotInA, na * d * dtype_bytes);
    void *db = self ? da : slot_alloc_impl(c, st, kSlotInB, nb * d * dtype_bytes);
    if (!da || !db) return fail(HJ_ERR_OOM, "out of device memory");
    cudaMemcpyAsync(da, a, na * d * dtype_bytes, cudaMemcpyHostToDevice, st);
    if (!self) cudaMemcpyAsync(db, b, nb * d * dtype_bytes, cudaMemcpyHostToDevice, st);
    if (int r = check_cuda("host to device copy")) return r;
    JoinIn in{da, db, na, self ? na : nb, dtype_bytes, d, eps, self};
    return run_pairs(c, in, opts, pairs, capacity, n_pairs, stats, c->ev[0]);
}

// Device EGO sort of one host set; perm (and sorted rows) copied back.
static int ego_sort_host(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts, uint64_t *perm,
                         double *sorted) {
    tl_error.clear();
    if (!perm || (n && !pts)) return fail(HJ_ERR_INVALID_ARG, "null pointer");
    if (int r = validate(n, n, d, eps)) return r;
    Ctx *c;
    if (int r = get_ctx(opts ? opts->device : -1, &c)) return r;
    if (n == 0) return HJ_OK;
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;
    void *dx = slot_alloc_impl(c, st, kSlotInA, n * d * 8);
    DimStats *ds = (DimStats *)slot_alloc_impl(c, st, kSlotDimStats, d * sizeof(DimStats));
    if (!dx || !ds) return fail(HJ_ERR_OOM, "out of device memory");
    cudaMemcpyAsync(dx, pts, n * d * 8, cudaMemcpyHostToDevice, st);
    unsigned long long *d_maxabs = c->d_small + 0;
    uint32_t *d_bad = reinterpret_cast<uint32_t *>(c->d_small + 1);
    launch_dim_stats_init(ds, d, d_maxabs, d_bad, st);
    launch_dim_stats(dx, 8, n, d, eps, ds, d_maxabs, d_bad, st);
    std::vector<DimStats> hds(d);
    cudaMemcpyAsync(hds.data(), ds, d * sizeof(DimStats), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(c->h_small, c->d_small, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("cell statistics");
    if ((uint32_t)c->h_small[1]) return fail(HJ_ERR_INVALID_ARG, "non-finite coordinate or cell out of range");
    double maxabs;
    std::memcpy(&maxabs, &c->h_small[0], 8);
    Grid g;
    if (int r = plan_grid(hds, d, eps, maxabs, {}, &g)) return r;
    GridDev gd;
    gd.off = (long long *)slot_alloc_impl(c, st, kSlotGridOff, d * 8);
    gd.bits = (uint32_t *)slot_alloc_impl(c, st, kSlotGridBits, d * 4);
    gd.word = (uint32_t *)slot_alloc_impl(c, st, kSlotGridWord, d * 4);
    gd.shift = (uint32_t *)slot_alloc_impl(c, st, kSlotGridShift, d * 4);
    uint32_t *keys_wm = (uint32_t *)slot_alloc_impl(c, st, kSlotKeysWmA, n * g.W * 4);
    uint32_t *dperm = (uint32_t *)slot_alloc_impl(c, st, kSlotPermA, n * 4);
    void *rs = slot_alloc_impl(c, st, kSlotHist, radix_scratch_bytes(n));
    void *rows = sorted ? slot_alloc_impl(c, st, kSlotRowsA, n * d * 8) : nullptr;
    if (!gd.off || !gd.bits || !gd.word || !gd.shift || !keys_wm || !dperm || !rs || (sorted && !rows))
        return fail(HJ_ERR_OOM, "out of device memory");
    cudaMemcpyAsync(gd.off, g.off.data(), d * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(gd.bits, g.bits.data(), d * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(gd.word, g.word.data(), d * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(gd.shift, g.shift.data(), d * 4, cudaMemcpyHostToDevice, st);
    int launches = 0;
    launch_pack_keys(dx, 8, n, d, eps, gd, g.W, keys_wm, st);
    radix_sort_perm(keys_wm, n, g.passes, dperm, rs, st, &launches);
    if (sorted) {
        SortedSet s;
        s.rows = rows;
        launch_gather(dx, 8, n, d, dperm, keys_wm, g.W, s, kGatherRows, st, &launches);
    }
    std::vector<uint32_t> hp(n);
    cudaMemcpyAsync(hp.data(), dperm, n * 4, cudaMemcpyDeviceToHost, st);
    if (sorted) cudaMemcpyAsync(sorted, rows, n * d * 8, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("EGO sort");
    if (int r = check_cuda("EGO sort")) return r;
    for (uint64_t i = 0; i < n; ++i) perm[i] = hp[i];
    return HJ_OK;
}

static int dim_order_host(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts,
                          int32_t *reorder_dim, uint64_t *costs_out) {
    tl_error.clear();
    if (!reorder_dim || (n && !pts)) return fail(HJ_ERR_INVALID_ARG, "null pointer");
    if (int r = validate(n, n, d, eps)) return r;
    Ctx *c;
    if (int r = get_ctx(opts ? opts->device : -1, &c)) return r;
    if (n == 0) {
        for (uint32_t t = 0; t < d; ++t) reorder_dim[t] = (int32_t)t;
        if (costs_out)
            for (uint32_t t = 0; t < d; ++t) costs_out[t] = 0;
        return HJ_OK;
    }
    cudaStream_t st = (opts && opts->stream) ? (cudaStream_t)opts->stream : c->stream;
    void *dx = slot_alloc_impl(c, st, kSlotInA, n * d * 8);
    DimStats *ds = (DimStats *)slot_alloc_impl(c, st, kSlotDimStats, d * sizeof(DimStats));
    if (!dx || !ds) return fail(HJ_ERR_OOM, "out of device memory");
    cudaMemcpyAsync(dx, pts, n * d * 8, cudaMemcpyHostToDevice, st);
    unsigned long long *d_maxabs = c->d_small + 0;
    uint32_t *d_bad = reinterpret_cast<uint32_t *>(c->d_small + 1);
    launch_dim_stats_init(ds, d, d_maxabs, d_bad, st);
    launch_dim_stats(dx, 8, n, d, eps, ds, d_maxabs, d_bad, st);
    cudaMemcpyAsync(c->h_small, c->d_small, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return check_cuda("cell statistics");
    if ((uint32_t)c->h_small[1]) return fail(HJ_ERR_INVALID_ARG, "non-finite coordinate or cell out of range");
    std::vector<uint32_t> ord;
    std::vector<unsigned long long> costs;
    if (int r = dim_order_by_cost(c, st, dx, 8, n, d, eps, ds, &ord, &costs)) return r;
    for (uint32_t pos = 0; pos < d; ++pos) reorder_dim[ord[pos]] = (int32_t)pos;
    if (costs_out)
        for (uint32_t t = 0; t < d; ++t) costs_out[t] = costs[t];
    return HJ_OK;
}

int engine_fail(int code, const std::string &msg) { return fail(code, msg); }

void engine_clear_error() { tl_error.clear(); }

uint64_t engine_ctx_bytes(int device) {
    auto it = tl_ctx.find(device);
    if (it == tl_ctx.end()) return 0;
    uint64_t b = 0;
    for (const auto &s : it->second->slots) b += s.second;
    return b;
}

void engine_ctx_trim(int device, cudaStream_t st) {
    auto it = tl_ctx.find(device);
    if (it == tl_ctx.end()) return;
    Ctx *c = it->second;
    cudaSetDevice(device);
    if (st) cudaStreamSynchronize(st);
    cudaStreamSynchronize(c->stream);
    for (auto &s : c->slots) {
        if (s.first) cudaFree(s.first);
        s = {nullptr, 0};
    }
    cudaGetLastError();
}

// Device memory one join takes in the calling thread's context, from the
// buffers prepare_set, the index and run_join allocate, with the key width
// bounded by 6 bits per dim (cell ranges up to 60 cells per dim; wider key
// words are rare and are measured after the join) and the band queue at its
// first size (a larger band regrows it; the server measures that too).
uint64_t engine_join_bytes_estimate(uint64_t na, uint64_t nb, uint32_t d, int dtype_bytes, int form, bool self,
                                    bool block_centring) {
    const uint64_t W = (6ull * d + 31) / 32 + 1;
    const bool tc = form_is_tc(form) || form == HJ_FORM_AUTO;
    const bool bc = block_centring && form != HJ_FORM_PLAIN_FP64 && d <= kBcMaxDim;
    auto per_set = [&](uint64_t n) -> uint64_t {
        const uint64_t npad = hj_ceil_div(std::max<uint64_t>(n, 1), kTcTileB) * kTcTileB;
        uint64_t b = n * d * (uint64_t)dtype_bytes;          // sorted rows
        b += n * (2 * W + 1) * 4 + n * 8;                     // packed keys (both layouts), permutation
        b += npad * d * 8;                                    // plain FP64 tiles (plain form or routed items)
        if (tc) b += npad * (hj_ceil_div(d, 64) * 64) * 4 + npad * 8;  // operands (widest form), norms
        if (bc)  // block-centred operand rows, q, |h|, blocks
            b += npad * 4 * bc_dp(d, HJ_FORM_TC_TF32) * 4 + npad * 8 + (npad / kBcBlock) * (16 + kBcCentStride * 4);
        // (TF32 rows, 4 bytes a column, bound the BF16 hi + lo pair too)
        return b;
    };
    uint64_t b = per_set(na) + (self ? 0 : per_set(nb));
    const uint64_t nmax = std::max(na, nb);
    b += radix_scratch_bytes(nmax) + 2 * radix_scratch_bytes(1);
    // work list: per A tile up to kMaxCombos runs, items of a few B tiles; the
    // A rows' packed bound keys (two of W words)
    const uint64_t tiles = hj_ceil_div(std::max<uint64_t>(na, 1), kPlainTile);
    b += tiles * (uint64_t)kMaxCombos * 8 + tiles * 64 * 16 + na * W * 8;
    if (tc) {
        const double cand = (double)na * (double)nb;
        b += (uint64_t)std::max(1048576.0, cand / (bc ? (form == HJ_FORM_TC_BF16X3 ? 256.0 : 512.0) : 4096.0)) *
             kBandEntryBytes;
    }
    return b + (16ull << 20);
}

int engine_prepare_job(cudaStream_t st_in, const void *a, const void *b, uint64_t na, uint64_t nb, int dtype_bytes,
                       uint32_t d, double eps, bool self, const hj_opts *opts, int form, PreparedJob *out) {
    if (!form_is_tc(form)) return fail(HJ_ERR_INVALID_ARG, "a batch runs a tensor-core form");
    if (dtype_bytes != 4 && dtype_bytes != 8) return fail(HJ_ERR_INVALID_ARG, "dtype_bytes must be 4 or 8");
    if (!a || (!self && !b) || na == 0 || (!self && nb == 0)) return fail(HJ_ERR_INVALID_ARG, "empty or null job");
    if (int r = validate(na, nb, d, eps)) return r;
    Ctx *c;
    if (int r = get_ctx(opts ? opts->device : -1, &c)) return r;
    cudaStream_t st = st_in ? st_in : c->stream;
    JoinIn in{a, self ? a : b, na, self ? na : nb, dtype_bytes, d, eps, self};
    Prepared P;
    if (int r = prepare_join(c, st, in, opts, form, &P)) return r;
    PreparedJob &J = *out;
    J = PreparedJob();
    J.A = P.A;
    J.B = P.B;
    J.na_eff = P.na_eff;
    J.nb_eff = P.nb_eff;
    J.op_scale = P.A.op_scale;
    J.maxabs = P.maxabs;
    J.form = P.form;
    J.num_sms = c->num_sms;
    int launches = P.launches;
    tc_band_constants(P.form, d, P.maxabs, &J.c_rel, &J.c_abs);
    const double T_tc = eps * eps * J.op_scale * J.op_scale;
    AllocCtx actx{c, st};
    int sr = split_items_by_precision(P.idx, J.A, J.B, J.c_rel, J.c_abs, 0.5 * T_tc, nullptr, slot_alloc_cb, &actx,
                                      st, &J.idx_tc, &J.idx_fp);
    if (sr == 2) return fail(HJ_ERR_OOM, "out of device memory (work list split)");
    if (sr) return check_cuda("work list split");
    launches += 2;
    if (J.idx_fp.n_items) {
        if (int rr = ensure_plain_tiles(c, st, &J.A, false, &launches)) return rr;
        if (self)
            J.B.tiles64 = J.A.tiles64, J.B.n_tiles64 = J.A.n_tiles64;
        else if (int rr = ensure_plain_tiles(c, st, &J.B, true, &launches))
            return rr;
    }
    J.launches = launches;
    return check_cuda("batch job preparation");
}

static int stripes_to_active_dims(int stripes) {
    int s = 0, p3 = 1;
    while (s < kMaxActiveDims && (p3 + 1) / 2 < stripes) {
        ++s;
        p3 *= 3;
    }
    return s;
}

}  // namespace hj

using namespace hj;

extern "C" {

void hj_opts_init(hj_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->form = HJ_FORM_PLAIN_FP64;
    o->active_dims = -1;
    o->device = -1;
}

const char *hj_status_str(int s) {
    switch (s) {
        case HJ_OK: return "ok";
        case HJ_ERR_INVALID_ARG: return "invalid argument";
        case HJ_ERR_OOM: return "out of device memory";
        case HJ_ERR_CUDA: return "CUDA error";
        case HJ_ERR_TIMEOUT: return "device wait timed out";
        case HJ_ERR_BAND_OVERFLOW: return "band queue overflow";
        case HJ_ERR_NO_DEVICE: return "no usable device";
        case HJ_ERR_UNSUPPORTED: return "unsupported input for this form";
        case HJ_ERR_BUSY: return "rejected by admission";
        case HJ_ERR_NOT_FOUND: return "not found";
        case HJ_ERR_CAPACITY: return "output buffer too small";
        default: return "unknown status";
    }
}

const char *hj_last_error(void) { return hj::tl_error.c_str(); }

const char *hj_version(void) { return "hj 1.0.0 sm_100a"; }

int hj_device_sm_count(int device) {
    int dev = device, sms = 0;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return sms;
}

int hj_self_join_count(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts, uint64_t *count,
                       hj_stats *stats) {
    return join_host(pts, n, pts, n, 8, d, eps, true, opts, count, stats);
}

int hj_self_join_count_f32(const float *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts,
                           uint64_t *count, hj_stats *stats) {
    return join_host(pts, n, pts, n, 4, d, eps, true, opts, count, stats);
}

int hj_join_count(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d, double eps,
                  const hj_opts *opts, uint64_t *count, hj_stats *stats) {
    return join_host(A, nA, B, nB, 8, d, eps, false, opts, count, stats);
}

int hj_join_count_f32(const float *A, uint64_t nA, const float *B, uint64_t nB, uint32_t d, double eps,
                      const hj_opts *opts, uint64_t *count, hj_stats *stats) {
    return join_host(A, nA, B, nB, 4, d, eps, false, opts, count, stats);
}

int hj_self_join_pairs(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts, uint64_t *pairs,
                       uint64_t capacity, uint64_t *n_pairs, hj_stats *stats) {
    return pairs_host(pts, n, pts, n, 8, d, eps, true, opts, pairs, capacity, n_pairs, stats);
}

int hj_self_join_pairs_f32(const float *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts,
                           uint64_t *pairs, uint64_t capacity, uint64_t *n_pairs, hj_stats *stats) {
    return pairs_host(pts, n, pts, n, 4, d, eps, true, opts, pairs, capacity, n_pairs, stats);
}

int hj_join_pairs(const double *A, uint64_t nA, const double *B, uint64_t nB, uint32_t d, double eps,
                  const hj_opts *opts, uint64_t *pairs, uint64_t capacity, uint64_t *n_pairs, hj_stats *stats) {
    return pairs_host(A, nA, B, nB, 8, d, eps, false, opts, pairs, capacity, n_pairs, stats);
}

int hj_join_pairs_f32(const float *A, uint64_t nA, const float *B, uint64_t nB, uint32_t d, double eps,
                      const hj_opts *opts, uint64_t *pairs, uint64_t capacity, uint64_t *n_pairs, hj_stats *stats) {
    return pairs_host(A, nA, B, nB, 4, d, eps, false, opts, pairs, capacity, n_pairs, stats);
}

int hj_dim_order(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts, int32_t *reorder_dim,
                 uint64_t *costs) {
    return dim_order_host(pts, n, d, eps, opts, reorder_dim, costs);
}

int hj_ego_sort(const double *pts, uint64_t n, uint32_t d, double eps, const hj_opts *opts, uint64_t *perm,
                double *sorted) {
    return ego_sort_host(pts, n, d, eps, opts, perm, sorted);
}

int hj_debug_tc_estimates(const float *A, uint64_t nA, const float *B, uint64_t nB, uint32_t d, int form,
                          float *out) {
    return hj_debug_tc_estimates_ex(A, nA, B, nB, d, form, HJ_CENTRING_GLOBAL, 0.0, out, nullptr);
}

int hj_debug_tc_estimates_ex(const float *A, uint64_t nA, const float *B, uint64_t nB, uint32_t d, int form,
                             int centring, double eps, float *out, hj_stats *stats) {
    tl_error.clear();
    if (!A || !B || !out || nA == 0 || nB == 0) return fail(HJ_ERR_INVALID_ARG, "null pointer or empty set");
    if (!form_is_tc(form)) return fail(HJ_ERR_INVALID_ARG, "not a tensor-core form");
    Ctx *c;
    if (int r = get_ctx(-1, &c)) return r;
    float *dbg = nullptr;
    if (cudaMalloc(&dbg, nA * nB * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        return fail(HJ_ERR_OOM, "out of device memory");
    }
    cudaMemset(dbg, 0xff, nA * nB * sizeof(float));  // NaN: pairs outside the work list
    double mx = 0;
    for (uint64_t i = 0; i < nA * d; ++i) mx = std::fmax(mx, std::fabs((double)A[i]));
    for (uint64_t i = 0; i < nB * d; ++i) mx = std::fmax(mx, std::fabs((double)B[i]));
    hj_opts o;
    hj_opts_init(&o);
    o.form = form;
    o.active_dims = 0;
    o.tc_centring = centring;
    uint64_t cnt;
    set_tc_debug_output(dbg);
    const double e = eps > 0 ? eps : 4.0 * (mx + 1.0) * std::sqrt((double)d);
    int r = hj_join_count_f32(A, nA, B, nB, d, e, &o, &cnt, stats);
    set_tc_debug_output(nullptr);
    if (r == HJ_OK && cudaMemcpy(out, dbg, nA * nB * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        r = check_cuda("debug copy");
    cudaFree(dbg);
    return r;
}

int hj_debug_set_wait_gate(uint64_t gate_ns) {
    tl_error.clear();
    if (gate_ns > kWaitLimitNs) return fail(HJ_ERR_INVALID_ARG, "gate longer than the wait limit");
    set_tc_wait_gate(gate_ns);
    return HJ_OK;
}

int hj_self_join_count_device(const void *pts, int dtype_bytes, uint64_t n, uint32_t d, double eps,
                              const hj_opts *opts, uint64_t *count, hj_stats *stats) {
    return join_device(pts, n, pts, n, dtype_bytes, d, eps, true, opts, count, stats);
}

int hj_join_count_device(const void *A, uint64_t nA, const void *B, uint64_t nB, int dtype_bytes, uint32_t d,
                         double eps, const hj_opts *opts, uint64_t *count, hj_stats *stats) {
    return join_device(A, nA, B, nB, dtype_bytes, d, eps, false, opts, count, stats);
}

void hj_test_ego_loop3_macro(size_t n, size_t d, double epsilon, double *array, size_t *countresult, int stripes,
                             double *sortTime, double *indextime, double *loadpercent) {
    hj_opts o;
    hj_opts_init(&o);
    o.ref_compat = 1;
    o.active_dims = stripes_to_active_dims(stripes);
    hj_stats s;
    uint64_t c = 0;
    int r = hj_self_join_count(array, n, (uint32_t)d, epsilon, &o, &c, &s);
    if (countresult) *countresult = r == HJ_OK ? (size_t)c : 0;
    if (sortTime) *sortTime = r == HJ_OK ? s.sort_ms / 1e3 : 0.0;
    if (indextime) *indextime = r == HJ_OK ? s.index_ms / 1e3 : 0.0;
    if (loadpercent) *loadpercent = r == HJ_OK ? s.loadpercent : 0.0;
}

void hj_test_ego_loop3_noself(const size_t nA, const size_t nB, const int d, const double epsilon, double *arrayA,
                              double *arrayB, size_t *countresult, const int activedims, double *sortTime,
                              double *indextime, double *loadpercent) {
    (void)activedims;
    hj_opts o;
    hj_opts_init(&o);
    o.ref_compat = 1;
    o.active_dims = 2;
    hj_stats s;
    uint64_t c = 0;
    int r = hj_join_count(arrayA, nA, arrayB, nB, (uint32_t)d, epsilon, &o, &c, &s);
    if (countresult) *countresult = r == HJ_OK ? (size_t)c : 0;
    if (sortTime) *sortTime = r == HJ_OK ? s.sort_ms / 1e3 : 0.0;
    if (indextime) *indextime = r == HJ_OK ? s.index_ms / 1e3 : 0.0;
    if (loadpercent) *loadpercent = r == HJ_OK ? s.loadpercent : 0.0;
}

}  // extern "C"
