// hj_internal.h -- declarations shared by the engine's translation units:
// device-side set layouts, the cell grid, and the kernel launch wrappers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string.h>

#include <string>
#include <vector>

#include "../../include/hj.h"

namespace hj {

// Point-tile sizes of the two distance kernels.
constexpr int kPlainTile = 64;   // plain FP64 kernel: 64 x 64 point tiles
constexpr int kTcTileA = 128;    // tensor-core kernel: 128 A rows (UMMA M) ...
constexpr int kTcTileB = 256;    // ... against 256 B rows (UMMA N)
constexpr int kMaxActiveDims = 5;
constexpr int kMaxCombos = 243;  // 3^kMaxActiveDims
constexpr uint32_t kMaxDim = 1024;

// Per-dimension summary of one set (or of the union of two sets) computed on
// the device: cell index range and the largest |coordinate|.
struct DimStats {
    long long cmin, cmax;
    unsigned long long xmin, xmax;  // coordinate range, order-preserving encoding of the FP64 bits
};

// FP64 <-> unsigned integer with the same order (for atomic min/max).
__host__ __device__ inline unsigned long long ordered_from_double(double v) {
    unsigned long long u;
    memcpy(&u, &v, 8);
    return (u >> 63) ? ~u : (u | (1ull << 63));
}
__host__ __device__ inline double double_from_ordered(unsigned long long u) {
    u = (u >> 63) ? (u & ~(1ull << 63)) : ~u;
    double v;
    memcpy(&v, &u, 8);
    return v;
}

// The epsilon grid shared by the sets of one join. Cell of a coordinate x in
// dim t: c = floor(x / eps) (FP64). A packed key stores per dim the field
// digit = clamp(c - off[t], 0, 2^bits[t] - 1), fields placed from the most
// significant bit of word 0 downward in dim order (never split across words),
// so comparing keys word by word as unsigned integers is the lexicographic
// comparison of cell vectors (the EGO order of hilbertjoin/egojoin.cpp:9-17).
// off[t] = min cell - 2 leaves room for the neighbour-cell queries (cell - 1,
// cell + 1, and one more for cells that jitter at borders).
struct Grid {
    uint32_t d = 0;
    double eps = 0, eps_wide = 0, maxabs = 0;
    uint32_t W = 0;                    // 32-bit words per key
    std::vector<long long> off;        // per dim
    std::vector<uint32_t> bits, word, shift;
    std::vector<long long> range;      // max cell - min cell per dim
    // radix passes: (word, low bit) of each 8-bit digit window that can vary
    std::vector<std::pair<uint32_t, uint32_t>> passes;
    // key position -> dim: fields are packed, and stripes take their active
    // dims, in this order (identity unless the dims are reordered)
    std::vector<uint32_t> ord;
};

// Device copy of the grid's per-dim packing tables (indexed by dim) and of the
// position order (nullptr = identity).
struct GridDev {
    long long *off = nullptr;
    uint32_t *bits = nullptr, *word = nullptr, *shift = nullptr;
    uint32_t *ord = nullptr;
};
__host__ __device__ inline uint32_t grid_dim_at(const GridDev &g, uint32_t pos) { return g.ord ? g.ord[pos] : pos; }

// Dimension cost for reordering: per dim, the number of unordered pairs of a
// fixed sample (min(n, kCostSample) points at floor(s n / S)) whose cells are
// equal or adjacent. One block per dim; cost[d] zeroed by the kernel.
constexpr uint32_t kCostSample = 8192;
void launch_dim_cost(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, const DimStats *ds,
                     unsigned long long *cost, cudaStream_t st);

// A point set after EGO sorting, in every layout the kernels need. Rows are
// in EGO rank order; `perm[r]` is the input index of rank r.
struct SortedSet {
    uint64_t n = 0;
    uint32_t d = 0;
    int dtype_bytes = 8;         // precision of the input (8 = FP64, 4 = FP32)
    const void *src = nullptr;   // the input rows (device), in input order
    const void *rows = nullptr;  // sorted rows, input precision, [n][d]
    uint32_t *keys = nullptr;    // sorted packed keys, [n][W]
    uint32_t *perm = nullptr;
    // plain FP64 kernel layout: [tile][d][64] (tile = 64 ranks), zero padded
    double *tiles64 = nullptr;
    uint64_t n_tiles64 = 0;
    // tensor-core layouts: [npad][kpad] with npad a multiple of 256
    float *tf32 = nullptr;       // TF32-rounded values in FP32 containers, kpad = roundup(d, 32)
    uint16_t *bf_hi = nullptr;   // BF16 split (or the FP16 operand), kpad16 = roundup(d, 64)
    uint16_t *bf_lo = nullptr;
    const double *center = nullptr;  // per-dim shift of the tensor-core operands (shared by A and B)
    double op_scale = 1.0;       // FP16 form: power of two applied to operands (norms: its square)
    float *norms = nullptr;      // FP32(|x - center|^2 in FP64); padding rows hold kPadNorm
    float *tile_maxnorm_a = nullptr;  // per kTcTileA-row tile
    float *tile_maxnorm_b = nullptr;  // per 256-row tile
    float *group_minnorm = nullptr;   // per 32-row group: min |x - center|^2
    uint64_t npad_tc = 0;
    uint32_t kpad_tf32 = 0, kpad_bf16 = 0;
    // per-block centring of the FP16 / TF32 operands (HJ_CENTRING_BLOCK; see
    // BcConsts): [npad][4 bc_dp] rows (FP16, or TF32 values in FP32 containers);
    // the B operand is the window at column 0, the A operand the window at column
    // bc_dp, both 3 bc_dp wide
    void *bc_op = nullptr;
    void *bc_op_lo = nullptr;  // BF16x3: the low BF16 halves of the same rows
    uint32_t bc_dp = 0;
    int bc_form = 0;
    float *bc_norms = nullptr;    // q = |h|^2 + 2 h.c per rank (FP32; padding rows kPadNorm)
    float *bc_xn = nullptr;       // |h| per rank, rounded up
    float4 *bc_blk = nullptr;     // per 128-rank block: {max |h|, |c|, max |q|, 0}, rounded up
    float *bc_cent = nullptr;     // per block: c in FP32 (FP16 values), kBcCentStride floats, zero padded
};

// Per-block centring of the tensor-core operands (FP16, TF32, or BF16 hi + lo
// pairs). Every 128-rank block of a sorted set (one A tile, half a B tile) gets
// a centre c whose coordinates are values of the operand type in the operand
// units ((x - center) * scale, the largest coordinate below 2^10), the
// midpoint of the block's range rounded; every rank is stored as that centre
// plus its residual h = fl(x - c), rounded to the operand type. With
// q = |h|^2 + 2 h.c per rank and three pieces of q / 2 (FP16: m1 2^15 +
// m2 2^4 + m3 2^-7; TF32 and BF16: m1 + m2 + m3; to 2^-33 |q|), a row holds four
// blocks of dp = roundup(d + 3, 8) columns (TF32: roundup(d + 3, 4); zero padded),
//     [h | h | c m1 m2 m3 | h a1 a2 a3],   (a1, a2, a3) = (-2^15, -2^4, -2^-7) (else -1, -1, -1),
// and the operands are two windows of 3 dp columns of the same rows:
//     B = columns [0, 3dp) = [h | h | c m],   A = columns [dp, 4dp) = [h | c m | h a].
// Column by column the products are h_i.h_j, c_i.h_j (m_i meets B's zero pad),
// h_i.c_j and a.m_j, so one MMA gives, for the operand points x' = c + h,
//     w_ij = h_i.h_j + c_i.h_j + h_i.c_j - q_j / 2 = x'_i.x'_j - c_i.c_j - q_j / 2,
//     dist2(x'_i, x'_j) = q_i + |c_i - c_j|^2 - 2 w_ij.
// (The A window's last atom reaches past the row end: the TMA fills zeros.)
// The accumulator alone orders the columns of a row (no per-column norm), so
// the epilogue's maximum over 32 columns is exact. The only rounding of the
// points is h's (relative 2^-11 per coordinate for FP16 and TF32, 2^-17 for the
// BF16 pair): it moves a point by rho <= 2^-11 |h| (2^-17 |h| for the pair; plus
// the subnormal floor), and distances by rho_i + rho_j.
// The error bound (bc_tau) is therefore linear in the residual norms instead
// of quadratic in the distance from one global centre, which keeps clustered
// data with eps far below its spread on the tensor cores.
constexpr uint32_t kBcBlock = 128;      // ranks per centring block (= kTcTileA, = kTcTileB / 2)
constexpr uint32_t kBcMaxDim = 64;      // dp <= 72: windows of <= 216 columns
constexpr uint32_t kBcCentStride = 64;  // floats per block in bc_cent
constexpr int kBcScaleShift = 5;        // operand scale of the global form times 2^-5
// block width of the rows: 16-byte multiples (TMA column offsets), FP16 8, TF32 4 columns
inline uint32_t bc_dp(uint32_t d, int form) {
    const uint32_t g = form == HJ_FORM_TC_TF32 ? 4u : 8u;
    return (d + 3 + g - 1) / g * g;
}
inline uint32_t bc_cols(uint32_t d, int form) { return 3 * bc_dp(d, form); }  // columns of an operand window
inline uint32_t bc_elem_bytes(int form) { return form == HJ_FORM_TC_TF32 ? 4u : 2u; }
struct BcConsts {
    float kp21;     // 2 kpad_bc 2^-22: the MMA accumulation error of w per unit of S, doubled for s
    float eps;      // eps in operand units, rounded up
    float rho_u;    // rounding radius per unit of |h| (2^-11 with margin)
    float rho_c;    // rounding radius floor (FP16 subnormals, FP64 shift), per point
    float u_norm;   // FP32 rounding of q, and the FP16 split of q / 2 (relative, with margin)
    float u_d;      // FP32 rounding of D = |c_i - c_j|^2 (relative)
    float theta_t;  // rounding of the FP64 pair test near eps^2, twice, in operand units
};
// Half-width of the band of s around eps^2 for a pair of a row (|h| = xa, its
// block's |c| = ca, |q| = pa) and a B block (max |h| = xb, |c| = cb, max |q| =
// qb) at block-centre distance^2 D; *S_out = the bound on sum_k |A_ik B_jk|
// (Cauchy-Schwarz per column group, and |q_j| / 2 for the folded pieces).
// With E = |s - dist2(x'_i, x'_j)| <= kp21 S + u_norm (pa + qb) + u_d D and
// rho = rho_i + rho_j: dist2 <= s + E + 2 rho sqrt(s + E) + rho^2, and
// 2 rho sqrt(E) <= rho^2 + E, so near eps^2 the FP64 test agrees with
// "s + tau <= eps^2 is inside, s - tau > eps^2 is outside" for
// tau = 2 E + 2 eps rho + 2 rho^2 + theta_t (times 1.25 for the FP32 of this
// function).
__host__ __device__ inline float bc_tau(float xa, float ca, float pa, float xb, float cb, float qb, float D,
                                        const BcConsts &k, float *S_out) {
    const float S = fmaf(xa, xb + cb, fmaf(ca, xb, 0.5005f * qb));
    const float rho = fmaf(k.rho_u, xa + xb, 2.0f * k.rho_c);
    const float E = fmaf(k.kp21, S, fmaf(k.u_norm, pa + qb, k.u_d * D));
    if (S_out) *S_out = S;
    return 1.25f * fmaf(2.0f, E, fmaf(2.0f * k.eps, rho, fmaf(2.0f * rho, rho, k.theta_t)));
}
// Fills the constants for form (FP16 or TF32), dimension d, eps^2 = T (caller
// units) and the block-centred operand scale.
BcConsts bc_constants(int form, uint32_t d, double T, double op_scale);
// Block centres, the operand rows ([npad][4 dp]), q, |h| and block summaries
// of a sorted set from its sorted rows. center = the global per-dim shift,
// scale = the block-centred operand scale.
void launch_bc_prepare(const SortedSet &s, const double *center, double scale, void *op, void *op_lo, float *norms,
                       float *xn, float4 *blk, float *cent, cudaStream_t st, int *launches);

constexpr float kPadNorm = 1.0e30f;

// Work item of the persistent distance kernels: A tile `a` against the B tiles
// [b0, b1). Produced by the index stage in Hilbert order.
struct WorkItem {
    uint32_t a, b0, b1, pad;
};

// Splits a tensor-core work list (128 x 256 tiles) by precision: items whose
// error bound c_rel * (max |a|^2 + max |b|^2) + c_abs exceeds `limit` go, as
// 64 x 64 items, to the plain FP64 kernel. Order (Hilbert) is preserved in both
// lists. Synchronises once on `st`.
// First scratch-slot id of the index stage (build_index, the precision split,
// sharding); the engine's own slot ids stay below it.
constexpr int kSlotIndexFirst = 64;

struct IndexResult;
// With bc non-null the bound is the per-block-centred one (bc_tau with the
// sets' block summaries, D = 0) and c_rel / c_abs are unused.
int split_items_by_precision(const IndexResult &tc_in, const SortedSet &A, const SortedSet &B, double c_rel,
                             double c_abs, double limit, const BcConsts *bc,
                             void *(*alloc)(void *ctx, int slot, size_t bytes), void *actx, cudaStream_t st,
                             IndexResult *tc_out, IndexResult *fp_out);

// Restricts a work list to shard k of K: the contiguous item range whose
// cumulative tile-pair load lies in [k L / K, (k+1) L / K) (L = total load).
// Synchronises once on `st`.
int shard_items(const IndexResult &in, int k, int K, void *(*alloc)(void *ctx, int slot, size_t bytes), void *actx,
                cudaStream_t st, IndexResult *out);

struct IndexResult {
    WorkItem *items = nullptr;  // device, Hilbert ordered
    uint64_t n_items = 0;
    uint64_t tile_pairs = 0;
    uint64_t candidate_pairs = 0;
};

// Raises a kernel's dynamic shared memory limit to `bytes` on the current
// device, once, and never lowers it: the attribute is global to the function,
// so per-call values would race between host threads launching the same
// kernel with different sizes.
void ensure_max_dynamic_smem(const void *func, int bytes);

// ---- launch wrappers (all asynchronous on `st` unless noted) ----------------

// Per-dim min/max cell, max |x|, non-finite flag over a row-major set; results
// accumulate into dstats[d], d_maxabs_bits, d_bad (initialised by the caller).
void launch_dim_stats(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, DimStats *dstats,
                      unsigned long long *d_maxabs_bits, uint32_t *d_bad, cudaStream_t st);
void launch_dim_stats_init(DimStats *dstats, uint32_t d, unsigned long long *d_maxabs_bits, uint32_t *d_bad,
                           cudaStream_t st);

// Packed keys, word-major [W][n].
// With norm_key non-null, the quantised norm key (launch_norm_key) of every
// point is written in the same pass.
void launch_pack_keys(const void *x, int dtype_bytes, uint64_t n, uint32_t d, double eps, const GridDev &g,
                      uint32_t W, uint32_t *keys_wm, cudaStream_t st, const double *center = nullptr,
                      double norm_scale = 0.0, uint32_t *norm_key = nullptr);

// Quantised |x - center|^2 (16 bits, key = min(65535, floor(norm * scale))),
// the least significant sort key of the tensor-core forms: points of one cell
// end up ordered by norm, so that 32 consecutive ranks have near-equal norms.
void launch_norm_key(const void *x, int dtype_bytes, uint64_t n, uint32_t d, const double *center, double scale,
                     uint32_t *key_out, cudaStream_t st);

// Stable LSD radix sort of a permutation by 8-bit windows of word-major keys
// ([word][n]); `passes` = (word, shift) in order, least significant first.
// Needs radix_scratch_bytes(n) of 16-byte aligned device scratch. Result:
// perm_out[r] = input index of rank r (identity when there is no pass).
size_t radix_scratch_bytes(uint64_t n);
void radix_sort_perm(const uint32_t *keys_wm, uint64_t n, const std::pair<uint32_t, uint32_t> *passes, size_t np,
                     uint32_t *perm_out, void *scratch, cudaStream_t st, int *launches);
void radix_sort_perm(const uint32_t *keys_wm, uint64_t n, const std::vector<std::pair<uint32_t, uint32_t>> &passes,
                     uint32_t *perm_out, void *scratch, cudaStream_t st, int *launches);
void launch_iota(uint32_t *p, uint64_t n, cudaStream_t st);
// Exclusive scan of u32 entries in place; total into *total if non-null. With
// `tile_sums` (scan_scratch_bytes(count) of device scratch) it runs over many
// blocks, else in one block.
size_t scan_scratch_bytes(uint64_t count);
void launch_scan_u32(uint32_t *a, uint64_t count, unsigned long long *total, cudaStream_t st,
                     unsigned long long *tile_sums = nullptr);

// Gathers the sorted layouts of a set (flags select the layouts to build).
enum GatherFlags : uint32_t { kGatherRows = 1, kGatherKeys = 2, kGatherPlain = 4, kGatherTf32 = 8, kGatherBf16 = 16,
                              kGatherNorms = 32, kGatherF16 = 64 };
void launch_gather(const void *x, int dtype_bytes, uint64_t n, uint32_t d, const uint32_t *perm,
                   const uint32_t *keys_wm, uint32_t W, const SortedSet &out, uint32_t flags, cudaStream_t st,
                   int *launches);

// Index stage: per A tile the stripe ranges into B's EGO order, merged into
// runs of B tiles; expanded into work items of at most `chunk` B tiles and
// sorted in Hilbert order. Synchronises once on `st` (item count).
struct IndexScratch;
int build_index(const SortedSet &A, const SortedSet &B, const Grid &grid, const GridDev &gdev, bool self,
                uint64_t na_eff, uint64_t nb_eff, int tile_a, int tile_b, int active_dims, uint32_t chunk,
                void *(*alloc)(void *ctx, int slot, size_t bytes), void *alloc_ctx, cudaStream_t st,
                IndexResult *out, int *launches, std::string *err);

// Plain FP64 distance kernel over the work list. Adds into *d_count.
void launch_join_fp64(const SortedSet &A, const SortedSet &B, bool self, uint64_t na_eff, uint64_t nb_eff,
                      double T, const IndexResult &idx, unsigned long long *d_count, uint32_t *d_err,
                      int num_sms, cudaStream_t st);

// Pair materialisation on the FP64 kernel. out_i == nullptr: adds each item's
// pair count into item_cnt[item] (zeroed by the caller). Otherwise item_cnt
// holds each item's first output slot (exclusive scan of the counts) and the
// kernel writes the pairs of input indices there (self joins as i < j), in no
// particular order within an item.
void launch_pairs_fp64(const SortedSet &A, const SortedSet &B, bool self, uint64_t na_eff, uint64_t nb_eff,
                       double T, const IndexResult &idx, uint32_t *item_cnt, uint32_t *out_i, uint32_t *out_j,
                       uint32_t *d_err, int num_sms, cudaStream_t st);

// Tensor-core kernel + FP64 recheck of the band. Adds into each job's count;
// band slots reserved into *d_band_total (may exceed `band_cap`: then the
// caller regrows), of which *d_band_holes were left unused (the recheck skips
// them). Band entries are 16 bytes (kBandEntryBytes).
constexpr size_t kBandEntryBytes = 16;
// One join of a tensor-core launch. A launch runs the work items of one or
// more jobs (WorkItem.pad = job index) over operand matrices whose rows hold
// all jobs' sets; rows are global ranks of those matrices.
struct TcJob {
    uint64_t a_row0, a_end;       // counted A ranks: [a_row0, a_end)
    uint64_t b_row0, b_end;       // counted B ranks: [b_row0, b_end)
    double T;                     // eps^2 (FP64), for the recheck
    unsigned long long *count;    // where the job's count accumulates
    const void *rows_a, *rows_b;  // sorted rows (input precision); rank r at (r - row0) * d
    float T_lo, T_hi;             // eps^2 in operand units, rounded down / up to FP32
    float c_rel_f, c_abs_f;       // error bound constants, rounded up to FP32
    float s_unscale;              // 1 / op_scale^2 (exact): estimates back to the caller's units
    uint32_t self;                // unordered pairs within one set (A = B)
    uint32_t ka;                  // K atoms of this job's operands
    uint32_t ksteps;              // MMA K steps of this job (16 columns each; TF32 8): the columns
                                  // holding data, rounded up; zero columns beyond are not multiplied
    uint32_t d;
};
// Fills a job for form `form`, dimension d, eps^2 = T, FP16 operand scale
// op_scale (1 for other forms), largest |coordinate| maxabs. Returns the
// error-bound constants through c_rel / c_abs (operand units) if non-null.
void fill_tc_job(TcJob *j, int form, uint32_t d, double T, double op_scale, double maxabs, uint64_t a_row0,
                 uint64_t na_eff, uint64_t b_row0, uint64_t nb_eff, bool self, unsigned long long *count,
                 const void *rows_a, const void *rows_b, double *c_rel, double *c_abs);

// Launches the tensor-core kernel over `idx` with the job table d_jobs (device).
// A and B describe the operand matrices (layout pointers, npad_tc rows, kpad,
// norms and their tile maxima and group minima); their d is the largest of the
// jobs'. na0 / nb0: job 0's counted ranks (debug output only).
// With bc non-null (FP16 or TF32 form, one job): the per-block-centred
// operands of A and B (their windows) and summaries; the job's ka and ksteps
// must be the ones of bc_cols(d, form) columns (tc_atoms, tc_ksteps).
int launch_join_tc(const SortedSet &A, const SortedSet &B, int form, const TcJob *d_jobs, uint64_t na0, uint64_t nb0,
                   const IndexResult &idx, uint2 *band, uint64_t band_cap, unsigned long long *d_band_total,
                   uint32_t *d_err, int num_sms, cudaStream_t st, std::string *err, const BcConsts *bc = nullptr,
                   unsigned long long *d_band_holes = nullptr);
// K atoms (128-byte operand column groups) of a form's operand rows of kcols columns.
uint32_t tc_atoms(int form, uint32_t kcols);
// MMA K steps that cover kcols columns (16 per kind::f16 instruction, 8 per kind::tf32),
// and the product terms K they sum (the accumulation error model's K).
uint32_t tc_ksteps(int form, uint32_t kcols);
uint32_t tc_kterms(int form, uint32_t kcols);
// FP64 recheck of the band pairs, each against its job's rows and eps^2.
// vec_rows: every job's rows are 16-byte aligned with d * dtype_bytes a
// multiple of 16 (then the rows are read with 16-byte loads).
void launch_recheck(const TcJob *d_jobs, int dtype_bytes, const uint2 *band, const unsigned long long *d_band_total,
                    uint64_t band_cap, unsigned int *d_max_err_bits, cudaStream_t st, bool vec_rows = false);
// Test hook: when non-null, the tensor-core kernel writes its dist^2 estimate
// of every pair to dbg[ia * nb + jb] (EGO ranks). Not thread-safe.
void set_tc_debug_output(float *dbg);
// Test hook: with ns > 0 the tensor-core kernel's epilogue first waits ns on a
// barrier that nothing arrives on, then raises kErrTimeout (0 = off).
void set_tc_wait_gate(uint64_t ns);
// Error-bound constant of a tensor-core form for dimension d.
void tc_band_constants(int form, uint32_t d, double maxabs, double *c_rel, double *c_abs);

// ---------------------------------------------------------------- batching
// One job prepared by the engine for a batched tensor-core launch: its sorted
// sets in every layout the kernels need and its work list split by precision.
// All pointers live in the calling thread's engine buffers and stay valid
// only until that thread's next engine call.
struct PreparedJob {
    SortedSet A, B;
    IndexResult idx_tc, idx_fp;  // tensor-core items; items routed to the FP64 kernel (64 x 64 tiles)
    uint64_t na_eff = 0, nb_eff = 0;
    double op_scale = 1.0, maxabs = 0.0, c_rel = 0.0, c_abs = 0.0;
    int form = 0;
    int launches = 0;
    int num_sms = 0;
};
// Prepares one join (device inputs) for tensor-core form `form` on the current
// device: cell statistics, EGO sort, layouts, index, precision split, and
// the plain FP64 tiles when items were routed to the FP64 kernel. Synchronises
// `st` a few times (planning read-backs). Returns an hj_status.
int engine_prepare_job(cudaStream_t st, const void *a, const void *b, uint64_t na, uint64_t nb, int dtype_bytes,
                       uint32_t d, double eps, bool self, const hj_opts *opts, int form, PreparedJob *out);
// Candidate pairs of every job of a planned batch (server statistics).
int batch_job_candidates(const hj_batch *b, uint64_t *out);
// Sets the calling thread's last error text and returns code.
int engine_fail(int code, const std::string &msg);
// Clears this host thread's error text (hj_last_error) at the start of a call.
void engine_clear_error();
// Device memory held by the calling thread's engine context on `device`
// (its reusable buffers), and their release once `st` and the context's own
// stream have drained.
uint64_t engine_ctx_bytes(int device);
void engine_ctx_trim(int device, cudaStream_t st);
// Upper estimate of the device memory one join takes in a context; with
// block_centring the per-block-centred operands and their first band queue
// are counted where that centring can be chosen (FP16 or auto form, d <= 64).
uint64_t engine_join_bytes_estimate(uint64_t na, uint64_t nb, uint32_t d, int dtype_bytes, int form, bool self,
                                    bool block_centring);
// Norm summaries over a row-major norm array of npad rows (padding rows hold
// kPadNorm): per A-tile and per B-tile maxima, per 32-row minima.
void launch_norm_summaries(const float *norms, uint64_t npad, float *tmax_a, float *tmax_b, float *gmin32,
                           cudaStream_t st);

}  // namespace hj
