// hj_batch.cu -- many joins in one persistent tensor-core launch.
//
// A batch holds joins of uneven n, d and eps (self-joins and two-set joins).
// Planning (hj_batch_create) prepares every job with the engine's own
// pipeline -- cell statistics, EGO sort, layouts, stripe index, Hilbert-ordered
// work list, precision split -- and copies what the distance kernels need into
// buffers the batch owns:
//   * one operand matrix holding every set's rows (row blocks of 256, in the
//     order A0, B0, A1, B1, ...; a self-join has one block), padded to the
//     largest K of the batch with zeros, which add nothing to a dot product;
//   * the sets' norms, with their per-tile maxima and 32-row minima;
//   * the sorted rows in input precision (for the FP64 recheck);
//   * one work list: each job's items, tile indices rebased onto the matrix,
//     the job index in WorkItem.pad;
//   * a job table (TcJob): counted rank ranges, eps^2 and bound constants in
//     the job's operand units (FP16 scale per job), K atoms, count target.
// Running (hj_batch_run) enqueues, without any host synchronisation: the
// count reset, ONE launch of the tensor-core kernel over the whole work list,
// the FP64 recheck of the band, and the FP64 kernel for the few jobs whose
// items were routed to it. A run can therefore be captured into a CUDA graph
// and replayed. hj_batch_counts waits for the last run and returns the counts.
//
// The reference has no counterpart: it runs one join per process
// (hilbertjoin/egojoin.cpp:777-907).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hj.h"
#include "hj_common.cuh"
#include "hj_internal.h"

using namespace hj;

namespace {

__global__ void k_fill_f32(float *p, uint64_t n, float v) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

__global__ void k_rebase_items(const WorkItem *__restrict__ in, uint64_t n, uint32_t a_off, uint32_t b_off,
                               uint32_t job, WorkItem *__restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const WorkItem w = in[i];
    out[i] = WorkItem{w.a + a_off, w.b0 + b_off, w.b1 + b_off, job};
}

// Items routed to the FP64 kernel, per job (rare: ill-conditioned jobs).
struct FpJob {
    uint32_t job = 0;
    SortedSet A, B;  // tiles64 (owned by the batch) and d
    IndexResult idx;
    uint64_t na_eff = 0, nb_eff = 0;
    bool self = false;
    double T = 0;
};

}  // namespace

struct hj_batch {
    int device = 0;
    int form = HJ_FORM_TC_FP16;
    int dtype = 4;
    int num_sms = 0;
    uint32_t n_jobs = 0, d_max = 0;
    cudaStream_t own = nullptr, last = nullptr;
    SortedSet ops;  // operand matrix view (A and B maps both use it)
    IndexResult idx;
    TcJob *d_jobs = nullptr;
    unsigned long long *d_counts = nullptr;
    uint2 *band = nullptr;
    uint64_t band_cap = 0;
    unsigned long long *d_band_total = nullptr;
    uint32_t *d_err = nullptr;
    unsigned int *d_maxerr = nullptr;
    std::vector<FpJob> fp;
    std::vector<void *> allocs;
    cudaStream_t alloc_stream = nullptr;  // planning stream: buffers are stream-ordered on it
    uint64_t candidate_pairs = 0, fp64_items = 0;
    std::vector<uint64_t> job_candidates;

    // Stream-ordered allocations (cudaMallocAsync): no device-wide
    // synchronisation, so batches built by concurrent server workers do not
    // stall each other's kernels.
    void *alloc(size_t bytes) {
        void *p = nullptr;
        if (cudaMallocAsync(&p, bytes ? bytes : 16, alloc_stream) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        allocs.push_back(p);
        return p;
    }
    ~hj_batch() {
        cudaStream_t fs = last ? last : alloc_stream;
        for (void *p : allocs) cudaFreeAsync(p, fs);
        if (fs) cudaStreamSynchronize(fs);
        if (own) cudaStreamDestroy(own);
    }
};

static int batch_enqueue(hj_batch *b, cudaStream_t st) {
    cudaMemsetAsync(b->d_counts, 0, b->n_jobs * sizeof(unsigned long long), st);
    cudaMemsetAsync(b->d_band_total, 0, 2 * sizeof(unsigned long long), st);  // slots reserved, left unused
    cudaMemsetAsync(b->d_err, 0, sizeof(uint32_t), st);
    cudaMemsetAsync(b->d_maxerr, 0, sizeof(unsigned int), st);
    std::string err;
    if (launch_join_tc(b->ops, b->ops, b->form, b->d_jobs, 0, 0, b->idx, b->band, b->band_cap, b->d_band_total,
                       b->d_err, b->num_sms, st, &err, nullptr, b->d_band_total + 1))
        return engine_fail(HJ_ERR_CUDA, err);
    launch_recheck(b->d_jobs, b->dtype, b->band, b->d_band_total, b->band_cap, b->d_maxerr, st);
    for (const FpJob &f : b->fp)
        launch_join_fp64(f.A, f.B, f.self, f.na_eff, f.nb_eff, f.T, f.idx, b->d_counts + f.job, b->d_err,
                         b->num_sms, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return engine_fail(HJ_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
    b->last = st;
    return HJ_OK;
}

// Waits for the last run; reports the device error word and band overflow.
static int batch_finish(hj_batch *b, uint64_t *band_total) {
    if (cudaStreamSynchronize(b->last) != cudaSuccess) {
        cudaError_t e = cudaGetLastError();
        return engine_fail(HJ_ERR_CUDA, std::string("batch run: ") + cudaGetErrorString(e));
    }
    uint32_t err = 0;
    unsigned long long bt[2] = {0, 0};
    cudaMemcpy(&err, b->d_err, sizeof(err), cudaMemcpyDeviceToHost);
    cudaMemcpy(bt, b->d_band_total, sizeof(bt), cudaMemcpyDeviceToHost);
    if (err & kErrTimeout) return engine_fail(HJ_ERR_TIMEOUT, "a bounded device-side wait timed out");
    if (err) return engine_fail(HJ_ERR_CUDA, "device error word set");
    if (band_total) *band_total = bt[0] - std::min(bt[0], bt[1]);  // band pairs: reserved slots less the unused
    if (bt[0] > b->band_cap) return engine_fail(HJ_ERR_BAND_OVERFLOW, "band queue overflow");
    return HJ_OK;
}

static uint64_t npad_rows(uint64_t n) { return hj_ceil_div(std::max<uint64_t>(n, 1), kTcTileB) * kTcTileB; }

static int batch_plan(const hj_batch_job *jobs, uint32_t n_jobs, int dtype_bytes, const hj_opts *opts,
                      hj_batch *b) {
    int form = opts ? opts->form : HJ_FORM_AUTO;
    if (form == HJ_FORM_AUTO) form = HJ_FORM_TC_FP16;
    if (form != HJ_FORM_TC_FP16 && form != HJ_FORM_TC_TF32 && form != HJ_FORM_TC_BF16X3)
        return engine_fail(HJ_ERR_UNSUPPORTED, "a batch runs a tensor-core form (fp16, tf32, bf16x3 or auto)");
    if (opts && opts->shard_count > 1) return engine_fail(HJ_ERR_UNSUPPORTED, "a batch is not sharded");
    if (dtype_bytes != 4 && dtype_bytes != 8) return engine_fail(HJ_ERR_INVALID_ARG, "dtype_bytes must be 4 or 8");
    if (n_jobs == 0 || !jobs) return engine_fail(HJ_ERR_INVALID_ARG, "no jobs");
    b->form = form;
    b->dtype = dtype_bytes;
    b->n_jobs = n_jobs;
    int dev = opts && opts->device >= 0 ? opts->device : -1;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) return engine_fail(HJ_ERR_NO_DEVICE, "no CUDA device");
    if (cudaSetDevice(dev) != cudaSuccess) return engine_fail(HJ_ERR_NO_DEVICE, "no CUDA device");
    b->device = dev;
    {
        // keep freed batch buffers in the device's default pool between batches
        // (the default threshold returns them to the system at every sync)
        static std::once_flag once[64];
        if (dev < 64)
            std::call_once(once[dev], [dev] {
                cudaMemPool_t pool;
                if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
                    uint64_t keep = ~0ull;
                    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
                }
                cudaGetLastError();
            });
    }
    cudaStream_t st = opts && opts->stream ? (cudaStream_t)opts->stream : nullptr;
    if (cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) != cudaSuccess)
        return engine_fail(HJ_ERR_CUDA, "cudaStreamCreate failed");
    if (!st) st = b->own;
    b->last = st;
    b->alloc_stream = st;
    b->job_candidates.assign(n_jobs, 0);

    // row layout of the operand matrix
    std::vector<uint64_t> a_row0(n_jobs), b_row0(n_jobs), rows_off_a(n_jobs), rows_off_b(n_jobs);
    uint64_t rows = 0, row_bytes = 0;
    for (uint32_t j = 0; j < n_jobs; ++j) {
        const hj_batch_job &J = jobs[j];
        const bool self = J.b == nullptr;
        if (!J.a || J.na == 0 || (!self && J.nb == 0)) return engine_fail(HJ_ERR_INVALID_ARG, "empty job");
        if (J.d == 0 || J.d > 256) return engine_fail(HJ_ERR_UNSUPPORTED, "batched jobs need 1 <= d <= 256");
        if (J.na >= (1ull << 31) || J.nb >= (1ull << 31)) return engine_fail(HJ_ERR_INVALID_ARG, "n below 2^31");
        b->d_max = std::max(b->d_max, J.d);
        a_row0[j] = rows;
        rows += npad_rows(J.na);
        b_row0[j] = self ? a_row0[j] : rows;
        if (!self) rows += npad_rows(J.nb);
        rows_off_a[j] = row_bytes;
        row_bytes += J.na * J.d * (uint64_t)dtype_bytes;
        rows_off_b[j] = self ? rows_off_a[j] : row_bytes;
        if (!self) row_bytes += J.nb * J.d * (uint64_t)dtype_bytes;
        row_bytes = (row_bytes + 255) / 256 * 256;
    }
    if (rows >= (1ull << 31)) return engine_fail(HJ_ERR_INVALID_ARG, "batch too large (2^31 rows)");
    const bool tf32 = form == HJ_FORM_TC_TF32, bf = form == HJ_FORM_TC_BF16X3;
    const uint32_t kpad = tf32 ? (uint32_t)hj_ceil_div(b->d_max, 32) * 32 : (uint32_t)hj_ceil_div(b->d_max, 64) * 64;
    const size_t esz = tf32 ? 4 : 2;
    SortedSet &O = b->ops;
    O.n = rows;
    O.d = b->d_max;
    O.dtype_bytes = dtype_bytes;
    O.npad_tc = rows;
    O.kpad_tf32 = kpad;
    O.kpad_bf16 = kpad;
    void *hi = b->alloc(rows * kpad * esz);
    void *lo = bf ? b->alloc(rows * kpad * esz) : nullptr;
    O.norms = (float *)b->alloc(rows * 4);
    O.tile_maxnorm_a = (float *)b->alloc((rows / kTcTileA) * 4);
    O.tile_maxnorm_b = (float *)b->alloc((rows / kTcTileB) * 4);
    O.group_minnorm = (float *)b->alloc((rows / 32) * 4);
    char *srows = (char *)b->alloc(row_bytes);
    b->d_jobs = (TcJob *)b->alloc(n_jobs * sizeof(TcJob));
    b->d_counts = (unsigned long long *)b->alloc(n_jobs * 8);
    b->d_band_total = (unsigned long long *)b->alloc(16);
    b->d_err = (uint32_t *)b->alloc(4);
    b->d_maxerr = (unsigned int *)b->alloc(4);
    if (!hi || (bf && !lo) || !O.norms || !O.tile_maxnorm_a || !O.tile_maxnorm_b || !O.group_minnorm || !srows ||
        !b->d_jobs || !b->d_counts || !b->d_band_total || !b->d_err || !b->d_maxerr)
        return engine_fail(HJ_ERR_OOM, "out of device memory (batch)");
    if (tf32)
        O.tf32 = (float *)hi;
    else
        O.bf_hi = (uint16_t *)hi, O.bf_lo = (uint16_t *)lo;
    cudaMemsetAsync(hi, 0, rows * kpad * esz, st);
    if (lo) cudaMemsetAsync(lo, 0, rows * kpad * esz, st);
    k_fill_f32<<<(unsigned)hj_ceil_div(rows, 256), 256, 0, st>>>(O.norms, rows, kPadNorm);

    std::vector<TcJob> hjobs(n_jobs);
    std::vector<std::pair<WorkItem *, uint64_t>> parts;
    uint64_t n_items = 0;
    for (uint32_t j = 0; j < n_jobs; ++j) {
        const hj_batch_job &J = jobs[j];
        const bool self = J.b == nullptr;
        PreparedJob P;
        if (int r = engine_prepare_job(st, J.a, J.b, J.na, self ? J.na : J.nb, dtype_bytes, J.d, J.eps, self, opts,
                                       form, &P))
            return r;
        b->num_sms = P.num_sms;
        // operands, norms and sorted rows into the batch's buffers; the engine's
        // buffers are reused by the next job, but all copies are ordered on `st`
        const uint32_t kj = tf32 ? P.A.kpad_tf32 : P.A.kpad_bf16;
        auto copy_set = [&](const SortedSet &S, uint64_t row0, uint64_t roff) {
            const void *src_hi = tf32 ? (const void *)S.tf32 : (const void *)S.bf_hi;
            cudaMemcpy2DAsync((char *)hi + row0 * kpad * esz, kpad * esz, src_hi, kj * esz, kj * esz, S.npad_tc,
                              cudaMemcpyDeviceToDevice, st);
            if (bf)
                cudaMemcpy2DAsync((char *)lo + row0 * kpad * esz, kpad * esz, S.bf_lo, kj * esz, kj * esz, S.npad_tc,
                                  cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(O.norms + row0, S.norms, S.npad_tc * 4, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(srows + roff, S.rows, S.n * S.d * (uint64_t)dtype_bytes, cudaMemcpyDeviceToDevice, st);
        };
        copy_set(P.A, a_row0[j], rows_off_a[j]);
        if (!self) copy_set(P.B, b_row0[j], rows_off_b[j]);
        fill_tc_job(&hjobs[j], form, J.d, J.eps * J.eps, P.op_scale, P.maxabs, a_row0[j], P.na_eff, b_row0[j],
                    P.nb_eff, self, b->d_counts + j, srows + rows_off_a[j], srows + rows_off_b[j], nullptr, nullptr);
        // work items rebased onto the matrix
        if (P.idx_tc.n_items) {
            WorkItem *w = (WorkItem *)b->alloc(P.idx_tc.n_items * sizeof(WorkItem));
            if (!w) return engine_fail(HJ_ERR_OOM, "out of device memory (batch items)");
            k_rebase_items<<<(unsigned)hj_ceil_div(P.idx_tc.n_items, 256), 256, 0, st>>>(
                P.idx_tc.items, P.idx_tc.n_items, (uint32_t)(a_row0[j] / kTcTileA), (uint32_t)(b_row0[j] / kTcTileB),
                j, w);
            parts.push_back({w, P.idx_tc.n_items});
            n_items += P.idx_tc.n_items;
        }
        b->candidate_pairs += P.idx_tc.candidate_pairs;
        b->job_candidates[j] = P.idx_tc.candidate_pairs + P.idx_fp.candidate_pairs;
        // items routed to the FP64 kernel keep their own plain tiles
        if (P.idx_fp.n_items) {
            FpJob f;
            f.job = j;
            f.self = self;
            f.na_eff = P.na_eff;
            f.nb_eff = P.nb_eff;
            f.T = J.eps * J.eps;
            const size_t ta = P.A.n_tiles64 * J.d * kPlainTile * 8;
            f.A.d = J.d;
            f.A.n_tiles64 = P.A.n_tiles64;
            f.A.tiles64 = (double *)b->alloc(ta);
            f.idx = P.idx_fp;
            f.idx.items = (WorkItem *)b->alloc(P.idx_fp.n_items * sizeof(WorkItem));
            if (!f.A.tiles64 || !f.idx.items) return engine_fail(HJ_ERR_OOM, "out of device memory (batch)");
            cudaMemcpyAsync(f.A.tiles64, P.A.tiles64, ta, cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(f.idx.items, P.idx_fp.items, P.idx_fp.n_items * sizeof(WorkItem),
                            cudaMemcpyDeviceToDevice, st);
            if (self) {
                f.B = f.A;
            } else {
                const size_t tb = P.B.n_tiles64 * J.d * kPlainTile * 8;
                f.B.d = J.d;
                f.B.n_tiles64 = P.B.n_tiles64;
                f.B.tiles64 = (double *)b->alloc(tb);
                if (!f.B.tiles64) return engine_fail(HJ_ERR_OOM, "out of device memory (batch)");
                cudaMemcpyAsync(f.B.tiles64, P.B.tiles64, tb, cudaMemcpyDeviceToDevice, st);
            }
            b->fp64_items += P.idx_fp.n_items;
            b->fp.push_back(f);
        }
        if (cudaGetLastError() != cudaSuccess) return engine_fail(HJ_ERR_CUDA, "batch planning copy failed");
    }
    // one work list
    b->idx.items = (WorkItem *)b->alloc(std::max<uint64_t>(n_items, 1) * sizeof(WorkItem));
    if (!b->idx.items) return engine_fail(HJ_ERR_OOM, "out of device memory (batch items)");
    uint64_t off = 0;
    for (auto &pt : parts) {
        cudaMemcpyAsync(b->idx.items + off, pt.first, pt.second * sizeof(WorkItem), cudaMemcpyDeviceToDevice, st);
        off += pt.second;
    }
    b->idx.n_items = n_items;
    launch_norm_summaries(O.norms, rows, O.tile_maxnorm_a, O.tile_maxnorm_b, O.group_minnorm, st);
    cudaMemcpyAsync(b->d_jobs, hjobs.data(), n_jobs * sizeof(TcJob), cudaMemcpyHostToDevice, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        cudaError_t e = cudaGetLastError();
        return engine_fail(HJ_ERR_CUDA, std::string("batch planning: ") + cudaGetErrorString(e));
    }
    // size the band queue with one run (regrown once if it overflows)
    b->band_cap = std::max<uint64_t>(1ull << 20, b->candidate_pairs / 4096);
    for (int attempt = 0; attempt < 3; ++attempt) {
        b->band = (uint2 *)b->alloc(b->band_cap * kBandEntryBytes);
        if (!b->band) return engine_fail(HJ_ERR_OOM, "out of device memory (band queue)");
        if (int r = batch_enqueue(b, st)) return r;
        uint64_t bt = 0;
        int r = batch_finish(b, &bt);
        if (r == HJ_OK) return HJ_OK;
        if (r != HJ_ERR_BAND_OVERFLOW) return r;
        b->band_cap = bt + bt / 4 + 4096;
    }
    return engine_fail(HJ_ERR_BAND_OVERFLOW, "band queue overflow");
}

namespace hj {
int batch_job_candidates(const hj_batch *b, uint64_t *out) {
    for (uint32_t j = 0; j < b->n_jobs; ++j) out[j] = b->job_candidates[j];
    return HJ_OK;
}
}  // namespace hj

extern "C" {

int hj_batch_create(const hj_batch_job *jobs, uint32_t n_jobs, int dtype_bytes, const hj_opts *opts,
                    hj_batch **out) {
    if (!out) return engine_fail(HJ_ERR_INVALID_ARG, "null pointer");
    *out = nullptr;
    hj_batch *b = new hj_batch();
    int r = batch_plan(jobs, n_jobs, dtype_bytes, opts, b);
    if (r != HJ_OK) {
        cudaStreamSynchronize(b->last);
        delete b;
        return r;
    }
    *out = b;
    return HJ_OK;
}

int hj_batch_run(hj_batch *b, void *stream) {
    if (!b) return engine_fail(HJ_ERR_INVALID_ARG, "null batch");
    cudaSetDevice(b->device);
    return batch_enqueue(b, stream ? (cudaStream_t)stream : b->own);
}

int hj_batch_counts(hj_batch *b, uint64_t *counts, hj_stats *stats) {
    if (!b || !counts) return engine_fail(HJ_ERR_INVALID_ARG, "null pointer");
    cudaSetDevice(b->device);
    uint64_t bt = 0;
    if (int r = batch_finish(b, &bt)) return r;
    std::vector<unsigned long long> h(b->n_jobs);
    if (cudaMemcpy(h.data(), b->d_counts, b->n_jobs * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return engine_fail(HJ_ERR_CUDA, "count read-back failed");
    for (uint32_t j = 0; j < b->n_jobs; ++j) counts[j] = h[j];
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        unsigned int eb = 0;
        cudaMemcpy(&eb, b->d_maxerr, 4, cudaMemcpyDeviceToHost);
        float ef;
        std::memcpy(&ef, &eb, 4);
        stats->candidate_pairs = b->candidate_pairs;
        stats->work_items = b->idx.n_items;
        stats->band_pairs = bt;
        stats->band_fraction = b->candidate_pairs ? (double)bt / (double)b->candidate_pairs : 0.0;
        stats->max_abs_err_band = ef;
        stats->fp64_items = b->fp64_items;
        stats->form_used = b->form;
        stats->kernel_launches = 2 + (int)b->fp.size();
    }
    return HJ_OK;
}

int hj_batch_destroy(hj_batch *b) {
    if (!b) return HJ_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->last);
    delete b;
    return HJ_OK;
}

int hj_batch_count_device(const hj_batch_job *jobs, uint32_t n_jobs, int dtype_bytes, const hj_opts *opts,
                          uint64_t *counts, hj_stats *stats) {
    if (!counts) return engine_fail(HJ_ERR_INVALID_ARG, "null pointer");
    hj_batch *b = nullptr;
    if (int r = hj_batch_create(jobs, n_jobs, dtype_bytes, opts, &b)) return r;
    // planning ran the batch once to size the band queue: its counts stand
    int r = hj_batch_counts(b, counts, stats);
    hj_batch_destroy(b);
    return r;
}

}  // extern "C"
