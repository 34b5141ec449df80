// hb_capi.cu -- the C ABI (include/hermite_b200.h): context, host mirror,
// uploads, launch-shape selection and error reporting.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "hermite_b200.h"
#include "hb_common.cuh"
#include "hb_internal.h"

namespace hb {
// compiled launch shapes per order and precision (hb_force_table.cuh)
constexpr int kNumVariants = 20;
const ForceVariant *force_variant_64(int order, int v);
const ForceVariant *force_variant_mixed(int order, int v);

int force_variant_count(int order, bool mixed)
{
    return (order == 4 || order == 6 || order == 8 || (order == 9 && !mixed)) ? kNumVariants : 0;
}

const ForceVariant *force_variant(int order, bool mixed, int v)
{
    return mixed ? force_variant_mixed(order, v) : force_variant_64(order, v);
}
}  // namespace hb

using namespace hb;

namespace {
constexpr int kMaxBody = 1 << 24;
// hb_set_jp_records of at least this many bytes uploads at once, in chunks.
constexpr size_t kEagerUploadBytes = (size_t)4 << 20, kUploadChunkBytes = (size_t)2 << 20;
// HB_ENGINE_AUTO takes the team engine up to this many particles.
constexpr int kTeamAutoMaxBody = 3072;

int rec_words(int order) { return 8 + 3 * (order - 2); }
int force_words(int order) { return 3 * (order / 2); }
int pred64_ncomp(int order) { return 7 + 3 * (order / 2 - 2) + (order == 9 ? 3 : 0); }
int predmx_ncomp(int order) { return 10 + 3 * (order / 2 - 2); }
}  // namespace

struct hb_ctx {
    int order = 0, nbody = 0, npad = 0;
    int precision = HB_FP64;        // used by the next predict_all
    int pred_precision = -1;        // precision of the last predict_all
    double tsys = 0.0;              // time of the last predict_all
    bool pred_stale = true;         // the predicted array is not at tsys yet
    int R = 0, F = 0;
    int device = 0, nsm = 0;
    cudaStream_t own_stream = nullptr, stream = nullptr;

    double *h_jp = nullptr, *h_force = nullptr, *h_pot = nullptr;
    double *h_force_dev = nullptr;  // device address of the mapped h_force
    double *d_jp = nullptr, *d_force = nullptr, *d_pot = nullptr, *d_posm = nullptr;
    double *d_partial = nullptr;
    void *d_pred = nullptr;
    unsigned *d_counter = nullptr;
    int *h_err = nullptr, *d_err = nullptr;
    size_t partial_cap = 0;         // doubles

    std::atomic<int> dirty_lo{INT_MAX}, dirty_hi{0};
    std::atomic<bool> upload_pending{false};
    cudaEvent_t ev_upload = nullptr;

    int njpsend = 0;                // the reference's bookkeeping (previous nact)
    long long launches = 0;
    int variant_override = -1, jsplit_override = 0;
    unsigned wait_limit = kSpinLimit;   // force kernel's tile waits (hb_set_wait_limit)

    // device-resident integration (hb_integrator_*)
    Sched *h_sched = nullptr;       // host copy of the scheduler (set-up only)
    Sched *d_sched = nullptr;       // device scheduler
    IntStatus *h_status = nullptr, *d_status = nullptr;   // mapped pinned
    double *d_dt = nullptr;
    int *d_ilist = nullptr;
    double *d_epart = nullptr, *h_eout = nullptr, *d_eout = nullptr;
    cudaGraph_t int_graph = nullptr;
    cudaGraphExec_t int_exec = nullptr;
    bool int_ready = false;
    // team engine (hb_team.cu)
    int engine = HB_ENGINE_AUTO, team_ctas = 0;
    TeamSys *d_team_sys = nullptr;
    double *d_aux = nullptr;          // per-slot dump derivatives
    TeamState *d_team_state = nullptr;
    int *d_team_next = nullptr;
    // persistent engine
    unsigned *d_gbar = nullptr;       // grid barrier words, zero between launches
    IntegratorLaunch int_L{};         // the step's buffers and work-item target
    int persist_grid = 0;             // resident CTAs of the persistent kernel
    int blocks_per_sm[2][kNumVariants] = {};
    bool smem_set[2][kNumVariants] = {};
    std::string err;
};

namespace {

int fail(hb_ctx *c, int status, const char *fmt, ...)
{
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return status;
}

#define HB_CK(call)                                                                  \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess)                                                       \
            return fail(ctx, HB_ERR_CUDA, "%s failed: %s (%s:%d)", #call,            \
                        cudaGetErrorString(e_), __FILE__, __LINE__);                 \
    } while (0)

void mark_dirty(hb_ctx *c, int lo, int hi)
{
    int cur = c->dirty_lo.load(std::memory_order_relaxed);
    while (lo < cur && !c->dirty_lo.compare_exchange_weak(cur, lo, std::memory_order_relaxed)) {}
    cur = c->dirty_hi.load(std::memory_order_relaxed);
    while (hi > cur && !c->dirty_hi.compare_exchange_weak(cur, hi, std::memory_order_relaxed)) {}
}

// A slot may be rewritten only after the DMA of the previous upload is done.
void wait_upload(hb_ctx *c)
{
    if (c->upload_pending.load(std::memory_order_acquire)) cudaEventSynchronize(c->ev_upload);
}

// Host copies of megabytes (bulk records in, forces and potentials out) are
// memory-bandwidth work: split over up to 8 host threads.
void host_copy(void *dst, const void *src, size_t bytes)
{
    constexpr size_t kParallel = (size_t)1 << 20, kPerThread = (size_t)256 << 10;
    if (bytes < kParallel) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const int nt = (int)std::min<size_t>(8, bytes / kPerThread);
    const size_t per = (bytes + nt - 1) / nt;
#pragma omp parallel for num_threads(nt) schedule(static, 1)
    for (int t = 0; t < nt; ++t) {
        const size_t o = (size_t)t * per;
        if (o < bytes)
            std::memcpy(static_cast<char *>(dst) + o, static_cast<const char *>(src) + o,
                        std::min(per, bytes - o));
    }
}

int do_upload(hb_ctx *ctx)
{
    const int lo = ctx->dirty_lo.exchange(INT_MAX);
    const int hi = ctx->dirty_hi.exchange(0);
    if (hi > lo) {
        const size_t off = (size_t)lo * ctx->R, words = (size_t)(hi - lo) * ctx->R;
        HB_CK(cudaMemcpyAsync(ctx->d_jp + off, ctx->h_jp + off, words * sizeof(double),
                              cudaMemcpyHostToDevice, ctx->stream));
        HB_CK(cudaEventRecord(ctx->ev_upload, ctx->stream));
        ctx->upload_pending.store(true, std::memory_order_release);
    }
    return HB_OK;
}

// Device-side waits that gave up leave a code in the mapped flag.
int check_device_flag(hb_ctx *ctx)
{
    volatile int *f = ctx->h_err;
    if (*f != kErrNone) {
        const int code = *f;
        *f = kErrNone;
        // the i-tile counters of an abandoned launch are not reset by it
        cudaMemsetAsync(ctx->d_counter, 0, sizeof(unsigned) * (ctx->npad / 32 + 1), ctx->stream);
        cudaStreamSynchronize(ctx->stream);
        return fail(ctx, HB_ERR_DEVICE_TIMEOUT,
                    "a bounded device-side wait gave up (code %d); results discarded", code);
    }
    return HB_OK;
}

int sync_stream(hb_ctx *ctx)
{
    HB_CK(cudaStreamSynchronize(ctx->stream));
    ctx->upload_pending.store(false, std::memory_order_release);
    return check_device_flag(ctx);
}

// Launch shapes measured by hermite_b200/autotune.py on a B200, keyed by
// (order, precision, log2 N bucket, log2 nact bucket).
struct TuneEntry {
    int order, mixed, log2n, log2nact, variant, jsplit;
};
const TuneEntry kTune[] = {
#if __has_include("hb_tuning.inc")
#include "hb_tuning.inc"
#endif
    {0, 0, 0, 0, 0, 0}   // end
};

// Nearest measured bucket: first the nearest N, then the nearest nact.
const TuneEntry *lookup_tuning(int order, bool mixed, int n, int nact)
{
    const double ln = std::log2((double)n), la = std::log2((double)std::max(nact, 1));
    const TuneEntry *best = nullptr;
    double bn = 1e30, ba = 1e30;
    for (const TuneEntry &e : kTune) {
        if (e.order != order || e.mixed != (mixed ? 1 : 0)) continue;
        const double dn = std::fabs(e.log2n - ln), da = std::fabs(e.log2nact - la);
        if (dn < bn - 1e-9 || (dn < bn + 1e-9 && da < ba)) {
            best = &e;
            bn = dn;
            ba = da;
        }
    }
    return best;
}

// Launch shape for the force kernel: the tuned variant and j-slice count of
// the nearest bucket (the slice count rescaled to keep the measured number
// of CTAs), else a heuristic; then the slice count is clamped so that each
// CTA keeps at least 8 chunks and the partials fit in the scratch buffer.
int pick_variant(const hb_ctx *c, int nact, int *jsplit_hint)
{
    *jsplit_hint = 0;
    if (c->variant_override >= 0) return c->variant_override;
    const bool mixed = c->pred_precision == HB_MIXED;
    // double-double (order 9) uses the 8th-order measurements
    if (const TuneEntry *e = lookup_tuning(c->order == 9 ? 8 : c->order, mixed, c->nbody, nact)) {
        const ForceVariant *fv = force_variant(c->order, mixed, e->variant);
        if (fv) {
            const long long gx_bucket = ((1LL << e->log2nact) + fv->ti - 1) / fv->ti;
            const long long gx = (nact + fv->ti - 1) / fv->ti;
            const long long ctas = gx_bucket * e->jsplit;
            *jsplit_hint = (int)std::max<long long>(1, (ctas + gx - 1) / gx);
            return e->variant;
        }
    }
    if (nact <= 32) return 2;
    if (nact <= 64) return 3;
    if (nact <= c->nsm * 256) return 0;
    return 1;
}

// Force records up to this size are written by the kernel straight into the
// mapped pinned buffer (no device->host copy in the block step).
constexpr size_t kZeroCopyBytes = 256 << 10;

int run_force(hb_ctx *ctx, int nact, double eps2, double *force_out_dev)
{
    if (nact == 0) return HB_OK;
    const bool mixed = ctx->pred_precision == HB_MIXED;
    if (!mixed && ctx->order != 9 && nact <= kLanesMaxAct && ctx->variant_override < 0) {
        // a handful of active particles: lanes share an i-particle
        ForceArgs a{};
        a.jp = ctx->d_jp;
        a.tsys = ctx->tsys;
        a.nbody = ctx->nbody;
        a.nchunk = ctx->npad / 32;
        a.nact = nact;
        a.eps2 = eps2;
        a.force = force_out_dev;
        a.partial = ctx->d_partial;
        a.counter = ctx->d_counter;
        a.err = ctx->d_err;
        a.spin = ctx->wait_limit;
        HB_CK(launch_force_lanes(ctx->order, a, ctx->nsm, ctx->stream));
        ctx->launches++;
        return HB_OK;
    }
    int jsplit_hint = 0;
    const int v = pick_variant(ctx, nact, &jsplit_hint);
    const ForceVariant *fv = force_variant(ctx->order, mixed, v);
    if (!fv) return fail(ctx, HB_ERR_INVALID, "force variant %d does not exist", v);
    const int m = mixed ? 1 : 0;
    const int threads = fv->nw * 32;
    if (!ctx->smem_set[m][v]) {
        HB_CK(cudaFuncSetAttribute(fv->kern, cudaFuncAttributeMaxDynamicSharedMemorySize, fv->smem));
        int nb = 0;
        HB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fv->kern, threads, fv->smem));
        ctx->blocks_per_sm[m][v] = std::max(nb, 1);
        ctx->smem_set[m][v] = true;
    }
    const int nchunk = ctx->npad / 32;
    const int gx = (nact + fv->ti - 1) / fv->ti;
    int S = ctx->jsplit_override > 0 ? ctx->jsplit_override : jsplit_hint;
    if (S <= 0) {
        const int target = ctx->nsm * ctx->blocks_per_sm[m][v];
        S = gx >= target ? 1 : (target + gx - 1) / gx;
        // at least 8 chunks (256 j) per CTA and 2 chunks per j-warp
        S = std::min(S, std::max(1, nchunk / std::max(8, 2 * fv->wj)));
    }
    S = std::max(1, std::min(S, ctx->jsplit_override > 0 ? nchunk : std::max(1, nchunk / 8)));
    if (S > 1) {
        const size_t need_per_slice = (size_t)gx * fv->ti * ctx->F;
        const size_t smax = ctx->partial_cap / need_per_slice;
        if ((size_t)S > smax) S = (int)std::max<size_t>(1, smax);
    }
    if (!fv->fused && ctx->pred_stale) {
        // two-pass shape: the predictor kernel first
        HB_CK(launch_predict(ctx->order, mixed, ctx->d_jp, ctx->nbody, ctx->npad, ctx->tsys,
                             ctx->d_pred, ctx->d_err, ctx->stream));
        ctx->launches++;
        ctx->pred_stale = false;
    }
    ForceArgs a{};
    a.pred = ctx->d_pred;
    a.jp = ctx->d_jp;
    a.tsys = ctx->tsys;
    a.nbody = ctx->nbody;
    a.nchunk = nchunk;
    a.nact = nact;
    a.eps2 = eps2;
    a.force = force_out_dev;
    a.partial = ctx->d_partial;
    a.counter = ctx->d_counter;
    a.err = ctx->d_err;
    a.spin = ctx->wait_limit;
    fv->kern<<<dim3(gx, S), threads, fv->smem, ctx->stream>>>(a);
    HB_CK(cudaGetLastError());
    ctx->launches++;
    return HB_OK;
}

bool valid_order(int order) { return order == 4 || order == 6 || order == 8; }

}  // namespace

// ===========================================================================
extern "C" {

const char *hb_status_string(int s)
{
    switch (s) {
    case HB_OK: return "ok";
    case HB_ERR_INVALID: return "invalid argument";
    case HB_ERR_CUDA: return "CUDA runtime error";
    case HB_ERR_ALLOC: return "allocation failed";
    case HB_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case HB_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case HB_ERR_STATE: return "call out of order";
    case HB_ERR_TOO_LARGE: return "size exceeds a fixed capacity";
    case HB_ERR_IO: return "file could not be written or parsed";
    }
    return "unknown status";
}

const char *hb_last_error(const hb_ctx *ctx)
{
    if (!ctx) return "null context";
    return ctx->err.c_str();
}

int hb_destroy(hb_ctx *ctx)
{
    if (!ctx) return HB_OK;
    if (ctx->own_stream) cudaStreamSynchronize(ctx->own_stream);
    if (ctx->stream && ctx->stream != ctx->own_stream) cudaStreamSynchronize(ctx->stream);
    cudaFreeHost(ctx->h_jp);
    cudaFreeHost(ctx->h_force);
    cudaFreeHost(ctx->h_pot);
    cudaFreeHost(ctx->h_err);
    cudaFree(ctx->d_jp);
    cudaFree(ctx->d_force);
    cudaFree(ctx->d_pot);
    cudaFree(ctx->d_posm);
    cudaFree(ctx->d_partial);
    cudaFree(ctx->d_pred);
    cudaFree(ctx->d_counter);
    if (ctx->int_exec) cudaGraphExecDestroy(ctx->int_exec);
    if (ctx->int_graph) cudaGraphDestroy(ctx->int_graph);
    delete ctx->h_sched;
    cudaFree(ctx->d_sched);
    cudaFreeHost(ctx->h_status);
    cudaFreeHost(ctx->h_eout);
    cudaFree(ctx->d_dt);
    cudaFree(ctx->d_ilist);
    cudaFree(ctx->d_epart);
    cudaFree(ctx->d_team_sys);
    cudaFree(ctx->d_aux);
    cudaFree(ctx->d_team_state);
    cudaFree(ctx->d_team_next);
    cudaFree(ctx->d_gbar);
    if (ctx->ev_upload) cudaEventDestroy(ctx->ev_upload);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return HB_OK;
}

int hb_create(int order, int nbody, int precision, hb_ctx **out)
{
    if (!out) return HB_ERR_INVALID;
    *out = nullptr;
    // HB_FP64_DD: 8th order with double-double positions, internal order 9
    const bool dd = precision == HB_FP64_DD;
    if (!valid_order(order) || nbody < 1 || nbody > kMaxBody ||
        (precision != HB_FP64 && precision != HB_MIXED && !(dd && order == 8)))
        return HB_ERR_INVALID;
    if (dd) {
        order = 9;
        precision = HB_FP64;
    }

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return HB_ERR_NO_DEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return HB_ERR_NO_DEVICE;
    if (prop.major != 10 || prop.minor != 0) return HB_ERR_NO_DEVICE;

    hb_ctx *ctx = new hb_ctx;
    ctx->order = order;
    ctx->nbody = nbody;
    ctx->npad = (nbody + kSlotPad - 1) / kSlotPad * kSlotPad;
    ctx->precision = precision;
    ctx->R = rec_words(order);
    ctx->F = force_words(order);
    ctx->device = dev;
    ctx->nsm = prop.multiProcessorCount;
    ctx->njpsend = nbody;

    const size_t np = ctx->npad;
    const size_t pred_bytes = std::max(np * pred64_ncomp(order) * sizeof(double),
                                       np * predmx_ncomp(order) * sizeof(float));
    ctx->partial_cap = (size_t)2 * ctx->nsm * 8 * 256 * ctx->F;
    bool ok = true;
    ok = ok && cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaEventCreateWithFlags(&ctx->ev_upload, cudaEventDisableTiming) == cudaSuccess;
    ok = ok && cudaHostAlloc((void **)&ctx->h_jp, np * ctx->R * sizeof(double), cudaHostAllocPortable) == cudaSuccess;
    ok = ok && cudaHostAlloc((void **)&ctx->h_force, np * ctx->F * sizeof(double),
                             cudaHostAllocMapped | cudaHostAllocPortable) == cudaSuccess;
    ok = ok && cudaHostAlloc((void **)&ctx->h_pot, np * sizeof(double), cudaHostAllocPortable) == cudaSuccess;
    ok = ok && cudaHostAlloc((void **)&ctx->h_err, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_jp, np * ctx->R * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_force, np * ctx->F * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_pot, np * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_posm, np * (order == 9 ? 7 : 4) * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_partial, ctx->partial_cap * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&ctx->d_pred, pred_bytes) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_counter, (np / 32 + 1) * sizeof(unsigned)) == cudaSuccess;
    if (ok) {
        ok = cudaHostGetDevicePointer((void **)&ctx->d_err, ctx->h_err, 0) == cudaSuccess &&
             cudaHostGetDevicePointer((void **)&ctx->h_force_dev, ctx->h_force, 0) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();   // clear the sticky-free error state of the failed call
        hb_destroy(ctx);
        return HB_ERR_ALLOC;
    }
    ctx->stream = ctx->own_stream;
    *ctx->h_err = kErrNone;
    std::memset(ctx->h_jp, 0, np * ctx->R * sizeof(double));
    if (cudaMemsetAsync(ctx->d_counter, 0, (np / 32 + 1) * sizeof(unsigned), ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(ctx->d_jp, 0, np * ctx->R * sizeof(double), ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        hb_destroy(ctx);
        return HB_ERR_CUDA;
    }
    // like the reference's first predict_all (njpsend = nbody), the first
    // upload covers every slot
    ctx->dirty_lo = 0;
    ctx->dirty_hi = nbody;
    *out = ctx;
    return HB_OK;
}

int hb_set_jp(hb_ctx *ctx, int addr, const double pos[3], double mass, const double vel[3],
              double tlast, const double *derivs)
{
    if (!ctx || addr < 0 || addr >= ctx->nbody || !pos || !vel || !derivs) return HB_ERR_INVALID;
    wait_upload(ctx);
    double *r = ctx->h_jp + (size_t)addr * ctx->R;
    r[0] = pos[0]; r[1] = pos[1]; r[2] = pos[2];
    r[3] = mass;
    r[4] = vel[0]; r[5] = vel[1]; r[6] = vel[2];
    r[7] = tlast;
    std::memcpy(r + 8, derivs, sizeof(double) * 3 * (ctx->order - 2));
    mark_dirty(ctx, addr, addr + 1);
    return HB_OK;
}

int hb_set_jp_records(hb_ctx *ctx, int addr0, int count, const double *records)
{
    if (!ctx || addr0 < 0 || count < 0 || (count > 0 && !records) ||
        (long long)addr0 + count > ctx->nbody)
        return HB_ERR_INVALID;
    if (count == 0) return HB_OK;
    wait_upload(ctx);
    const size_t off = (size_t)addr0 * ctx->R, bytes = sizeof(double) * (size_t)count * ctx->R;
    if (bytes < kEagerUploadBytes) {
        host_copy(ctx->h_jp + off, records, bytes);
        mark_dirty(ctx, addr0, addr0 + count);
        return HB_OK;
    }
    // A bulk set: copy into the pinned mirror chunk by chunk and upload each
    // chunk while the next one is copied (stream-ordered after any force
    // still reading the device copy).  These slots need no later upload.
    const char *src = reinterpret_cast<const char *>(records);
    char *hm = reinterpret_cast<char *>(ctx->h_jp + off);
    char *dm = reinterpret_cast<char *>(ctx->d_jp + off);
    for (size_t o = 0; o < bytes; o += kUploadChunkBytes) {
        const size_t len = std::min(kUploadChunkBytes, bytes - o);
        host_copy(hm + o, src + o, len);
        HB_CK(cudaMemcpyAsync(dm + o, hm + o, len, cudaMemcpyHostToDevice, ctx->stream));
    }
    HB_CK(cudaEventRecord(ctx->ev_upload, ctx->stream));
    ctx->upload_pending.store(true, std::memory_order_release);
    return HB_OK;
}

int hb_upload(hb_ctx *ctx)
{
    if (!ctx) return HB_ERR_INVALID;
    return do_upload(ctx);
}

int hb_predict_all_device(hb_ctx *ctx, double tsys)
{
    if (!ctx) return HB_ERR_INVALID;
    // The prediction itself runs with the next force launch: inside the fused
    // force kernel, or as a predictor pass ahead of a two-pass force kernel.
    ctx->tsys = tsys;
    ctx->pred_precision = ctx->precision;
    ctx->pred_stale = true;
    return HB_OK;
}

int hb_predict_pass(hb_ctx *ctx)
{
    if (!ctx) return HB_ERR_INVALID;
    if (ctx->pred_precision < 0) return fail(ctx, HB_ERR_STATE, "predictor pass before any predict_all");
    HB_CK(launch_predict(ctx->order, ctx->pred_precision == HB_MIXED, ctx->d_jp, ctx->nbody, ctx->npad,
                         ctx->tsys, ctx->d_pred, ctx->d_err, ctx->stream));
    ctx->launches++;
    ctx->pred_stale = false;
    return HB_OK;
}

int hb_predict_all(hb_ctx *ctx, double tsys)
{
    if (!ctx) return HB_ERR_INVALID;
    int s = do_upload(ctx);
    if (s != HB_OK) return s;
    return hb_predict_all_device(ctx, tsys);
}

int hb_force_device(hb_ctx *ctx, int nact, double eps2)
{
    if (!ctx) return HB_ERR_INVALID;
    if (nact < 0 || nact > ctx->nbody)
        return fail(ctx, HB_ERR_INVALID, "nact=%d outside [0, %d]", nact, ctx->nbody);
    if (!(eps2 >= 0.0)) return fail(ctx, HB_ERR_INVALID, "eps2 must be >= 0");
    if (ctx->pred_precision < 0)
        return fail(ctx, HB_ERR_STATE, "calc_force_on_first_nact before any predict_all");
    return run_force(ctx, nact, eps2, ctx->d_force);
}

int hb_download_forces(hb_ctx *ctx, int nact, double *force_out)
{
    if (!ctx || nact < 0 || nact > ctx->nbody || (nact > 0 && !force_out)) return HB_ERR_INVALID;
    if (nact > 0) {
        HB_CK(cudaMemcpyAsync(ctx->h_force, ctx->d_force, sizeof(double) * (size_t)nact * ctx->F,
                              cudaMemcpyDeviceToHost, ctx->stream));
    }
    int s = sync_stream(ctx);
    if (s != HB_OK) return s;
    if (nact > 0) host_copy(force_out, ctx->h_force, sizeof(double) * (size_t)nact * ctx->F);
    return HB_OK;
}

int hb_force_first_nact(hb_ctx *ctx, int nact, double eps2, double *force_out)
{
    if (!ctx) return HB_ERR_INVALID;
    if (nact > 0 && !force_out) return fail(ctx, HB_ERR_INVALID, "force_out is NULL");
    int s;
    if ((size_t)nact * ctx->F * sizeof(double) <= kZeroCopyBytes) {
        // small block step: the kernel writes the records into pinned host
        // memory itself; only the stream synchronisation remains
        if (nact < 0 || nact > ctx->nbody)
            return fail(ctx, HB_ERR_INVALID, "nact=%d outside [0, %d]", nact, ctx->nbody);
        if (!(eps2 >= 0.0)) return fail(ctx, HB_ERR_INVALID, "eps2 must be >= 0");
        if (ctx->pred_precision < 0)
            return fail(ctx, HB_ERR_STATE, "calc_force_on_first_nact before any predict_all");
        s = run_force(ctx, nact, eps2, ctx->h_force_dev);
        if (s == HB_OK) s = sync_stream(ctx);
        if (s != HB_OK) return s;
        if (nact > 0) std::memcpy(force_out, ctx->h_force, sizeof(double) * (size_t)nact * ctx->F);
    } else {
        s = hb_force_device(ctx, nact, eps2);
        if (s == HB_OK) s = hb_download_forces(ctx, nact, force_out);
        if (s != HB_OK) return s;
    }
    ctx->njpsend = nact;
    return HB_OK;
}

int hb_potential(hb_ctx *ctx, double eps2, double *pot_out)
{
    if (!ctx) return HB_ERR_INVALID;
    if (!pot_out) return fail(ctx, HB_ERR_INVALID, "pot_out is NULL");
    if (!(eps2 >= 0.0)) return fail(ctx, HB_ERR_INVALID, "eps2 must be >= 0");
    int s = do_upload(ctx);
    if (s != HB_OK) return s;
    HB_CK(launch_potential(ctx->order, ctx->d_jp, ctx->nbody, ctx->npad, eps2, ctx->d_posm,
                           ctx->d_pot, ctx->d_err, ctx->stream));
    ctx->launches += 2;
    HB_CK(cudaMemcpyAsync(ctx->h_pot, ctx->d_pot, sizeof(double) * ctx->nbody,
                          cudaMemcpyDeviceToHost, ctx->stream));
    s = sync_stream(ctx);
    if (s != HB_OK) return s;
    host_copy(pot_out, ctx->h_pot, sizeof(double) * ctx->nbody);
    return HB_OK;
}

int hb_set_precision(hb_ctx *ctx, int precision)
{
    if (!ctx) return HB_ERR_INVALID;
    if (ctx->order == 9) {
        if (precision != HB_FP64_DD && precision != HB_FP64)
            return fail(ctx, HB_ERR_INVALID, "a double-double context stays double-double");
        return HB_OK;
    }
    if (precision != HB_FP64 && precision != HB_MIXED)
        return fail(ctx, HB_ERR_INVALID, "precision %d unknown", precision);
    ctx->precision = precision;
    return HB_OK;
}

int hb_get_precision(const hb_ctx *ctx)
{
    return ctx ? (ctx->order == 9 ? HB_FP64_DD : ctx->precision) : -1;
}

int hb_set_stream(hb_ctx *ctx, void *cuda_stream)
{
    if (!ctx) return HB_ERR_INVALID;
    int s = sync_stream(ctx);
    if (s != HB_OK) return s;
    ctx->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->own_stream;
    return HB_OK;
}

int hb_synchronize(hb_ctx *ctx)
{
    if (!ctx) return HB_ERR_INVALID;
    return sync_stream(ctx);
}

const double *hb_device_forces(const hb_ctx *ctx) { return ctx ? ctx->d_force : nullptr; }

long long hb_launch_count(const hb_ctx *ctx) { return ctx ? ctx->launches : -1; }

int hb_set_force_shape(hb_ctx *ctx, int variant, int jsplit)
{
    if (!ctx) return HB_ERR_INVALID;
    if (variant >= kNumVariants || jsplit < 0)
        return fail(ctx, HB_ERR_INVALID, "variant %d / jsplit %d out of range", variant, jsplit);
    ctx->variant_override = variant;   // < 0: automatic
    ctx->jsplit_override = jsplit;     // 0: automatic
    return HB_OK;
}

int hb_set_wait_limit(hb_ctx *ctx, long long polls)
{
    if (!ctx) return HB_ERR_INVALID;
    ctx->wait_limit = polls < 0 ? kSpinLimit
                                : (unsigned)std::min<long long>(polls, (long long)kSpinLimit);
    return HB_OK;
}

int hb_force_variant_count(int order, int precision)
{
    if (!valid_order(order)) return 0;
    if (precision == HB_FP64_DD) return order == 8 ? force_variant_count(9, false) : 0;
    if (precision != HB_FP64 && precision != HB_MIXED) return 0;
    return force_variant_count(order, precision == HB_MIXED);
}

int hb_force_variant_info(int order, int precision, int variant, int *threads, int *i_per_thread,
                          int *j_warps)
{
    if (!valid_order(order)) return HB_ERR_INVALID;
    if (precision == HB_FP64_DD) {
        if (order != 8) return HB_ERR_INVALID;
        order = 9;
        precision = HB_FP64;
    }
    if (precision != HB_FP64 && precision != HB_MIXED) return HB_ERR_INVALID;
    const ForceVariant *fv = force_variant(order, precision == HB_MIXED, variant);
    if (!fv) return HB_ERR_INVALID;
    if (threads) *threads = fv->nw * 32;
    if (i_per_thread) *i_per_thread = fv->ni;
    if (j_warps) *j_warps = fv->wj;
    return HB_OK;
}

// ---- device-resident integration -------------------------------------------
namespace {
constexpr int kStepsPerGraph = 32;
constexpr int kEnergyParts = 256;

int integrator_alloc(hb_ctx *ctx)
{
    if (ctx->h_sched) return HB_OK;
    const size_t np = ctx->npad;
    bool ok = cudaMalloc((void **)&ctx->d_sched, sizeof(Sched)) == cudaSuccess &&
              cudaHostAlloc((void **)&ctx->h_status, sizeof(IntStatus), cudaHostAllocMapped) == cudaSuccess &&
              cudaHostGetDevicePointer((void **)&ctx->d_status, ctx->h_status, 0) == cudaSuccess &&
              cudaHostAlloc((void **)&ctx->h_eout, 2 * sizeof(double), cudaHostAllocMapped) == cudaSuccess &&
              cudaHostGetDevicePointer((void **)&ctx->d_eout, ctx->h_eout, 0) == cudaSuccess &&
              cudaMalloc((void **)&ctx->d_dt, np * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&ctx->d_ilist, np * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&ctx->d_epart, 2 * kEnergyParts * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&ctx->d_aux, np * kAuxWords * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&ctx->d_team_sys, sizeof(TeamSys)) == cudaSuccess &&
              cudaMalloc((void **)&ctx->d_team_state, sizeof(TeamState)) == cudaSuccess &&
              cudaMalloc((void **)&ctx->d_team_next, sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&ctx->d_gbar, 2 * sizeof(unsigned)) == cudaSuccess &&
              cudaMemset(ctx->d_gbar, 0, 2 * sizeof(unsigned)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return fail(ctx, HB_ERR_ALLOC, "integrator buffers could not be allocated");
    }
    ctx->h_sched = new Sched;
    return HB_OK;
}
}  // namespace

namespace {
// Scheduler state and the captured block-step graph for the records, dt and
// dump derivatives now on the device (after init_step or a restore).
int setup_integrator(hb_ctx *ctx, double tsys, double eps2, double eta, double dtmax,
                     long long particle_steps, long long block_steps)
{
    Sched &sc = *ctx->h_sched;
    std::memset(&sc, 0, sizeof(Sched));
    sc.tnext_bits = 0x7ff0000000000000ull;
    sc.tsys = tsys;
    sc.tend = tsys;
    sc.eps2 = eps2;
    // set_run_params (SRC/nbodysystem.h:472); the double-double scheme is 8th order
    sc.etapow = std::pow(eta, 2.0 * ((ctx->order == 9 ? 8 : ctx->order) - 3));
    sc.dtmax = dtmax;
    sc.particle_steps = particle_steps;
    sc.block_steps = block_steps;
    sc.status = ctx->d_status;
    std::memset(ctx->h_status, 0, sizeof(IntStatus));
    ctx->h_status->tsys = tsys;
    ctx->h_status->particle_steps = particle_steps;
    ctx->h_status->block_steps = block_steps;
    HB_CK(cudaMemcpy(ctx->d_sched, &sc, sizeof(Sched), cudaMemcpyHostToDevice));
    const TeamSys ts{0, ctx->nbody, 0, eps2};
    HB_CK(cudaMemcpy(ctx->d_team_sys, &ts, sizeof(TeamSys), cudaMemcpyHostToDevice));

    IntegratorLaunch L;
    L.jp = ctx->d_jp;
    L.dt = ctx->d_dt;
    L.aux = ctx->d_aux;
    L.ilist = ctx->d_ilist;
    L.sched = ctx->d_sched;
    L.force = ctx->d_force;
    L.partial = ctx->d_partial;
    L.counter = ctx->d_counter;
    L.err = ctx->d_err;
    L.n = ctx->nbody;
    L.nchunk = ctx->npad / 32;
    L.nsm = ctx->nsm;
    L.partial_cap = ctx->partial_cap;
    L.mixed = ctx->precision == HB_MIXED;
    int smem = 0, per_sm = 0, big_per_sm = 0;
    HB_CK(integrator_kernel_setup(ctx->order, L.mixed, &smem, &per_sm, &big_per_sm));
    L.smem_fp64 = L.smem_mixed = smem;
    L.items_grid = ctx->nsm * std::max(1, per_sm);
    L.big_grid = ctx->nsm * std::max(1, big_per_sm);
    L.target_items = 2 * L.items_grid;
    ctx->int_L = L;
    int psmem = 0, p_per_sm = 0;
    HB_CK(persistent_setup(ctx->order, L.mixed, &psmem, &p_per_sm));
    ctx->persist_grid = ctx->nsm * p_per_sm;

    if (ctx->stream == nullptr) return fail(ctx, HB_ERR_STATE, "integrator needs a non-default stream");
    HB_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaSuccess;
    for (int k = 0; k < kStepsPerGraph && ce == cudaSuccess; ++k)
        ce = integrator_step_launch(ctx->order, L, ctx->stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &graph);
    if (ce != cudaSuccess || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return fail(ctx, HB_ERR_CUDA, "capturing the block-step graph failed: %s",
                    cudaGetErrorString(ce != cudaSuccess ? ce : ee));
    }
    ctx->int_graph = graph;
    HB_CK(cudaGraphInstantiate(&ctx->int_exec, graph, 0));
    ctx->int_ready = true;
    ctx->pred_precision = ctx->precision;
    return HB_OK;
}

int reset_integrator(hb_ctx *ctx)
{
    int s = integrator_alloc(ctx);
    if (s == HB_OK) s = sync_stream(ctx);
    if (s != HB_OK) return s;
    if (ctx->int_exec) { cudaGraphExecDestroy(ctx->int_exec); ctx->int_exec = nullptr; }
    if (ctx->int_graph) { cudaGraphDestroy(ctx->int_graph); ctx->int_graph = nullptr; }
    ctx->int_ready = false;
    return HB_OK;
}

bool power_of_two(double x) { return x > 0.0 && std::log2(x) == std::floor(std::log2(x)); }
}  // namespace

int hb_integrator_init(hb_ctx *ctx, double tsys, double eps2, double eta, double eta_s, double dtmax)
{
    if (!ctx) return HB_ERR_INVALID;
    if (!(eps2 >= 0.0) || !(eta > 0.0) || !(eta_s > 0.0) || !power_of_two(dtmax) || !(tsys >= 0.0))
        return fail(ctx, HB_ERR_INVALID, "integrator_init: need eps2 >= 0, eta, eta_s > 0, "
                                         "dtmax a power of two, tsys >= 0");
    int s = reset_integrator(ctx);
    if (s != HB_OK) return s;

    // initial conditions: the mirror's pos, mass, vel at tlast = tsys, all
    // derivatives zero (the reference's Particle constructor), as in
    // NbodySystem::init_step (SRC/nbodysystem.h:565-631)
    for (int i = 0; i < ctx->nbody; ++i) {
        double *r = ctx->h_jp + (size_t)i * ctx->R;
        r[7] = tsys;
        std::memset(r + 8, 0, sizeof(double) * (ctx->R - 8));
    }
    mark_dirty(ctx, 0, ctx->nbody);
    s = do_upload(ctx);
    if (s != HB_OK) return s;
    HB_CK(cudaMemsetAsync(ctx->d_aux, 0, sizeof(double) * ctx->npad * kAuxWords, ctx->stream));
    const int passes = ctx->order > 4 ? 2 : 1;   // higher derivatives bootstrap
    for (int p = 0; p < passes; ++p) {
        hb_predict_all_device(ctx, tsys);
        s = run_force(ctx, ctx->nbody, eps2, ctx->d_force);
        if (s != HB_OK) return s;
        HB_CK(integrator_assign(ctx->order, ctx->d_jp, ctx->d_dt, ctx->d_force, ctx->nbody,
                                p == passes - 1, eta_s, dtmax, ctx->stream));
        ctx->launches++;
    }
    s = sync_stream(ctx);
    if (s != HB_OK) return s;
    return setup_integrator(ctx, tsys, eps2, eta, dtmax, 0, 0);
}

int hb_integrator_dump(hb_ctx *ctx, const char *path, int dumpid, double init_energy,
                       double prev_energy)
{
    if (!ctx || !path) return HB_ERR_INVALID;
    if (!ctx->int_ready) return fail(ctx, HB_ERR_STATE, "hb_integrator_dump before hb_integrator_init");
    int s = sync_stream(ctx);
    if (s != HB_OK) return s;
    const size_t n = ctx->nbody;
    std::vector<double> rec(n * ctx->R), aux(n * kAuxWords);
    HB_CK(cudaMemcpy(rec.data(), ctx->d_jp, rec.size() * sizeof(double), cudaMemcpyDeviceToHost));
    HB_CK(cudaMemcpy(aux.data(), ctx->d_aux, aux.size() * sizeof(double), cudaMemcpyDeviceToHost));
    const volatile IntStatus *st = ctx->h_status;
    const double tsys = st->tsys;
    for (size_t i = 0; i < n; ++i)
        if (rec[i * ctx->R + 7] != tsys)
            return fail(ctx, HB_ERR_STATE, "dump at t = %.17g: slot %zu is at %.17g (dump at a multiple "
                                           "of dtmax, where every particle is at the block time)",
                        tsys, i, rec[i * ctx->R + 7]);
    s = hb_dump_write(path, ctx->order, dumpid, ctx->nbody, tsys, init_energy, prev_energy,
                      st->particle_steps, st->block_steps, nullptr, rec.data(), aux.data());
    return s == HB_OK ? HB_OK : fail(ctx, s, "cannot write the dump file %s", path);
}

int hb_integrator_restore(hb_ctx *ctx, const char *path, double eps2, double eta, double dtmax,
                          int *dumpid, double *init_energy, double *prev_energy)
{
    if (!ctx || !path) return HB_ERR_INVALID;
    if (!(eps2 >= 0.0) || !(eta > 0.0) || !power_of_two(dtmax))
        return fail(ctx, HB_ERR_INVALID, "integrator_restore: need eps2 >= 0, eta > 0, dtmax a power of two");
    int order = 0, did = 0, nb = 0;
    double tsys = 0.0, e0 = 0.0, e1 = 0.0;
    long long steps = 0, bsteps = 0;
    int s = hb_dump_read_header(path, &order, &did, &nb, &tsys, &e0, &e1, &steps, &bsteps);
    if (s != HB_OK) return fail(ctx, s, "cannot read the dump header of %s", path);
    if (order != (ctx->order == 9 ? 8 : ctx->order) || nb != ctx->nbody)
        return fail(ctx, HB_ERR_INVALID, "the dump holds order %d, N = %d; the context order %d, N = %d",
                    order, nb, ctx->order, ctx->nbody);
    s = reset_integrator(ctx);
    if (s != HB_OK) return s;
    const size_t n = nb;
    std::vector<double> rec(n * ctx->R), aux(n * kAuxWords), dt(n);
    s = hb_dump_read(path, ctx->order, nb, nullptr, rec.data(), aux.data());
    if (s != HB_OK) return fail(ctx, s, "cannot read the dump particles of %s", path);
    // NbodySystem::restore + reinitialize_steps (SRC/nbodysystem.h:429-458):
    // tlast = tsys, dt from recalc_dt
    for (size_t i = 0; i < n; ++i) {
        rec[i * ctx->R + 7] = tsys;
        dt[i] = recalc_dt(ctx->order, rec.data() + i * ctx->R, aux.data() + i * kAuxWords, eta, dtmax);
    }
    wait_upload(ctx);
    std::memcpy(ctx->h_jp, rec.data(), rec.size() * sizeof(double));
    mark_dirty(ctx, 0, nb);
    s = do_upload(ctx);
    if (s != HB_OK) return s;
    HB_CK(cudaMemcpyAsync(ctx->d_aux, aux.data(), aux.size() * sizeof(double), cudaMemcpyHostToDevice,
                          ctx->stream));
    HB_CK(cudaMemcpyAsync(ctx->d_dt, dt.data(), dt.size() * sizeof(double), cudaMemcpyHostToDevice,
                          ctx->stream));
    s = sync_stream(ctx);
    if (s != HB_OK) return s;
    if (dumpid) *dumpid = did;
    if (init_energy) *init_energy = e0;
    if (prev_energy) *prev_energy = e1;
    return setup_integrator(ctx, tsys, eps2, eta, dtmax, steps, bsteps);
}

namespace {
constexpr long long kTeamStepsPerLaunch = 1LL << 14;

// The team size for one system of n slots: about kTeamChunksPerCta 32-slot
// chunks per CTA, at most 16 CTAs (8 where the device cannot co-schedule a
// 16-CTA cluster with this kernel's shared memory).
constexpr int kTeamChunksPerCta = 2;

int team_config_for(hb_ctx *ctx, int n, int want_ctas, TeamConfig *cfg)
{
    const int nch = (n + 31) / 32;
    int ctas = want_ctas > 0 ? want_ctas
                             : std::min(16, std::max(1, (nch + kTeamChunksPerCta - 1) / kTeamChunksPerCta));
    for (;;) {
        const cudaError_t e = team_setup(ctx->order, ctas, cfg);
        if (e == cudaSuccess && cfg->max_teams >= 1) break;
        cudaGetLastError();
        if (want_ctas > 0 || ctas <= 8) return fail(ctx, HB_ERR_CUDA, "a team of %d CTAs cannot be scheduled", ctas);
        ctas = 8;
    }
    if ((long long)((nch + ctas - 1) / ctas) * 32 > cfg->jl_cap_g)
        return fail(ctx, HB_ERR_TOO_LARGE, "%d slots do not fit a team of %d CTAs (%d slots each)", n,
                    ctas, cfg->jl_cap_g);
    return HB_OK;
}

// The engine the next hb_integrator_run uses.
int resolve_engine(hb_ctx *ctx, TeamConfig *cfg)
{
    if (ctx->engine == HB_ENGINE_GRAPH) return HB_ENGINE_GRAPH;
    if (ctx->engine == HB_ENGINE_PERSISTENT) return HB_ENGINE_PERSISTENT;
    const bool fp64 = ctx->precision == HB_FP64;
    if (ctx->engine == HB_ENGINE_TEAM) {
        if (!fp64) return -fail(ctx, HB_ERR_INVALID, "the team engine integrates in FP64 only");
        const int s = team_config_for(ctx, ctx->nbody, ctx->team_ctas, cfg);
        return s == HB_OK ? HB_ENGINE_TEAM : -s;
    }
    if (!fp64 || ctx->nbody > kTeamAutoMaxBody) return HB_ENGINE_GRAPH;
    return team_config_for(ctx, ctx->nbody, ctx->team_ctas, cfg) == HB_OK ? HB_ENGINE_TEAM
                                                                          : HB_ENGINE_GRAPH;
}

int run_team(hb_ctx *ctx, const TeamConfig &cfg, double tend, long long max_block_steps)
{
    volatile IntStatus *st = ctx->h_status;
    HB_CK(team_sched_sync(ctx->d_sched, ctx->d_team_state, true, ctx->stream));
    TeamLaunch L;
    L.jp = ctx->d_jp;
    L.dt = ctx->d_dt;
    L.aux = ctx->d_aux;
    L.sys = ctx->d_team_sys;
    L.st = ctx->d_team_state;
    L.next_sys = ctx->d_team_next;
    L.nsys = 1;
    if (team_shape(ctx->order, cfg, ctx->nbody, &L) != 0)
        return fail(ctx, HB_ERR_TOO_LARGE, "the system does not fit a team of %d CTAs", cfg.ctas);
    L.tend = tend;
    L.etapow = ctx->h_sched->etapow;
    L.dtmax = ctx->h_sched->dtmax;
    const long long first_steps = st->block_steps;
    long long last_steps = st->block_steps;
    while (st->tsys < tend) {
        long long budget = kTeamStepsPerLaunch;
        if (max_block_steps > 0) {
            const long long left = max_block_steps - (st->block_steps - first_steps);
            if (left <= 0)
                return fail(ctx, HB_ERR_STATE, "block-step limit %lld reached at t = %.17g",
                            max_block_steps, st->tsys);
            budget = std::min(budget, left);
        }
        L.max_steps = budget;
        HB_CK(cudaMemsetAsync(ctx->d_team_next, 0, sizeof(int), ctx->stream));
        HB_CK(team_launch(ctx->order, L, 1, ctx->stream));
        HB_CK(team_sched_sync(ctx->d_sched, ctx->d_team_state, false, ctx->stream));
        ctx->launches += 1;
        const int s = sync_stream(ctx);
        if (s != HB_OK) return s;
        if (st->error) return fail(ctx, HB_ERR_STATE, "a timestep underflowed (< 2^-48)");
        if (st->block_steps == last_steps && st->tsys < tend)
            return fail(ctx, HB_ERR_STATE, "integration stalled at t = %.17g", st->tsys);
        last_steps = st->block_steps;
    }
    return HB_OK;
}

// The persistent engine: one cooperative launch per kPersistStepsPerLaunch
// block steps; the host reads the mapped status between launches.
constexpr long long kPersistStepsPerLaunch = 4096;

int run_persistent(hb_ctx *ctx, double tend, long long max_block_steps)
{
    if (ctx->persist_grid <= 0)
        return fail(ctx, HB_ERR_CUDA, "the persistent kernel cannot be resident on this device");
    volatile IntStatus *st = ctx->h_status;
    const long long first_steps = st->block_steps;
    long long last_steps = st->block_steps;
    while (st->tsys < tend) {
        long long budget = kPersistStepsPerLaunch;
        if (max_block_steps > 0) {
            const long long left = max_block_steps - (st->block_steps - first_steps);
            if (left <= 0)
                return fail(ctx, HB_ERR_STATE, "block-step limit %lld reached at t = %.17g",
                            max_block_steps, st->tsys);
            budget = std::min(budget, left);
        }
        HB_CK(persistent_launch(ctx->order, ctx->int_L, ctx->d_gbar, budget, ctx->wait_limit,
                                ctx->persist_grid, ctx->stream));
        ctx->launches += 1;
        const int s = sync_stream(ctx);
        if (s != HB_OK) {
            // a barrier or tile wait gave up: the barrier words are left mid-use
            cudaMemsetAsync(ctx->d_gbar, 0, 2 * sizeof(unsigned), ctx->stream);
            cudaStreamSynchronize(ctx->stream);
            return s;
        }
        if (st->error)
            return fail(ctx, st->error == 2 ? HB_ERR_DEVICE_TIMEOUT : HB_ERR_STATE,
                        st->error == 2 ? "a device-side wait gave up" : "a timestep underflowed (< 2^-48)");
        if (st->block_steps == last_steps && st->tsys < tend)
            return fail(ctx, HB_ERR_STATE, "integration stalled at t = %.17g", st->tsys);
        last_steps = st->block_steps;
    }
    return HB_OK;
}
}  // namespace

int hb_integrator_set_engine(hb_ctx *ctx, int engine, int team_ctas)
{
    if (!ctx || engine < HB_ENGINE_AUTO || engine > HB_ENGINE_PERSISTENT || team_ctas < 0 ||
        team_ctas > 16)
        return HB_ERR_INVALID;
    ctx->engine = engine;
    ctx->team_ctas = team_ctas;
    return HB_OK;
}

int hb_integrator_engine(hb_ctx *ctx, int *engine, int *team_ctas)
{
    if (!ctx) return HB_ERR_INVALID;
    TeamConfig cfg{};
    const int r = resolve_engine(ctx, &cfg);
    if (r < 0) return -r;
    if (engine) *engine = r;
    if (team_ctas) *team_ctas = r == HB_ENGINE_TEAM ? cfg.ctas : 0;
    return HB_OK;
}

int hb_integrator_run(hb_ctx *ctx, double tend, long long max_block_steps)
{
    if (!ctx) return HB_ERR_INVALID;
    if (!ctx->int_ready) return fail(ctx, HB_ERR_STATE, "hb_integrator_run before hb_integrator_init");
    int s = sync_stream(ctx);
    if (s != HB_OK) return s;
    volatile IntStatus *st = ctx->h_status;
    if (!(tend >= st->tsys)) return fail(ctx, HB_ERR_INVALID, "tend %g is before tsys %g", tend, st->tsys);
    HB_CK(cudaMemcpy(&ctx->d_sched->tend, &tend, sizeof(double), cudaMemcpyHostToDevice));
    TeamConfig cfg{};
    const int engine = resolve_engine(ctx, &cfg);
    if (engine < 0) return -engine;
    if (engine == HB_ENGINE_TEAM) return run_team(ctx, cfg, tend, max_block_steps);
    if (engine == HB_ENGINE_PERSISTENT) return run_persistent(ctx, tend, max_block_steps);
    long long last_steps = st->block_steps;
    const long long first_steps = st->block_steps;
    while (st->tsys < tend) {
        if (max_block_steps > 0 && st->block_steps - first_steps >= max_block_steps)
            return fail(ctx, HB_ERR_STATE, "block-step limit %lld reached at t = %.17g",
                        max_block_steps, st->tsys);
        HB_CK(cudaGraphLaunch(ctx->int_exec, ctx->stream));
        ctx->launches += 5LL * kStepsPerGraph;
        s = sync_stream(ctx);
        if (s != HB_OK) return s;
        if (st->error)
            return fail(ctx, st->error == 2 ? HB_ERR_DEVICE_TIMEOUT : HB_ERR_STATE,
                        st->error == 2 ? "a device-side wait gave up" : "a timestep underflowed (< 2^-48)");
        if (st->block_steps == last_steps && st->tsys < tend)
            return fail(ctx, HB_ERR_STATE, "integration stalled at t = %.17g", st->tsys);
        last_steps = st->block_steps;
    }
    return HB_OK;
}

int hb_integrator_stats(const hb_ctx *ctx, long long *particle_steps, long long *block_steps,
                        double *tsys)
{
    if (!ctx || !ctx->h_status) return HB_ERR_INVALID;
    const volatile IntStatus *st = ctx->h_status;
    if (particle_steps) *particle_steps = st->particle_steps;
    if (block_steps) *block_steps = st->block_steps;
    if (tsys) *tsys = st->tsys;
    return HB_OK;
}

int hb_energy(hb_ctx *ctx, double eps2, double *kinetic, double *potential)
{
    if (!ctx || !kinetic || !potential) return HB_ERR_INVALID;
    if (!(eps2 >= 0.0)) return fail(ctx, HB_ERR_INVALID, "eps2 must be >= 0");
    int s = integrator_alloc(ctx);
    if (s == HB_OK) s = do_upload(ctx);
    if (s != HB_OK) return s;
    HB_CK(launch_potential(ctx->order, ctx->d_jp, ctx->nbody, ctx->npad, eps2, ctx->d_posm,
                           ctx->d_pot, ctx->d_err, ctx->stream));
    HB_CK(integrator_energy(ctx->order, ctx->d_jp, ctx->d_pot, ctx->nbody, ctx->d_epart,
                            ctx->d_eout, ctx->stream));
    ctx->launches += 4;
    s = sync_stream(ctx);
    if (s != HB_OK) return s;
    *kinetic = ctx->h_eout[0];
    *potential = ctx->h_eout[1];
    return HB_OK;
}

int hb_get_records(hb_ctx *ctx, int addr0, int count, double *records_out, double *dt_out)
{
    if (!ctx || addr0 < 0 || count < 0 || (long long)addr0 + count > ctx->nbody ||
        (count > 0 && !records_out))
        return HB_ERR_INVALID;
    int s = sync_stream(ctx);
    if (s != HB_OK || count == 0) return s;
    HB_CK(cudaMemcpy(records_out, ctx->d_jp + (size_t)addr0 * ctx->R,
                     sizeof(double) * (size_t)count * ctx->R, cudaMemcpyDeviceToHost));
    if (dt_out) {
        if (!ctx->d_dt) return fail(ctx, HB_ERR_STATE, "no timesteps before hb_integrator_init");
        HB_CK(cudaMemcpy(dt_out, ctx->d_dt + addr0, sizeof(double) * (size_t)count,
                         cudaMemcpyDeviceToHost));
    }
    return HB_OK;
}

int hb_measure_fma_peak(int precision, double *gflops)
{
    if (!gflops || precision < 0 || precision > 2) return HB_ERR_INVALID;
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return HB_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return HB_ERR_NO_DEVICE;
    // precision: 0 = FP64, 1 = FP32 scalar FMA, 2 = FP32 packed (f32x2) FMA
    return run_fma_peak(precision, nsm, gflops) == cudaSuccess ? HB_OK : HB_ERR_CUDA;
}

}  // extern "C"
