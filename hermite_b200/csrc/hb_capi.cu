// hb_capi.cu -- the C ABI (include/hermite_b200.h): context, host mirror,
// uploads, launch-shape selection and error reporting.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "hermite_b200.h"
#include "hb_common.cuh"
#include "hb_internal.h"

namespace hb {
const ForceVariant *force_variant_64(int order, int v);
const ForceVariant *force_variant_mixed(int order, int v);

int force_variant_count(int order, bool) { return (order == 4 || order == 6 || order == 8) ? 5 : 0; }

const ForceVariant *force_variant(int order, bool mixed, int v)
{
    return mixed ? force_variant_mixed(order, v) : force_variant_64(order, v);
}
}  // namespace hb

using namespace hb;

namespace {
constexpr int kMaxBody = 1 << 24;
constexpr int kNumVariants = 5;

int rec_words(int order) { return 8 + 3 * (order - 2); }
int force_words(int order) { return 3 * (order / 2); }
int pred64_ncomp(int order) { return 7 + 3 * (order / 2 - 2); }
int predmx_ncomp(int order) { return 10 + 3 * (order / 2 - 2); }
}  // namespace

struct hb_ctx {
    int order = 0, nbody = 0, npad = 0;
    int precision = HB_FP64;        // used by the next predict_all
    int pred_precision = -1;        // layout of the current predicted array
    int R = 0, F = 0;
    int device = 0, nsm = 0;
    cudaStream_t own_stream = nullptr, stream = nullptr;

    double *h_jp = nullptr, *h_force = nullptr, *h_pot = nullptr;
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

// Launch shape for the force kernel: variant by nact, then the number of
// j-slices so that the grid fills the device, each CTA keeps at least a few
// chunks per warp, and the partials fit in the scratch buffer.
int pick_variant(const hb_ctx *c, int nact)
{
    if (c->variant_override >= 0) return c->variant_override;
    if (nact <= 32) return 2;
    if (nact <= 64) return 3;
    if (nact <= c->nsm * 256) return 0;
    return 1;
}

int run_force(hb_ctx *ctx, int nact, double eps2)
{
    if (nact == 0) return HB_OK;
    const bool mixed = ctx->pred_precision == HB_MIXED;
    const int v = pick_variant(ctx, nact);
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
    int S = ctx->jsplit_override;
    if (S <= 0) {
        const int target = ctx->nsm * ctx->blocks_per_sm[m][v];
        S = gx >= target ? 1 : (target + gx - 1) / gx;
        // at least 8 chunks (256 j) per CTA and 2 chunks per j-warp
        S = std::min(S, std::max(1, nchunk / std::max(8, 2 * fv->wj)));
    }
    S = std::max(1, std::min(S, nchunk));
    if (S > 1) {
        const size_t need_per_slice = (size_t)gx * fv->ti * ctx->F;
        const size_t smax = ctx->partial_cap / need_per_slice;
        if ((size_t)S > smax) S = (int)std::max<size_t>(1, smax);
    }
    ForceArgs a;
    a.pred = ctx->d_pred;
    a.nchunk = nchunk;
    a.nact = nact;
    a.eps2 = eps2;
    a.force = ctx->d_force;
    a.partial = ctx->d_partial;
    a.counter = ctx->d_counter;
    a.err = ctx->d_err;
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
    if (ctx->ev_upload) cudaEventDestroy(ctx->ev_upload);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return HB_OK;
}

int hb_create(int order, int nbody, int precision, hb_ctx **out)
{
    if (!out) return HB_ERR_INVALID;
    *out = nullptr;
    if (!valid_order(order) || nbody < 1 || nbody > kMaxBody ||
        (precision != HB_FP64 && precision != HB_MIXED))
        return HB_ERR_INVALID;

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
    ok = ok && cudaHostAlloc((void **)&ctx->h_force, np * ctx->F * sizeof(double), cudaHostAllocPortable) == cudaSuccess;
    ok = ok && cudaHostAlloc((void **)&ctx->h_pot, np * sizeof(double), cudaHostAllocPortable) == cudaSuccess;
    ok = ok && cudaHostAlloc((void **)&ctx->h_err, sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_jp, np * ctx->R * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_force, np * ctx->F * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_pot, np * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_posm, np * 4 * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_partial, ctx->partial_cap * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&ctx->d_pred, pred_bytes) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&ctx->d_counter, (np / 32 + 1) * sizeof(unsigned)) == cudaSuccess;
    if (ok) {
        ok = cudaHostGetDevicePointer((void **)&ctx->d_err, ctx->h_err, 0) == cudaSuccess;
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
    std::memcpy(ctx->h_jp + (size_t)addr0 * ctx->R, records,
                sizeof(double) * (size_t)count * ctx->R);
    mark_dirty(ctx, addr0, addr0 + count);
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
    const bool mixed = ctx->precision == HB_MIXED;
    HB_CK(launch_predict(ctx->order, mixed, ctx->d_jp, ctx->nbody, ctx->npad, tsys, ctx->d_pred,
                         ctx->d_err, ctx->stream));
    ctx->launches++;
    ctx->pred_precision = ctx->precision;
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
    return run_force(ctx, nact, eps2);
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
    if (nact > 0) std::memcpy(force_out, ctx->h_force, sizeof(double) * (size_t)nact * ctx->F);
    return HB_OK;
}

int hb_force_first_nact(hb_ctx *ctx, int nact, double eps2, double *force_out)
{
    if (!ctx) return HB_ERR_INVALID;
    if (nact > 0 && !force_out) return fail(ctx, HB_ERR_INVALID, "force_out is NULL");
    int s = hb_force_device(ctx, nact, eps2);
    if (s != HB_OK) return s;
    s = hb_download_forces(ctx, nact, force_out);
    if (s != HB_OK) return s;
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
    std::memcpy(pot_out, ctx->h_pot, sizeof(double) * ctx->nbody);
    return HB_OK;
}

int hb_set_precision(hb_ctx *ctx, int precision)
{
    if (!ctx) return HB_ERR_INVALID;
    if (precision != HB_FP64 && precision != HB_MIXED)
        return fail(ctx, HB_ERR_INVALID, "precision %d unknown", precision);
    ctx->precision = precision;
    return HB_OK;
}

int hb_get_precision(const hb_ctx *ctx) { return ctx ? ctx->precision : -1; }

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

int hb_force_variant_count(int order, int precision)
{
    if (!valid_order(order) || (precision != HB_FP64 && precision != HB_MIXED)) return 0;
    return force_variant_count(order, precision == HB_MIXED);
}

int hb_force_variant_info(int order, int precision, int variant, int *threads, int *i_per_thread,
                          int *j_warps)
{
    if (!valid_order(order) || (precision != HB_FP64 && precision != HB_MIXED)) return HB_ERR_INVALID;
    const ForceVariant *fv = force_variant(order, precision == HB_MIXED, variant);
    if (!fv) return HB_ERR_INVALID;
    if (threads) *threads = fv->nw * 32;
    if (i_per_thread) *i_per_thread = fv->ni;
    if (j_warps) *j_warps = fv->wj;
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
