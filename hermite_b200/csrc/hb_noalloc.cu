// hb_noalloc.cu -- force on predicted j-particles with no memory allocation.
//
// For callers that cannot call cudaMalloc: code embedded in a host framework
// that owns every device allocation through its own pool (an allocation behind
// the pool's back breaks its accounting or fails against its reservation),
// and fixed-budget jobs on a shared GPU that must not grow their footprint
// after start-up.  They own the input and output buffers; the only
// scratch the force kernel needs (the j-slice partial sums and the per-i-tile
// arrival counters) lives in the file-scope device array below, which the
// library holds on every GPU it is loaded on until the process exits.
#include <algorithm>
#include <mutex>

#include "hermite_b200.h"
#include "hb_common.cuh"
#include "hb_internal.h"

namespace {

// Limits of the shared scratch.
constexpr int kNoAllocMaxSlots = 1 << 20;                        // predicted slots
constexpr int kCounterWords = kNoAllocMaxSlots / 32;            // one per i-tile
constexpr size_t kCounterBytes = kCounterWords * sizeof(unsigned);   // 128 KiB
constexpr size_t kPartialDoubles = (size_t)1 << 19;             // 4 MiB of partials
constexpr size_t kScratchBytes = kCounterBytes + kPartialDoubles * sizeof(double);
constexpr int kMaxDevices = 64;

// counters at offset 0, FP64 partials after them (256-byte aligned)
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DeviceScratch {
    std::mutex mu;
    unsigned char *base = nullptr;   // device address of g_noalloc_scratch
    int nsm = 0;
};
DeviceScratch g_dev[kMaxDevices];

// With device `dev` current: the device address of the scratch array (its
// host-side name is only a stand-in) and the SM count, looked up on the first
// successful call for that device and kept from then on.  A failed lookup is
// returned and not kept, so a later call tries again.
cudaError_t scratch_for_device(int dev, DeviceScratch *&out)
{
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    DeviceScratch &d = g_dev[dev];
    std::lock_guard<std::mutex> lock(d.mu);
    if (!d.base) {
        void *p = nullptr;
        int nsm = 0;
        cudaError_t st = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (st == cudaSuccess) st = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (st != cudaSuccess) return st;
        d.nsm = nsm;
        d.base = static_cast<unsigned char *>(p);
    }
    out = &d;
    return cudaSuccess;
}

bool valid_order(int order) { return order == 4 || order == 6 || order == 8; }

}  // namespace

extern "C" int hb_force_predicted_noalloc(int order, int precision, const void *pred, int nslots,
                                          int nact, double eps2, double *force, void *stream)
{
    if (!valid_order(order) || (precision != HB_FP64 && precision != HB_MIXED)) return HB_ERR_INVALID;
    if (nslots < 1 || nslots % hb::kSlotPad != 0 || nact < 0 || nact > nslots || !(eps2 >= 0.0) ||
        !pred || (nact > 0 && !force))
        return HB_ERR_INVALID;
    if (nslots > kNoAllocMaxSlots) return HB_ERR_TOO_LARGE;
    if (nact == 0) return HB_OK;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return HB_ERR_NO_DEVICE;
    DeviceScratch *ds = nullptr;
    if (scratch_for_device(dev, ds) != cudaSuccess) return HB_ERR_CUDA;

    const bool mixed = precision == HB_MIXED;
    // launch shape: as the context path picks it, with the slice count bounded
    // by the shared partial buffer
    const int v = nact <= 32 ? 2 : nact <= 64 ? 3 : nact <= ds->nsm * 256 ? 0 : 1;
    const hb::ForceVariant *fv = hb::force_variant(order, mixed, v);
    if (!fv) return HB_ERR_INVALID;
    if (fv->smem > 48 * 1024 &&
        cudaFuncSetAttribute(fv->kern, cudaFuncAttributeMaxDynamicSharedMemorySize, fv->smem) != cudaSuccess)
        return HB_ERR_CUDA;
    const int nchunk = nslots / 32;
    const int gx = (nact + fv->ti - 1) / fv->ti;
    const int target = ds->nsm * 4;
    int S = gx >= target ? 1 : (target + gx - 1) / gx;
    S = std::min(S, std::max(1, nchunk / std::max(8, 2 * fv->wj)));
    const size_t per_slice = (size_t)gx * fv->ti * (3 * (order / 2));
    S = (int)std::max<size_t>(1, std::min<size_t>((size_t)S, kPartialDoubles / per_slice));

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned *counter = reinterpret_cast<unsigned *>(ds->base);
    // The scratch keeps the previous call's contents: the arrival counters of
    // the i-tiles this launch uses must start at zero.
    if (S > 1 && cudaMemsetAsync(counter, 0, sizeof(unsigned) * gx, s) != cudaSuccess) return HB_ERR_CUDA;

    hb::ForceArgs a{};
    a.pred = pred;
    a.nchunk = nchunk;
    a.nact = nact;
    a.eps2 = eps2;
    a.force = force;
    a.partial = reinterpret_cast<double *>(ds->base + kCounterBytes);
    a.counter = counter;
    a.err = nullptr;
    a.spin = hb::kSpinLimit;
    // cudaLaunchKernel returns this launch's own status, so an earlier,
    // unrelated error on the caller's thread is neither blamed on this call
    // nor cleared by it.
    void *args[] = {&a};
    const cudaError_t st = cudaLaunchKernel(reinterpret_cast<const void *>(fv->kern), dim3(gx, S),
                                            dim3(fv->nw * 32), args, (size_t)fv->smem, s);
    return st == cudaSuccess ? HB_OK : HB_ERR_CUDA;
}
