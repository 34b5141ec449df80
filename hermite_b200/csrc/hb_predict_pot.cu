// hb_predict_pot.cu -- predictor, potential and the FMA-peak probe.
#include <type_traits>
#include "hb_internal.h"
#include "hb_math.cuh"

namespace hb {

// ---------------------------------------------------------------------------
// Predictor (replaces predict_kernel, SRC/hermite4-titan.cu:80-99,
// SRC/hermite6-titan.cu:113-133, SRC/hermite8-titan.cu:153-172).
// One thread per slot.  The CTA's 128 contiguous AoS records are brought into
// shared memory by one bulk async copy; the outputs are written per
// component into the AoSoA32 predicted layout (full 128/256-byte stores).
// Slots in [n, npad) are written as zero-mass far-away padding.
constexpr int kPredThreads = 128;

template <int ORDER, bool MIXED>
__global__ void __launch_bounds__(kPredThreads)
predict_kernel(const double *__restrict__ jp, int n, int npad, double tsys,
               void *__restrict__ pred, int *err)
{
    constexpr int R = Rec<ORDER>::words;
    __shared__ __align__(128) double rec[kPredThreads * R];
    __shared__ __align__(8) uint64_t bar;
    const int tid = threadIdx.x;
    const int base = blockIdx.x * kPredThreads;
    const int cnt = min(kPredThreads, n - base);

    if (cnt > 0) {
        if (tid == 0) {
            mbar_init(&bar, 1);
            fence_mbar_init();
        }
        __syncthreads();
        if (tid == 0) {
            // a bulk copy moves a multiple of 16 bytes: with 29-word records
            // (ORDER 9) a partial last block rounds up by 8 bytes, which stay
            // inside the padded record array and the staging buffer
            const uint32_t bytes = (uint32_t)((cnt * R * 8 + 15) & ~15);
            mbar_arrive_expect_tx(&bar, bytes);
            bulk_load(rec, jp + (size_t)base * R, bytes, &bar);
        }
        const bool ok = mbar_wait_bounded(&bar, 0);
        if (!__syncthreads_and(ok)) {
            if (tid == 0) {
                raise_error(err, kErrWaitTimeout);
                mbar_wait_bounded(&bar, 0);
            }
            return;
        }
    }
    const int slot = base + tid;
    if (slot >= npad) return;
    double x[3], v[3], a[3] = {0, 0, 0}, jk[3] = {0, 0, 0}, xl[3] = {0, 0, 0}, m;
    if (tid < cnt) {
        const double *r = rec + tid * R;
        predict_slot<ORDER>(r, tsys, x, v, a, jk, xl);
        m = r[3];
    } else {
        for (int k = 0; k < 3; ++k) { x[k] = pad_position(slot, k); v[k] = 0.0; }
        m = 0.0;
    }
    const int ci = slot >> 5, lane = slot & 31;
    if constexpr (MIXED) {
        constexpr int NC = PredMx<ORDER>::ncomp;
        float *c = static_cast<float *>(pred) + (size_t)ci * NC * 32 + lane;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float hi = __double2float_rn(x[k]);
            c[(PMX_XH + k) * 32] = hi;
            c[(PMX_XL + k) * 32] = __double2float_rn(x[k] - (double)hi);
            c[(PMX_V + k) * 32] = __double2float_rn(v[k]);
            if constexpr (ORDER >= 6) c[(PMX_A + k) * 32] = __double2float_rn(a[k]);
            if constexpr (ORDER == 8) c[(PMX_J + k) * 32] = __double2float_rn(jk[k]);
        }
        c[PMX_M * 32] = __double2float_rn(m);
    } else {
        constexpr int NC = Pred64<ORDER>::ncomp;
        double *c = static_cast<double *>(pred) + (size_t)ci * NC * 32 + lane;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            c[(P64_X + k) * 32] = x[k];
            c[(P64_V + k) * 32] = v[k];
            if constexpr (ORDER >= 6) c[(P64_A + k) * 32] = a[k];
            if constexpr (ORDER >= 8) c[(P64_J + k) * 32] = jk[k];
            if constexpr (ORDER == 9) c[(P64_XL + k) * 32] = xl[k];
        }
        c[P64_M * 32] = m;
    }
}

template <int ORDER, bool MIXED>
static cudaError_t launch_predict_t(const double *jp, int n, int npad, double tsys,
                                    void *pred, int *err, cudaStream_t s)
{
    const int grid = npad / kPredThreads;   // npad is a multiple of 256
    predict_kernel<ORDER, MIXED><<<grid, kPredThreads, 0, s>>>(jp, n, npad, tsys, pred, err);
    return cudaGetLastError();
}

cudaError_t launch_predict(int order, bool mixed, const double *jp, int n, int npad,
                           double tsys, void *pred, int *err, cudaStream_t s)
{
    switch (order * 2 + (mixed ? 1 : 0)) {
    case 8:  return launch_predict_t<4, false>(jp, n, npad, tsys, pred, err, s);
    case 9:  return launch_predict_t<4, true>(jp, n, npad, tsys, pred, err, s);
    case 12: return launch_predict_t<6, false>(jp, n, npad, tsys, pred, err, s);
    case 13: return launch_predict_t<6, true>(jp, n, npad, tsys, pred, err, s);
    case 16: return launch_predict_t<8, false>(jp, n, npad, tsys, pred, err, s);
    case 17: return launch_predict_t<8, true>(jp, n, npad, tsys, pred, err, s);
    case 18: return launch_predict_t<9, false>(jp, n, npad, tsys, pred, err, s);
    }
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// Potential (replaces pot_kernel + calc_potential, SRC/pot-titan.hu:80-171).
// Pass 1 packs (x, y, z, m) of the un-predicted records into AoSoA32;
// pass 2 sums phi_i = -sum_{j != i} m_j / sqrt(r^2 + eps2) in FP64 with the
// same bulk-copy ring as the force kernel.  Each 32-slot chunk is summed
// separately and then added to the running total (two-level blocked sum;
// the reference uses a four-level cascade, SRC/pot-titan.hu:103-114).
// ORDER 9 (double-double positions) packs (x, y, z, m, xL, yL, zL) and takes
// the separation as (xj - xi) + (xLj - xLi) (calc_potential,
// SRC/hermite8dd.h:397-416).
template <int ORDER> constexpr int posm_comps() { return ORDER == 9 ? 7 : 4; }

template <int ORDER>
__global__ void pack_posm_kernel(const double *__restrict__ jp, int n, int npad,
                                 double *__restrict__ posm)
{
    constexpr int R = Rec<ORDER>::words, NC = posm_comps<ORDER>();
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= npad) return;
    double *c = posm + (size_t)(slot >> 5) * NC * 32 + (slot & 31);
    if (slot < n) {
        const double *r = jp + (size_t)slot * R;
        for (int k = 0; k < 4; ++k) c[k * 32] = r[k];
        if constexpr (NC == 7)
            for (int k = 0; k < 3; ++k) c[(4 + k) * 32] = r[kRecPosL + k];
    } else {
        for (int k = 0; k < 3; ++k) c[k * 32] = pad_position(slot, k);
        c[3 * 32] = 0.0;
        if constexpr (NC == 7)
            for (int k = 0; k < 3; ++k) c[(4 + k) * 32] = 0.0;
    }
}

constexpr int kPotThreads = 128;
constexpr int kPotTileChunks = 8;

template <int NC>
__global__ void __launch_bounds__(kPotThreads)
potential_kernel(const double *__restrict__ posm, int nchunk, int n, double eps2,
                 double *__restrict__ pot, int *err)
{
    constexpr int kPosmChunkBytes = NC * 32 * 8;
    constexpr int TB = kPotTileChunks * kPosmChunkBytes;
    __shared__ __align__(128) unsigned char ring[2 * TB];
    __shared__ __align__(8) uint64_t bar[2];
    const int tid = threadIdx.x;
    const int i = blockIdx.x * kPotThreads + tid;   // < npad always
    const double *ci = posm + (size_t)(i >> 5) * NC * 32 + (i & 31);
    const double xi = ci[0], yi = ci[32], zi = ci[64];
    double xli = 0.0, yli = 0.0, zli = 0.0;
    if constexpr (NC == 7) {
        xli = ci[128];
        yli = ci[160];
        zli = ci[192];
    }
    const int ntile = (nchunk + kPotTileChunks - 1) / kPotTileChunks;

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t) {
        const int cnt = min(kPotTileChunks, nchunk - t * kPotTileChunks);
        const uint32_t bytes = (uint32_t)(cnt * kPosmChunkBytes);
        mbar_arrive_expect_tx(&bar[t & 1], bytes);
        bulk_load(ring + (t & 1) * TB,
                  reinterpret_cast<const unsigned char *>(posm) + (size_t)t * TB, bytes, &bar[t & 1]);
    };
    if (tid == 0) {
        issue(0);
        if (ntile > 1) issue(1);
    }
    double total = 0.0;
    for (int t = 0; t < ntile; ++t) {
        const bool got = mbar_wait_bounded(&bar[t & 1], (uint32_t)((t >> 1) & 1));
        if (!__syncthreads_and(got)) {
            if (tid == 0) {
                raise_error(err, kErrWaitTimeout);
                for (int u = t; u < ntile && u < t + 2; ++u)
                    mbar_wait_bounded(&bar[u & 1], (uint32_t)((u >> 1) & 1));
            }
            return;
        }
        const int cnt = min(kPotTileChunks, nchunk - t * kPotTileChunks);
        const double *tile = reinterpret_cast<const double *>(ring + (t & 1) * TB);
        for (int q = 0; q < cnt; ++q) {
            const double *cp = tile + q * NC * 32;
            const int jbase = (t * kPotTileChunks + q) * 32;
            double part = 0.0;
#pragma unroll 8
            for (int jl = 0; jl < 32; ++jl) {
                double dx = cp[jl] - xi, dy = cp[32 + jl] - yi, dz = cp[64 + jl] - zi;
                if constexpr (NC == 7) {
                    dx = dx + (cp[128 + jl] - xli);
                    dy = dy + (cp[160 + jl] - yli);
                    dz = dz + (cp[192 + jl] - zli);
                }
                const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
                const double mj = (jbase + jl == i) ? 0.0 : cp[96 + jl];
                part = fma(-mj, rsqrt_fp64(r2), part);
            }
            total += part;
        }
        __syncthreads();
        if (tid == 0 && t + 2 < ntile) issue(t + 2);
    }
    if (i < n) pot[i] = total;
}

cudaError_t launch_potential(int order, const double *jp, int n, int npad, double eps2,
                             double *posm, double *pot, int *err, cudaStream_t s)
{
    const int g = npad / 128;
    switch (order) {
    case 4: pack_posm_kernel<4><<<g, 128, 0, s>>>(jp, n, npad, posm); break;
    case 6: pack_posm_kernel<6><<<g, 128, 0, s>>>(jp, n, npad, posm); break;
    case 8: pack_posm_kernel<8><<<g, 128, 0, s>>>(jp, n, npad, posm); break;
    case 9: pack_posm_kernel<9><<<g, 128, 0, s>>>(jp, n, npad, posm); break;
    default: return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (order == 9)
        potential_kernel<7><<<npad / kPotThreads, kPotThreads, 0, s>>>(posm, npad / 32, n, eps2, pot, err);
    else
        potential_kernel<4><<<npad / kPotThreads, kPotThreads, 0, s>>>(posm, npad / 32, n, eps2, pot, err);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FMA-pipe peak probe: independent register-resident FMA chains, no memory
// traffic inside the timed loop.  mode 0 = FP64 (DFMA), 1 = FP32 (FFMA),
// 2 = packed FP32 (f32x2 FMA, two FMAs per instruction).
constexpr int kPeakChains = 8;
constexpr int kPeakIters = 4096;

template <int MODE>
__global__ void __launch_bounds__(256) fma_peak_kernel(float seed, double *sink)
{
    if constexpr (MODE == 0) {
        double r[kPeakChains];
        for (int c = 0; c < kPeakChains; ++c) r[c] = seed + threadIdx.x + c;
        const double a = 0.999999, b = 1e-7;
#pragma unroll 4
        for (int it = 0; it < kPeakIters; ++it)
#pragma unroll
            for (int c = 0; c < kPeakChains; ++c) r[c] = fma(r[c], a, b);
        double s = 0;
        for (int c = 0; c < kPeakChains; ++c) s += r[c];
        if (s == 12345.678) sink[0] = s;
    } else if constexpr (MODE == 1) {
        float r[kPeakChains];
        for (int c = 0; c < kPeakChains; ++c) r[c] = seed + threadIdx.x + c;
        const float a = 0.999999f, b = 1e-7f;
#pragma unroll 4
        for (int it = 0; it < kPeakIters; ++it)
#pragma unroll
            for (int c = 0; c < kPeakChains; ++c) r[c] = fmaf(r[c], a, b);
        float s = 0;
        for (int c = 0; c < kPeakChains; ++c) s += r[c];
        if (s == 12345.678f) sink[0] = s;
    } else {
        float2 r[kPeakChains];
        for (int c = 0; c < kPeakChains; ++c) r[c] = make_float2(seed + threadIdx.x + c, seed - c);
        const float2 a = f2(0.999999f), b = f2(1e-7f);
#pragma unroll 4
        for (int it = 0; it < kPeakIters; ++it)
#pragma unroll
            for (int c = 0; c < kPeakChains; ++c) r[c] = fma2(r[c], a, b);
        float s = 0;
        for (int c = 0; c < kPeakChains; ++c) s += r[c].x + r[c].y;
        if (s == 12345.678f) sink[0] = s;
    }
}

cudaError_t run_fma_peak(int mode, int nsm, double *gflops)
{
    double *sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, sizeof(double));
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int grid = nsm * 8, block = 256;
    auto launch = [&]() {
        if (mode == 0) fma_peak_kernel<0><<<grid, block>>>(1.0f, sink);
        else if (mode == 1) fma_peak_kernel<1><<<grid, block>>>(1.0f, sink);
        else fma_peak_kernel<2><<<grid, block>>>(1.0f, sink);
    };
    for (int w = 0; w < 3; ++w) launch();
    float best_ms = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        launch();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) best_ms = ms;
    }
    e = cudaGetLastError();
    const double fmas = (double)grid * block * kPeakIters * kPeakChains * (mode == 2 ? 2 : 1);
    *gflops = 2.0 * fmas / (best_ms * 1e-3) * 1e-9;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return e;
}

}  // namespace hb
