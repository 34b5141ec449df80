// hb_force.cuh -- direct-summation force kernel (FP64 and mixed precision).
//
// Replaces force_kernel + reduce_kernel of the reference's CUDA path
// (SRC/hermite4-titan.cu:189-238,303-327; SRC/hermite6-titan.cu:245-299,
// 302-326; SRC/hermite8-titan.cu:304-364,367-391) with one kernel:
//
//   grid  = (i-tiles, j-slices S); block = NW warps.
//   * j-particles stream through shared memory in tiles of TCH 32-slot
//     chunks, brought in by bulk async copies (cp.async.bulk, non-multicast)
//     into a two-stage ring completed on mbarriers; every wait is bounded.
//   * a warp owns NI 32-slot chunks of i-particles (register blocking);
//     the CTA's NW warps form WI = NW/WJ i-groups, and the WJ warps of an
//     i-group split each j tile between them (small-nact occupancy).
//   * j-slices of one i-tile are separate CTAs (blockIdx.y), as the
//     reference's NJBLOCK; their FP64 partials meet in a scratch buffer and
//     the last CTA of the i-tile to finish adds them in slice order -- no
//     second launch, and the sum order is fixed, so results are
//     deterministic for a given launch shape.
#pragma once
#include <type_traits>
#include "hb_common.cuh"
#include "hb_internal.h"
#include "hb_math.cuh"

namespace hb {


template <int ORDER, bool MIXED>
struct Layout {
    static constexpr int ncomp = MIXED ? PredMx<ORDER>::ncomp : Pred64<ORDER>::ncomp;
    static constexpr int chunk_bytes = MIXED ? PredMx<ORDER>::chunk_bytes
                                             : Pred64<ORDER>::chunk_bytes;
};

template <int ORDER, bool MIXED, int NW, int NI, int WJ, int TCH, bool FUSED = false>
struct ForceShape {
    static constexpr int F = Frc<ORDER>::words;
    static constexpr int WI = NW / WJ;
    static constexpr int TI = WI * 32 * NI;         // i per CTA
    static constexpr int STG = 2;
    static constexpr int CB = Layout<ORDER, MIXED>::chunk_bytes;
    // two-pass: the ring holds predicted tiles; fused: the ring holds raw
    // records and one predicted tile sits after it
    static constexpr int tile_bytes = FUSED ? TCH * 32 * Rec<ORDER>::bytes : TCH * CB;
    static constexpr int ring_bytes = STG * tile_bytes;
    static constexpr int ptile_bytes = FUSED ? TCH * CB : 0;
    static constexpr int red_bytes = (WJ - 1) * WI * NI * F * 32 * 8;
    static constexpr int work_bytes = ring_bytes + ptile_bytes;
    static constexpr int body_bytes = work_bytes > red_bytes ? work_bytes : red_bytes;
    static constexpr int smem_bytes = body_bytes + 64;   // + mbarriers
    static_assert(NW % WJ == 0, "WJ must divide NW");
    static_assert(256 % TI == 0, "i-tile must divide the slot padding");
    static_assert(!FUSED || TI <= TCH * 32, "fused: the i-tile must fit one raw stage");
};

// Predicts nslot consecutive records (raw, AoS) to tsys into the predicted
// AoSoA32 layout at `out` (FP64 or hi/lo mixed), slots >= n as padding.
// One out-of-line copy serves both the i- and the j-particles of the fused
// kernel, so a particle's two predicted states are bit-identical and its
// self term stays exactly zero.
template <int ORDER, bool MIXED>
__device__ __noinline__ void predict_tile(const double *raw, int nslot, int slot0, int n,
                                          double tsys, void *out)
{
    constexpr int R = Rec<ORDER>::words;
    for (int q = threadIdx.x; q < nslot; q += blockDim.x) {
        double x[3], v[3], a[3] = {0, 0, 0}, jk[3] = {0, 0, 0}, xl[3] = {0, 0, 0}, m;
        const int slot = slot0 + q;
        if (slot < n) {
            const double *r = raw + (size_t)q * R;
            predict_slot<ORDER>(r, tsys, x, v, a, jk, xl);
            m = r[3];
        } else {
            for (int k = 0; k < 3; ++k) { x[k] = pad_position(slot, k); v[k] = 0.0; }
            m = 0.0;
        }
        const int ci = q >> 5, lane = q & 31;
        if constexpr (MIXED) {
            constexpr int NC = PredMx<ORDER>::ncomp;
            float *c = static_cast<float *>(out) + ci * NC * 32 + lane;
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
            double *c = static_cast<double *>(out) + ci * NC * 32 + lane;
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
}

// Loads the i-particles of lane `lane` in chunk `ci` from the predicted array.
template <int ORDER>
__device__ __forceinline__ void load_i64(const double *pred, int ci, int lane, Body64 &b)
{
    constexpr int NC = Pred64<ORDER>::ncomp;
    const double *c = pred + (size_t)ci * NC * 32 + lane;
#pragma unroll
    for (int k = 0; k < 3; ++k) { b.x[k] = c[(P64_X + k) * 32]; b.v[k] = c[(P64_V + k) * 32]; }
    b.m = c[P64_M * 32];
    if constexpr (ORDER >= 6) {
#pragma unroll
        for (int k = 0; k < 3; ++k) b.a[k] = c[(P64_A + k) * 32];
    }
    if constexpr (ORDER >= 8) {
#pragma unroll
        for (int k = 0; k < 3; ++k) b.jk[k] = c[(P64_J + k) * 32];
    }
    if constexpr (ORDER == 9) {
#pragma unroll
        for (int k = 0; k < 3; ++k) b.xl[k] = c[(P64_XL + k) * 32];
    }
}

template <int ORDER>
__device__ __forceinline__ void load_i_mixed(const float *pred, int ci, int lane, NegI32 &b)
{
    constexpr int NC = PredMx<ORDER>::ncomp;
    const float *c = pred + (size_t)ci * NC * 32 + lane;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        b.xh[k] = f2(-c[(PMX_XH + k) * 32]);
        b.xl[k] = f2(-c[(PMX_XL + k) * 32]);
        b.v[k] = f2(-c[(PMX_V + k) * 32]);
        if constexpr (ORDER >= 6) b.a[k] = f2(-c[(PMX_A + k) * 32]);
        if constexpr (ORDER == 8) b.jk[k] = f2(-c[(PMX_J + k) * 32]);
    }
}

// Compensated (Kahan) accumulation of FP64 partial sums: `tot` carries the
// running sum of a long j range and `cmp` its lost low-order part, so the
// sum over all j stays within a few ulp of exact however long the range.
// (Plain sequential FP64 over 2^20 terms of one sign drifts by ~1e-14
// relative -- at a particle far outside the cluster, 4e-14 against 3e-16
// for 84 blocks of 2^20/84 -- and the 8th-order corrector amplifies the
// step-to-step part of that by up to dt^-7.)  `part` is added and cleared.
template <int NI, int F>
__device__ __forceinline__ void kahan_fold(double (&tot)[NI][F], double (&cmp)[NI][F],
                                           double (&part)[NI][F])
{
#pragma unroll
    for (int n = 0; n < NI; ++n)
#pragma unroll
        for (int c = 0; c < F; ++c) {
            const double y = __dsub_rn(part[n][c], cmp[n][c]);
            const double t = __dadd_rn(tot[n][c], y);
            cmp[n][c] = __dsub_rn(__dsub_rn(t, tot[n][c]), y);
            tot[n][c] = t;
            part[n][c] = 0.0;
        }
}

// The FP64 j-sums of the 8th-order schemes are Kahan-compensated per tile:
// their corrector turns step-to-step rounding noise of the force into the
// timestep criterion with factors up to dt^-7 (an outer particle of the
// 8th-order N = 2^20 configuration reached a timestep below 2^-48 on plain
// sums over 2^20 terms).  Lower orders keep plain sums and their occupancy.
template <int ORDER, bool MIXED>
constexpr bool kKahan = !MIXED && ORDER >= 8;

// One 32-slot j chunk (in shared memory) against this thread's NI i-particles.
template <int ORDER, int NI>
__device__ __forceinline__ void chunk64(const double *cp, const Body64 (&I)[NI],
                                        double eps2, double (&f)[NI][Frc<ORDER>::words])
{
#pragma unroll 2
    for (int jl = 0; jl < 32; jl += 2) {
        Body64 J0, J1;
        double2 w;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            w = *reinterpret_cast<const double2 *>(cp + (P64_X + k) * 32 + jl); J0.x[k] = w.x; J1.x[k] = w.y;
            w = *reinterpret_cast<const double2 *>(cp + (P64_V + k) * 32 + jl); J0.v[k] = w.x; J1.v[k] = w.y;
            if constexpr (ORDER >= 6) {
                w = *reinterpret_cast<const double2 *>(cp + (P64_A + k) * 32 + jl); J0.a[k] = w.x; J1.a[k] = w.y;
            }
            if constexpr (ORDER >= 8) {
                w = *reinterpret_cast<const double2 *>(cp + (P64_J + k) * 32 + jl); J0.jk[k] = w.x; J1.jk[k] = w.y;
            }
            if constexpr (ORDER == 9) {
                w = *reinterpret_cast<const double2 *>(cp + (P64_XL + k) * 32 + jl); J0.xl[k] = w.x; J1.xl[k] = w.y;
            }
        }
        w = *reinterpret_cast<const double2 *>(cp + P64_M * 32 + jl); J0.m = w.x; J1.m = w.y;
#pragma unroll
        for (int n = 0; n < NI; ++n) {
            interact64<ORDER>(I[n], J0, eps2, f[n]);
            interact64<ORDER>(I[n], J1, eps2, f[n]);
        }
    }
}

// Small blocks (FP64): the lanes of a warp form groups of G = 2^LOG2G lanes;
// the lanes of group p share i-particle p and lane g of the group adds
// j = g, g + G, ... of the chunk.  lanes_log2g picks G = 32 / P for P = nact
// rounded up to a power of two (nact <= 16, so G >= 2).
__host__ __device__ __forceinline__ int lanes_log2g(int nact)
{
    int lg = 5;
    while ((1 << (5 - lg)) < nact) --lg;
    return lg;
}

template <int ORDER, int LOG2G>
__device__ __forceinline__ void chunk64_lanes(const double *cp, const Body64 &I, double eps2,
                                              double (&f)[Frc<ORDER>::words])
{
    constexpr int G = 1 << LOG2G, P = 32 / G;
    const int g = threadIdx.x & (G - 1);
#pragma unroll
    for (int k = 0; k < P; ++k) {
        Body64 J;
        load_i64<ORDER>(cp, 0, g + k * G, J);
        interact64<ORDER>(I, J, eps2, f);
    }
}

template <int ORDER>
__device__ __forceinline__ void chunk64_lanes(int log2g, const double *cp, const Body64 &I,
                                              double eps2, double (&f)[Frc<ORDER>::words])
{
    switch (log2g) {
    case 1: chunk64_lanes<ORDER, 1>(cp, I, eps2, f); break;
    case 2: chunk64_lanes<ORDER, 2>(cp, I, eps2, f); break;
    case 3: chunk64_lanes<ORDER, 3>(cp, I, eps2, f); break;
    case 4: chunk64_lanes<ORDER, 4>(cp, I, eps2, f); break;
    default: chunk64_lanes<ORDER, 5>(cp, I, eps2, f); break;
    }
}

// After the j sums of a small block: the G lanes of each group add theirs in
// a fixed butterfly, then lane p takes group p's sum (lanes p >= 32/G keep
// group 0's), so the results sit where the one-i-per-lane code has them.
template <int F>
__device__ __forceinline__ void lanes_gather(int log2g, double (&f)[F])
{
    const int G = 1 << log2g, lane = threadIdx.x & 31;
    for (int o = G >> 1; o > 0; o >>= 1)
#pragma unroll
        for (int q = 0; q < F; ++q) f[q] += __shfl_xor_sync(0xffffffffu, f[q], o);
    const int src = (lane < (32 >> log2g) ? lane : 0) << log2g;
#pragma unroll
    for (int q = 0; q < F; ++q) f[q] = __shfl_sync(0xffffffffu, f[q], src);
}

template <int ORDER, int NI, bool REFINE>
__device__ __forceinline__ void chunk_mixed(const float *cp, const NegI32 (&I)[NI], float2 eps2,
                                            double (&f)[NI][Frc<ORDER>::words])
{
    constexpr int FS = Frc<ORDER>::words;
    float2 s[NI][FS];
#pragma unroll
    for (int n = 0; n < NI; ++n)
#pragma unroll
        for (int c = 0; c < FS; ++c) s[n][c] = make_float2(0.f, 0.f);

#pragma unroll 2
    for (int jl = 0; jl < 32; jl += 2) {
        JPair32 J;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            J.xh[k] = *reinterpret_cast<const float2 *>(cp + (PMX_XH + k) * 32 + jl);
            J.xl[k] = *reinterpret_cast<const float2 *>(cp + (PMX_XL + k) * 32 + jl);
            J.v[k] = *reinterpret_cast<const float2 *>(cp + (PMX_V + k) * 32 + jl);
            if constexpr (ORDER >= 6) J.a[k] = *reinterpret_cast<const float2 *>(cp + (PMX_A + k) * 32 + jl);
            if constexpr (ORDER == 8) J.jk[k] = *reinterpret_cast<const float2 *>(cp + (PMX_J + k) * 32 + jl);
        }
        J.m = *reinterpret_cast<const float2 *>(cp + PMX_M * 32 + jl);
#pragma unroll
        for (int n = 0; n < NI; ++n) interact_mixed<ORDER, REFINE>(I[n], J, eps2, s[n]);
    }
    // flush the FP32 partial sums (16 pairs per lane half) into the FP64
    // accumulators
#pragma unroll
    for (int n = 0; n < NI; ++n)
#pragma unroll
        for (int c = 0; c < FS; ++c) f[n][c] += (double)s[n][c].x + (double)s[n][c].y;
}

// The end of a force launch, shared by the kernels below: the WJ warps of an
// i-group add their FP64 sums (fixed order, through shared memory); with one
// j-slice the sums are the forces; otherwise each slice publishes its
// partial and the last CTA of the i-tile to arrive (threadfence + arrival
// counter) adds the S partials in slice order and resets the counter.
template <int ORDER, int NW, int NI, int WJ, int WI, int TI>
__device__ __forceinline__ void force_epilogue(double (&f)[NI][Frc<ORDER>::words],
                                               unsigned char *smem, const ForceArgs &a,
                                               int ig, int jg, int ichunk0)
{
    constexpr int F = Frc<ORDER>::words;
    __shared__ unsigned s_last;
    const int tid = threadIdx.x, lane = tid & 31;
    const int S = gridDim.y, sl = blockIdx.y;
    // Combine the WJ warps of each i-group (fixed order), through the ring.
    if constexpr (WJ > 1) {
        double *red = reinterpret_cast<double *>(smem);
        if (jg > 0) {
#pragma unroll
            for (int n = 0; n < NI; ++n)
#pragma unroll
                for (int c = 0; c < F; ++c)
                    red[((((jg - 1) * WI + ig) * NI + n) * F + c) * 32 + lane] = f[n][c];
        }
        __syncthreads();
        if (jg == 0) {
            for (int g = 1; g < WJ; ++g)
#pragma unroll
                for (int n = 0; n < NI; ++n)
#pragma unroll
                    for (int c = 0; c < F; ++c)
                        f[n][c] += red[((((g - 1) * WI + ig) * NI + n) * F + c) * 32 + lane];
        }
    }

    if (S == 1) {
        if (jg == 0) {
#pragma unroll
            for (int n = 0; n < NI; ++n) {
                const int i = (ichunk0 + n) * 32 + lane;
                if (i < a.nact) {
#pragma unroll
                    for (int c = 0; c < F; ++c) a.force[(size_t)i * F + c] = f[n][c];
                }
            }
        }
        return;
    }

    // j-split across CTAs: publish this slice's partial, last CTA reduces.
    const size_t ispan = (size_t)gridDim.x * TI;
    if (jg == 0) {
#pragma unroll
        for (int n = 0; n < NI; ++n) {
            const int i = (ichunk0 + n) * 32 + lane;
#pragma unroll
            for (int c = 0; c < F; ++c) a.partial[((size_t)sl * ispan + i) * F + c] = f[n][c];
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(&a.counter[blockIdx.x], 1u) == (unsigned)(S - 1));
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // Sum the S slice partials of this i-tile.  With few values per tile the
    // slices are split among thread groups (g, g+G, g+2G, ...) and the group
    // sums are added in group order; the order is fixed either way.
    constexpr int T = NW * 32;
    const int i0 = blockIdx.x * TI;
    const int V = min(TI, a.nact - i0) * F;
    const size_t sstride = ispan * F;
    const double *pbase = a.partial + (size_t)i0 * F;
    if (V >= T / 2) {
        for (int e = tid; e < V; e += T) {
            double sum = 0.0;
            int s = 0;
            for (; s + 4 <= S; s += 4) {
                const double p0 = __ldcg(pbase + (size_t)(s + 0) * sstride + e);
                const double p1 = __ldcg(pbase + (size_t)(s + 1) * sstride + e);
                const double p2 = __ldcg(pbase + (size_t)(s + 2) * sstride + e);
                const double p3 = __ldcg(pbase + (size_t)(s + 3) * sstride + e);
                sum += p0; sum += p1; sum += p2; sum += p3;
            }
            for (; s < S; ++s) sum += __ldcg(pbase + (size_t)s * sstride + e);
            a.force[(size_t)i0 * F + e] = sum;
        }
    } else {
        const int G = T / V;
        const int g = tid / V, e = tid % V;
        double *red = reinterpret_cast<double *>(smem);   // the ring is idle now
        if (g < G) {
            double sum = 0.0;
            for (int s = g; s < S; s += G) sum += __ldcg(pbase + (size_t)s * sstride + e);
            red[tid] = sum;
        }
        __syncthreads();
        if (tid < V) {
            double sum = red[tid];
            for (int gg = 1; gg < G; ++gg) sum += red[gg * V + tid];
            a.force[(size_t)i0 * F + tid] = sum;
        }
    }
    if (tid == 0) a.counter[blockIdx.x] = 0u;
}

// Mixed precision: one Newton step on the hardware rsqrt measured no more
// accurate on B200 (acc error max 4.4e-7 vs 5.0e-7, median 5.5e-8 vs 2.0e-8
// without it, 6th order N=262144) and 8% slower, so it is off by default.
#ifndef HB_MIXED_REFINE
#define HB_MIXED_REFINE 0
#endif

template <int ORDER, bool MIXED, int NW, int NI, int WJ, int TCH, int MINB, bool FUSED = false,
          bool REFINE = (HB_MIXED_REFINE != 0)>
__global__ void __launch_bounds__(NW * 32, MINB)
force_kernel(ForceArgs a)
{
    using Sh = ForceShape<ORDER, MIXED, NW, NI, WJ, TCH, FUSED>;
    constexpr int F = Sh::F, WI = Sh::WI, TI = Sh::TI, STG = Sh::STG, CB = Sh::CB;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + Sh::body_bytes);
    unsigned char *ptile = smem + Sh::ring_bytes;          // fused only
    constexpr int RB = Rec<ORDER>::bytes;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ig = warp % WI, jg = warp / WI;
    const int S = gridDim.y, sl = blockIdx.y;
    const int c0 = (int)(((long long)sl * a.nchunk) / S);
    const int c1 = (int)(((long long)(sl + 1) * a.nchunk) / S);
    const int ntile = (c1 - c0 + TCH - 1) / TCH;
    const int ichunk0 = (blockIdx.x * TI) / 32 + ig * NI;   // first i chunk of this warp

    // i-particles and accumulators (8th order FP64: per-tile sums in f,
    // Kahan-folded into tot/cmp)
    constexpr bool KAHAN = kKahan<ORDER, MIXED>;
    double f[NI][F], tot[NI][F], cmp[NI][F];
#pragma unroll
    for (int n = 0; n < NI; ++n)
#pragma unroll
        for (int c = 0; c < F; ++c) f[n][c] = tot[n][c] = cmp[n][c] = 0.0;

    using IBody = typename std::conditional<MIXED, NegI32, Body64>::type;
    IBody I[NI];

    if (tid == 0) {
#pragma unroll
        for (int st = 0; st < STG + 1; ++st) mbar_init(&bar[st], 1);
        fence_mbar_init();
    }
    __syncthreads();

    if constexpr (FUSED) {
        // this CTA's i-records -> raw stage 0 -> predicted tile -> registers
        if (tid == 0) {
            const uint32_t bytes = (uint32_t)(TI * RB);
            mbar_arrive_expect_tx(&bar[STG], bytes);
            bulk_load(smem, a.jp + (size_t)blockIdx.x * TI * Rec<ORDER>::words, bytes, &bar[STG]);
        }
        const bool got = mbar_wait_bounded(&bar[STG], 0, a.spin);
        if (!__syncthreads_and(got)) {
            if (tid == 0) {
                raise_error(a.err, kErrWaitTimeout);
                mbar_wait_bounded(&bar[STG], 0);
            }
            return;
        }
        predict_tile<ORDER, MIXED>(reinterpret_cast<const double *>(smem), TI, blockIdx.x * TI,
                                   a.nbody, a.tsys, ptile);
        __syncthreads();
#pragma unroll
        for (int n = 0; n < NI; ++n) {
            if constexpr (MIXED) load_i_mixed<ORDER>(reinterpret_cast<const float *>(ptile), ig * NI + n, lane, I[n]);
            else load_i64<ORDER>(reinterpret_cast<const double *>(ptile), ig * NI + n, lane, I[n]);
        }
        __syncthreads();
    } else {
#pragma unroll
        for (int n = 0; n < NI; ++n) {
            if constexpr (MIXED) load_i_mixed<ORDER>(static_cast<const float *>(a.pred), ichunk0 + n, lane, I[n]);
            else load_i64<ORDER>(static_cast<const double *>(a.pred), ichunk0 + n, lane, I[n]);
        }
    }

    auto issue = [&](int t) {   // thread 0 only
        const int st = t % STG;
        const int cs = c0 + t * TCH;
        const int cnt = min(TCH, c1 - cs);
        if constexpr (FUSED) {
            const uint32_t bytes = (uint32_t)(cnt * 32 * RB);
            mbar_arrive_expect_tx(&bar[st], bytes);
            bulk_load(smem + st * Sh::tile_bytes, a.jp + (size_t)cs * 32 * Rec<ORDER>::words,
                      bytes, &bar[st]);
        } else {
            const uint32_t bytes = (uint32_t)(cnt * CB);
            mbar_arrive_expect_tx(&bar[st], bytes);
            bulk_load(smem + st * Sh::tile_bytes,
                      static_cast<const unsigned char *>(a.pred) + (size_t)cs * CB, bytes, &bar[st]);
        }
    };
    if (tid == 0)
        for (int t = 0; t < STG && t < ntile; ++t) issue(t);

    const float2 eps2f = f2((float)a.eps2);
    int failed_at = -1;
    for (int t = 0; t < ntile; ++t) {
        const int st = t % STG;
        const bool got = mbar_wait_bounded(&bar[st], (uint32_t)((t / STG) & 1), a.spin);
        if (!__syncthreads_and(got)) { failed_at = t; break; }
        const int cnt = min(TCH, c1 - (c0 + t * TCH));
        const unsigned char *tile = smem + st * Sh::tile_bytes;
        if constexpr (FUSED) {
            predict_tile<ORDER, MIXED>(reinterpret_cast<const double *>(tile), cnt * 32,
                                       (c0 + t * TCH) * 32, a.nbody, a.tsys, ptile);
            __syncthreads();
            if (tid == 0 && t + STG < ntile) issue(t + STG);   // the raw stage is free
            tile = ptile;
        }
        for (int q = jg; q < cnt; q += WJ) {
            if constexpr (MIXED)
                chunk_mixed<ORDER, NI, REFINE>(reinterpret_cast<const float *>(tile + q * CB), I, eps2f, f);
            else
                chunk64<ORDER, NI>(reinterpret_cast<const double *>(tile + q * CB), I, a.eps2, f);
        }
        if constexpr (KAHAN) kahan_fold<NI, F>(tot, cmp, f);
        __syncthreads();
        if (!FUSED && tid == 0 && t + STG < ntile) issue(t + STG);
    }
    if (failed_at >= 0) {
        // Leave no bulk copy writing into this CTA's shared memory after exit.
        if (tid == 0) {
            raise_error(a.err, kErrWaitTimeout);
            for (int t = failed_at; t < ntile && t < failed_at + STG; ++t)
                mbar_wait_bounded(&bar[t % STG], (uint32_t)((t / STG) & 1));
        }
        return;
    }
    if constexpr (KAHAN) {
#pragma unroll
        for (int n = 0; n < NI; ++n)
#pragma unroll
            for (int c = 0; c < F; ++c) f[n][c] = __dsub_rn(tot[n][c], cmp[n][c]);
    }

    force_epilogue<ORDER, NW, NI, WJ, WI, TI>(f, smem, a, ig, jg, ichunk0);
}



}  // namespace hb
