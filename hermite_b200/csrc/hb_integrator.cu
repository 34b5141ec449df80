// hb_integrator.cu -- block-timestep Hermite integration resident on the GPU.
//
// The reference integrates on the host: per block step NbodySystem finds the
// next block time and the active set (calc_dtlim / count_nact over a
// dt-sorted array, SRC/nbodysystem.h:652-690), calls the force calculator,
// corrects the active particles and re-sorts them (:693-765).  Here the whole
// step stays on the device, four phases per step, replayed from a captured
// CUDA graph (no host round trip per step):
//   1. next block time  = min over slots of (tlast + dt)   (grid reduction)
//   2. active set       = slots with tlast + dt == tnext    (compaction),
//                         dtlim from tnext                  (calc_dtlim)
//   3. force            = fused predict + force on the active set, work items
//                         (i-tile, j-slice) sized on the device from nact
//   4. corrector        = Particle::correct + quantised Aarseth dt
// Slots are never re-sorted; the j summation order is the slot order.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "hermite_b200.h"
#include "hb_common.cuh"
#include "hb_corrector.cuh"
#include "hb_force.cuh"
#include "hb_internal.h"

namespace hb {

constexpr unsigned long long kInfBits = 0x7ff0000000000000ull;   // +inf
// Steps with more active slots than this use the large-step force kernel
// (measured on N = 65536, 4th order: 512 and 2048 lose to the 32-slot items,
// 4096 gains a few per cent).
#ifndef HB_BIG_NACT
#define HB_BIG_NACT 4096
#endif
constexpr int kBigNact = HB_BIG_NACT;
// Small steps: j-slices of at least this many 32-slot chunks, and a slice
// count aimed at this percentage of the launch's work-item target.
#ifndef HB_ITEMS_MIN_CHUNKS
#define HB_ITEMS_MIN_CHUNKS 8
#endif
#ifndef HB_ITEMS_TARGET_PCT
#define HB_ITEMS_TARGET_PCT 100
#endif

// Programmatic dependent launch: let the next kernel of the step be
// scheduled now, then wait until the previous kernel's results are visible.
// (The step's kernels are launched with programmatic stream serialisation;
// without it both instructions are no-ops.)
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ---------------------------------------------------------------------------
template <int ORDER>
__device__ __forceinline__ void min_phase(const double *__restrict__ jp, const double *__restrict__ dt,
                                          int n, Sched *s)
{
    constexpr int R = Rec<ORDER>::words;
    double m = __longlong_as_double((long long)kInfBits);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = fmin(m, dt[i] + jp[(size_t)i * R + 7]);
    for (int o = 16; o; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : __longlong_as_double((long long)kInfBits);
        for (int o = 16; o; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) atomicMin(&s->tnext_bits, (unsigned long long)__double_as_longlong(m));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        s->nact = 0;
        s->work = 0;
    }
}

template <int ORDER>
__global__ void sched_min_kernel(const double *__restrict__ jp, const double *__restrict__ dt,
                                 int n, Sched *s)
{
    pdl_enter();
    min_phase<ORDER>(jp, dt, n, s);
}

// Active set and dtlim.  Positive doubles order like their bit patterns.
// Returns whether the step is live (tnext within tend and no error): the same
// answer in every thread of the grid.
template <int ORDER>
__device__ __forceinline__ bool compact_phase(const double *__restrict__ jp,
                                              const double *__restrict__ dt, int n, Sched *s,
                                              int *__restrict__ ilist)
{
    constexpr int R = Rec<ORDER>::words;
    const double tnext = __longlong_as_double((long long)s->tnext_bits);
    const bool live = tnext <= s->tend && s->error == 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        // calc_dtlim (SRC/nbodysystem.h:652-661): the largest power-of-two
        // fraction of dtmax that tnext is a multiple of
        double dtlim = s->dtmax, q = tnext / s->dtmax;
        for (int k = 0; k < 64 && q != trunc(q); ++k) {
            q *= 2.0;
            dtlim *= 0.5;
        }
        s->tnext = tnext;
        s->dtlim = dtlim;
    }
    if (!live) return false;
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int i = base + threadIdx.x;
        const bool act = i < n && dt[i] + jp[(size_t)i * R + 7] == tnext;
        const unsigned ballot = __ballot_sync(0xffffffffu, act);
        int off = 0;
        if ((threadIdx.x & 31) == 0 && ballot) off = atomicAdd(&s->nact, __popc(ballot));
        off = __shfl_sync(0xffffffffu, off, 0);
        if (act) ilist[off + __popc(ballot & ((1u << (threadIdx.x & 31)) - 1u))] = i;
    }
    return true;
}

template <int ORDER>
__global__ void sched_compact_kernel(const double *__restrict__ jp, const double *__restrict__ dt,
                                     int n, Sched *s, int *__restrict__ ilist)
{
    pdl_enter();
    compact_phase<ORDER>(jp, dt, n, s, ilist);
}

// Sum of the S slice partials of one i-tile (V values, slice stride sstride
// doubles) by the T threads of the last CTA to finish it.  Every value is
// summed in the same association whatever V is: kGroups interleaved partial
// sums (slices g, g + kGroups, ...), each in slice order, then added in group
// order.  (The tile a particle lands in, and so V, depends on the order of
// the active list, which the compaction does not fix; the association must
// not.)  With few values the groups of one value go to different threads
// and meet in red[]; the result is the same bits either way.
constexpr int kGroups = 8;

template <int T>
__device__ __forceinline__ void sum_slices(const double *pbase, size_t sstride, int S, int V,
                                           double *out, double *red)
{
    const int tid = threadIdx.x;
    if (V * kGroups <= T) {
        const int g = tid / V, e = tid % V;
        if (g < kGroups) {
            double sum = 0.0;
            for (int s = g; s < S; s += kGroups) sum += __ldcg(pbase + (size_t)s * sstride + e);
            red[tid] = sum;
        }
        __syncthreads();
        if (tid < V) {
            double sum = red[tid];
#pragma unroll
            for (int gg = 1; gg < kGroups; ++gg) sum += red[gg * V + tid];
            out[tid] = sum;
        }
    } else {
        for (int e = tid; e < V; e += T) {
            double acc[kGroups];
#pragma unroll
            for (int g = 0; g < kGroups; ++g) acc[g] = 0.0;
            int s = 0;
            for (; s + kGroups <= S; s += kGroups) {
#pragma unroll
                for (int g = 0; g < kGroups; ++g) acc[g] += __ldcg(pbase + (size_t)(s + g) * sstride + e);
            }
#pragma unroll
            for (int g = 0; g < kGroups; ++g)
                if (s + g < S) acc[g] += __ldcg(pbase + (size_t)(s + g) * sstride + e);
            double sum = acc[0];
#pragma unroll
            for (int g = 1; g < kGroups; ++g) sum += acc[g];
            out[e] = sum;
        }
    }
}

// Fused predict + force over work items (i-tile of 32 active slots, j-slice),
// taken from a device counter by a grid sized once; one warp per quarter of
// every j tile (the 32 i are shared by the CTA's 4 warps).
struct ItemsArgs {
    const double *jp;
    const int *ilist;
    Sched *s;
    double *force;      // [nact][F], indexed by position in ilist
    double *partial;    // [S][gx*32][F]
    unsigned *counter;  // [gx]
    int *err;
    int n, nchunk;
    size_t partial_cap;
    int target_items;
    int big_nact;       // steps with more active slots take the large-step kernel
};

template <int ORDER, bool MIXED>
using ItemsShape = ForceShape<ORDER, MIXED, 4, 1, 4, 4, true>;

// (8th-order FP64 j-sums are Kahan-compensated per tile: kKahan, hb_force.cuh)

// The work items of one step with 1..big_nact active slots, taken by this CTA
// until none are left.  smem: ItemsShape's layout; bar: two initialised
// mbarriers whose phases continue from g (tiles issued by this CTA before).
// Returns false when a wait gave up (the error is raised, the CTA's copies
// drained).
template <int ORDER, bool MIXED>
__device__ __forceinline__ bool items_phase(const ItemsArgs &a, unsigned char *smem, uint64_t *bar,
                                            unsigned &g)
{
    constexpr int NW = 4, WJ = 4, TCH = 4, STG = 2, TI = 32;
    constexpr int F = Frc<ORDER>::words, R = Rec<ORDER>::words, RB = Rec<ORDER>::bytes;
    using Sh = ItemsShape<ORDER, MIXED>;
    constexpr int CB = Sh::CB;
    unsigned char *ptile = smem + Sh::ring_bytes;
    __shared__ int s_item;
    __shared__ unsigned s_last;

    const int nact = a.s->nact;
    const double tsys = a.s->tnext, eps2 = a.s->eps2;
    const int tid = threadIdx.x, lane = tid & 31, jg = tid >> 5;
    const int gx = (nact + TI - 1) / TI;
    const int target = (int)((long long)a.target_items * HB_ITEMS_TARGET_PCT / 100);
    int S = (target + gx - 1) / gx;
    S = max(1, min(S, max(1, a.nchunk / HB_ITEMS_MIN_CHUNKS)));
    while (S > 1 && (size_t)S * gx * TI * F > a.partial_cap) --S;
    const int items = gx * S;
    const size_t ispan = (size_t)gx * TI;
    // FP64 steps of at most kLanesMaxAct active slots: lanes share an
    // i-particle and split each chunk's j (lanes_log2g, hb_force.cuh)
    constexpr bool kLaneSplit = !MIXED && ORDER != 9;
    const int lg = kLaneSplit && nact <= kLanesMaxAct ? lanes_log2g(nact) : 0;

    const float2 eps2f = f2((float)eps2);
    for (;;) {
        if (tid == 0) s_item = atomicAdd(&a.s->work, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= items) break;
        const int itile = item / S, sl = item % S;

        // gather the 32 i-records of this tile and predict them
        double *raw = reinterpret_cast<double *>(smem);
        for (int w = tid; w < TI * R; w += NW * 32) {
            const int q = w / R, k = itile * TI + q;
            const int slot = a.ilist[k < nact ? k : nact - 1];
            raw[w] = a.jp[(size_t)slot * R + (w - q * R)];
        }
        __syncthreads();
        predict_tile<ORDER, MIXED>(raw, TI, 0, 0x7fffffff, tsys, ptile);
        __syncthreads();
        using IBody = typename std::conditional<MIXED, NegI32, Body64>::type;
        IBody I[1];
        if constexpr (MIXED) load_i_mixed<ORDER>(reinterpret_cast<const float *>(ptile), 0, lane, I[0]);
        else load_i64<ORDER>(reinterpret_cast<const double *>(ptile), 0, lg ? min(lane >> lg, nact - 1) : lane, I[0]);
        __syncthreads();

        double f[1][F], tot[1][F], cmp[1][F];   // FP64: per-tile sums, Kahan-folded
#pragma unroll
        for (int c = 0; c < F; ++c) f[0][c] = tot[0][c] = cmp[0][c] = 0.0;
        const int c0 = (int)(((long long)sl * a.nchunk) / S);
        const int c1 = (int)(((long long)(sl + 1) * a.nchunk) / S);
        const int ntile = (c1 - c0 + TCH - 1) / TCH;
        auto issue = [&](int t) {
            const unsigned gt = g + t;
            const int st = gt % STG;
            const int cs = c0 + t * TCH, cnt = min(TCH, c1 - cs);
            const uint32_t bytes = (uint32_t)(cnt * 32 * RB);
            mbar_arrive_expect_tx(&bar[st], bytes);
            bulk_load(smem + st * Sh::tile_bytes, a.jp + (size_t)cs * 32 * R, bytes, &bar[st]);
        };
        if (tid == 0)
            for (int t = 0; t < STG && t < ntile; ++t) issue(t);
        int failed_at = -1;
        for (int t = 0; t < ntile; ++t) {
            const unsigned gt = g + t;
            const int st = gt % STG;
            const bool got = mbar_wait_bounded(&bar[st], (gt / STG) & 1u);
            if (!__syncthreads_and(got)) { failed_at = t; break; }
            const int cnt = min(TCH, c1 - (c0 + t * TCH));
            predict_tile<ORDER, MIXED>(reinterpret_cast<const double *>(smem + st * Sh::tile_bytes),
                                       cnt * 32, (c0 + t * TCH) * 32, a.n, tsys, ptile);
            __syncthreads();
            if (tid == 0 && t + STG < ntile) issue(t + STG);
            for (int q = jg; q < cnt; q += WJ) {
                if constexpr (MIXED) {
                    chunk_mixed<ORDER, 1, (HB_MIXED_REFINE != 0)>(reinterpret_cast<const float *>(ptile + q * CB), I, eps2f, f);
                } else {
                    if (kLaneSplit && lg)
                        chunk64_lanes<ORDER>(lg, reinterpret_cast<const double *>(ptile + q * CB), I[0], eps2, f[0]);
                    else
                        chunk64<ORDER, 1>(reinterpret_cast<const double *>(ptile + q * CB), I, eps2, f);
                }
            }
            if constexpr (kKahan<ORDER, MIXED>) kahan_fold<1, F>(tot, cmp, f);
            __syncthreads();
        }
        if (failed_at >= 0) {
            if (tid == 0) {
                raise_error(a.err, kErrWaitTimeout);
                for (int t = failed_at; t < ntile && t < failed_at + STG; ++t)
                    mbar_wait_bounded(&bar[(g + t) % STG], ((g + t) / STG) & 1u);
            }
            a.s->error = 2;
            return false;
        }
        g += ntile;
        if constexpr (kKahan<ORDER, MIXED>) {
#pragma unroll
            for (int c = 0; c < F; ++c) f[0][c] = __dsub_rn(tot[0][c], cmp[0][c]);
        }
        if (kLaneSplit && lg) lanes_gather<F>(lg, f[0]);

        // the 4 warps' j quarters, in warp order
        double *red = reinterpret_cast<double *>(smem);
        if (jg > 0)
#pragma unroll
            for (int c = 0; c < F; ++c) red[((jg - 1) * F + c) * 32 + lane] = f[0][c];
        __syncthreads();
        const int k = itile * TI + lane;
        if (jg == 0) {
            for (int w = 1; w < WJ; ++w)
#pragma unroll
                for (int c = 0; c < F; ++c) f[0][c] += red[((w - 1) * F + c) * 32 + lane];
            if (S == 1) {
                if (k < nact)
#pragma unroll
                    for (int c = 0; c < F; ++c) a.force[(size_t)k * F + c] = f[0][c];
            } else {
#pragma unroll
                for (int c = 0; c < F; ++c) a.partial[((size_t)sl * ispan + k) * F + c] = f[0][c];
            }
        }
        if (S > 1) {
            __threadfence();
            __syncthreads();
            if (tid == 0) s_last = (atomicAdd(&a.counter[itile], 1u) == (unsigned)(S - 1));
            __syncthreads();
            if (s_last) {
                __threadfence();
                sum_slices<NW * 32>(a.partial + (size_t)itile * TI * F, ispan * F, S,
                                    min(TI, nact - itile * TI) * F, a.force + (size_t)itile * TI * F,
                                    reinterpret_cast<double *>(smem));
                if (tid == 0) a.counter[itile] = 0u;
            }
        }
        __syncthreads();
    }
    return true;
}

template <int ORDER, bool MIXED>
__global__ void __launch_bounds__(128)
force_items_kernel(ItemsArgs a)
{
    pdl_enter();
    using Sh = ItemsShape<ORDER, MIXED>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + Sh::body_bytes);
    const int nact = a.s->nact;
    if (nact == 0 || nact > a.big_nact) return;   // large steps: force_items_big_kernel
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned g = 0;   // tiles issued by this CTA so far (mbarrier phases)
    items_phase<ORDER, MIXED>(a, smem, bar, g);
}

// The same work for steps with many active slots: items of 4 warps x NI
// i-chunks of 32 (NI = 2 at 4th order, 1 above, as the all-active tuning
// chose), every warp over every j tile (no in-CTA j-split).  The raw
// i-records fit the two stages of the j ring.
template <int ORDER, bool MIXED>
struct BigShape {
    static constexpr int NW = 4, NI = ORDER == 4 ? 2 : 1, TCH = 4, STG = 2, TI = NW * NI * 32;
    static constexpr int RB = Rec<ORDER>::bytes, CB = Layout<ORDER, MIXED>::chunk_bytes;
    static constexpr int tile_bytes = TCH * 32 * RB;                 // one raw j stage
    static constexpr int ring_bytes = STG * tile_bytes;
    static constexpr int ptile_bytes = (TI / 32 > TCH ? TI / 32 : TCH) * CB;
    static constexpr int smem_bytes = ring_bytes + ptile_bytes + 64;
    static_assert(TI * RB <= ring_bytes, "the raw i-tile must fit the ring");
};

// Large-step counterpart of items_phase (smem: BigShape's layout).
template <int ORDER, bool MIXED>
__device__ __forceinline__ bool big_phase(const ItemsArgs &a, unsigned char *smem, uint64_t *bar,
                                          unsigned &g)
{
    using B = BigShape<ORDER, MIXED>;
    constexpr int NW = B::NW, NI = B::NI, TCH = B::TCH, STG = B::STG, TI = B::TI, CB = B::CB;
    constexpr int F = Frc<ORDER>::words, R = Rec<ORDER>::words, RB = Rec<ORDER>::bytes;
    unsigned char *ptile = smem + B::ring_bytes;
    __shared__ int s_item;
    __shared__ unsigned s_last;

    const int nact = a.s->nact;
    const double tsys = a.s->tnext, eps2 = a.s->eps2;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int gx = (nact + TI - 1) / TI;
    int S = (a.target_items + gx - 1) / gx;
    S = max(1, min(S, max(1, a.nchunk / 8)));
    while (S > 1 && (size_t)S * gx * TI * F > a.partial_cap) --S;
    const int items = gx * S;
    const size_t ispan = (size_t)gx * TI;
    // FP64 steps of at most kLanesMaxAct active slots: lanes share an
    // i-particle and split each chunk's j (lanes_log2g, hb_force.cuh)
    constexpr bool kLaneSplit = !MIXED && ORDER != 9;
    const int lg = kLaneSplit && nact <= kLanesMaxAct ? lanes_log2g(nact) : 0;

    const float2 eps2f = f2((float)eps2);
    for (;;) {
        if (tid == 0) s_item = atomicAdd(&a.s->work, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= items) break;
        const int itile = item / S, sl = item % S;

        // gather the TI i-records of this tile into the ring, predict them
        double *raw = reinterpret_cast<double *>(smem);
        for (int w = tid; w < TI * R; w += NW * 32) {
            const int q = w / R, k = itile * TI + q;
            const int slot = a.ilist[k < nact ? k : nact - 1];
            raw[w] = a.jp[(size_t)slot * R + (w - q * R)];
        }
        __syncthreads();
        predict_tile<ORDER, MIXED>(raw, TI, 0, 0x7fffffff, tsys, ptile);
        __syncthreads();
        using IBody = typename std::conditional<MIXED, NegI32, Body64>::type;
        IBody I[NI];
#pragma unroll
        for (int n = 0; n < NI; ++n) {
            if constexpr (MIXED) load_i_mixed<ORDER>(reinterpret_cast<const float *>(ptile), warp * NI + n, lane, I[n]);
            else load_i64<ORDER>(reinterpret_cast<const double *>(ptile), warp * NI + n, lane, I[n]);
        }
        __syncthreads();

        double f[NI][F], tot[NI][F], cmp[NI][F];   // FP64: per-tile sums, Kahan-folded
#pragma unroll
        for (int n = 0; n < NI; ++n)
#pragma unroll
            for (int c = 0; c < F; ++c) f[n][c] = tot[n][c] = cmp[n][c] = 0.0;
        const int c0 = (int)(((long long)sl * a.nchunk) / S);
        const int c1 = (int)(((long long)(sl + 1) * a.nchunk) / S);
        const int ntile = (c1 - c0 + TCH - 1) / TCH;
        auto issue = [&](int t) {
            const unsigned gt = g + t;
            const int st = gt % STG;
            const int cs = c0 + t * TCH, cnt = min(TCH, c1 - cs);
            const uint32_t bytes = (uint32_t)(cnt * 32 * RB);
            mbar_arrive_expect_tx(&bar[st], bytes);
            bulk_load(smem + st * B::tile_bytes, a.jp + (size_t)cs * 32 * R, bytes, &bar[st]);
        };
        if (tid == 0)
            for (int t = 0; t < STG && t < ntile; ++t) issue(t);
        int failed_at = -1;
        for (int t = 0; t < ntile; ++t) {
            const unsigned gt = g + t;
            const int st = gt % STG;
            const bool got = mbar_wait_bounded(&bar[st], (gt / STG) & 1u);
            if (!__syncthreads_and(got)) { failed_at = t; break; }
            const int cnt = min(TCH, c1 - (c0 + t * TCH));
            predict_tile<ORDER, MIXED>(reinterpret_cast<const double *>(smem + st * B::tile_bytes),
                                       cnt * 32, (c0 + t * TCH) * 32, a.n, tsys, ptile);
            __syncthreads();
            if (tid == 0 && t + STG < ntile) issue(t + STG);
            for (int q = 0; q < cnt; ++q) {
                if constexpr (MIXED)
                    chunk_mixed<ORDER, NI, (HB_MIXED_REFINE != 0)>(reinterpret_cast<const float *>(ptile + q * CB), I, eps2f, f);
                else
                    chunk64<ORDER, NI>(reinterpret_cast<const double *>(ptile + q * CB), I, eps2, f);
            }
            if constexpr (kKahan<ORDER, MIXED>) kahan_fold<NI, F>(tot, cmp, f);
            __syncthreads();
        }
        if (failed_at >= 0) {
            if (tid == 0) {
                raise_error(a.err, kErrWaitTimeout);
                for (int t = failed_at; t < ntile && t < failed_at + STG; ++t)
                    mbar_wait_bounded(&bar[(g + t) % STG], ((g + t) / STG) & 1u);
            }
            a.s->error = 2;
            return false;
        }
        g += ntile;
        if constexpr (kKahan<ORDER, MIXED>) {
#pragma unroll
            for (int n = 0; n < NI; ++n)
#pragma unroll
                for (int c = 0; c < F; ++c) f[n][c] = __dsub_rn(tot[n][c], cmp[n][c]);
        }

        if (S == 1) {
#pragma unroll
            for (int n = 0; n < NI; ++n) {
                const int k = itile * TI + (warp * NI + n) * 32 + lane;
                if (k < nact)
#pragma unroll
                    for (int c = 0; c < F; ++c) a.force[(size_t)k * F + c] = f[n][c];
            }
        } else {
#pragma unroll
            for (int n = 0; n < NI; ++n) {
                const int k = itile * TI + (warp * NI + n) * 32 + lane;
#pragma unroll
                for (int c = 0; c < F; ++c) a.partial[((size_t)sl * ispan + k) * F + c] = f[n][c];
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) s_last = (atomicAdd(&a.counter[itile], 1u) == (unsigned)(S - 1));
            __syncthreads();
            if (s_last) {
                __threadfence();
                sum_slices<NW * 32>(a.partial + (size_t)itile * TI * F, ispan * F, S,
                                    min(TI, nact - itile * TI) * F, a.force + (size_t)itile * TI * F,
                                    reinterpret_cast<double *>(smem));
                if (tid == 0) a.counter[itile] = 0u;
            }
        }
        __syncthreads();
    }
    return true;
}

template <int ORDER, bool MIXED>
__global__ void __launch_bounds__(128)
force_items_big_kernel(ItemsArgs a)
{
    pdl_enter();
    using B = BigShape<ORDER, MIXED>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + B::ring_bytes + B::ptile_bytes);
    if (a.s->nact <= a.big_nact) return;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned g = 0;   // tiles issued by this CTA so far (mbarrier phases)
    big_phase<ORDER, MIXED>(a, smem, bar, g);
}

template <int ORDER>
__device__ __forceinline__ void correct_phase(double *__restrict__ jp, double *__restrict__ dt,
                                              const double *__restrict__ force,
                                              const int *__restrict__ ilist, Sched *s,
                                              double *__restrict__ aux)
{
    constexpr int R = Rec<ORDER>::words, F = Frc<ORDER>::words;
    const int nact = s->nact;
    const double dtlim = s->dtlim, etapow = s->etapow;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nact; k += gridDim.x * blockDim.x) {
        const int i = ilist[k];
        const double dtn = correct_particle<ORDER>(jp + (size_t)i * R, force + (size_t)k * F, dt[i],
                                                   etapow, dtlim, aux + (size_t)i * kAuxWords);
        if (!(dtn >= 0x1p-48)) s->error = 1;   // timestep underflow (or NaN)
        dt[i] = dtn;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (nact > 0) {
            s->tsys = s->tnext;
            s->particle_steps += nact;
            s->block_steps += 1;
        }
        s->tnext_bits = kInfBits;
        IntStatus *st = s->status;
        st->tsys = s->tsys;
        st->particle_steps = s->particle_steps;
        st->block_steps = s->block_steps;
        st->error = s->error;
    }
}

template <int ORDER>
__global__ void correct_kernel(double *__restrict__ jp, double *__restrict__ dt,
                               const double *__restrict__ force, const int *__restrict__ ilist,
                               Sched *s, double *__restrict__ aux)
{
    pdl_enter();
    correct_phase<ORDER>(jp, dt, force, ilist, s, aux);
}

// ---------------------------------------------------------------------------
// Persistent engine: the four phases of a block step (next block time, active
// set, force, corrector) in one cooperative kernel, its CTAs all resident,
// separated by grid barriers in place of kernel boundaries; up to max_steps
// steps per launch.  The phases are the graph engine's own code, and the
// force phases take the same work items (same target), so both engines give
// the same block steps and records bit for bit.
struct PersistArgs {
    ItemsArgs it;
    int *ilist;              // writable views of it.ilist and it.jp
    double *jp;
    double *dt, *aux;
    unsigned *gbar;          // grid barrier: [0] arrivals, [1] generation
    long long max_steps;
    unsigned spin;           // poll limit of one barrier wait
};

template <int ORDER, bool MIXED>
struct PersistSmem {
    static constexpr int items = ItemsShape<ORDER, MIXED>::body_bytes;
    static constexpr int big = BigShape<ORDER, MIXED>::ring_bytes + BigShape<ORDER, MIXED>::ptile_bytes;
    static constexpr int bar_off = ((items > big ? items : big) + 15) / 16 * 16;
    static constexpr int bytes = bar_off + 64;
};

// Barrier over a co-resident grid.  Thread 0 of each CTA reads the generation
// word, then arrives on the counter (acquire-release); the last CTA to arrive
// resets the counter and advances the generation (release), which the others
// poll (acquire).  The CTA barriers on both sides carry the ordering to the
// CTA's other threads, so every write made before the barrier anywhere in the
// grid is visible to every read after it, the bulk copies that thread 0
// issues included (proxy fences).  A wait is bounded: after `spin` polls the CTA reports false (the
// caller raises the error and returns; the other CTAs then give up at their
// next barrier).
__device__ __forceinline__ unsigned ld_relaxed_gpu(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ bool grid_barrier(unsigned *gbar, unsigned spin)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        // The phases read records with bulk copies (async proxy) that other
        // CTAs wrote with ordinary stores (generic proxy): proxy fences on
        // both sides of the barrier order the two.
        fence_proxy_async_global();
        const unsigned my = ld_relaxed_gpu(gbar + 1);
        unsigned old;
        asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;"
                     : "=r"(old) : "l"(gbar) : "memory");
        int ok = 1;
        if (old == gridDim.x - 1) {
            asm volatile("st.relaxed.gpu.global.u32 [%0], 0;" :: "l"(gbar) : "memory");
            asm volatile("red.release.gpu.global.add.u32 [%0], 1;" :: "l"(gbar + 1) : "memory");
        } else {
            ok = 0;
            for (unsigned it = 0; it < spin; ++it) {
                if (ld_acquire_gpu(gbar + 1) != my) {
                    ok = 1;
                    break;
                }
                __nanosleep(64);
            }
        }
        fence_proxy_async_global();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <int ORDER, bool MIXED>
__global__ void __launch_bounds__(128)
persistent_kernel(PersistArgs p)
{
    using P = PersistSmem<ORDER, MIXED>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + P::bar_off);
    const ItemsArgs &a = p.it;
    Sched *s = a.s;
    if (threadIdx.x == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned g = 0;   // tiles issued by this CTA so far (mbarrier phases)
    bool gave_up = false;
    for (long long k = 0; k < p.max_steps && !gave_up; ++k) {
        min_phase<ORDER>(a.jp, p.dt, a.n, s);
        if (!grid_barrier(p.gbar, p.spin)) { gave_up = true; break; }
        const bool live = compact_phase<ORDER>(a.jp, p.dt, a.n, s, p.ilist);
        if (!grid_barrier(p.gbar, p.spin)) { gave_up = true; break; }
        if (!live) {                     // every CTA reads the same state
            // as the graph engine leaves a step past tend
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                s->tnext_bits = kInfBits;
                s->status->error = s->error;   // an error set after the last status write
            }
            return;
        }
        const int nact = s->nact;
        if (nact > 0) {
            const bool ok = nact <= a.big_nact ? items_phase<ORDER, MIXED>(a, smem, bar, g)
                                               : big_phase<ORDER, MIXED>(a, smem, bar, g);
            if (!ok) return;             // raised; the others give up at the next barrier
        }
        if (!grid_barrier(p.gbar, p.spin)) { gave_up = true; break; }
        correct_phase<ORDER>(p.jp, p.dt, a.force, a.ilist, s, p.aux);
        if (!grid_barrier(p.gbar, p.spin)) { gave_up = true; break; }
    }
    if (gave_up && threadIdx.x == 0) {   // a barrier wait gave up
        s->error = 2;
        raise_error(a.err, kErrWaitTimeout);
    }
}

// Initialisation: write the force of all slots into the records (assign_force)
// and, on the last pass, the initial dt (init_dt).
template <int ORDER>
__global__ void assign_kernel(double *__restrict__ jp, double *__restrict__ dt,
                              const double *__restrict__ force, int n, int set_dt, double eta_s,
                              double dtmax)
{
    constexpr int R = Rec<ORDER>::words, F = Frc<ORDER>::words;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *r = jp + (size_t)i * R;
    const double *f = force + (size_t)i * F;
    for (int c = 0; c < F; ++c) r[8 + c] = f[c];
    if (set_dt) dt[i] = initial_dt<ORDER>(f, eta_s, dtmax);
}

// 0.5*sum m v^2 and 0.5*sum m phi, per-block partials then one block, in a
// fixed order.
template <int ORDER>
__global__ void energy_partial_kernel(const double *__restrict__ jp, const double *__restrict__ pot,
                                      int n, double *__restrict__ part)
{
    constexpr int R = Rec<ORDER>::words;
    double ke = 0.0, pe = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double *r = jp + (size_t)i * R;
        ke += r[3] * (r[4] * r[4] + r[5] * r[5] + r[6] * r[6]);
        pe += r[3] * pot[i];
    }
    __shared__ double sk[256], sp[256];
    sk[threadIdx.x] = ke;
    sp[threadIdx.x] = pe;
    __syncthreads();
    for (int o = blockDim.x / 2; o; o >>= 1) {
        if (threadIdx.x < o) {
            sk[threadIdx.x] += sk[threadIdx.x + o];
            sp[threadIdx.x] += sp[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sk[0];
        part[2 * blockIdx.x + 1] = sp[0];
    }
}

__global__ void energy_final_kernel(const double *part, int nblk, double *out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double ke = 0.0, pe = 0.0;
        for (int b = 0; b < nblk; ++b) {
            ke += part[2 * b];
            pe += part[2 * b + 1];
        }
        out[0] = 0.5 * ke;
        out[1] = 0.5 * pe;
    }
}

constexpr int kEnergyBlocks = 256;

template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kern)(KArgs...), int grid, int block, int smem, cudaStream_t s,
                              Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

template <int ORDER>
static cudaError_t launch_step(const IntegratorLaunch &L, cudaStream_t s)
{
    const int nb = std::min((L.n + 255) / 256, L.nsm * 8);
    cudaError_t e = launch_pdl(sched_min_kernel<ORDER>, nb, 256, 0, s, (const double *)L.jp,
                               (const double *)L.dt, L.n, L.sched);
    if (e == cudaSuccess)
        e = launch_pdl(sched_compact_kernel<ORDER>, nb, 256, 0, s, (const double *)L.jp,
                       (const double *)L.dt, L.n, L.sched, L.ilist);
    ItemsArgs a{L.jp, L.ilist, L.sched, L.force, L.partial, L.counter, L.err, L.n, L.nchunk,
                L.partial_cap, L.target_items, kBigNact};
    // both force shapes are in every step; the one not meant for this step's
    // nact (known on the device only) returns at once
    if constexpr (ORDER == 9) {   // double-double positions: FP64 only
        if (e == cudaSuccess)
            e = launch_pdl(force_items_kernel<ORDER, false>, L.items_grid, 128, L.smem_fp64, s, a);
        if (e == cudaSuccess)
            e = launch_pdl(force_items_big_kernel<ORDER, false>, L.big_grid, 128,
                           BigShape<ORDER, false>::smem_bytes, s, a);
    } else {
        if (e == cudaSuccess) {
            if (L.mixed)
                e = launch_pdl(force_items_kernel<ORDER, true>, L.items_grid, 128, L.smem_mixed, s, a);
            else
                e = launch_pdl(force_items_kernel<ORDER, false>, L.items_grid, 128, L.smem_fp64, s, a);
        }
        if (e == cudaSuccess) {
            if (L.mixed)
                e = launch_pdl(force_items_big_kernel<ORDER, true>, L.big_grid, 128,
                               BigShape<ORDER, true>::smem_bytes, s, a);
            else
                e = launch_pdl(force_items_big_kernel<ORDER, false>, L.big_grid, 128,
                               BigShape<ORDER, false>::smem_bytes, s, a);
        }
    }
    if (e == cudaSuccess)
        e = launch_pdl(correct_kernel<ORDER>, std::max(1, std::min(nb, L.nsm * 4)), 256, 0, s, L.jp,
                       L.dt, (const double *)L.force, (const int *)L.ilist, L.sched, L.aux);
    return e;
}

cudaError_t integrator_step_launch(int order, const IntegratorLaunch &L, cudaStream_t s)
{
    switch (order) {
    case 4: return launch_step<4>(L, s);
    case 6: return launch_step<6>(L, s);
    case 8: return launch_step<8>(L, s);
    case 9: return launch_step<9>(L, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t integrator_kernel_setup(int order, bool mixed, int *smem, int *grid_per_sm,
                                    int *big_per_sm)
{
    const void *k = nullptr;
    int sm = 0;
#define HB_ITEMS(O, M)                                                                        \
    k = (const void *)&force_items_kernel<O, M>;                                                \
    sm = ForceShape<O, M, 4, 1, 4, 4, true>::smem_bytes;
    switch (order * 2 + (mixed ? 1 : 0)) {
    case 8: HB_ITEMS(4, false) break;
    case 9: HB_ITEMS(4, true) break;
    case 12: HB_ITEMS(6, false) break;
    case 13: HB_ITEMS(6, true) break;
    case 16: HB_ITEMS(8, false) break;
    case 17: HB_ITEMS(8, true) break;
    case 18: HB_ITEMS(9, false) break;
    default: return cudaErrorInvalidValue;
    }
#undef HB_ITEMS
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    *smem = sm;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(grid_per_sm, k, 128, sm);
    if (e != cudaSuccess) return e;
    // the large-step kernel
#define HB_BIG(O, M)                                                                          \
    k = (const void *)&force_items_big_kernel<O, M>;                                            \
    sm = BigShape<O, M>::smem_bytes;
    switch (order * 2 + (mixed ? 1 : 0)) {
    case 8: HB_BIG(4, false) break;
    case 9: HB_BIG(4, true) break;
    case 12: HB_BIG(6, false) break;
    case 13: HB_BIG(6, true) break;
    case 16: HB_BIG(8, false) break;
    case 18: HB_BIG(9, false) break;
    default: HB_BIG(8, true) break;
    }
#undef HB_BIG
    e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(big_per_sm, k, 128, sm);
}

template <int ORDER, bool MIXED>
static cudaError_t persistent_setup_t(int *smem, int *per_sm)
{
    const void *k = (const void *)&persistent_kernel<ORDER, MIXED>;
    *smem = PersistSmem<ORDER, MIXED>::bytes;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, *smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, 128, *smem);
    return e;
}

cudaError_t persistent_setup(int order, bool mixed, int *smem, int *per_sm)
{
    switch (order * 2 + (mixed ? 1 : 0)) {
    case 8: return persistent_setup_t<4, false>(smem, per_sm);
    case 9: return persistent_setup_t<4, true>(smem, per_sm);
    case 12: return persistent_setup_t<6, false>(smem, per_sm);
    case 13: return persistent_setup_t<6, true>(smem, per_sm);
    case 16: return persistent_setup_t<8, false>(smem, per_sm);
    case 17: return persistent_setup_t<8, true>(smem, per_sm);
    case 18: return persistent_setup_t<9, false>(smem, per_sm);
    }
    return cudaErrorInvalidValue;
}

template <int ORDER, bool MIXED>
static cudaError_t persistent_launch_t(const PersistArgs &p, int grid, cudaStream_t s)
{
    PersistArgs arg = p;
    void *args[] = {&arg};
    return cudaLaunchCooperativeKernel((const void *)&persistent_kernel<ORDER, MIXED>, dim3(grid),
                                       dim3(128), args, (size_t)PersistSmem<ORDER, MIXED>::bytes, s);
}

cudaError_t persistent_launch(int order, const IntegratorLaunch &L, unsigned *gbar,
                              long long max_steps, unsigned spin, int grid, cudaStream_t s)
{
    PersistArgs p;
    p.it = ItemsArgs{L.jp, L.ilist, L.sched, L.force, L.partial, L.counter, L.err, L.n, L.nchunk,
                     L.partial_cap, L.target_items, kBigNact};
    p.ilist = L.ilist;
    p.jp = L.jp;
    p.dt = L.dt;
    p.aux = L.aux;
    p.gbar = gbar;
    p.max_steps = max_steps;
    p.spin = spin;
    const bool mixed = L.mixed && order != 9;
    switch (order * 2 + (mixed ? 1 : 0)) {
    case 8: return persistent_launch_t<4, false>(p, grid, s);
    case 9: return persistent_launch_t<4, true>(p, grid, s);
    case 12: return persistent_launch_t<6, false>(p, grid, s);
    case 13: return persistent_launch_t<6, true>(p, grid, s);
    case 16: return persistent_launch_t<8, false>(p, grid, s);
    case 17: return persistent_launch_t<8, true>(p, grid, s);
    case 18: return persistent_launch_t<9, false>(p, grid, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t integrator_assign(int order, double *jp, double *dt, const double *force, int n,
                              int set_dt, double eta_s, double dtmax, cudaStream_t s)
{
    const int g = (n + 127) / 128;
    switch (order) {
    case 4: assign_kernel<4><<<g, 128, 0, s>>>(jp, dt, force, n, set_dt, eta_s, dtmax); break;
    case 6: assign_kernel<6><<<g, 128, 0, s>>>(jp, dt, force, n, set_dt, eta_s, dtmax); break;
    case 8: assign_kernel<8><<<g, 128, 0, s>>>(jp, dt, force, n, set_dt, eta_s, dtmax); break;
    case 9: assign_kernel<9><<<g, 128, 0, s>>>(jp, dt, force, n, set_dt, eta_s, dtmax); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t integrator_energy(int order, const double *jp, const double *pot, int n, double *part,
                              double *out, cudaStream_t s)
{
    switch (order) {
    case 4: energy_partial_kernel<4><<<kEnergyBlocks, 256, 0, s>>>(jp, pot, n, part); break;
    case 6: energy_partial_kernel<6><<<kEnergyBlocks, 256, 0, s>>>(jp, pot, n, part); break;
    case 8: energy_partial_kernel<8><<<kEnergyBlocks, 256, 0, s>>>(jp, pot, n, part); break;
    case 9: energy_partial_kernel<9><<<kEnergyBlocks, 256, 0, s>>>(jp, pot, n, part); break;
    default: return cudaErrorInvalidValue;
    }
    energy_final_kernel<<<1, 32, 0, s>>>(part, kEnergyBlocks, out);
    return cudaGetLastError();
}

}  // namespace hb
