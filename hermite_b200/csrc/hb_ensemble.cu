// hb_ensemble.cu -- batched ensembles of independent clusters on one GPU.
//
// Many small N-body systems (different N, masses, softenings) advanced
// together: one global block-step loop over the union of their particles,
// each particle interacting only with its own cluster.  Clusters are laid
// end to end in one record array, each padded to a multiple of 128 slots
// with inert padding (zero mass, far-away positions, dt = +inf, so never
// active and contributing exactly zero).  Per block step, all on the device
// and replayed from a captured CUDA graph:
//   1. tnext = min over all slots of (tlast + dt), from a compact per-slot
//      copy the corrector keeps (the records are 112..208 bytes a slot);
//      per-cluster counters reset
//   2. active slots compacted into their cluster's own slot range
//      (ilist[off_c + k]), then one CTA turns the per-cluster counts into
//      i-tile offsets
//   3. one work-item force launch over every cluster's i-tiles x j-slices,
//      each tile against its own cluster's j range and softening
//   4. the Hermite corrector (shared with the single-system integrator)
// This is the batching form of the reference's integrator: no reference
// counterpart exists (the reference runs one system per process).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hermite_b200.h"
#include "hb_common.cuh"
#include "hb_corrector.cuh"
#include "hb_force.cuh"
#include "hb_internal.h"

namespace hb {
namespace {

constexpr int kClusterPad = 128;
constexpr int kMaxClusters = 4096;
constexpr unsigned long long kInf = 0x7ff0000000000000ull;

struct Cluster {
    int off, n, npad, pad;
    double eps2;
};

// Clusters integrated by team kernels of one size: systems [first,
// first + count) of the team system table.
struct TeamGroup {
    int ctas, first, count, nmax;
    TeamConfig cfg;
};

// Programmatic dependent launch (see hb_integrator.cu): schedule the next
// kernel now, wait for the previous kernel's results.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// host-visible mirror, written once per block step (mapped pinned memory)
struct EnsStatus {
    double tsys, interactions;
    long long particle_steps, block_steps;
    int error, pad;
};

// scheduler state in device memory (its atomics stay on the device)
struct EnsSched {
    unsigned long long tnext_bits;
    int work, error, total_tiles, nact;
    double tnext, dtlim, tsys, tend;
    double etapow, dtmax;
    long long particle_steps, block_steps;
    double interactions;
    EnsStatus *status;
};

struct EnsLaunch {
    double *jp, *dt, *force, *partial;
    double *tn;                        // per slot tlast + dt (a compact copy for steps 1, 2a)
    int *ilist, *ccnt, *tile_base;     // tile_base[nclusters + 1]
    int *item_base, *pitem_base;       // per-cluster force items / partial slots, prefix sums
    unsigned *counter;
    const Cluster *cl;
    const int *slot_cluster;           // per 128-slot block
    TeamState *cst;                    // per-cluster state and counters
    EnsSched *s;
    int *err;
    int nslot, nclusters, nsm;
    size_t partial_cap;
    int target_items, items_grid, smem;
};

// j-slices of one i-tile of a cluster with cnt active slots in npad slots:
// a function of the cluster alone (up to kEnsSplit (tile, slice) items when
// it has few active tiles, no slice thinner than 4 chunks), so that a
// cluster's forces -- and its block steps -- do not depend on the other
// clusters of the ensemble.  Measured on the batched-ensemble shapes (256
// clusters, N 1024..32768, 6th order): 16 / 32 / 64 / 128 / 256 items gave
// 179 / 190 / 194 / 196 / 197 Gint/s; steps with few active particles fill
// the GPU only with fine slices.
constexpr int kEnsSplit = 128;
__device__ __forceinline__ int ens_split(int cnt, int npad)
{
    const int tiles = (cnt + 31) / 32;
    if (tiles == 0) return 0;
    return max(1, min(kEnsSplit / tiles, npad / 128));
}

// 1. next block time; reset the per-cluster counters
template <int ORDER>
__global__ void ens_min_kernel(EnsLaunch L)
{
    pdl_enter();
    double m = __longlong_as_double((long long)kInf);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.nslot; i += gridDim.x * blockDim.x)
        m = fmin(m, L.tn[i]);
    for (int o = 16; o; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double wm[32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? wm[threadIdx.x] : __longlong_as_double((long long)kInf);
        for (int o = 16; o; o >>= 1) m = fmin(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) atomicMin(&L.s->tnext_bits, (unsigned long long)__double_as_longlong(m));
    }
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < L.nclusters; c += gridDim.x * blockDim.x)
        L.ccnt[c] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) L.s->work = 0;
}

// 2a. active slots into their cluster's range
template <int ORDER>
__global__ void ens_compact_kernel(EnsLaunch L)
{
    pdl_enter();
    const double tnext = __longlong_as_double((long long)L.s->tnext_bits);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double dtlim = L.s->dtmax, q = tnext / L.s->dtmax;
        for (int k = 0; k < 64 && q != trunc(q); ++k) {
            q *= 2.0;
            dtlim *= 0.5;
        }
        L.s->tnext = tnext;
        L.s->dtlim = dtlim;
    }
    if (!(tnext <= L.s->tend) || L.s->error) return;
    for (int base = blockIdx.x * blockDim.x; base < L.nslot; base += gridDim.x * blockDim.x) {
        const int i = base + threadIdx.x;   // blockDim 128: one cluster per block
        const int c = L.slot_cluster[base / kClusterPad];
        const bool act = i < L.nslot && L.tn[i] == tnext;
        const unsigned ballot = __ballot_sync(0xffffffffu, act);
        int off = 0;
        if ((threadIdx.x & 31) == 0 && ballot) off = atomicAdd(&L.ccnt[c], __popc(ballot));
        off = __shfl_sync(0xffffffffu, off, 0);
        if (act) L.ilist[L.cl[c].off + off + __popc(ballot & ((1u << (threadIdx.x & 31)) - 1u))] = i;
    }
}

// 2b. per-cluster i-tile offsets (one CTA)
__global__ void ens_tiles_kernel(EnsLaunch L)
{
    pdl_enter();
    __shared__ int part[1024], ipart[1024], ppart[1024];
    const int per = (L.nclusters + blockDim.x - 1) / blockDim.x;
    const int c0 = threadIdx.x * per, c1 = min(L.nclusters, c0 + per);
    int tiles = 0, act = 0, items = 0, pitems = 0;
    const double tnext = L.s->tnext;
    for (int c = c0; c < c1; ++c) {
        const int k = L.ccnt[c];
        const int tl = (k + 31) / 32, sc = ens_split(k, L.cl[c].npad);
        tiles += tl;
        items += tl * sc;
        pitems += sc > 1 ? tl * sc : 0;
        act += k;
        if (k > 0) {   // this cluster takes a block step at tnext
            TeamState &t = L.cst[c];
            t.tsys = tnext;
            t.particle_steps += k;
            t.block_steps += 1;
            t.interactions += (double)k * L.cl[c].n;
        }
    }
    part[threadIdx.x] = tiles;
    ipart[threadIdx.x] = items;
    ppart[threadIdx.x] = pitems;
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0, irun = 0, prun = 0;
        for (int t = 0; t < (int)blockDim.x; ++t) {
            const int v = part[t], iv = ipart[t], pv = ppart[t];
            part[t] = run;
            ipart[t] = irun;
            ppart[t] = prun;
            run += v;
            irun += iv;
            prun += pv;
        }
        L.s->total_tiles = run;
    }
    __syncthreads();
    int run = part[threadIdx.x], irun = ipart[threadIdx.x], prun = ppart[threadIdx.x];
    for (int c = c0; c < c1; ++c) {
        const int k = L.ccnt[c];
        const int tl = (k + 31) / 32, sc = ens_split(k, L.cl[c].npad);
        L.tile_base[c] = run;
        L.item_base[c] = irun;
        L.pitem_base[c] = prun;
        run += tl;
        irun += tl * sc;
        prun += sc > 1 ? tl * sc : 0;
    }
    if (threadIdx.x == blockDim.x - 1) {
        L.tile_base[L.nclusters] = run;
        L.item_base[L.nclusters] = irun;
        L.pitem_base[L.nclusters] = prun;
    }
    // totals for the statistics
    __shared__ int sact[1024];
    sact[threadIdx.x] = act;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long tot = 0;
        double inter = 0.0;
        for (int t = 0; t < (int)blockDim.x; ++t) tot += sact[t];
        for (int c = 0; c < L.nclusters; ++c) inter += (double)L.ccnt[c] * L.cl[c].n;
        L.s->nact = (int)tot;
        if (tot > 0) {
            L.s->particle_steps += tot;
            L.s->block_steps += 1;
            L.s->interactions += inter;
        }
    }
}

// Sums of the per-cluster counters (fixed order), minimum time, any error.
struct EnsTotals {
    double tmin, interactions;
    long long particle_steps, block_steps;
    int error, pad;
};

__global__ void ens_totals_kernel(const TeamState *st, const int *idx, int n, EnsTotals *out)
{
    __shared__ double s_t[256], s_i[256];
    __shared__ long long s_p[256], s_b[256];
    __shared__ int s_e[256];
    double t = __longlong_as_double(0x7ff0000000000000ll), in = 0.0;
    long long ps = 0, bs = 0;
    int er = 0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const TeamState &x = st[idx ? idx[k] : k];
        t = fmin(t, x.tsys);
        in += x.interactions;
        ps += x.particle_steps;
        bs += x.block_steps;
        er |= x.error;
    }
    s_t[threadIdx.x] = t;
    s_i[threadIdx.x] = in;
    s_p[threadIdx.x] = ps;
    s_b[threadIdx.x] = bs;
    s_e[threadIdx.x] = er;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)blockDim.x; ++k) {
            t = fmin(t, s_t[k]);
            in += s_i[k];
            ps += s_p[k];
            bs += s_b[k];
            er |= s_e[k];
        }
        out->tmin = t;
        out->interactions = in;
        out->particle_steps = ps;
        out->block_steps = bs;
        out->error = er;
    }
}

// 3. fused predict + force over (tile, j-slice) items of all clusters
template <int ORDER, bool MIXED>
__global__ void __launch_bounds__(128)
ens_force_kernel(EnsLaunch L)
{
    pdl_enter();
    constexpr int NW = 4, WJ = 4, TCH = 4, STG = 2, TI = 32;
    constexpr int F = Frc<ORDER>::words, R = Rec<ORDER>::words, RB = Rec<ORDER>::bytes;
    using Sh = ForceShape<ORDER, MIXED, NW, 1, WJ, TCH, true>;
    constexpr int CB = Sh::CB;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + Sh::body_bytes);
    unsigned char *ptile = smem + Sh::ring_bytes;
    __shared__ int s_item;
    __shared__ unsigned s_last;

    const int items = L.item_base[L.nclusters];
    if (items == 0) return;
    const double tsys = L.s->tnext;
    const int tid = threadIdx.x, lane = tid & 31, jg = tid >> 5;

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned g = 0;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(&L.s->work, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= items) break;
        // the item's cluster: last c with item_base[c] <= item
        int lo = 0, hi = L.nclusters - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (L.item_base[mid] <= item) lo = mid; else hi = mid - 1;
        }
        const int c = lo;
        const Cluster cl = L.cl[c];
        const int cnt = L.ccnt[c];
        const int S = ens_split(cnt, cl.npad);
        const int li = item - L.item_base[c], tl = li / S, sl = li - tl * S;
        const int tile = L.tile_base[c] + tl;
        const size_t pslot = (size_t)L.pitem_base[c] + (size_t)tl * S;   // partials of this tile
        const int k0 = tl * TI;
        const double eps2 = cl.eps2;

        double *raw = reinterpret_cast<double *>(smem);
        for (int w = tid; w < TI * R; w += NW * 32) {
            const int q = w / R, k = k0 + q;
            const int slot = L.ilist[cl.off + (k < cnt ? k : cnt - 1)];
            raw[w] = L.jp[(size_t)slot * R + (w - q * R)];
        }
        __syncthreads();
        predict_tile<ORDER, MIXED>(raw, TI, 0, INT_MAX, tsys, ptile);
        __syncthreads();
        using IBody = typename std::conditional<MIXED, NegI32, Body64>::type;
        IBody I[1];
        if constexpr (MIXED) load_i_mixed<ORDER>(reinterpret_cast<const float *>(ptile), 0, lane, I[0]);
        else load_i64<ORDER>(reinterpret_cast<const double *>(ptile), 0, lane, I[0]);
        __syncthreads();

        double f[1][F], tot[1][F], cmp[1][F];   // 8th order FP64: Kahan-folded per tile
#pragma unroll
        for (int q = 0; q < F; ++q) f[0][q] = tot[0][q] = cmp[0][q] = 0.0;
        const int cb = cl.off / 32, nch = cl.npad / 32;
        const int c0 = cb + (int)(((long long)sl * nch) / S);
        const int c1 = cb + (int)(((long long)(sl + 1) * nch) / S);
        const int ntile = (c1 - c0 + TCH - 1) / TCH;
        auto issue = [&](int t) {
            const unsigned gt = g + t;
            const int st = gt % STG;
            const int cs = c0 + t * TCH, cc = min(TCH, c1 - cs);
            const uint32_t bytes = (uint32_t)(cc * 32 * RB);
            mbar_arrive_expect_tx(&bar[st], bytes);
            bulk_load(smem + st * Sh::tile_bytes, L.jp + (size_t)cs * 32 * R, bytes, &bar[st]);
        };
        if (tid == 0)
            for (int t = 0; t < STG && t < ntile; ++t) issue(t);
        const float2 eps2f = f2((float)eps2);
        int failed_at = -1;
        for (int t = 0; t < ntile; ++t) {
            const unsigned gt = g + t;
            const int st = gt % STG;
            const bool got = mbar_wait_bounded(&bar[st], (gt / STG) & 1u);
            if (!__syncthreads_and(got)) { failed_at = t; break; }
            const int cc = min(TCH, c1 - (c0 + t * TCH));
            // padding records are inert (zero mass, far away): no slot test
            predict_tile<ORDER, MIXED>(reinterpret_cast<const double *>(smem + st * Sh::tile_bytes),
                                       cc * 32, 0, INT_MAX, tsys, ptile);
            __syncthreads();
            if (tid == 0 && t + STG < ntile) issue(t + STG);
            for (int q = jg; q < cc; q += WJ) {
                if constexpr (MIXED)
                    chunk_mixed<ORDER, 1, (HB_MIXED_REFINE != 0)>(reinterpret_cast<const float *>(ptile + q * CB), I, eps2f, f);
                else
                    chunk64<ORDER, 1>(reinterpret_cast<const double *>(ptile + q * CB), I, eps2, f);
            }
            if constexpr (kKahan<ORDER, MIXED>) kahan_fold<1, F>(tot, cmp, f);
            __syncthreads();
        }
        if (failed_at >= 0) {
            if (tid == 0) {
                raise_error(L.err, kErrWaitTimeout);
                for (int t = failed_at; t < ntile && t < failed_at + STG; ++t)
                    mbar_wait_bounded(&bar[(g + t) % STG], ((g + t) / STG) & 1u);
            }
            L.s->error = 2;
            return;
        }
        g += ntile;
        if constexpr (kKahan<ORDER, MIXED>) {
#pragma unroll
            for (int q = 0; q < F; ++q) f[0][q] = __dsub_rn(tot[0][q], cmp[0][q]);
        }

        double *red = reinterpret_cast<double *>(smem);
        if (jg > 0)
#pragma unroll
            for (int q = 0; q < F; ++q) red[((jg - 1) * F + q) * 32 + lane] = f[0][q];
        __syncthreads();
        const int k = k0 + lane;
        const size_t pos = (size_t)cl.off + k;   // force row = ilist position
        if (jg == 0) {
            for (int w = 1; w < WJ; ++w)
#pragma unroll
                for (int q = 0; q < F; ++q) f[0][q] += red[((w - 1) * F + q) * 32 + lane];
            if (S == 1) {
                if (k < cnt)
#pragma unroll
                    for (int q = 0; q < F; ++q) L.force[pos * F + q] = f[0][q];
            } else {
#pragma unroll
                for (int q = 0; q < F; ++q)
                    L.partial[((pslot + sl) * TI + lane) * F + q] = f[0][q];
            }
        }
        if (S > 1) {
            __threadfence();
            __syncthreads();
            if (tid == 0) s_last = (atomicAdd(&L.counter[tile], 1u) == (unsigned)(S - 1));
            __syncthreads();
            if (s_last) {
                __threadfence();
                const int V = min(TI, cnt - k0) * F;
                const double *pbase = L.partial + pslot * TI * F;
                for (int e = tid; e < V; e += NW * 32) {
                    double sum = 0.0;
                    for (int s2 = 0; s2 < S; ++s2) sum += __ldcg(pbase + (size_t)s2 * TI * F + e);
                    L.force[((size_t)cl.off + k0) * F + e] = sum;
                }
                if (tid == 0) L.counter[tile] = 0u;
            }
        }
        __syncthreads();
    }
}

// 4. corrector over every cluster's active list
template <int ORDER>
__global__ void ens_correct_kernel(EnsLaunch L)
{
    pdl_enter();
    constexpr int R = Rec<ORDER>::words, F = Frc<ORDER>::words;
    const int T = L.s->total_tiles;
    const double dtlim = L.s->dtlim, etapow = L.s->etapow;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < T * 32; p += gridDim.x * blockDim.x) {
        const int tile = p >> 5;
        int lo = 0, hi = L.nclusters - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (L.tile_base[mid] <= tile) lo = mid; else hi = mid - 1;
        }
        const int k = (tile - L.tile_base[lo]) * 32 + (p & 31);
        if (k >= L.ccnt[lo]) continue;
        const size_t pos = (size_t)L.cl[lo].off + k;
        const int i = L.ilist[pos];
        const double dtn = correct_particle<ORDER>(L.jp + (size_t)i * R, L.force + pos * F, L.dt[i],
                                                   etapow, dtlim);
        if (!(dtn >= 0x1p-48)) L.s->error = 1;
        L.dt[i] = dtn;
        L.tn[i] = L.jp[(size_t)i * R + 7] + dtn;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (L.s->nact > 0) L.s->tsys = L.s->tnext;
        L.s->tnext_bits = kInf;
        EnsStatus *st = L.s->status;
        st->tsys = L.s->tsys;
        st->interactions = L.s->interactions;
        st->particle_steps = L.s->particle_steps;
        st->block_steps = L.s->block_steps;
        st->error = L.s->error;
    }
}

// initialisation: every real slot active (no dt yet), forces written into the
// records, dt from init_dt on the last pass
__global__ void ens_all_active_kernel(EnsLaunch L)
{
    for (int c = blockIdx.x; c < L.nclusters; c += gridDim.x) {
        const Cluster cl = L.cl[c];
        for (int k = threadIdx.x; k < cl.n; k += blockDim.x) L.ilist[cl.off + k] = cl.off + k;
        if (threadIdx.x == 0) L.ccnt[c] = cl.n;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) L.s->work = 0;
}

// tn = tlast + dt for every slot (padding: dt = +inf), before a run of the
// lockstep engine: the team engine and the host set-up write records and dt
// without it
template <int ORDER>
__global__ void ens_tn_kernel(EnsLaunch L)
{
    constexpr int R = Rec<ORDER>::words;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.nslot; i += gridDim.x * blockDim.x)
        L.tn[i] = L.dt[i] + L.jp[(size_t)i * R + 7];
}

template <int ORDER>
__global__ void ens_assign_kernel(EnsLaunch L, int set_dt, double eta_s)
{
    constexpr int R = Rec<ORDER>::words, F = Frc<ORDER>::words;
    for (int c = blockIdx.x; c < L.nclusters; c += gridDim.x) {
        const Cluster cl = L.cl[c];
        for (int k = threadIdx.x; k < cl.n; k += blockDim.x) {
            const size_t i = (size_t)cl.off + k;
            for (int q = 0; q < F; ++q) L.jp[i * R + 8 + q] = L.force[i * F + q];
            if (set_dt) L.dt[i] = initial_dt<ORDER>(L.force + i * F, eta_s, L.s->dtmax);
        }
    }
}

// potential per cluster (FP64), then per-cluster kinetic / potential sums
template <int ORDER>
__global__ void ens_potential_kernel(EnsLaunch L, double *pot)
{
    constexpr int R = Rec<ORDER>::words;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;       // blockDim 128
    const Cluster cl = L.cl[L.slot_cluster[blockIdx.x * blockDim.x / kClusterPad]];
    const double *ri = L.jp + (size_t)i * R;
    double sum = 0.0;
    for (int j = cl.off; j < cl.off + cl.n; ++j) {
        const double *rj = L.jp + (size_t)j * R;
        const double dx = rj[0] - ri[0], dy = rj[1] - ri[1], dz = rj[2] - ri[2];
        const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, cl.eps2)));
        if (j != i) sum = fma(-rj[3], rsqrt_fp64(r2), sum);
    }
    pot[i] = sum;
}

template <int ORDER>
__global__ void ens_energy_kernel(EnsLaunch L, const double *pot, double *out)
{
    constexpr int R = Rec<ORDER>::words;
    const Cluster cl = L.cl[blockIdx.x];
    double ke = 0.0, pe = 0.0;
    for (int k = threadIdx.x; k < cl.n; k += blockDim.x) {
        const double *r = L.jp + (size_t)(cl.off + k) * R;
        ke += r[3] * (r[4] * r[4] + r[5] * r[5] + r[6] * r[6]);
        pe += r[3] * pot[cl.off + k];
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
        out[2 * blockIdx.x] = 0.5 * sk[0];
        out[2 * blockIdx.x + 1] = 0.5 * sp[0];
    }
}

template <typename K>
cudaError_t launch_pdl(K kern, int grid, int block, int smem, cudaStream_t s, const EnsLaunch &L)
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
    return cudaLaunchKernelEx(&cfg, kern, L);
}

template <int ORDER>
cudaError_t ens_step(const EnsLaunch &L, bool mixed, cudaStream_t s)
{
    const int nb = std::max(1, std::min((L.nslot + 127) / 128, L.nsm * 8));
    cudaError_t e = launch_pdl(ens_min_kernel<ORDER>, nb, 256, 0, s, L);
    if (e == cudaSuccess) e = launch_pdl(ens_compact_kernel<ORDER>, nb, 128, 0, s, L);
    if (e == cudaSuccess) e = launch_pdl(ens_tiles_kernel, 1, 256, 0, s, L);
    if (e == cudaSuccess)
        e = mixed ? launch_pdl(ens_force_kernel<ORDER, true>, L.items_grid, 128, L.smem, s, L)
                  : launch_pdl(ens_force_kernel<ORDER, false>, L.items_grid, 128, L.smem, s, L);
    if (e == cudaSuccess) e = launch_pdl(ens_correct_kernel<ORDER>, L.nsm * 4, 128, 0, s, L);
    return e;
}

template <int ORDER>
cudaError_t ens_force_all(const EnsLaunch &L, bool mixed, int set_dt, double eta_s, cudaStream_t s)
{
    ens_all_active_kernel<<<std::min(L.nclusters, 1024), 256, 0, s>>>(L);
    ens_tiles_kernel<<<1, 256, 0, s>>>(L);
    if (mixed) ens_force_kernel<ORDER, true><<<L.items_grid, 128, L.smem, s>>>(L);
    else ens_force_kernel<ORDER, false><<<L.items_grid, 128, L.smem, s>>>(L);
    ens_assign_kernel<ORDER><<<std::min(L.nclusters, 1024), 256, 0, s>>>(L, set_dt, eta_s);
    return cudaGetLastError();
}

template <int ORDER>
cudaError_t ens_energy(const EnsLaunch &L, double *pot, double *out, cudaStream_t s)
{
    ens_potential_kernel<ORDER><<<L.nslot / 128, 128, 0, s>>>(L, pot);
    ens_energy_kernel<ORDER><<<L.nclusters, 256, 0, s>>>(L, pot, out);
    return cudaGetLastError();
}

template <int ORDER, bool M>
cudaError_t ens_setup(int *smem, int *per_sm)
{
    const void *k = (const void *)&ens_force_kernel<ORDER, M>;
    *smem = ForceShape<ORDER, M, 4, 1, 4, 4, true>::smem_bytes;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, *smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, 128, *smem);
}

}  // namespace
}  // namespace hb

using namespace hb;

struct hb_ens {
    int order = 0, precision = 0, nclusters = 0, nslot = 0, R = 0, F = 0, nsm = 0;
    std::vector<Cluster> cl;
    cudaStream_t stream = nullptr;
    double *d_jp = nullptr, *d_dt = nullptr, *d_tn = nullptr, *d_force = nullptr, *d_partial = nullptr,
           *d_pot = nullptr, *h_eout = nullptr, *d_eout = nullptr;
    int *d_ilist = nullptr, *d_ccnt = nullptr, *d_tile_base = nullptr, *d_slot_cluster = nullptr;
    int *d_item_base = nullptr, *d_pitem_base = nullptr;
    unsigned *d_counter = nullptr;
    Cluster *d_cl = nullptr;
    EnsSched *h_s = nullptr, *d_s = nullptr;       // host copy (set-up) / device
    EnsStatus *h_st = nullptr, *d_st = nullptr;    // mapped
    int *h_err = nullptr, *d_err = nullptr;
    size_t partial_cap = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool ready = false;
    std::string err;
    EnsLaunch L;
    // per-cluster state (both engines) and the team engine
    TeamState *d_cstate = nullptr;
    EnsTotals *h_tot = nullptr, *d_tot = nullptr;   // mapped
    TeamSys *d_tsys = nullptr;                      // team systems, grouped by team size
    int *d_tidx = nullptr;                          // their cluster indices
    int *d_team_next = nullptr;
    int engine = HB_ENGINE_AUTO, team_ctas = 0;
    std::vector<TeamGroup> groups;                  // built for (engine, team_ctas)
    std::vector<int> cluster_ctas;                  // per cluster: team size, 0 = lockstep engine
    bool groups_ready = false;
};

namespace {
constexpr int kEnsStepsPerGraph = 32;

int ens_fail(hb_ens *e, int status, const char *msg, cudaError_t ce = cudaSuccess)
{
    if (e) {
        e->err = msg;
        if (ce != cudaSuccess) {
            e->err += ": ";
            e->err += cudaGetErrorString(ce);
        }
    }
    return status;
}

// Team size for a cluster of n particles: at least n / kEnsTeamSlots CTAs
// (a power of two), more if its slots do not fit the CTAs' shared memory.
constexpr int kEnsTeamSlots = 512;
constexpr long long kEnsTeamStepsPerLaunch = 1LL << 14;

int build_groups(hb_ens *e)
{
    if (e->groups_ready) return HB_OK;
    e->groups.clear();
    e->cluster_ctas.assign(e->nclusters, 0);
    if (e->engine == HB_ENGINE_GRAPH) {
        e->groups_ready = true;
        return HB_OK;
    }
    if (e->precision != HB_FP64) {
        if (e->engine == HB_ENGINE_TEAM)
            return ens_fail(e, HB_ERR_INVALID, "the team engine integrates in FP64 only");
        e->groups_ready = true;
        return HB_OK;
    }
    TeamConfig cfgs[17] = {};
    bool tried[17] = {};
    auto cfg_for = [&](int C) -> const TeamConfig * {
        if (!tried[C]) {
            tried[C] = true;
            if (team_setup(e->order, C, &cfgs[C]) != cudaSuccess || cfgs[C].max_teams < 1) {
                cudaGetLastError();
                cfgs[C].ctas = 0;
            }
        }
        return cfgs[C].ctas ? &cfgs[C] : nullptr;
    };
    std::vector<std::vector<int>> by(17);
    for (int c = 0; c < e->nclusters; ++c) {
        const int n = e->cl[c].n, nch = (n + 31) / 32;
        int C = e->team_ctas;
        if (C == 0) {
            C = 1;
            while (C < 16 && (long long)C * kEnsTeamSlots < n) C <<= 1;
        }
        for (;;) {
            const TeamConfig *cf = cfg_for(C);
            // the automatic choice takes only clusters whose records fit in
            // shared memory (larger ones run faster on the lockstep engine:
            // measured on 256 clusters of N <= 32768, 16.3 s team vs 12.5 s)
            const int cap = cf ? (e->engine == HB_ENGINE_TEAM ? cf->jl_cap_g : cf->jl_cap) : 0;
            if (cf && (long long)((nch + C - 1) / C) * 32 <= cap) break;
            if (e->team_ctas > 0 || C >= 16) {
                C = 0;
                break;
            }
            C <<= 1;
        }
        if (C == 0) continue;   // the lockstep engine takes it
        by[C].push_back(c);
        e->cluster_ctas[c] = C;
    }
    if (e->engine == HB_ENGINE_AUTO) {
        // all or nothing: a team phase followed by a lockstep phase for the
        // rest would leave most of the GPU idle in the tail of each
        bool all = true;
        for (int C : e->cluster_ctas) all &= C > 0;
        if (!all) {
            e->cluster_ctas.assign(e->nclusters, 0);
            e->groups_ready = true;
            return HB_OK;
        }
    }
    std::vector<TeamSys> ts;
    std::vector<int> idx;
    for (int C = 1; C <= 16; ++C) {
        if (by[C].empty()) continue;
        std::vector<int> &v = by[C];
        // largest systems first: the queue's tail is short
        std::stable_sort(v.begin(), v.end(), [&](int a, int b) { return e->cl[a].n > e->cl[b].n; });
        TeamGroup g;
        g.ctas = C;
        g.first = (int)ts.size();
        g.count = (int)v.size();
        g.nmax = e->cl[v.front()].n;
        g.cfg = cfgs[C];
        for (int c : v) {
            TeamSys t;
            t.off = e->cl[c].off;
            t.n = e->cl[c].n;
            t.id = c;
            t.eps2 = e->cl[c].eps2;
            ts.push_back(t);
            idx.push_back(c);
        }
        e->groups.push_back(g);
    }
    if (!ts.empty()) {
        cudaError_t ce = cudaMemcpy(e->d_tsys, ts.data(), ts.size() * sizeof(TeamSys), cudaMemcpyHostToDevice);
        if (ce == cudaSuccess)
            ce = cudaMemcpy(e->d_tidx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "team system table", ce);
    }
    e->groups_ready = true;
    return HB_OK;
}

// Sums of the per-cluster counters over `count` clusters (all when idx is null).
int totals(hb_ens *e, const int *idx, int count)
{
    ens_totals_kernel<<<1, 256, 0, e->stream>>>(e->d_cstate, idx, count, e->d_tot);
    cudaError_t ce = cudaGetLastError();
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? HB_OK : ens_fail(e, HB_ERR_CUDA, "cluster totals", ce);
}

// Every team-engine cluster integrated to tend, one group of team size at a time.
int run_teams(hb_ens *e, double tend, long long max_block_steps)
{
    for (const TeamGroup &g : e->groups) {
        TeamLaunch L;
        L.jp = e->d_jp;
        L.dt = e->d_dt;
        L.aux = nullptr;
        L.sys = e->d_tsys + g.first;
        L.st = e->d_cstate;
        L.next_sys = e->d_team_next;
        L.nsys = g.count;
        if (team_shape(e->order, g.cfg, g.nmax, &L) != 0)
            return ens_fail(e, HB_ERR_TOO_LARGE, "a cluster does not fit its team");
        L.tend = tend;
        L.etapow = e->h_s->etapow;
        L.dtmax = e->h_s->dtmax;
        L.max_steps = max_block_steps > 0 ? max_block_steps : kEnsTeamStepsPerLaunch;
        const int teams = std::min(g.cfg.max_teams, g.count);
        double last = -1.0;
        for (;;) {
            cudaError_t ce = cudaMemsetAsync(e->d_team_next, 0, sizeof(int), e->stream);
            if (ce == cudaSuccess) ce = team_launch(e->order, L, teams, e->stream);
            if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "team launch", ce);
            const int s = totals(e, e->d_tidx + g.first, g.count);
            if (s != HB_OK) return s;
            const volatile EnsTotals *t = e->h_tot;
            if (t->error) return ens_fail(e, HB_ERR_STATE, "a timestep underflowed (< 2^-48)");
            if (t->tmin >= tend) break;
            if (max_block_steps > 0) return ens_fail(e, HB_ERR_STATE, "block-step limit reached");
            if (t->tmin == last) return ens_fail(e, HB_ERR_STATE, "ensemble integration stalled");
            last = t->tmin;
        }
    }
    return HB_OK;
}

cudaError_t dispatch_step(hb_ens *e)
{
    const bool m = e->precision == HB_MIXED;
    switch (e->order) {
    case 4: return ens_step<4>(e->L, m, e->stream);
    case 6: return ens_step<6>(e->L, m, e->stream);
    case 8: return ens_step<8>(e->L, m, e->stream);
    }
    return cudaErrorInvalidValue;
}
}  // namespace

extern "C" {

int hb_ens_destroy(hb_ens *e)
{
    if (!e) return HB_OK;
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->graph) cudaGraphDestroy(e->graph);
    cudaFree(e->d_jp);
    cudaFree(e->d_dt);
    cudaFree(e->d_tn);
    cudaFree(e->d_force);
    cudaFree(e->d_partial);
    cudaFree(e->d_pot);
    cudaFree(e->d_ilist);
    cudaFree(e->d_ccnt);
    cudaFree(e->d_tile_base);
    cudaFree(e->d_item_base);
    cudaFree(e->d_pitem_base);
    cudaFree(e->d_slot_cluster);
    cudaFree(e->d_counter);
    cudaFree(e->d_cl);
    delete e->h_s;
    cudaFree(e->d_s);
    cudaFreeHost(e->h_st);
    cudaFreeHost(e->h_eout);
    cudaFreeHost(e->h_err);
    cudaFree(e->d_cstate);
    cudaFreeHost(e->h_tot);
    cudaFree(e->d_tsys);
    cudaFree(e->d_tidx);
    cudaFree(e->d_team_next);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return HB_OK;
}

int hb_ens_create(int order, int nclusters, const int *sizes, int precision, hb_ens **out)
{
    if (!out) return HB_ERR_INVALID;
    *out = nullptr;
    if ((order != 4 && order != 6 && order != 8) || nclusters < 1 || nclusters > kMaxClusters ||
        !sizes || (precision != HB_FP64 && precision != HB_MIXED))
        return HB_ERR_INVALID;
    long long total = 0;
    for (int c = 0; c < nclusters; ++c) {
        if (sizes[c] < 1) return HB_ERR_INVALID;
        total += (sizes[c] + kClusterPad - 1) / kClusterPad * kClusterPad;
    }
    if (total > (1LL << 26)) return HB_ERR_TOO_LARGE;
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess ||
        prop.major != 10 || prop.minor != 0)
        return HB_ERR_NO_DEVICE;

    hb_ens *e = new hb_ens;
    e->order = order;
    e->precision = precision;
    e->nclusters = nclusters;
    e->nslot = (int)total;
    e->R = 8 + 3 * (order - 2);
    e->F = 3 * (order / 2);
    e->nsm = prop.multiProcessorCount;
    int off = 0;
    std::vector<int> slot_cluster(total / kClusterPad);
    for (int c = 0; c < nclusters; ++c) {
        Cluster k;
        k.off = off;
        k.n = sizes[c];
        k.npad = (sizes[c] + kClusterPad - 1) / kClusterPad * kClusterPad;
        k.pad = 0;
        k.eps2 = 0.0;
        for (int b = off / kClusterPad; b < (off + k.npad) / kClusterPad; ++b) slot_cluster[b] = c;
        e->cl.push_back(k);
        off += k.npad;
    }
    const size_t ns = e->nslot;
    // a cluster with j-split tiles has at most kEnsSplit (tile, slice) items
    e->partial_cap = (size_t)kEnsSplit * nclusters * 32 * e->F;
    bool ok = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc((void **)&e->d_jp, ns * e->R * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_dt, ns * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_tn, ns * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_force, ns * e->F * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_partial, e->partial_cap * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_pot, ns * sizeof(double)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_ilist, ns * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_ccnt, nclusters * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_tile_base, (nclusters + 1) * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_item_base, (nclusters + 1) * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_pitem_base, (nclusters + 1) * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_slot_cluster, slot_cluster.size() * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_counter, (ns / 32 + nclusters + 1) * sizeof(unsigned)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_cl, nclusters * sizeof(Cluster)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_s, sizeof(EnsSched)) == cudaSuccess &&
              cudaHostAlloc((void **)&e->h_st, sizeof(EnsStatus), cudaHostAllocMapped) == cudaSuccess &&
              cudaHostGetDevicePointer((void **)&e->d_st, e->h_st, 0) == cudaSuccess &&
              cudaHostAlloc((void **)&e->h_eout, 2 * nclusters * sizeof(double), cudaHostAllocMapped) == cudaSuccess &&
              cudaHostGetDevicePointer((void **)&e->d_eout, e->h_eout, 0) == cudaSuccess &&
              cudaHostAlloc((void **)&e->h_err, sizeof(int), cudaHostAllocMapped) == cudaSuccess &&
              cudaHostGetDevicePointer((void **)&e->d_err, e->h_err, 0) == cudaSuccess &&
              cudaMalloc((void **)&e->d_cstate, nclusters * sizeof(TeamState)) == cudaSuccess &&
              cudaHostAlloc((void **)&e->h_tot, sizeof(EnsTotals), cudaHostAllocMapped) == cudaSuccess &&
              cudaHostGetDevicePointer((void **)&e->d_tot, e->h_tot, 0) == cudaSuccess &&
              cudaMalloc((void **)&e->d_tsys, nclusters * sizeof(TeamSys)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_tidx, nclusters * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&e->d_team_next, sizeof(int)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        hb_ens_destroy(e);
        return HB_ERR_ALLOC;
    }
    *e->h_err = 0;
    e->h_s = new EnsSched;
    std::memset(e->h_s, 0, sizeof(EnsSched));
    e->h_s->tnext_bits = kInf;
    e->h_s->status = e->d_st;
    std::memset(e->h_st, 0, sizeof(EnsStatus));
    // inert padding everywhere until clusters are set
    std::vector<double> pad(ns * e->R, 0.0);
    std::vector<double> dt(ns, INFINITY);
    for (size_t i = 0; i < ns; ++i)
        for (int k = 0; k < 3; ++k) pad[i * e->R + k] = 1099511627776.0 + (double)(i * 3 + k);
    ok = cudaMemcpy(e->d_jp, pad.data(), pad.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(e->d_dt, dt.data(), dt.size() * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(e->d_slot_cluster, slot_cluster.data(), slot_cluster.size() * sizeof(int),
                    cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(e->d_counter, 0, (ns / 32 + nclusters + 1) * sizeof(unsigned)) == cudaSuccess;
    if (!ok) {
        hb_ens_destroy(e);
        return HB_ERR_CUDA;
    }
    EnsLaunch &L = e->L;
    L.jp = e->d_jp;
    L.dt = e->d_dt;
    L.tn = e->d_tn;
    L.force = e->d_force;
    L.partial = e->d_partial;
    L.ilist = e->d_ilist;
    L.ccnt = e->d_ccnt;
    L.tile_base = e->d_tile_base;
    L.item_base = e->d_item_base;
    L.pitem_base = e->d_pitem_base;
    L.counter = e->d_counter;
    L.cl = e->d_cl;
    L.slot_cluster = e->d_slot_cluster;
    L.cst = e->d_cstate;
    L.s = e->d_s;
    L.err = e->d_err;
    L.nslot = e->nslot;
    L.nclusters = nclusters;
    L.nsm = e->nsm;
    L.partial_cap = e->partial_cap;
    int smem = 0, per_sm = 0;
    cudaError_t ce;
    switch (order * 2 + (precision == HB_MIXED)) {
    case 8: ce = ens_setup<4, false>(&smem, &per_sm); break;
    case 9: ce = ens_setup<4, true>(&smem, &per_sm); break;
    case 12: ce = ens_setup<6, false>(&smem, &per_sm); break;
    case 13: ce = ens_setup<6, true>(&smem, &per_sm); break;
    case 16: ce = ens_setup<8, false>(&smem, &per_sm); break;
    default: ce = ens_setup<8, true>(&smem, &per_sm); break;
    }
    if (ce != cudaSuccess) {
        hb_ens_destroy(e);
        return HB_ERR_CUDA;
    }
    L.smem = smem;
    L.items_grid = e->nsm * std::max(1, per_sm);
    L.target_items = 2 * L.items_grid;
    *out = e;
    return HB_OK;
}

const char *hb_ens_last_error(const hb_ens *e) { return e ? e->err.c_str() : "null ensemble"; }

int hb_ens_cluster_offset(const hb_ens *e, int c)
{
    return (e && c >= 0 && c < e->nclusters) ? e->cl[c].off : -1;
}

int hb_ens_set_cluster(hb_ens *e, int c, const double *records, double eps2)
{
    if (!e || c < 0 || c >= e->nclusters || !records || !(eps2 >= 0.0)) return HB_ERR_INVALID;
    e->cl[c].eps2 = eps2;
    e->groups_ready = false;
    cudaError_t ce = cudaMemcpyAsync(e->d_jp + (size_t)e->cl[c].off * e->R, records,
                                     sizeof(double) * (size_t)e->cl[c].n * e->R,
                                     cudaMemcpyHostToDevice, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    return ce == cudaSuccess ? HB_OK : ens_fail(e, HB_ERR_CUDA, "hb_ens_set_cluster", ce);
}

int hb_ens_get_cluster(hb_ens *e, int c, double *records, double *dt)
{
    if (!e || c < 0 || c >= e->nclusters || !records) return HB_ERR_INVALID;
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpy(records, e->d_jp + (size_t)e->cl[c].off * e->R,
                        sizeof(double) * (size_t)e->cl[c].n * e->R, cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess && dt)
        ce = cudaMemcpy(dt, e->d_dt + e->cl[c].off, sizeof(double) * e->cl[c].n, cudaMemcpyDeviceToHost);
    return ce == cudaSuccess ? HB_OK : ens_fail(e, HB_ERR_CUDA, "hb_ens_get_cluster", ce);
}

int hb_ens_init(hb_ens *e, double tsys, double eta, double eta_s, double dtmax)
{
    if (!e) return HB_ERR_INVALID;
    if (!(eta > 0.0) || !(eta_s > 0.0) || !(dtmax > 0.0) ||
        std::log2(dtmax) != std::floor(std::log2(dtmax)) || !(tsys >= 0.0))
        return ens_fail(e, HB_ERR_INVALID, "hb_ens_init: eta, eta_s > 0, dtmax a power of two");
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "sync", ce);
    if (e->exec) { cudaGraphExecDestroy(e->exec); e->exec = nullptr; }
    if (e->graph) { cudaGraphDestroy(e->graph); e->graph = nullptr; }
    e->ready = false;
    // tlast = tsys, derivatives zero, for every real slot (device copy)
    std::vector<double> rec;
    for (int c = 0; c < e->nclusters; ++c) {
        const Cluster &k = e->cl[c];
        rec.resize((size_t)k.n * e->R);
        ce = cudaMemcpy(rec.data(), e->d_jp + (size_t)k.off * e->R, rec.size() * sizeof(double),
                        cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "init read", ce);
        for (int i = 0; i < k.n; ++i) {
            double *r = rec.data() + (size_t)i * e->R;
            r[7] = tsys;
            std::memset(r + 8, 0, sizeof(double) * (e->R - 8));
        }
        ce = cudaMemcpy(e->d_jp + (size_t)k.off * e->R, rec.data(), rec.size() * sizeof(double),
                        cudaMemcpyHostToDevice);
        if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "init write", ce);
    }
    ce = cudaMemcpy(e->d_cl, e->cl.data(), e->cl.size() * sizeof(Cluster), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "cluster table", ce);
    EnsSched &s = *e->h_s;
    std::memset(&s, 0, sizeof(EnsSched));
    s.tnext_bits = kInf;
    s.tsys = tsys;
    s.tend = tsys;
    s.tnext = tsys;       // the init force is evaluated at tsys
    s.etapow = std::pow(eta, 2.0 * (e->order - 3));
    s.dtmax = dtmax;
    s.status = e->d_st;
    ce = cudaMemcpy(e->d_s, &s, sizeof(EnsSched), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "scheduler upload", ce);
    const bool m = e->precision == HB_MIXED;
    const int passes = e->order > 4 ? 2 : 1;
    for (int p = 0; p < passes && ce == cudaSuccess; ++p) {
        switch (e->order) {
        case 4: ce = ens_force_all<4>(e->L, m, p == passes - 1, eta_s, e->stream); break;
        case 6: ce = ens_force_all<6>(e->L, m, p == passes - 1, eta_s, e->stream); break;
        default: ce = ens_force_all<8>(e->L, m, p == passes - 1, eta_s, e->stream); break;
        }
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce == cudaSuccess) ce = cudaMemcpy(&s, e->d_s, sizeof(EnsSched), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "init forces", ce);
    if (*e->h_err || s.error) return ens_fail(e, HB_ERR_DEVICE_TIMEOUT, "a device-side wait gave up");
    s.particle_steps = s.block_steps = 0;
    s.interactions = 0.0;
    s.tnext_bits = kInf;
    s.tsys = tsys;
    ce = cudaMemcpy(e->d_s, &s, sizeof(EnsSched), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "scheduler upload", ce);
    std::memset(e->h_st, 0, sizeof(EnsStatus));
    e->h_st->tsys = tsys;
    std::vector<TeamState> cs(e->nclusters);
    for (TeamState &t : cs) {
        std::memset(&t, 0, sizeof t);
        t.tsys = tsys;
    }
    ce = cudaMemcpy(e->d_cstate, cs.data(), cs.size() * sizeof(TeamState), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "cluster state", ce);
    e->groups_ready = false;
    ce = cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "capture", ce);
    cudaError_t le = cudaSuccess;
    for (int k = 0; k < kEnsStepsPerGraph && le == cudaSuccess; ++k) le = dispatch_step(e);
    cudaGraph_t g = nullptr;
    ce = cudaStreamEndCapture(e->stream, &g);
    if (le != cudaSuccess || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return ens_fail(e, HB_ERR_CUDA, "capturing the ensemble step graph",
                        le != cudaSuccess ? le : ce);
    }
    e->graph = g;
    ce = cudaGraphInstantiate(&e->exec, g, 0);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "instantiate", ce);
    e->ready = true;
    return HB_OK;
}

int hb_ens_run(hb_ens *e, double tend, long long max_block_steps)
{
    if (!e) return HB_ERR_INVALID;
    if (!e->ready) return ens_fail(e, HB_ERR_STATE, "hb_ens_run before hb_ens_init");
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "sync", ce);
    int s0 = build_groups(e);
    if (s0 == HB_OK) s0 = totals(e, nullptr, e->nclusters);
    if (s0 != HB_OK) return s0;
    if (!(tend >= e->h_tot->tmin)) return ens_fail(e, HB_ERR_INVALID, "tend is before tsys");
    s0 = run_teams(e, tend, max_block_steps);
    if (s0 != HB_OK) return s0;
    bool lockstep = false;
    for (int c : e->cluster_ctas) lockstep |= c == 0;
    if (!lockstep) return HB_OK;

    // the lockstep engine: the other clusters (those already at tend have
    // no active particles until tend)
    volatile EnsStatus *st = e->h_st;
    if (!(tend >= st->tsys)) return ens_fail(e, HB_ERR_INVALID, "tend is before tsys");
    ce = cudaMemcpy(&e->d_s->tend, &tend, sizeof(double), cudaMemcpyHostToDevice);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "tend upload", ce);
    {
        const int nb = std::max(1, std::min((e->nslot + 255) / 256, e->nsm * 8));
        switch (e->order) {
        case 4: ens_tn_kernel<4><<<nb, 256, 0, e->stream>>>(e->L); break;
        case 6: ens_tn_kernel<6><<<nb, 256, 0, e->stream>>>(e->L); break;
        default: ens_tn_kernel<8><<<nb, 256, 0, e->stream>>>(e->L); break;
        }
        ce = cudaGetLastError();
        if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "tlast + dt", ce);
    }
    long long last = st->block_steps;
    const long long first = st->block_steps;
    while (st->tsys < tend) {
        if (max_block_steps > 0 && st->block_steps - first >= max_block_steps)
            return ens_fail(e, HB_ERR_STATE, "block-step limit reached");
        ce = cudaGraphLaunch(e->exec, e->stream);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
        if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "graph launch", ce);
        if (*e->h_err || st->error)
            return ens_fail(e, st->error == 1 ? HB_ERR_STATE : HB_ERR_DEVICE_TIMEOUT,
                            st->error == 1 ? "a timestep underflowed (< 2^-48)"
                                           : "a device-side wait gave up");
        if (st->block_steps == last && st->tsys < tend)
            return ens_fail(e, HB_ERR_STATE, "ensemble integration stalled");
        last = st->block_steps;
    }
    return HB_OK;
}

int hb_ens_stats(hb_ens *e, long long *particle_steps, long long *block_steps, double *tsys,
                 double *interactions)
{
    if (!e) return HB_ERR_INVALID;
    const int s = totals(e, nullptr, e->nclusters);
    if (s != HB_OK) return s;
    const volatile EnsTotals *t = e->h_tot;
    if (particle_steps) *particle_steps = t->particle_steps;
    if (block_steps) *block_steps = t->block_steps;
    if (tsys) *tsys = t->tmin;
    if (interactions) *interactions = t->interactions;
    return HB_OK;
}

int hb_ens_cluster_stats(hb_ens *e, int c, long long *particle_steps, long long *block_steps,
                         double *tsys)
{
    if (!e || c < 0 || c >= e->nclusters) return HB_ERR_INVALID;
    TeamState t;
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce == cudaSuccess) ce = cudaMemcpy(&t, e->d_cstate + c, sizeof t, cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "cluster stats", ce);
    if (particle_steps) *particle_steps = t.particle_steps;
    if (block_steps) *block_steps = t.block_steps;
    if (tsys) *tsys = t.tsys;
    return HB_OK;
}

int hb_ens_set_engine(hb_ens *e, int engine, int team_ctas)
{
    if (!e || engine < HB_ENGINE_AUTO || engine > HB_ENGINE_TEAM || team_ctas < 0 || team_ctas > 16)
        return HB_ERR_INVALID;
    e->engine = engine;
    e->team_ctas = team_ctas;
    e->groups_ready = false;
    return HB_OK;
}

int hb_ens_cluster_engine(hb_ens *e, int c, int *engine, int *team_ctas)
{
    if (!e || c < 0 || c >= e->nclusters) return HB_ERR_INVALID;
    const int s = build_groups(e);
    if (s != HB_OK) return s;
    const int C = e->cluster_ctas[c];
    if (engine) *engine = C ? HB_ENGINE_TEAM : HB_ENGINE_GRAPH;
    if (team_ctas) *team_ctas = C;
    return HB_OK;
}

int hb_ens_energy(hb_ens *e, double *kinetic, double *potential)
{
    if (!e || !kinetic || !potential) return HB_ERR_INVALID;
    cudaError_t ce = cudaMemcpy(e->d_cl, e->cl.data(), e->cl.size() * sizeof(Cluster),
                                cudaMemcpyHostToDevice);
    if (ce == cudaSuccess) {
        switch (e->order) {
        case 4: ce = ens_energy<4>(e->L, e->d_pot, e->d_eout, e->stream); break;
        case 6: ce = ens_energy<6>(e->L, e->d_pot, e->d_eout, e->stream); break;
        default: ce = ens_energy<8>(e->L, e->d_pot, e->d_eout, e->stream); break;
        }
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return ens_fail(e, HB_ERR_CUDA, "energy", ce);
    for (int c = 0; c < e->nclusters; ++c) {
        kinetic[c] = e->h_eout[2 * c];
        potential[c] = e->h_eout[2 * c + 1];
    }
    return HB_OK;
}

}  // extern "C"
