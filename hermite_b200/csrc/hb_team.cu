// hb_team.cu -- block-timestep integration of small systems by one
// thread-block cluster ("team") per system, the whole block-step loop inside
// one kernel.
//
// The reference's host loop (NbodySystem::integrate_one_block,
// SRC/nbodysystem.h:693-765: next block time, active set, predict, force,
// correct) costs a few microseconds of launch and synchronisation per step
// when each step is its own set of kernels; for N of a few thousand the
// force itself is smaller than that.  Here C CTAs of one cluster own the
// system's slots in C contiguous 32-slot-aligned ranges and run every step
// with three cluster barriers and no grid-wide synchronisation:
//
//   A  each CTA: minimum of tlast + dt over its own slots       -> barrier 1
//   B  every CTA reads the C minima (distributed shared memory): tnext;
//      each CTA lists its own active slots (slot order) and predicts its own
//      slots to tnext into shared memory                        -> barrier 2
//   C  every CTA gathers the predicted states of all active slots from
//      their owners and sums them against its own slots (a j-split across
//      the team), partial forces in its shared memory           -> barrier 3
//      each owner adds the C partials of its active slots in rank order and
//      runs the corrector (Particle::correct + the quantised Aarseth step)
//
// Steps with more active slots than the push regions hold are processed in
// rounds pulled from the owners.
// Teams take systems from a device counter, so one launch integrates a whole
// ensemble with every system on its own block-time sequence (no lockstep),
// or a single system.  The per-system state is the same record array and dt
// array that the multi-kernel engine uses.  FP64 throughout.
//
// Every decision that controls a barrier (system index, tnext, error flag,
// step count, round count) is computed identically by every thread of the
// team from the same shared data, so all threads take the same barriers.
// No thread spins on memory: the only waits are cluster and CTA barriers.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>

#include "hb_common.cuh"
#include "hb_corrector.cuh"
#include "hb_force.cuh"
#include "hb_internal.h"

namespace hb {
namespace {

namespace cg = cooperative_groups;

constexpr int kTeamWarps = 16;

struct TeamXch {
    double m;     // minimum of tlast + dt over the sender's own slots
    int k;        // the sender's own slots at that minimum (candidates)
    int err;      // a corrector of the sender produced a timestep underflow
};

// Shared-memory carve-up for jl own slots per CTA and im i-states per round;
// the own records are in shared memory (RSMEM) or stay in global memory.
template <int ORDER>
struct TeamSmem {
    static constexpr int R = Rec<ORDER>::words, P = Pred64<ORDER>::ncomp, F = Frc<ORDER>::words;
    // per i-state: ibuf [P], part [F] (doubles); gq, gc (ints)
    static constexpr size_t per_i = (size_t)(P + F) * 8 + 2 * 4;
    // per slot: [record], predicted state, tlast + dt, dt (doubles); candidate (int)
    static constexpr size_t per_slot(bool rsmem) { return (size_t)((rsmem ? R : 0) + P + 2) * 8 + 4; }
    // xa [16], koff [48], misc [4], alignment
    static constexpr size_t fixed = 16 * sizeof(TeamXch) + (48 + 4) * 4 + 64;
    static size_t bytes(int jl, int im, bool rsmem)
    {
        return fixed + per_i * (size_t)im + per_slot(rsmem) * (size_t)jl;
    }
};
// Smallest round with the records in global memory (larger systems).
constexpr int kTeamIMinGlobal = 64;

__device__ __forceinline__ double warp_min(double v)
{
    for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// calc_dtlim (SRC/nbodysystem.h:652-661): dtmax halved until tnext is a
// multiple of it, at most 64 times.  For a power-of-two dtmax = 2^D this is
// 2^(D-k) with k = clamp(D - e, 0, 64), e the exponent of the lowest set
// bit of tnext (tnext = 0 is a multiple of everything): the same value the
// reference's loop reaches, from the exponent and significand bits.
__device__ __forceinline__ double team_dtlim(double tnext, double dtmax)
{
    if (!(tnext > 0.0)) return dtmax;
    const long long b = __double_as_longlong(tnext);
    const int ex = (int)((b >> 52) & 0x7ff);
    const long long sig = (b & 0xfffffffffffffll) | (ex ? (1ll << 52) : 0ll);
    const int e = (ex ? ex : 1) - 1075 + (__ffsll(sig) - 1);
    const int D = (int)((__double_as_longlong(dtmax) >> 52) & 0x7ff) - 1023;
    const int k = max(0, min(64, D - e));
    return __longlong_as_double(__double_as_longlong(dtmax) - ((long long)k << 52));
}

// Partial forces of nr i-particles (ibuf, AoSoA32, at positions idx(gi))
// against this CTA's JL own predicted slots.  G lanes (a power of two)
// share NI i-particles, each lane summing every G-th own slot, and their
// sums meet in a fixed xor-shuffle tree; out(gi, f) is called by the first
// lane of each group.  NW * 32 / G * NI >= nr i-slots.
template <int ORDER, int NI, typename Idx, typename Out>
__device__ __forceinline__ void team_force_ni(const double *ibuf, const double *pred, int JL, int nr,
                                              double eps2, Idx idx, Out out)
{
    constexpr int NW = kTeamWarps, F = Frc<ORDER>::words;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int G = 32;
    while (G > 1 && NW * (32 / G) * NI < nr) G >>= 1;
    const int gp = w * (32 / G) + lane / G, js = lane & (G - 1);
    double f[NI][F];
#pragma unroll
    for (int n = 0; n < NI; ++n)
#pragma unroll
        for (int c = 0; c < F; ++c) f[n][c] = 0.0;
    if (gp * NI < nr) {
        Body64 I[NI];
#pragma unroll
        for (int n = 0; n < NI; ++n) {
            const int x = idx(gp * NI + n < nr ? gp * NI + n : gp * NI);   // a missing pair partner repeats the first
            load_i64<ORDER>(ibuf, x >> 5, x & 31, I[n]);
        }
#pragma unroll 2
        for (int j = js; j < JL; j += G) {
            Body64 J;
            load_i64<ORDER>(pred, j >> 5, j & 31, J);
#pragma unroll
            for (int n = 0; n < NI; ++n) interact64<ORDER>(I[n], J, eps2, f[n]);
        }
    }
    for (int o = G >> 1; o; o >>= 1)
#pragma unroll
        for (int n = 0; n < NI; ++n)
#pragma unroll
            for (int c = 0; c < F; ++c) f[n][c] += __shfl_xor_sync(0xffffffffu, f[n][c], o);
    if (js == 0)
#pragma unroll
        for (int n = 0; n < NI; ++n)
            if (gp * NI + n < nr) out(gp * NI + n, f[n]);
}

// Two i per lane (two independent chains per j load) at 4th order, where the
// registers allow it, once the round is large enough for the lane groups to
// stay narrow; one otherwise.  The choice depends on nr only, so every CTA
// of a team sums in the same order.
template <int ORDER, typename Idx, typename Out>
__device__ __forceinline__ void team_force(const double *ibuf, const double *pred, int JL, int nr,
                                           double eps2, Idx idx, Out out)
{
    if constexpr (ORDER == 4) {
        if (nr > 128) {
            team_force_ni<ORDER, 2>(ibuf, pred, JL, nr, eps2, idx, out);
            return;
        }
    }
    team_force_ni<ORDER, 1>(ibuf, pred, JL, nr, eps2, idx, out);
}

template <int ORDER, bool RSMEM>
__global__ void __launch_bounds__(kTeamWarps * 32, 1) team_kernel(TeamLaunch L)
{
    constexpr int T = kTeamWarps * 32;
    constexpr int R = Rec<ORDER>::words, F = Frc<ORDER>::words, P = Pred64<ORDER>::ncomp;
    cg::cluster_group team = cg::this_cluster();
    const int C = (int)team.num_blocks(), rank = (int)team.block_rank();
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int jl_cap = L.jl_cap;   // own slots per CTA
    const int IM = L.im;           // i states per round (<= NW * 32)
    const int KM = IM / C;         // i states one rank pushes per step (its region of ibuf)

    extern __shared__ __align__(16) unsigned char smem[];
    double *rec_s = reinterpret_cast<double *>(smem);             // [jl_cap][R] own records (RSMEM)
    double *pred = rec_s + (RSMEM ? (size_t)jl_cap * R : 0);      // [jl_cap/32][P][32]
    double *ibuf = pred + (size_t)jl_cap * P;                     // [IM/32][P][32] i states
    double *part = ibuf + IM * P;                                 // [IM][F] partial forces
    double *tn = part + IM * F;                                   // [jl_cap] tlast + dt
    double *dts = tn + jl_cap;                                    // [jl_cap] dt
    TeamXch *xa = reinterpret_cast<TeamXch *>(dts + jl_cap);      // [16] every rank's (m, k, err)
    int *cand = reinterpret_cast<int *>(xa + 16);                 // [jl_cap] candidates, slot order
    int *gq = cand + jl_cap;                                      // [IM]
    int *gc = gq + IM;                                            // [IM]
    int *koff = gc + IM;                                          // [48] koff[c] = actives below rank c
    int *misc = koff + 48;                                        // [0] system (rank 0), [1] own error

    const double inf = __longlong_as_double(0x7ff0000000000000ll);

    for (;;) {
        if (rank == 0 && tid == 0) misc[0] = atomicAdd(L.next_sys, 1);
        team.sync();
        const int sidx = team.map_shared_rank(misc, 0)[0];
        if (sidx >= L.nsys) {
            team.sync();   // no CTA leaves while another still reads its shared memory
            break;
        }
        const TeamSys S = L.sys[sidx];
        const int n = S.n;
        const double eps2 = S.eps2;
        double *jp = L.jp + (size_t)S.off * R;
        double *dtg = L.dt + S.off;
        const int nch = (n + 31) >> 5;
        const int c0 = (int)((long long)rank * nch / C), c1 = (int)((long long)(rank + 1) * nch / C);
        const int lo = c0 * 32, JL = (c1 - c0) * 32;
        // own records: a copy in shared memory, or in place in global memory
        double *rec = RSMEM ? rec_s : jp + (size_t)lo * R;

        if constexpr (RSMEM)
            for (int e = tid; e < JL * R; e += T) {
                const int q = e / R, slot = lo + q;
                rec[e] = slot < n ? jp[(size_t)lo * R + e] : 0.0;
            }
        for (int q = tid; q < JL; q += T) {
            const int slot = lo + q;
            if (slot < n) {
                const double d = dtg[slot];
                dts[q] = d;
                tn[q] = d + jp[(size_t)slot * R + 7];
            } else {
                dts[q] = 0.0;
                tn[q] = inf;
            }
        }
        if (tid == 0) misc[1] = 0;
        double tsys = L.st[S.id].tsys;
        const bool dead = L.st[S.id].error != 0;   // a system that failed stays stopped
        long long steps = 0, psteps = 0;
        double inter = 0.0;
        int err = 0;
        __syncthreads();

        // Warp 0, before every barrier 1: the own minimum, its candidates (in
        // slot order), their states predicted to it pushed into region `rank`
        // of every CTA's ibuf, and (m, k, err) into every CTA's xa[rank].
        auto announce = [&]() {
            double m = inf;
            for (int q = lane; q < JL; q += 32) m = fmin(m, tn[q]);
            m = warp_min(m);
            int k = 0;
            if (m < inf) {
                for (int base = 0; base < JL; base += 32) {
                    const int q = base + lane;
                    const bool act = q < JL && tn[q] == m;
                    const unsigned b = __ballot_sync(0xffffffffu, act);
                    if (act) cand[k + __popc(b & ((1u << lane) - 1u))] = q;
                    k += __popc(b);
                }
            }
            __syncwarp();
            // the candidates' states predicted to m, pushed by one lane each
            // into region `rank` of every CTA's ibuf (store instructions of
            // one lane go to one rank back to back, from registers)
            const int kp = min(k, KM);
            for (int a = lane; a < kp; a += 32) {
                const double *r = rec + (size_t)cand[a] * R;
                double x[3], v[3], ac[3] = {0.0, 0.0, 0.0}, jk[3] = {0.0, 0.0, 0.0};
                double xl[3] = {0.0, 0.0, 0.0};
                predict_slot<ORDER>(r, m, x, v, ac, jk, xl);
                const double mass = r[3];
                const int g = rank * KM + a;
                const int off = (g >> 5) * P * 32 + (g & 31);
                for (int c = 0; c < C; ++c) {
                    double *d = team.map_shared_rank(ibuf, c) + off;
#pragma unroll
                    for (int kk = 0; kk < 3; ++kk) {
                        d[(P64_X + kk) * 32] = x[kk];
                        d[(P64_V + kk) * 32] = v[kk];
                        if constexpr (ORDER >= 6) d[(P64_A + kk) * 32] = ac[kk];
                        if constexpr (ORDER >= 8) d[(P64_J + kk) * 32] = jk[kk];
                        if constexpr (ORDER == 9) d[(P64_XL + kk) * 32] = xl[kk];
                    }
                    d[P64_M * 32] = mass;
                }
            }
            if (lane < C) {
                TeamXch *d = team.map_shared_rank(xa, lane) + rank;
                d->m = m;
                d->k = k;
                d->err = misc[1];
            }
        };
        if (w == 0) announce();

        for (;;) {
            team.sync();   // barrier 1: every rank's (m, k, err) and pushed states are here

            double mc = inf;
            int kc = 0, ec = 0;
            if (lane < C) {
                mc = xa[lane].m;
                kc = xa[lane].k;
                ec = xa[lane].err;
            }
            const double tnext = warp_min(mc);
            err = __any_sync(0xffffffffu, ec != 0);
            const int kk = (lane < C && mc == tnext) ? kc : 0;     // actives of rank `lane`
            const bool over = __any_sync(0xffffffffu, kk > KM);
            int incl = kk;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const int nact = __shfl_sync(0xffffffffu, incl, 31);
            const int kact = __shfl_sync(0xffffffffu, kk, rank);
            const int myoff = __shfl_sync(0xffffffffu, incl, rank) - kact;
            if (dead || err || !(tnext <= L.tend) || steps >= L.max_steps) break;
            const double dtlim = team_dtlim(tnext, L.dtmax);
            if (w == 0) {
                koff[lane + 1] = incl;
                if (lane == 0) koff[0] = 0;
            }

            // own slots predicted to tnext (the j side)
            for (int q = tid; q < JL; q += T) {
                const int slot = lo + q;
                double x[3], v[3], a[3] = {0.0, 0.0, 0.0}, jk[3] = {0.0, 0.0, 0.0}, mass;
                double xl[3] = {0.0, 0.0, 0.0};
                if (slot < n) {
                    const double *r = rec + (size_t)q * R;
                    predict_slot<ORDER>(r, tnext, x, v, a, jk, xl);
                    mass = r[3];
                } else {
#pragma unroll
                    for (int k = 0; k < 3; ++k) { x[k] = pad_position(slot, k); v[k] = 0.0; }
                    mass = 0.0;
                }
                double *c = pred + (size_t)(q >> 5) * P * 32 + (q & 31);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    c[(P64_X + k) * 32] = x[k];
                    c[(P64_V + k) * 32] = v[k];
                    if constexpr (ORDER >= 6) c[(P64_A + k) * 32] = a[k];
                    if constexpr (ORDER >= 8) c[(P64_J + k) * 32] = jk[k];
                    if constexpr (ORDER == 9) c[(P64_XL + k) * 32] = xl[k];
                }
                c[P64_M * 32] = mass;
            }
            __syncthreads();

            if (!over && nact <= IM) {
                // the active states are the pushed ones: position gi of rank c
                // sits at ibuf[c * KM + a]; partials go to the owner's part
                // at [rank * KM + a]
                team_force<ORDER>(
                    ibuf, pred, JL, nact, eps2,
                    [&](int gi) {
                        int c = 0;
                        while (c + 1 < C && gi >= koff[c + 1]) ++c;
                        return c * KM + (gi - koff[c]);
                    },
                    [&](int gi, const double *f) {
                        int c = 0;
                        while (c + 1 < C && gi >= koff[c + 1]) ++c;
                        double *d = team.map_shared_rank(part, c) + (size_t)(rank * KM + gi - koff[c]) * F;
#pragma unroll
                        for (int k = 0; k < F; ++k) d[k] = f[k];
                    });
                team.sync();   // barrier 3: every partial is with its owner

                if (w == 0) {
                    for (int a = lane; a < kact; a += 32) {
                        double f[F];
#pragma unroll
                        for (int k = 0; k < F; ++k) f[k] = 0.0;
                        for (int src = 0; src < C; ++src)
#pragma unroll
                            for (int k = 0; k < F; ++k) f[k] += part[(size_t)(src * KM + a) * F + k];
                        const int q = cand[a];
                        double *r = rec + (size_t)q * R;
                        const double dtn = correct_particle<ORDER>(
                            r, f, dts[q], L.etapow, dtlim,
                            L.aux ? L.aux + (size_t)(S.off + lo + q) * kAuxWords : nullptr);
                        if (!(dtn >= 0x1p-48)) misc[1] = 1;   // timestep underflow (or NaN)
                        dts[q] = dtn;
                        tn[q] = dtn + r[7];
                    }
                    __syncwarp();
                    announce();
                }
            } else {
                // many actives: rounds of IM pulled from the owners
                team.sync();   // barrier 2: predicted states and candidate lists complete
                for (int base = 0; base < nact; base += IM) {
                    const int nr = min(IM, nact - base);
                    for (int i = tid; i < nr; i += T) {
                        const int g = base + i;
                        int c = 0;
                        while (c + 1 < C && g >= koff[c + 1]) ++c;
                        gq[i] = team.map_shared_rank(cand, c)[g - koff[c]];
                        gc[i] = c;
                    }
                    __syncthreads();
                    for (int e2 = tid; e2 < nr * P; e2 += T) {
                        const int comp = e2 / nr, i = e2 - comp * nr, q = gq[i];
                        ibuf[(i >> 5) * P * 32 + comp * 32 + (i & 31)] =
                            team.map_shared_rank(pred, gc[i])[(size_t)(q >> 5) * P * 32 + comp * 32 + (q & 31)];
                    }
                    __syncthreads();
                    team_force<ORDER>(
                        ibuf, pred, JL, nr, eps2, [](int gi) { return gi; },
                        [&](int gi, const double *f) {
#pragma unroll
                            for (int k = 0; k < F; ++k) part[gi * F + k] = f[k];
                        });
                    team.sync();   // barrier 3: every partial of the round is visible

                    const int a0 = max(0, base - myoff), a1 = min(kact, base + nr - myoff);
                    for (int a = a0 + tid; a < a1; a += T) {
                        const int i = myoff + a - base;
                        double f[F];
#pragma unroll
                        for (int k = 0; k < F; ++k) f[k] = 0.0;
                        for (int src = 0; src < C; ++src) {
                            const double *pp = team.map_shared_rank(part, src) + i * F;
#pragma unroll
                            for (int k = 0; k < F; ++k) f[k] += pp[k];
                        }
                        const int q = cand[a];
                        double *r = rec + (size_t)q * R;
                        const double dtn = correct_particle<ORDER>(
                            r, f, dts[q], L.etapow, dtlim,
                            L.aux ? L.aux + (size_t)(S.off + lo + q) * kAuxWords : nullptr);
                        if (!(dtn >= 0x1p-48)) misc[1] = 1;
                        dts[q] = dtn;
                        tn[q] = dtn + r[7];
                    }
                    if (base + IM < nact) team.sync();   // part and ibuf are reused by the next round
                }
                __syncthreads();
                if (w == 0) announce();
            }
            ++steps;
            psteps += nact;
            inter += (double)nact * (double)n;
            tsys = tnext;
        }

        if constexpr (RSMEM)
            for (int e = tid; e < JL * R; e += T)
                if (lo + e / R < n) jp[(size_t)lo * R + e] = rec[e];
        for (int q = tid; q < JL; q += T)
            if (lo + q < n) dtg[lo + q] = dts[q];
        if (rank == 0 && tid == 0) {
            TeamState &st = L.st[S.id];
            st.tsys = tsys;
            st.particle_steps += psteps;
            st.block_steps += steps;
            st.interactions += inter;
            if (err) st.error = 1;
        }
        __syncthreads();
    }
}

template <int ORDER>
cudaError_t team_setup_t(int ctas, TeamConfig *cfg)
{
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    const int avail = optin - 1024;
    // slots per CTA: records in shared memory with the smallest round of
    // kTeamIMax i-states, or records in global memory with kTeamIMinGlobal
    using SM = TeamSmem<ORDER>;
    auto cap = [&](bool rsmem, int im) {
        const long long c = ((long long)avail - (long long)SM::fixed - (long long)SM::per_i * im) /
                            (long long)SM::per_slot(rsmem);
        return (int)std::min<long long>(c & ~31LL, kTeamMaxSlotsPerCta);
    };
    const int jl_cap = cap(true, kTeamIMax), jl_cap_g = cap(false, kTeamIMinGlobal);
    if (jl_cap < 32) return cudaErrorInvalidValue;
    const int smem = avail;
    for (const void *k : {(const void *)&team_kernel<ORDER, true>, (const void *)&team_kernel<ORDER, false>}) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e == cudaSuccess && ctas > 8)
            e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(ctas);
    lc.blockDim = dim3(kTeamWarps * 32);
    lc.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    int teams = 0;
    e = cudaOccupancyMaxActiveClusters(&teams, (void *)&team_kernel<ORDER, true>, &lc);
    if (e != cudaSuccess) return e;
    cfg->ctas = ctas;
    cfg->jl_cap = jl_cap;
    cfg->jl_cap_g = std::max(jl_cap, jl_cap_g);
    cfg->smem = smem;
    cfg->max_teams = teams;
    return cudaSuccess;
}

// Launch shape for systems of up to nmax particles: the own slots per CTA
// they need, and as many i-states per round (a multiple of 32, at most one
// per thread) as the rest of the shared memory holds.
template <int ORDER>
int team_shape_t(const TeamConfig &cfg, int nmax, TeamLaunch *L)
{
    using SM = TeamSmem<ORDER>;
    const int nch = (nmax + 31) / 32;
    const int jl = (nch + cfg.ctas - 1) / cfg.ctas * 32;
    const bool rsmem = jl <= cfg.jl_cap;   // records in shared memory when they fit
    if (!rsmem && jl > cfg.jl_cap_g) return -1;
    long long im = ((long long)cfg.smem - (long long)SM::fixed - (long long)SM::per_slot(rsmem) * jl) /
                   (long long)SM::per_i;
    im = std::min<long long>(im & ~31LL, kTeamWarps * 32);
    if (im < (rsmem ? kTeamIMax : kTeamIMinGlobal)) return -1;
    L->ctas = cfg.ctas;
    L->jl_cap = jl;
    L->im = (int)im;
    L->rsmem = rsmem;
    L->smem = (int)SM::bytes(jl, (int)im, rsmem);
    return 0;
}

template <int ORDER>
cudaError_t team_launch_t(const TeamLaunch &L, int teams, cudaStream_t s)
{
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(teams * L.ctas);
    lc.blockDim = dim3(kTeamWarps * 32);
    lc.dynamicSmemBytes = L.smem;
    lc.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = L.ctas;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    return L.rsmem ? cudaLaunchKernelEx(&lc, team_kernel<ORDER, true>, L)
                   : cudaLaunchKernelEx(&lc, team_kernel<ORDER, false>, L);
}

// Single-system bookkeeping: the multi-kernel engine's scheduler <-> the
// team's per-system state.
__global__ void team_from_sched_kernel(const Sched *s, TeamState *st)
{
    st->tsys = s->tsys;
    st->particle_steps = s->particle_steps;
    st->block_steps = s->block_steps;
    st->interactions = 0.0;
    st->error = s->error;
}

__global__ void team_to_sched_kernel(const TeamState *st, Sched *s)
{
    s->tsys = st->tsys;
    s->particle_steps = st->particle_steps;
    s->block_steps = st->block_steps;
    if (st->error) s->error = st->error;
    s->tnext_bits = 0x7ff0000000000000ull;
    IntStatus *o = s->status;
    o->tsys = s->tsys;
    o->particle_steps = s->particle_steps;
    o->block_steps = s->block_steps;
    o->error = s->error;
}

}  // namespace

cudaError_t team_setup(int order, int ctas, TeamConfig *cfg)
{
    if (ctas < 1 || ctas > 16) return cudaErrorInvalidValue;
    switch (order) {
    case 4: return team_setup_t<4>(ctas, cfg);
    case 6: return team_setup_t<6>(ctas, cfg);
    case 8: return team_setup_t<8>(ctas, cfg);
    case 9: return team_setup_t<9>(ctas, cfg);
    }
    return cudaErrorInvalidValue;
}

int team_shape(int order, const TeamConfig &cfg, int nmax, TeamLaunch *L)
{
    switch (order) {
    case 4: return team_shape_t<4>(cfg, nmax, L);
    case 6: return team_shape_t<6>(cfg, nmax, L);
    case 8: return team_shape_t<8>(cfg, nmax, L);
    case 9: return team_shape_t<9>(cfg, nmax, L);
    }
    return -1;
}

cudaError_t team_launch(int order, const TeamLaunch &L, int teams, cudaStream_t s)
{
    switch (order) {
    case 4: return team_launch_t<4>(L, teams, s);
    case 6: return team_launch_t<6>(L, teams, s);
    case 8: return team_launch_t<8>(L, teams, s);
    case 9: return team_launch_t<9>(L, teams, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t team_sched_sync(Sched *s, TeamState *st, bool to_team, cudaStream_t stream)
{
    if (to_team) team_from_sched_kernel<<<1, 1, 0, stream>>>(s, st);
    else team_to_sched_kernel<<<1, 1, 0, stream>>>(st, s);
    return cudaGetLastError();
}

}  // namespace hb
