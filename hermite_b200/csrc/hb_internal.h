// hb_internal.h -- host-side declarations shared by the library's units.
#pragma once
#include <cuda_runtime.h>

namespace hb {

struct ForceArgs {
    const void *pred;      // predicted slots, AoSoA32 (FP64 or mixed layout)
    int nchunk;            // number of 32-slot j chunks (padded slots / 32)
    int nact;              // i-particles: slots [0, nact)
    double eps2;
    double *force;         // [nact][F]
    double *partial;       // [S][gridDim.x*TI][F]  (only when S > 1)
    unsigned *counter;     // [gridDim.x], zero between launches
    int *err;              // mapped host flag
    unsigned spin;         // poll limit of the waits for incoming tiles
                           // (kSpinLimit; lowered only by hb_set_wait_limit)
    // fused predict + force only: raw j-particle records and the time to
    // predict them to (slots >= nbody are padding)
    const double *jp;
    double tsys;
    int nbody;
};

// One compiled launch shape of the force kernel.
struct ForceVariant {
    int nw;        // warps per CTA
    int ni;        // i-chunks (32 i each) per warp
    int wj;        // warps of an i-group that split the j tile
    int tch;       // 32-slot chunks per j tile
    int ti;        // i per CTA
    int smem;      // dynamic shared memory bytes
    bool fused;    // predicts j (and i) from the raw records itself
    void (*kern)(ForceArgs);
};

// Device-resident block-step integration (hb_integrator.cu).
// What the host reads between graph replays; written once per block step by
// one thread into mapped pinned memory (the scheduler itself stays in device
// memory: its atomics must not cross the host link).
struct IntStatus {
    double tsys;
    long long particle_steps, block_steps;
    int error;
    int pad;
};

struct Sched {
    unsigned long long tnext_bits;   // min(tlast + dt) as the bits of a positive double
    int nact;                        // active slots of the current step
    int work;                        // next force work item
    int error;                       // 1: a timestep underflowed, 2: a device wait gave up
    int pad;
    double tnext, dtlim, tsys, tend;
    double eps2, etapow, dtmax;
    long long particle_steps, block_steps;
    IntStatus *status;               // mapped mirror for the host
};

// Per slot, the two higher derivatives kept for dumps (see correct_particle).
constexpr int kAuxWords = 6;
// Particle::recalc_dt on the host, from a record and its aux row (hb_dump.cu).
double recalc_dt(int order, const double *rec, const double *aux, double eta, double dtmax);

struct IntegratorLaunch {
    double *jp;          // records (the state)
    double *dt;          // per-slot timestep
    double *aux;         // per-slot dump derivatives [kAuxWords]
    int *ilist;          // active slots
    Sched *sched;
    double *force, *partial;
    unsigned *counter;
    int *err;
    int n, nchunk, nsm;
    size_t partial_cap;
    int target_items, items_grid, smem_fp64, smem_mixed;
    int big_grid;       // grid of the large-step force kernel
    bool mixed;
};

cudaError_t integrator_step_launch(int order, const IntegratorLaunch &L, cudaStream_t s);

// Persistent engine (hb_integrator.cu): one cooperative launch runs up to
// max_steps block steps; gbar is two zeroed words (grid barrier); spin is the
// poll limit of a barrier wait.  setup: dynamic shared memory and resident
// CTAs per SM of the kernel.
cudaError_t persistent_setup(int order, bool mixed, int *smem, int *per_sm);
cudaError_t persistent_launch(int order, const IntegratorLaunch &L, unsigned *gbar,
                              long long max_steps, unsigned spin, int grid, cudaStream_t s);

// Team engine (hb_team.cu): one thread-block cluster of `ctas` CTAs runs the
// whole block-step loop of one system at a time inside one kernel.
constexpr int kTeamIMax = 256;              // smallest round of i-states
constexpr int kTeamMaxSlotsPerCta = 2048;
struct TeamSys {
    long long off;     // first slot of the system in the record / dt arrays
    int n;
    int id;            // index of the system's TeamState
    double eps2;
};
struct TeamState {     // per system, persistent across launches
    double tsys;
    long long particle_steps, block_steps;
    double interactions;
    int error, pad;
};
struct TeamConfig {
    int ctas;          // CTAs per team (cluster size)
    int jl_cap;        // slots per CTA with their records in shared memory (rounds of kTeamIMax)
    int jl_cap_g;      // slots per CTA with the records left in global memory
    int smem;          // dynamic shared memory available per CTA
    int max_teams;     // co-resident teams on this device
};
struct TeamLaunch {
    double *jp, *dt;
    double *aux;       // per-slot dump derivatives [kAuxWords], or null
    const TeamSys *sys;
    TeamState *st;     // indexed by TeamSys::id
    int *next_sys;     // work counter, zero at launch
    int nsys;
    int ctas, jl_cap, im, smem;   // from team_shape
    bool rsmem;                   // own records copied into shared memory
    double tend, etapow, dtmax;
    long long max_steps;   // per system and launch
};
cudaError_t team_setup(int order, int ctas, TeamConfig *cfg);
// Fills L's ctas, jl_cap, im and smem for systems of up to nmax particles;
// -1 when they do not fit a team of cfg.ctas CTAs.
int team_shape(int order, const TeamConfig &cfg, int nmax, TeamLaunch *L);
cudaError_t team_launch(int order, const TeamLaunch &L, int teams, cudaStream_t s);
cudaError_t team_sched_sync(Sched *s, TeamState *st, bool to_team, cudaStream_t stream);

cudaError_t integrator_kernel_setup(int order, bool mixed, int *smem, int *blocks_per_sm,
                                    int *big_per_sm);
cudaError_t integrator_assign(int order, double *jp, double *dt, const double *force, int n,
                              int set_dt, double eta_s, double dtmax, cudaStream_t s);
cudaError_t integrator_energy(int order, const double *jp, const double *pot, int n, double *part,
                              double *out, cudaStream_t s);

int force_variant_count(int order, bool mixed);
const ForceVariant *force_variant(int order, bool mixed, int v);

// FP64 force for block steps of at most kLanesMaxAct active particles
// (orders 4, 6, 8): lanes of a warp share an i-particle and split j
// (hb_force_lanes.cu).  Uses a.jp / a.tsys / a.nbody (it predicts the raw
// records itself), a.partial for S * kLanesMaxAct * F doubles, a.counter[0],
// and a.spin / a.err for its bounded waits on bulk copies.
constexpr int kLanesMaxAct = 16;
cudaError_t launch_force_lanes(int order, const ForceArgs &a, int nsm, cudaStream_t s);

cudaError_t launch_predict(int order, bool mixed, const double *jp, int n, int npad,
                           double tsys, void *pred, int *err, cudaStream_t s);
cudaError_t launch_potential(int order, const double *jp, int n, int npad, double eps2,
                             double *posm, double *pot, int *err, cudaStream_t s);
cudaError_t run_fma_peak(int mode, int nsm, double *gflops);

}  // namespace hb
