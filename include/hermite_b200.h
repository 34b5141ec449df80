/*
 * hermite_b200.h -- C ABI of the B200 (sm_100a) Hermite force calculator.
 *
 * This is the boundary that replaces the reference's CUDA force calculator,
 * the compile-time C++ `struct Gravity` of SRC/hermite{4,6,8}-titan.h that
 * SRC/hermite{4,6,8}.h select with -DCUDA_TITAN (e.g. SRC/hermite4.h:286-287)
 * and that the integrator drives (SRC/nbodysystem.h:308,326,565-765).  Each
 * entry point names the reference member it stands for.  The C++ drop-in that
 * maps `struct Gravity` onto these calls is hermite_b200/gravity/.
 *
 * Plain pointers and sizes only; no CUDA or torch types in the signatures.
 * Every function returns an int status (HB_OK == 0).  The reference has no
 * status codes (it prints and aborts through checkCudaErrors,
 * SRC/cuda_pointer.h:6-10); the C++ drop-in restores that behaviour.
 *
 * Data formats (doubles, little-endian host order):
 *   j-particle record, 8 + 3*(order-2) words (14 / 20 / 26):
 *     pos[3] mass vel[3] tlast acc[3] jrk[3] [snp[3] crk[3]] [d4a[3] d5a[3]]
 *     (the field order of the reference's GParticle, SRC/hermite4-titan.h:20-27,
 *      SRC/hermite6-titan.h:20-29, SRC/hermite8-titan.h:20-31)
 *   force record, 3*(order/2) words (6 / 9 / 12):
 *     acc[3] jrk[3] [snp[3]] [crk[3]]
 *     (the reference's `struct Force`, SRC/hermite4.h:4-14, SRC/hermite6.h:4-17,
 *      SRC/hermite8.h:8-24)
 *
 * Threading: hb_set_jp / hb_set_jp_records may be called concurrently from
 * several host threads on distinct slots (the integrator does so from OpenMP
 * workers, SRC/nbodysystem.h:753-756).  Every other call on one context must
 * come from one thread at a time.
 */
#ifndef HERMITE_B200_H
#define HERMITE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct hb_ctx hb_ctx;

enum hb_status {
    HB_OK = 0,
    HB_ERR_INVALID = 1,        /* an argument is out of range              */
    HB_ERR_CUDA = 2,           /* a CUDA runtime call failed               */
    HB_ERR_ALLOC = 3,          /* device or pinned host allocation failed  */
    HB_ERR_DEVICE_TIMEOUT = 4, /* a bounded device-side wait gave up       */
    HB_ERR_NO_DEVICE = 5,      /* no CUDA device, or not an sm_100 device  */
    HB_ERR_STATE = 6,          /* call out of order (e.g. force before any
                                  predict_all)                            */
    HB_ERR_TOO_LARGE = 7,      /* a size exceeds a fixed capacity (see
                                  hb_force_predicted_noalloc)             */
    HB_ERR_IO = 8              /* a file could not be written or parsed   */
};

enum hb_precision {
    HB_FP64 = 0,    /* plain FP64 interaction and accumulation (the default) */
    HB_MIXED = 1,   /* FP64 predictor; hi/lo FP32 relative positions; FP32
                       interaction; FP32 partial sums flushed into FP64
                       accumulators; FP64 crackle accumulation at 8th order  */
    HB_FP64_DD = 2  /* order 8 only: positions as double-double (posH +
                       posL), the reference's SRC/hermite8dd.h.  Records are
                       the 8th-order record followed by posL[3] (29 words;
                       hb_set_jp's derivs: acc jrk snp crk d4a d5a posL);
                       the predictor advances posL only; pair separations
                       are (posHj - posHi) + (posLj - posLi), pairs at zero
                       separation are skipped; FP64 arithmetic otherwise.
                       The file helpers below take order code 9 for it.  */
};

/* Gravity(int nbody) -- SRC/hermite4-titan.h:49-57 (also 6th/8th).
 * order is 4, 6 or 8; 1 <= nbody <= 1<<24.  Allocates device buffers and
 * pinned host mirrors once; nothing is allocated per call afterwards. */
int hb_create(int order, int nbody, int precision, hb_ctx **out);

/* ~Gravity() -- SRC/hermite4-titan.h:58-63.  NULL is accepted. */
int hb_destroy(hb_ctx *ctx);

/* Gravity::set_jp(int addr, const Particle p) -- SRC/hermite4-titan.h:70-78,
 * SRC/hermite6-titan.h:70-97, SRC/hermite8-titan.h:77-112.
 * Writes slot `addr` of the pinned host mirror only.  `derivs` holds
 * 3*(order-2) doubles: acc jrk [snp crk] [d4a d5a]. */
int hb_set_jp(hb_ctx *ctx, int addr, const double pos[3], double mass,
              const double vel[3], double tlast, const double *derivs);

/* Bulk form of set_jp: `count` consecutive records starting at slot addr0. */
int hb_set_jp_records(hb_ctx *ctx, int addr0, int count, const double *records);

/* Gravity::predict_all(double tsys) -- SRC/hermite4-titan.cu:102-116.
 * Uploads the slots changed since the last upload (the reference uploads the
 * first `njpsend` = previous nact slots, SRC/hermite4-titan.cu:103,411; this
 * also covers any other slot passed to set_jp), then predicts every slot to
 * tsys from its own tlast.  Asynchronous: returns once work is queued. */
int hb_predict_all(hb_ctx *ctx, double tsys);

/* Gravity::calc_force_on_first_nact(int nact, double eps2, Force force[]) --
 * SRC/hermite4-titan.cu:362-412, SRC/hermite6-titan.cu:362-405,
 * SRC/hermite8-titan.cu:428-473.  Force on slots [0,nact) from all slots,
 * self pair included (exactly zero for eps2 > 0).  Writes nact force records
 * to force_out and returns when they are there.  0 <= nact <= nbody. */
int hb_force_first_nact(hb_ctx *ctx, int nact, double eps2, double *force_out);

/* Gravity::calc_potential(double eps2, double potbuf[]) --
 * SRC/pot-titan.hu:131-171.  phi_i = -sum_{j != i} m_j / sqrt(r^2 + eps2)
 * on the un-predicted positions of the host mirror (pending set_jp slots are
 * uploaded first).  Writes nbody doubles to pot_out. */
int hb_potential(hb_ctx *ctx, double eps2, double *pot_out);

/* Switch between HB_FP64 and HB_MIXED.  Takes effect at the next
 * predict_all (the predicted layout differs). */
int hb_set_precision(hb_ctx *ctx, int precision);
int hb_get_precision(const hb_ctx *ctx);

/* Last error message of this context ("" if none); static text for NULL. */
const char *hb_last_error(const hb_ctx *ctx);
const char *hb_status_string(int status);

/* ---- device-resident forms (no host<->device copies) -------------------
 * For callers that keep inputs and results in HBM, and for timing the
 * kernels alone.  None of these has a reference counterpart; they split
 * predict_all / calc_force_on_first_nact at the copy boundaries. */

/* Run all later work of this context on the given cudaStream_t (NULL restores
 * the context's own stream). */
int hb_set_stream(hb_ctx *ctx, void *cuda_stream);
/* Upload pending set_jp slots now (the copy part of predict_all). */
int hb_upload(hb_ctx *ctx);
/* The kernel part of predict_all: predict every slot to tsys, no upload.
 * The prediction runs with the next force launch (inside the fused force
 * kernel, or as a predictor pass ahead of a two-pass one). */
int hb_predict_all_device(hb_ctx *ctx, double tsys);
/* Run the predictor pass now: every slot predicted to the tsys of the last
 * predict_all into the context's predicted array (the two-pass force shapes
 * read it; fused shapes predict for themselves).  The next two-pass force
 * launch then skips its own pass.  For timing the predictor alone. */
int hb_predict_pass(hb_ctx *ctx);
/* The kernel part of calc_force_on_first_nact: results stay in HBM
 * (hb_device_forces), nothing is copied back, no synchronisation. */
int hb_force_device(hb_ctx *ctx, int nact, double eps2);
/* Copy nact force records of the last hb_force_device to the host. */
int hb_download_forces(hb_ctx *ctx, int nact, double *force_out);
/* Device address of the force records (nbody x 3*(order/2) doubles). */
const double *hb_device_forces(const hb_ctx *ctx);
/* Wait for the context's queued work; reports device-side wait timeouts. */
int hb_synchronize(hb_ctx *ctx);
/* Number of kernels this context has launched so far. */
long long hb_launch_count(const hb_ctx *ctx);

/* Test hook: the poll limit of the force kernel's waits for incoming j tiles
 * (default and maximum 1<<22 polls; polls < 0 restores the default), and of
 * the persistent engine's grid-barrier waits.  A
 * limit of 0 makes every such wait give up at once, so a test can drive the
 * kernel's timeout path with no fault: the kernel raises its error flag, its
 * waits for the copies already in flight keep the full limit, the call
 * returns HB_ERR_DEVICE_TIMEOUT and the context stays usable.  No
 * counterpart in the reference, whose CUDA path only aborts on errors
 * (SRC/cuda_pointer.h:6-10). */
int hb_set_wait_limit(hb_ctx *ctx, long long polls);

/* Launch shape of the force kernel, picked per (order, precision, nbody,
 * nact) by the built-in tuning table unless overridden here.  variant
 * indexes the compiled kernel variants (see hb_force_variant_count);
 * jsplit is the number of j-slices (CTAs per i-tile); 0 means "auto".
 * With variant < 0 (automatic), FP64 block steps of at most 16 active
 * particles (orders 4, 6, 8) take a separate kernel in which the lanes of
 * a warp share an i-particle and split the j range; an explicit variant
 * always takes the tiled kernel. */
int hb_set_force_shape(hb_ctx *ctx, int variant, int jsplit);
int hb_force_variant_count(int order, int precision);
/* Describe a variant: threads per CTA, i per thread, warps splitting j. */
int hb_force_variant_info(int order, int precision, int variant,
                          int *threads, int *i_per_thread, int *j_warps);

/* ---- device-resident block-step integration ------------------------------
 * The reference runs the Hermite corrector and the block-timestep scheduler
 * on the host (NbodySystem::init_step / integrate_one_block,
 * SRC/nbodysystem.h:565-631,693-765; Particle::correct and init_dt,
 * SRC/hermite{4,6,8}.h).  These entry points run the same algorithm on the
 * device: next block time = min(tlast + dt), active set, dtlim, fused
 * predict + force on the active set, corrector with the quantised Aarseth
 * step, 32 block steps per replay of a captured CUDA graph, no host round
 * trip per step.  Slots are not re-sorted.  The state is the context's
 * j-particle records plus a per-slot dt. */

/* init_step: the current records' pos, mass and vel (set with set_jp) at
 * tlast = tsys with zero derivatives are the initial conditions; forces are
 * evaluated (twice for order > 4, to bootstrap snap/crackle), written into
 * the records, and the initial dt set from eta_s and dtmax (a power of two).
 * etapow = eta^(2*(order-3)) as the reference's set_run_params. */
int hb_integrator_init(hb_ctx *ctx, double tsys, double eps2, double eta, double eta_s,
                       double dtmax);
/* Engines for hb_integrator_run (same state, same algorithm):
 *  HB_ENGINE_GRAPH  four phases (five kernels) per block step over the whole GPU, 32 steps
 *                   per replay of a CUDA graph (any N, FP64 or mixed);
 *  HB_ENGINE_PERSISTENT  the graph engine's phases in one cooperative kernel
 *                   whose CTAs all stay resident, grid barriers (bounded
 *                   waits) between the phases, up to 4096 block steps per
 *                   launch; the same block steps and records as the graph
 *                   engine, bit for bit (any N, FP64 or mixed);
 *  HB_ENGINE_TEAM   one thread-block cluster of up to 16 CTAs runs the whole
 *                   block-step loop in one kernel, three cluster barriers per
 *                   step (FP64; N up to 16 x the slots one CTA holds in
 *                   shared memory, about 16k);
 *  HB_ENGINE_AUTO   the team engine for FP64 systems of up to 3072
 *                   particles, else the graph engine (the default).
 * team_ctas: CTAs per team (1..16), 0 = chosen from N. */
enum { HB_ENGINE_AUTO = 0, HB_ENGINE_GRAPH = 1, HB_ENGINE_TEAM = 2, HB_ENGINE_PERSISTENT = 3 };
int hb_integrator_set_engine(hb_ctx *ctx, int engine, int team_ctas);
/* The engine (HB_ENGINE_GRAPH, _TEAM or _PERSISTENT) and team size the next
 * hb_integrator_run uses; HB_ERR_TOO_LARGE / HB_ERR_INVALID when a forced
 * team engine cannot take this system. */
int hb_integrator_engine(hb_ctx *ctx, int *engine, int *team_ctas);
/* Integrate block steps on the device until the system time reaches tend
 * (a multiple of dtmax for a synchronised end state).  max_block_steps > 0
 * bounds the number of block steps of this call (HB_ERR_STATE when reached,
 * with the state consistent at the time reached); 0 = no bound. */
int hb_integrator_run(hb_ctx *ctx, double tend, long long max_block_steps);
/* Counters since hb_integrator_init: sum of nact over block steps, block
 * steps, and the current system time. */
int hb_integrator_stats(const hb_ctx *ctx, long long *particle_steps, long long *block_steps,
                        double *tsys);
/* Kinetic 0.5*sum m v^2 and potential 0.5*sum m phi of the records (the
 * reference's calc_energy, SRC/nbodysystem.h:633-650). */
int hb_energy(hb_ctx *ctx, double eps2, double *kinetic, double *potential);
/* Copy count records (and, if dt_out, their timesteps) from the device. */
int hb_get_records(hb_ctx *ctx, int addr0, int count, double *records_out, double *dt_out);

/* ---- checkpoints -----------------------------------------------------------
 * The reference's dump format (NbodySystem::dump / restore,
 * SRC/nbodysystem.h:405-446; Particle::dump / restore, SRC/hermite{4,6,8}.h):
 * a header (order, dumpid, nbody, tsys, initial and previous energy, particle
 * and block steps) and per particle id, mass, pos, vel, acc, jrk, snp, crk
 * [d4a d5a [d6a d7a]] in %A hex floats.  Files written here restore in the
 * reference's integrator and the reverse.
 *
 * Host-only helpers.  records: nbody j-particle records (tlast is not in a
 * dump; the reader sets it to tsys); aux: nbody x 6 doubles, the two vectors
 * beyond the record (snp crk at 4th order, d4a d5a at 6th, d6a d7a at 8th);
 * ids: nbody ids (null on write: the slot index; null on read: dropped). */
int hb_dump_write(const char *path, int order, int dumpid, int nbody, double tsys,
                  double init_energy, double prev_energy, long long steps, long long block_steps,
                  const long long *ids, const double *records, const double *aux);
int hb_dump_read_header(const char *path, int *order, int *dumpid, int *nbody, double *tsys,
                        double *init_energy, double *prev_energy, long long *steps,
                        long long *block_steps);
int hb_dump_read(const char *path, int order, int nbody, long long *ids, double *records,
                 double *aux);
/* Dump the device integrator's state.  Every particle must be at the block
 * time (tsys a multiple of dtmax), as in the reference's dump intervals. */
int hb_integrator_dump(hb_ctx *ctx, const char *path, int dumpid, double init_energy,
                       double prev_energy);
/* Restore a dump (order and N must match the context) and prepare the
 * integrator as the reference's restore + reinitialize_steps do
 * (SRC/nbodysystem.h:429-458): tlast = tsys for all, dt from recalc_dt(eta,
 * dtmax); the dumped forces are the corrector's previous forces, no force
 * evaluation.  Returns the dump id and the two energies. */
int hb_integrator_restore(hb_ctx *ctx, const char *path, double eps2, double eta, double dtmax,
                          int *dumpid, double *init_energy, double *prev_energy);

/* ---- snapshots -------------------------------------------------------------
 * The reference's snapshot text format (read_snapshot_masaki /
 * write_snapshot_masaki, SRC/nbodysystem.h:359-403): "%d\n%ld\n%f\n" (snapid,
 * nbody, time), then per particle id, mass, pos[3], vel[3], potential as
 * "%6ld    %A    %A %A %A    %A %A %A    %A".  Host only; the particle lines
 * are parsed and formatted on several host threads.  pos / vel: nbody x 3;
 * ids and pot may be null (write: slot index / 0). */
int hb_snapshot_read_header(const char *path, int *snapid, int *nbody, double *tsys);
int hb_snapshot_read(const char *path, int nbody, long long *ids, double *mass, double *pos,
                     double *vel, double *pot);
int hb_snapshot_write(const char *path, int snapid, int nbody, double tsys, const long long *ids,
                      const double *mass, const double *pos, const double *vel, const double *pot);

/* ---- batched ensembles ---------------------------------------------------
 * No reference counterpart (the reference integrates one system per
 * process).  Many independent clusters (any sizes, softenings, masses)
 * advanced together by one device-resident block-step loop over the union
 * of their particles; each particle interacts only with its own cluster.
 * All clusters share eta, eta_s and dtmax; each has its own eps2. */
typedef struct hb_ens hb_ens;
int hb_ens_create(int order, int nclusters, const int *sizes, int precision, hb_ens **out);
int hb_ens_destroy(hb_ens *ens);
const char *hb_ens_last_error(const hb_ens *ens);
/* Initial conditions of cluster c: sizes[c] j-particle records (pos, mass,
 * vel used; tlast and derivatives are reset by hb_ens_init) and its eps2. */
int hb_ens_set_cluster(hb_ens *ens, int c, const double *records, double eps2);
/* Current records (and dt) of cluster c. */
int hb_ens_get_cluster(hb_ens *ens, int c, double *records, double *dt_out);
/* Slot offset of cluster c in the ensemble's record array. */
int hb_ens_cluster_offset(const hb_ens *ens, int c);
/* init_step for every cluster (bootstrap forces, initial dt). */
int hb_ens_init(hb_ens *ens, double tsys, double eta, double eta_s, double dtmax);
/* Engines for hb_ens_run (HB_ENGINE_* as for hb_integrator_set_engine):
 *  HB_ENGINE_GRAPH  lockstep: one global block-step loop over the union of
 *                   all clusters, five kernels per step from a CUDA graph;
 *  HB_ENGINE_TEAM   every cluster that fits a team of up to 16 CTAs (about
 *                   33k particles at 6th order) on its own block-time
 *                   sequence: one thread-block cluster of team_ctas CTAs
 *                   (0: chosen per cluster from its size) integrates one
 *                   cluster at a time from a device queue, largest first
 *                   (FP64); the clusters that do not fit follow on the
 *                   lockstep engine;
 *  HB_ENGINE_AUTO   the team engine when every cluster fits a team with its
 *                   records in shared memory (about 11k particles at 6th
 *                   order), else the lockstep engine for all (the default).
 * Per cluster both engines integrate the same algorithm; a cluster's
 * result does not depend on the other clusters. */
int hb_ens_set_engine(hb_ens *ens, int engine, int team_ctas);
/* The engine (HB_ENGINE_TEAM / HB_ENGINE_GRAPH) and team size that
 * hb_ens_run uses for cluster c. */
int hb_ens_cluster_engine(hb_ens *ens, int c, int *engine, int *team_ctas);
/* Integrate all clusters until tend (max_block_steps as hb_integrator_run,
 * counted per cluster for the team engine). */
int hb_ens_run(hb_ens *ens, double tend, long long max_block_steps);
/* Sums over clusters since init: particle steps, block steps (each
 * cluster's own), the earliest cluster time, and interactions (sum over
 * block steps of nact_c * N_c). */
int hb_ens_stats(hb_ens *ens, long long *particle_steps, long long *block_steps,
                 double *tsys, double *interactions);
/* One cluster's particle steps, block steps and time. */
int hb_ens_cluster_stats(hb_ens *ens, int c, long long *particle_steps, long long *block_steps,
                         double *tsys);
/* Per-cluster kinetic and potential energy (arrays of nclusters). */
int hb_ens_energy(hb_ens *ens, double *kinetic, double *potential);

/* Measured peak of the FP32 (precision = HB_MIXED) or FP64 (HB_FP64) FMA
 * pipe on the current device, in GFLOP/s (2 flops per FMA), from a
 * register-resident FMA-chain kernel.  A roofline denominator for the force
 * kernels; no reference counterpart. */
int hb_measure_fma_peak(int precision, double *gflops);

/* ---- allocation-free force ---------------------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code inside a host framework that owns every device allocation through its
 * own pool (an allocation behind the pool's back breaks its accounting or
 * fails against its reservation), and fixed-budget jobs on a shared GPU that
 * must not grow their footprint after start-up.  hb_create allocates, so such
 * callers use this context-free entry point instead; it allocates nothing.
 *
 * Computes the force on slots [0,nact) from all nslots slots, like
 * hb_force_device, from predicted j-particles the caller already holds in
 * device memory, in the library's predicted layout ("AoSoA32": chunks of 32
 * slots, each chunk one 32-wide vector per component;
 *   HB_FP64:  x y z m vx vy vz [ax ay az] [jx jy jz]              (double)
 *   HB_MIXED: xh yh zh xl yl zl m vx vy vz [ax ay az] [jx jy jz]   (float,
 *             position = hi + lo)
 * with unused slots given zero mass at distinct far-away positions).  Writes
 * nact force records (3*(order/2) doubles each) to the device array `force`.
 * Asynchronous on `stream` (a cudaStream_t; NULL = the default stream).
 *
 * Limits: nslots a multiple of 256 and at most 1<<20 (HB_ERR_TOO_LARGE
 * beyond); larger nact get fewer j-slices, never a larger buffer.
 * Scratch: one file-scope device array of 4.125 MiB (4 MiB of j-slice
 * partial sums, 128 KiB of arrival counters) that every GPU loading the
 * library holds until the process exits.  The first call on each device (with
 * that device current) looks up that array's device address; make that first
 * call before any stream capture.  A lookup that fails returns HB_ERR_CUDA and
 * is tried again by the next call.  Every call shares the array and clears
 * the counters it uses on
 * its stream first; calls that overlap on the GPU (on different streams or
 * devices sharing a context) race on it and must be serialised by the caller.
 * A device-side wait that gives up is not reported by this entry point. */
int hb_force_predicted_noalloc(int order, int precision, const void *pred, int nslots,
                               int nact, double eps2, double *force, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HERMITE_B200_H */
