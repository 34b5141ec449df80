"""Benchmark of the Hermite force hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Headline workload: the 6th-order configuration of the metric -- Plummer
N = 262144, equal masses, Henon units, eps = 1/4096 -- in plain FP64, the
reference's own precision.  One "step" is one block step with every particle
active, the reference's "Init N square" step (SRC/nbodysystem.h:582-594):
predict_all over all N, then the force on all N (N^2 interactions, self pair
included, 97 flops each by the reference's convention, SRC/hermite6.h:22).
  value  -- Gint/s with inputs resident in HBM (predictor + force kernels),
            L2 flushed before every timed step.
  e2e    -- the same step through the C ABI with host buffers: set_jp of
            all N records, predict_all (host->device upload), force into host
            memory (device->host), all inside the timed region.
  mixed  -- the same step with the mixed-precision force kernel, its rate
            against the FP64 kernel's, and both precisions' force errors
            against the FP64 oracle on integrator states (4096 sampled i
            against all N).
Extra keys: the roofline of the force kernel against the FP64 FMA peak
measured in the same run; the reference's own AVX2 CPU Gravity (built from
its sources into oracle/_ref/) on a sample of the same step (set_jp and
predict_all of all N, the force on the first 8192 i against all N), repeated
for at least 10 s, as cpu_baseline; block-step times of the device-resident
integrator; the 8th-order configuration; batched ensembles; the force noise
of the mixed kernel against what the step criterion tolerates.

--impl reference times the reference's AVX2 Gravity (set_jp, predict_all,
calc_force_on_first_nact) on this host's cores on the same sample of the
step (K steps after W warm-up).  Under torchrun only rank 0 runs it.
--gpus N > 1 runs N independent replicas (the path does not shard across
GPUs in the reference; one process per GPU), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Gint/s & block-step time, mixed-prec vs FP64 kernel, 1 B200, at stated force/energy err"
UNIT = "Gint/s"
ORDER, N, EPS = 6, 262144, 1.0 / 4096
CPU_NACT = 8192            # i-particles of the CPU sample of the step
NSAMPLE = 4096             # i-particles of the accuracy sample
FLOPS = {4: 60, 6: 97, 8: 144}
L2_FLUSH_BYTES = 256 << 20


def workload_config(extra=None):
    cfg = {"workload": "Plummer N=262144 equal-mass Henon units, eps=1/4096, 6th-order Hermite, "
                       "plain FP64; one step = predict_all + force on all N (full block step)",
           "order": ORDER, "nbody": N, "nact": N, "eps": EPS, "precision": "fp64",
           "flops_per_interaction": FLOPS[ORDER], "l2": "flushed (256 MiB write) before each step",
           "parallelism": "replicas"}
    if extra:
        cfg.update(extra)
    return cfg


def plummer_records(order, n, seed=0):
    from hermite_b200.ic import plummer, records
    return records(plummer(n, seed), order)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
def host_threads() -> int:
    """CPUs this process may run on (libgomp's default team size)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_force_rate(order, n, nact, threads, rec=None, min_s=10.0, min_reps=3, max_reps=200):
    """The reference's AVX2 Gravity (oracle/_ref) on this host: Gint/s of
    set_jp of all n + predict_all + force on the first nact against all n,
    repeated until min_s seconds (at least min_reps, at most max_reps steps)
    after one warm-up."""
    from oracle import RefGravity
    os.environ["OMP_NUM_THREADS"] = str(threads)
    if rec is None:
        rec = plummer_records(order, n)
    g = RefGravity(order, n, "avx")
    eps2 = EPS * EPS
    g.set_jp_all(rec)
    g.predict_all(0.0)
    g.force(nact, eps2)                     # warm-up
    times = []
    while len(times) < max_reps and (len(times) < min_reps or sum(times) < min_s):
        t0 = time.perf_counter()
        g.set_jp_all(rec)
        g.predict_all(0.0)
        g.force(nact, eps2)
        times.append(time.perf_counter() - t0)
    g.close()
    return nact * n / (sum(times) / len(times)) * 1e-9, times


def cpu_sample_text(steps, extra=""):
    return (f"set_jp + predict_all of all {N} particles, force on the first {CPU_NACT} i "
            f"against all {N} j ({CPU_NACT * N:.3g} interactions per step), {steps} steps{extra}")


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = host_threads()
    from oracle import ref_available
    if not ref_available("avx", ORDER):
        print(json.dumps({"impl": "reference", "unavailable":
                          f"oracle/_ref/libref_avx{ORDER}.so not built (needs the reference sources)"}))
        return
    rec = plummer_records(ORDER, N)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import RefGravity
    g = RefGravity(ORDER, N, "avx")
    eps2 = EPS * EPS
    for _ in range(args.warmup):
        g.set_jp_all(rec)
        g.predict_all(0.0)
        g.force(CPU_NACT, eps2)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        g.set_jp_all(rec)
        g.predict_all(0.0)
        g.force(CPU_NACT, eps2)
    dt = time.perf_counter() - t0
    g.close()
    value = CPU_NACT * N * args.steps / dt * 1e-9
    sample = cpu_sample_text(args.steps, f" after {args.warmup} warm-up")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config({"impl": "reference AVX2 Gravity "
                                                        "(SRC/hermite6-avx.h) on host cores",
                                                        "nact_sampled": CPU_NACT}),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ---------------------------------------------------------------------------
def traffic_from_profiles(name):
    """dram bytes per force-kernel launch from a committed ncu summary."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1])
            except ValueError:
                return None
    return None


def tiled_shape(order, n, nact):
    """The tiled force kernel's shape (variant, j-slices) that the library
    takes from its tuning table for (order, FP64, n, nact): the nearest N
    bucket, then the nearest nact bucket, the slice count rescaled to the
    bucket's CTA count (hb_capi.cu, pick_variant)."""
    import ctypes
    import math
    from hermite_b200 import load_library
    best = None
    for line in (ROOT / "hermite_b200" / "csrc" / "hb_tuning.inc").read_text().splitlines():
        if not line.startswith("{"):
            continue
        o, m, ln, la, v, sp = (int(x) for x in line.strip("{},").split(","))
        if o != order or m != 0:
            continue
        key = (abs(ln - math.log2(n)), abs(la - math.log2(nact)))
        if best is None or key < best[0]:
            best = (key, la, v, sp)
    _, la, v, sp = best
    th, ni, wj = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    load_library().hb_force_variant_info(order, 0, v, ctypes.byref(th), ctypes.byref(ni), ctypes.byref(wj))
    ti = th.value // (32 * wj.value) * 32 * ni.value
    gx_bucket, gx = -(-(1 << la) // ti), -(-nact // ti)
    return v, max(1, -(-(gx_bucket * sp) // gx))


def timed_steps(g, stream, flush, steps, eps2, t0=0.0):
    """CUDA-event times (ms) of `steps` device-resident steps: L2 flush,
    predict_all to a new time, force on all N."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.zero_()
        e0, e1, e2 = ev[k]
        e0.record(stream)
        g.predict_all_device(t0 + 1e-6 * (k + 1))
        e1.record(stream)
        g.force_device(N, eps2)
        e2.record(stream)
    stream.synchronize()
    return ([a.elapsed_time(c) for a, b, c in ev], [a.elapsed_time(b) for a, b, c in ev],
            [b.elapsed_time(c) for a, b, c in ev])


def run_ours(args):
    import torch
    from hermite_b200 import Gravity, measure_fma_peak

    world, rank, local = dist_setup(args)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    rec = plummer_records(ORDER, N, seed=rank)
    eps2 = EPS * EPS
    nint = float(N) * N
    F = 3 * (ORDER // 2)

    with torch.cuda.stream(stream):
        g = Gravity(ORDER, N, "fp64")
        g.set_stream(stream.cuda_stream)
        g.set_jp_records(rec)
        g.upload()
        for _ in range(args.warmup):
            g.predict_all_device(0.0)
            g.force_device(N, eps2)
        stream.synchronize()

        # ---- device-resident timed region ----
        l0 = g.launch_count()
        dist_barrier(world)
        torch.cuda.synchronize(dev)
        with ClockSampler(local) as clk:
            step_ms, pred_ms, force_ms = timed_steps(g, stream, flush, args.steps, eps2)
            torch.cuda.synchronize(dev)
        dist_barrier(world)
        launches = g.launch_count() - l0
        total_ms = dist_max(sum(step_ms), world)
        value = nint * args.steps * world / (total_ms * 1e-3) * 1e-9

        # ---- end to end through the C ABI with host buffers ----
        out = np.empty((N, F))
        g.set_stream(None)
        for _ in range(2):
            g.set_jp_records(rec)
            g.predict_all(0.0)
            g.calc_force_on_first_nact(N, eps2, out)
        dist_barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            g.set_jp_records(rec)
            g.predict_all(0.0)
            g.calc_force_on_first_nact(N, eps2, out)
        e2e_s = dist_max(time.perf_counter() - t0, world)
        e2e = nint * args.steps * world / e2e_s * 1e-9

        # ---- block-step latency through the C ABI (set_jp + predict_all + force) ----
        def block_step_us(nact, reps):
            buf = np.empty((nact, F))
            for _ in range(3):
                g.predict_all(0.0)
                g.calc_force_on_first_nact(nact, eps2, buf)
            times = []
            for _ in range(reps):
                t0 = time.perf_counter()
                g.set_jp_records(rec[:nact])
                g.predict_all(0.0)
                g.calc_force_on_first_nact(nact, eps2, buf)
                times.append(time.perf_counter() - t0)
            return statistics.median(times) * 1e6
        block_us = {str(nact): block_step_us(nact, 200 if nact <= 8192 else 5)
                    for nact in (1, 4, 16, 32, 1024, 8192, 65536)}
        # the same small steps on the tiled kernel (the tuning table's shape),
        # against the lane-split kernel the automatic choice takes
        block_us_tiled = {}
        for nact in (1, 4, 16):
            v, S = tiled_shape(ORDER, N, nact)
            g.set_force_shape(v, S)
            block_us_tiled[str(nact)] = block_step_us(nact, 200)
        g.set_force_shape(-1, 0)
        g.close()

        # ---- the same step with the mixed-precision kernel ----
        gm = Gravity(ORDER, N, "mixed")
        gm.set_stream(stream.cuda_stream)
        gm.set_jp_records(rec)
        gm.upload()
        for _ in range(args.warmup):
            gm.predict_all_device(0.0)
            gm.force_device(N, eps2)
        stream.synchronize()
        mstep_ms, mpred_ms, mforce_ms = timed_steps(gm, stream, flush, args.steps, eps2)
        gm.close()

    fp64_peak = measure_fma_peak(0)      # GFLOP/s, same device, same run
    fp32_peak = measure_fma_peak(2)
    force_avg_ms = sum(force_ms) / len(force_ms)
    achieved = nint * FLOPS[ORDER] / (force_avg_ms * 1e-3) * 1e-12
    mforce_avg_ms = sum(mforce_ms) / len(mforce_ms)
    machieved = nint * FLOPS[ORDER] / (mforce_avg_ms * 1e-3) * 1e-12
    mvalue = nint * args.steps / (sum(mstep_ms) * 1e-3) * 1e-9
    traffic = traffic_from_profiles("force_fp64_o6_n262144.txt")
    mtraffic = traffic_from_profiles("force_mixed_o6_n262144.txt")

    # the accuracy, 8th-order, integrator, ensemble and CPU legs run on
    # single-GPU runs only (replicas add nothing to them)
    skip_mixed = args.skip_mixed or world > 1
    skip_integrator = args.skip_integrator or world > 1
    accuracy = accuracy_leg("c3") if not skip_mixed else None
    mixed = {
        "value": mvalue, "unit": UNIT, "ms_per_step": sum(mstep_ms) / args.steps,
        "speedup_vs_fp64": mvalue / value * world, "force_ms": mforce_avg_ms,
        "force_speedup_vs_fp64": force_avg_ms / mforce_avg_ms,
        "kernel_ms": {"predict": sum(mpred_ms) / len(mpred_ms), "force": mforce_avg_ms},
        "roofline": {"bound": "fp32", "achieved": machieved, "peak": fp32_peak * 1e-3,
                     "unit": "TFLOP/s", "frac": machieved / (fp32_peak * 1e-3), "traffic": mtraffic,
                     "kernel": "hb::force_kernel<6, MIXED>",
                     "peak_source": "packed-FP32 (f32x2) FMA-chain kernel measured in this run"},
        "force_error_vs_oracle": accuracy,
    }
    c4 = config_c4_leg() if not skip_mixed else None
    noise = noise_leg(accuracy) if not skip_mixed else None
    integ = device_integrator_leg() if not skip_integrator else None
    mixed_int = mixed_integration_leg() if not skip_integrator else None
    ref_gpu = reference_gpu_leg() if not skip_integrator else None
    ens = ensemble_leg() if not skip_integrator else None
    ens_small = small_ensemble_leg() if not skip_integrator else None
    pred = predictor_leg() if not skip_mixed else None

    if rank != 0:
        dist_barrier(world)
        return
    cpu = None
    if not args.skip_cpu and world == 1:
        try:
            from oracle import ref_available
            if ref_available("avx", ORDER):
                threads = host_threads()
                rate, times = reference_force_rate(ORDER, N, CPU_NACT, threads, rec)
                cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                       "sample": "reference AVX2 Gravity (SRC/hermite6-avx.h, built from source): "
                                 + cpu_sample_text(len(times), f", {sum(times):.1f} s total")}
        except Exception as e:          # the baseline is reported, not required
            cpu = {"value": None, "unit": UNIT, "cores": host_threads(), "kind": "reference",
                   "sample": f"failed: {e}"}
    ens_cpu = None
    if not args.skip_cpu and not skip_integrator:
        try:
            ens_cpu = ensemble_cpu_leg()
        except Exception as e:
            ens_cpu = {"failed": str(e)}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": N * (8 + 3 * (ORDER - 2)) * 8,
                "d2h_bytes_per_step": N * F * 8},
        "gpu_launches": launches,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak * 1e-3,
                     "unit": "TFLOP/s", "frac": achieved / (fp64_peak * 1e-3), "traffic": traffic,
                     "kernel": "hb::force_kernel<6, FP64>",
                     "peak_source": "FP64 FMA-chain kernel measured in this run "
                                    "(hb_measure_fma_peak); MEASURED_PEAKS.json has no FP64 figure",
                     "achieved_basis": f"N^2 x {FLOPS[ORDER]} flops per launch / mean CUDA-event "
                                       "duration of the force launch"},
        "kernel_ms": {"predict": sum(pred_ms) / len(pred_ms), "force": force_avg_ms},
        "fp32_peak_tflops": fp32_peak * 1e-3,
        "mixed": mixed,
        "block_step_us": {"order": ORDER, "nbody": N, "precision": "fp64",
                          "through": "set_jp(nact) + predict_all + calc_force_on_first_nact "
                                     "(Python ctypes calls; median of 200)",
                          "us": block_us, "us_tiled_kernel": block_us_tiled},
        "config_c4": c4,
        "mixed_force_noise": noise,
        "device_integrator": integ,
        "mixed_integration": mixed_int,
        "reference_gpu_recompiled": ref_gpu,
        "ensemble": ens,
        "ensemble_small_clusters": ens_small,
        "predictor_roofline": pred,
        "ensemble_cpu_reference": ens_cpu,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))
    dist_barrier(world)


# ---------------------------------------------------------------------------
STATE_CONFIGS = {
    # name -> (order, N, eps, eta, eta_s, dtmax, t_run)
    "c1": (4, 1024, 1 / 256, 0.01, 0.0025, 1 / 8, 1 / 8),
    "c3": (6, 262144, 1 / 4096, 0.1, 0.02, 1 / 32, 1 / 1024),
    "c4": (8, 1 << 20, 1 / 16384, 0.2, 0.04, 1 / 64, 1 / 4096),
}


def integrator_state(name):
    """Records (slot order), time and eps2 of the FP64 device integrator after
    its start-up and a short run: realistic acc/jrk/snp/crk and tlast."""
    from hermite_b200 import Gravity
    from hermite_b200.ic import plummer, records
    order, n, eps, eta, eta_s, dtmax, t_run = STATE_CONFIGS[name]
    with Gravity(order, n, "fp64") as g:
        g.set_jp_records(records(plummer(n, 0), order))
        g.integrator_init(0.0, eps * eps, eta, eta_s, dtmax)
        g.integrator_run(t_run)
        t = g.integrator_stats()[2]
        rec = g.get_records()
    return rec, t, eps * eps


def error_stats(got, ref):
    a = got.reshape(got.shape[0], -1, 3)
    b = ref.reshape(ref.shape[0], -1, 3)
    err = np.linalg.norm(a - b, axis=2) / np.linalg.norm(b, axis=2)
    names = ("acc", "jrk", "snp", "crk")[:err.shape[1]]
    return {nm: {"max": float(err[:, k].max()), "p99": float(np.quantile(err[:, k], 0.99)),
                 "median": float(np.median(err[:, k]))} for k, nm in enumerate(names)}


def accuracy_leg(name, nsample=NSAMPLE):
    """Per-derivative relative force errors of both precisions against the
    FP64 oracle (oracle/hermite_oracle.c, all host cores), on the first
    nsample slots of a random permutation of an integrator state, each
    against all N, predicted to the integrator's time."""
    from hermite_b200 import Gravity
    from oracle import Oracle
    order = STATE_CONFIGS[name][0]
    rec, t, eps2 = integrator_state(name)
    n = rec.shape[0]
    rng = np.random.default_rng(1)
    pick = rng.choice(n, size=nsample, replace=False)
    recp = np.ascontiguousarray(rec[np.concatenate([pick, np.setdiff1d(np.arange(n), pick)])])
    t0 = time.perf_counter()
    ref = Oracle().predict_force(order, recp, t, nsample, eps2)
    oracle_s = time.perf_counter() - t0
    out = {"config": name, "order": order, "nbody": n, "t": t, "sample_i": nsample,
           "state": "FP64 device integrator after start-up and a run to t",
           "oracle_s": oracle_s}
    for prec in ("fp64", "mixed"):
        with Gravity(order, n, prec) as g:
            g.set_jp_records(recp)
            g.predict_all(t)
            out[prec] = error_stats(g.calc_force_on_first_nact(nsample, eps2), ref)
    return out


def config_c4_leg(nrate=32768):
    """8th order, Plummer N = 2^20, eps = 1/16384 (the 8th-order
    configuration): both kernels' rates on the first nrate i against all N,
    and both precisions' errors against the oracle on an integrator state."""
    import torch
    from hermite_b200 import Gravity
    order, n, eps2 = 8, 1 << 20, (1.0 / 16384) ** 2
    rec = plummer_records(order, n, seed=11)
    res = {"order": order, "nbody": n, "eps": 1.0 / 16384, "rate_i": nrate}
    stream = torch.cuda.Stream()
    for prec in ("fp64", "mixed"):
        with torch.cuda.stream(stream):
            g = Gravity(order, n, prec)
            g.set_stream(stream.cuda_stream)
            g.set_jp_records(rec)
            g.upload()
            g.predict_all_device(0.0)
            g.force_device(nrate, eps2)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(2):
                g.force_device(nrate, eps2)
            e1.record(stream)
            stream.synchronize()
            ms = e0.elapsed_time(e1) / 2
            g.close()
        res[prec] = {"gint_s": nrate * n / (ms * 1e-3) * 1e-9, "force_ms": ms}
    res["speedup"] = res["mixed"]["gint_s"] / res["fp64"]["gint_s"]
    res["force_error_vs_oracle"] = accuracy_leg("c4")
    return res


def noise_leg(c3_accuracy):
    """The mixed kernel's force deviation from the FP64 kernel on the same
    predicted states, next to the force noise the reference's step criterion
    tolerates (measured on the CPU by tests/test_noise_tolerance.py: white
    noise of that relative size per derivative leaves the block steps within
    10 %; ten times more blows them up).  c1: all 1024 particles of the
    4th-order configuration after t = 1/8; c3: the accuracy sample."""
    from hermite_b200 import Gravity
    rec, t, eps2 = integrator_state("c1")
    n = rec.shape[0]
    f = {}
    for prec in ("fp64", "mixed"):
        with Gravity(4, n, prec) as g:
            g.set_jp_records(rec)
            g.predict_all(t)
            f[prec] = g.calc_force_on_first_nact(n, eps2)
    return {
        "c1_mixed_vs_fp64": error_stats(f["mixed"], f["fp64"]),
        "c3_mixed_vs_oracle": c3_accuracy["mixed"] if c3_accuracy else None,
        "tolerated_relative_noise": {
            "4th order, eta=0.01 (c1)": 1e-9, "4th order, eta=0.1 (RUN/inp.4th)": 1e-6,
            "6th order, eta=0.1 (c3 parameters, N=4096)": 1e-11},
        "source": "tests/test_noise_tolerance.py (reference integrator on the CPU, seeded "
                  "relative noise on the oracle's forces)"}


def mixed_integration_leg():
    """4th order at the reference's own run parameters (RUN/inp.4th: eta =
    0.1, eta_s = 0.01, dtmax = 1/16), Plummer N = 1024 and 65536 (eps = 4/N),
    t = 0..1/4 on the graph engine, FP64 and mixed forces: block steps,
    particle steps, time per block step and the energy error."""
    from hermite_b200 import Gravity
    from hermite_b200.ic import plummer, records
    out = {}
    for n in (1024, 65536):
        eps2 = (4.0 / n) ** 2
        rec = records(plummer(n, 0), 4)
        for prec in ("fp64", "mixed"):
            with Gravity(4, n, prec) as g:
                g.set_engine("graph")
                g.set_jp_records(rec)
                g.integrator_init(0.0, eps2, 0.1, 0.01, 1.0 / 16)
                ke0, pe0 = g.energy(eps2)
                t0 = time.perf_counter()
                g.integrator_run(0.25)
                wall = time.perf_counter() - t0
                ps, bs, _ = g.integrator_stats()
                ke, pe = g.energy(eps2)
            e0 = ke0 + pe0
            out[f"n{n}_{prec}"] = {"block_steps": bs, "particle_steps": ps,
                                   "us_per_block": wall / max(bs, 1) * 1e6,
                                   "gint_s": ps * n / wall * 1e-9,
                                   "de_global": (e0 - (ke + pe)) / e0}
    return out


def hbm_peak():
    """Measured HBM copy bandwidth of this pool's B200s (GB/s), else the
    earlier measurement on the same pool."""
    p = Path(__file__).resolve().parent / "MEASURED_PEAKS.json"
    try:
        v = json.loads(p.read_text()).get("hbm_gbs")
        if v:
            return float(v), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, ValueError):
        pass
    return 6650.0, "fallback (6.65 TB/s, earlier copy measurement on this pool)"


def predictor_leg(reps=50):
    """The predictor pass alone (hb_predict_pass), plain FP64, back to back:
    algorithmic bytes = N x (record read + predicted state written) =
    168 / 312 B per slot at 4th / 8th order, over the mean CUDA-event time of
    one pass.  8th order, N = 2^20 moves 327 MB per pass (above L2: HBM
    bound); 4th order, N = 65536 moves 11 MB (L2 resident, launch bound)."""
    import torch
    from hermite_b200 import Gravity
    peak, src = hbm_peak()
    out = {"peak_gb_s": peak, "peak_source": src}
    stream = torch.cuda.Stream()
    for order, n in ((4, 1 << 16), (8, 1 << 20)):
        rec = plummer_records(order, n, seed=3)
        with torch.cuda.stream(stream):
            g = Gravity(order, n, "fp64")
            g.set_stream(stream.cuda_stream)
            g.set_jp_records(rec)
            g.upload()
            g.predict_all_device(1e-3)
            for _ in range(3):
                g.predict_pass()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                g.predict_pass()
            e1.record(stream)
            stream.synchronize()
            us = e0.elapsed_time(e1) / reps * 1e3
            g.set_stream(None)
            g.close()
        nbytes = n * 8 * ({4: 14, 6: 20, 8: 26}[order] + {4: 7, 6: 10, 8: 13}[order])
        gbs = nbytes / (us * 1e-6) * 1e-9
        out[f"order{order}_n{n}"] = {"bytes_per_pass": nbytes, "us_per_pass": us, "gb_s": gbs,
                                     "frac": gbs / peak}
    return out


def ensemble_cpu_leg(nclusters=256, tend=1.0 / 16):
    """The reference's AVX2 integrator (oracle/_ref/avx2-6, all host cores) on
    a sample of the ensemble leg's clusters -- the smallest, median and
    largest whose N is a multiple of 4 (the AVX backend works on groups of
    4) -- over t = 0..tend (one dtmax, the app's shortest run):
    interactions per second of each run and of the sample (the CPU
    counterpart of the ensemble's Gint/s)."""
    from hermite_b200.ic import plummer, power_law_masses
    from run_app import APP, run
    if not Path(str(APP["cpu-ref"]).format(order=6)).exists():
        return None
    rng = np.random.default_rng(2024)
    sizes = [int(round(np.exp(rng.uniform(np.log(1024), np.log(32768))))) for _ in range(nclusters)]
    by4 = [int(c) for c in np.argsort(sizes) if sizes[c] % 4 == 0]
    pick = [by4[0], by4[len(by4) // 2], by4[-1]]
    runs, inter, wall = [], 0.0, 0.0
    for c in pick:
        n = sizes[c]
        snap = plummer(n, seed=c, masses=power_law_masses(n, np.random.default_rng(c)))
        r = run("c5", "cpu-ref", tend=tend, snapshot=snap, eps=4.0 / n)
        i = float(r["particle_steps"]) * n
        runs.append({"cluster": c, "n": n, "app_wtime_s": r.get("app_wtime_s"),
                     "gint_s": i / r["app_wtime_s"] * 1e-9 if r.get("app_wtime_s") else None})
        inter += i
        wall += r.get("app_wtime_s") or 0.0
    return {"binary": "oracle/_ref/avx2-6 (reference SRC/hermite6-avx.h, built from source)",
            "cores": os.cpu_count(), "window": f"t = 0..{tend}", "clusters": runs,
            "gint_s": inter / wall * 1e-9 if wall else None}


PROFILE_CASES = {
    # name -> (order, precision, N)
    "fp64_o6_c3": (6, "fp64", 262144), "mixed_o6_c3": (6, "mixed", 262144),
    "fp64_o4": (4, "fp64", 65536), "mixed_o6": (6, "mixed", 65536),
    "fp64_o6": (6, "fp64", 65536), "mixed_o8": (8, "mixed", 65536),
}


def run_profile_case(case: str):
    """One predict + two force launches on all N, for ncu captures:
    fp64_o6_c3 / mixed_o6_c3 = the headline force kernel and its mixed
    counterpart (6th order, N = 262144: 42 MB of records, 0.1-0.25 s per
    launch); the others at N = 65536; team_c1 = one team-kernel launch on c1
    (N = 1024, 16 CTAs, t = 0..1/128); ensemble_window = the ensemble leg's
    256 clusters on the lockstep engine, t = 0..1/128; lanes_o6_c3 = three
    block steps of one active particle at N = 262144 (the small-step kernel)."""
    from hermite_b200 import Gravity
    if case == "lanes_o6_c3":
        # the small-step kernel: nact = 1 against N = 262144 (6th order, FP64)
        g = Gravity(6, 262144, "fp64")
        g.set_jp_records(plummer_records(6, 262144))
        out = np.empty((1, 9))
        for k in range(3):
            g.predict_all(1e-6 * k)
            g.calc_force_on_first_nact(1, EPS * EPS, out)
        g.close()
        print("profile case lanes_o6_c3 done")
        return
    if case == "ensemble_window":
        print("profile case ensemble_window done", json.dumps(ensemble_leg(tend=1.0 / 128)))
        return
    if case == "team_c1":
        from hermite_b200.ic import plummer, records
        with Gravity(4, 1024, "fp64") as g:
            g.set_engine("team", 16)
            g.set_jp_records(records(plummer(1024, 0), 4))
            g.integrator_init(0.0, (1.0 / 256) ** 2, 0.01, 0.0025, 1.0 / 8)
            g.integrator_run(1.0 / 128)
            print("profile case team_c1 done", g.integrator_stats())
        return
    order, prec, n = PROFILE_CASES[case]
    g = Gravity(order, n, prec)
    g.set_jp_records(plummer_records(order, n))
    g.predict_all(0.0)
    for _ in range(2):
        g.force_device(n, EPS * EPS)
    g.synchronize()
    g.close()
    print(f"profile case {case} done")


def device_integrator_leg(configs=("c1", "c2", "c3")):
    """Block-step time of the device-resident integrator (corrector and
    scheduler on the GPU) on the configurations c1, c2 and c3 of run_app.py,
    plain FP64 (at c1/c2's eta = 0.01 and at 6th order the step criterion
    tolerates far less force noise than the mixed kernel leaves): wall time
    per block step, particle steps x N / time, and the energy error.  c1
    (N = 1024) runs on both engines: "team" (one thread-block cluster, the
    whole loop in one kernel; the automatic choice at this N) and "graph"
    (four phases, five kernels, per step over the whole GPU, 32 steps per CUDA-graph
    replay; the automatic choice for c2 and c3) and "persistent" (the same
    phases in one cooperative kernel, grid barriers between them).  c2 and c3
    run windows (t = 0..1/64 and 0..1/32)."""
    from hermite_b200 import Gravity
    from hermite_b200.ic import plummer, records
    from run_app import CONFIGS
    out = {}
    for name in configs:
        cfg = dict(CONFIGS[name])
        if name in ("c2", "c3"):
            # windows of the runs (c3: the reference CUDA leg's window)
            cfg["tend"] = 1.0 / 64 if name == "c2" else 1.0 / 32
        order, n = cfg["order"], cfg["n"]
        eps2 = cfg["eps"] ** 2
        engines = ("team", "graph", "persistent") if name == "c1" else ("graph", "persistent")
        for eng in engines:
            prec = "fp64"
            with Gravity(order, n, prec) as g:
                g.set_engine(eng)
                used = g.engine()
                g.set_jp_records(records(plummer(n, 0), order))
                g.integrator_init(0.0, eps2, cfg["eta"], cfg["eta_s"], 1.0 / cfg["dtmaxinv"])
                ke0, pe0 = g.energy(eps2)
                t0 = time.perf_counter()
                g.integrator_run(cfg["tend"], max_block_steps=2_000_000)
                wall = time.perf_counter() - t0
                ps, bs, t = g.integrator_stats()
                ke, pe = g.energy(eps2)
            e0 = ke0 + pe0
            key = f"{name}_{prec}_{used[0]}"
            out[key] = {
                "engine": used[0], "team_ctas": used[1],
                "order": order, "n": n, "tend": cfg["tend"], "block_steps": bs,
                "particle_steps": ps, "nact_mean": ps / max(bs, 1), "wall_s": wall,
                "us_per_block": wall / max(bs, 1) * 1e6, "gint_s": ps * n / wall * 1e-9,
                "de_global": (e0 - (ke + pe)) / e0}
    return out


def small_ensemble_leg(nclusters=256, tend=1.0 / 16):
    """256 clusters with N log-uniform in [256, 4096] (otherwise as the
    ensemble leg: power-law masses, eps = 4/N, 6th order FP64, eta = 0.1,
    dtmax = 1/16), t = 0..tend, on the lockstep engine and on the team
    engine (every cluster on its own block steps): wall time, Gint/s and the
    per-cluster block steps summed (equal on both engines)."""
    from hermite_b200 import Ensemble
    from hermite_b200.ic import plummer, power_law_masses, records
    rng = np.random.default_rng(2024)
    sizes = [int(round(np.exp(rng.uniform(np.log(256), np.log(4096))))) for _ in range(nclusters)]
    recs = [records(plummer(n, seed=c, masses=power_law_masses(n, np.random.default_rng(c))), 6)
            for c, n in enumerate(sizes)]
    out = {"clusters": nclusters, "n_total": int(sum(sizes)), "order": 6, "precision": "fp64",
           "eta": 0.1, "dtmax": 1.0 / 16, "tend": tend}
    for eng in ("graph", "team"):
        with Ensemble(6, sizes, "fp64") as ens:
            ens.set_engine(eng)
            for c, n in enumerate(sizes):
                ens.set_cluster(c, recs[c], (4.0 / n) ** 2)
            ens.init(0.0, 0.1, 0.02, 1.0 / 16)
            t0 = time.perf_counter()
            ens.run(tend, max_block_steps=400_000)
            wall = time.perf_counter() - t0
            ps, bs, t, inter = ens.stats()
        out["lockstep" if eng == "graph" else "team"] = {
            "wall_s": wall, "gint_s": inter / wall * 1e-9, "particle_steps": ps,
            "cluster_block_steps": bs}
    out["team_speedup"] = out["lockstep"]["wall_s"] / out["team"]["wall_s"]
    return out


def ensemble_leg(nclusters=256, tend=1.0 / 16, precision="fp64"):
    """Batched ensemble: 256 clusters with seeds 0..255, N
    log-uniform in [1024, 32768], power-law masses (slope -2.35 on [0.1, 100],
    total 1), eps = 4/N each, 6th order, eta = 0.1 (eta_s = eta/5),
    dtmax = 1/16, integrated by one device-resident loop; window
    t = 0..tend.  Interactions = sum over block steps and clusters of
    nact_c * N_c.  FP64: with mixed-precision forces the 6th-order
    corrector's Aarseth steps collapse at this eta (FP32 rounding noise
    amplified by its h^-3..h^-5 interpolation factors)."""
    from hermite_b200 import Ensemble
    from hermite_b200.ic import plummer, power_law_masses, records
    rng = np.random.default_rng(2024)
    sizes = [int(round(np.exp(rng.uniform(np.log(1024), np.log(32768))))) for _ in range(nclusters)]
    out = {"clusters": nclusters, "n_total": int(sum(sizes)), "order": 6, "precision": precision,
           "eta": 0.1, "eta_s": 0.02, "dtmax": 1.0 / 16, "tend": tend}
    with Ensemble(6, sizes, precision) as ens:
        engine = ens.cluster_engine(0)[0]    # clusters above ~11k fit no team: lockstep
        for c, n in enumerate(sizes):
            r = np.random.default_rng(c)
            snap = plummer(n, seed=c, masses=power_law_masses(n, r))
            ens.set_cluster(c, records(snap, 6), (4.0 / n) ** 2)
        ens.init(0.0, 0.1, 0.02, 1.0 / 16)
        ke0, pe0 = ens.energy()
        t0 = time.perf_counter()
        ens.run(tend, max_block_steps=400_000)
        wall = time.perf_counter() - t0
        ps, bs, t, inter = ens.stats()
        ke1, pe1 = ens.energy()
    de = (ke0 + pe0 - ke1 - pe1) / (ke0 + pe0)
    out.update({"engine": "lockstep" if engine == "graph" else "team", "wall_s": wall,
                "cluster_block_steps": bs, "particle_steps": ps, "gint_s": inter / wall * 1e-9,
                "de_global_max_abs": float(np.max(np.abs(de))),
                "de_global_median_abs": float(np.median(np.abs(de)))})
    return out


def reference_gpu_leg():
    """The reference's own FP64 CUDA force path (SRC/hermite6-titan.cu, written
    for sm_35) recompiled unmodified for sm_100a (oracle/_ref/titan-6), on the
    headline configuration: its own "## Init N square" report of one full
    N^2 force evaluation at N = 262144, and its app-level block-step rate over
    the window t = 0..1/32 of configuration c3."""
    from run_app import APP, run
    if not Path(str(APP["ref-gpu"]).format(order=6)).exists():
        return None
    r = run("c3", "ref-gpu", tend=1.0 / 32)
    return {"binary": "oracle/_ref/titan-6 (reference SRC/hermite6-titan.cu, sm_100a)",
            "init_n2_gint_s": r["init_n2_gflops"] / FLOPS[ORDER] if r["init_n2_gflops"] else None,
            "app_us_per_block": r.get("us_per_block"), "app_gint_s": r.get("app_gint_s"),
            "block_steps": r.get("block_steps"), "de_global": r.get("de_global"),
            "window": "c3 (N=262144, eps=1/4096, eta=0.1) t = 0..1/32"}


def main():
    ap = argparse.ArgumentParser(description="Hermite force hot-path benchmark")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--skip-cpu", action="store_true", help="omit the cpu_baseline leg")
    ap.add_argument("--skip-mixed", action="store_true",
                    help="omit the accuracy, 8th-order, noise and predictor legs")
    ap.add_argument("--skip-integrator", action="store_true",
                    help="omit the device-integrator block-step leg")
    ap.add_argument("--profile", choices=(*PROFILE_CASES, "team_c1", "ensemble_window", "lanes_o6_c3"),
                    help="run one case for an ncu capture and exit")
    args = ap.parse_args()
    if args.profile:
        run_profile_case(args.profile)
        return
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
