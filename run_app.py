"""Run the reference's own integrator on one of the benchmark configurations.

The integrator is the reference's SRC/compile.cpp + SRC/nbodysystem.h built
unmodified against the drop-in Gravity (hermite_b200/gravity/_build/
hb-app-{4,6,8}, this library, FP64 or mixed), or -- for the CPU comparison --
the reference's AVX2 build (oracle/_ref/avx2-{4,6,8}).  The run's own
reports are parsed:
  "## nbody wtime Gflops wtime/block(usec) nact"   (SRC/nbodysystem.h:146-150)
  " de(local/global) : ..."                         (SRC/nbodysystem.h:948-951)
  "ke = .., pe = .., e = .."                        (SRC/nbodysystem.h:644-647)

    python run_app.py --config c1 [--impl gpu|gpu-mixed|gpu-fast|cpu-ref|ref-gpu|
                                         device|device-mixed] [--tend T] [--n N]

--impl device[-mixed] runs the configuration on the library's device-resident
integrator instead of the reference's host loop.

Configurations (Plummer spheres from hermite_b200.ic, seed 0, equal masses,
G = M = 1, gen-plum's scaling E ~ -1/4):
  c1: 4th, N=1024,    eps=1/256,   eta=0.01, eta_s=0.0025, dtmax=1/8,  t 0->1
  c2: 4th, N=65536,   eps=1/1024,  eta=0.01, eta_s=0.0025, dtmax=1/16, t 0->0.25
  c3: 6th, N=262144,  eps=1/4096,  eta=0.1,  eta_s=0.02,   dtmax=1/32, t 0->0.125
  c4: 8th, N=1048576, eps=1/16384, eta=0.2,  eta_s=0.04,   dtmax=1/64, t 0->1/32
eta_s is not given for c2-c4; the ratios of RUN/inp.4th-style c1 (1/4) and
RUN/inp.6th (1/5) are used.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CONFIGS = {
    "c1": dict(order=4, n=1024, eps=1 / 256, eta=0.01, eta_s=0.0025, dtmaxinv=8, tend=1.0),
    "c2": dict(order=4, n=65536, eps=1 / 1024, eta=0.01, eta_s=0.0025, dtmaxinv=16, tend=0.25),
    "c3": dict(order=6, n=262144, eps=1 / 4096, eta=0.1, eta_s=0.02, dtmaxinv=32, tend=0.125),
    "c4": dict(order=8, n=1048576, eps=1 / 16384, eta=0.2, eta_s=0.04, dtmaxinv=64, tend=1 / 32),
    # one cluster of the batched ensemble (its N and eps = 4/N given per run)
    "c5": dict(order=6, n=1024, eps=4 / 1024, eta=0.1, eta_s=0.02, dtmaxinv=16, tend=0.25),
}

APP = {"gpu": ROOT / "hermite_b200" / "gravity" / "_build" / "hb-app-{order}",
       "gpu-mixed": ROOT / "hermite_b200" / "gravity" / "_build" / "hb-app-{order}",
       # the integrator's -DFAST_OMP_SYNC loop on the drop-in (make -C hermite_b200/gravity fast)
       "gpu-fast": ROOT / "hermite_b200" / "gravity" / "_build" / "hb-app-fast-{order}",
       "cpu-ref": ROOT / "oracle" / "_ref" / "avx2-{order}",
       # the reference's own FP64 CUDA path recompiled for sm_100a (oracle/Makefile ref-gpu)
       "ref-gpu": ROOT / "oracle" / "_ref" / "titan-{order}"}


def input_text(cfg, snap, log_interval):
    return (f"order {cfg['order']}\neta {cfg['eta']!r}\neta_s {cfg['eta_s']!r}\n"
            f"snapin {snap}\ntend {cfg['tend']!r}\ndtmaxinv {cfg['dtmaxinv']}\n"
            f"eps {cfg['eps']!r}\nlog_interval {log_interval!r}\n"
            f"snap_interval {2 * cfg['tend']!r}\ndump_interval {cfg['tend']!r}\n")


def run(config: str, impl: str = "gpu", tend: float | None = None, n: int | None = None,
        seed: int = 0, workdir: Path | None = None, threads: int | None = None,
        snapshot=None, eps: float | None = None) -> dict:
    """snapshot: initial conditions (an ic.Snapshot) instead of the seeded
    Plummer sphere; eps: softening instead of the configuration's."""
    from hermite_b200.ic import plummer, write_snapshot
    cfg = dict(CONFIGS[config])
    if tend is not None:
        cfg["tend"] = tend
    if n is not None:
        cfg["n"] = n
    if snapshot is not None:
        cfg["n"] = snapshot.n
    if eps is not None:
        cfg["eps"] = eps
    app = Path(str(APP[impl]).format(order=cfg["order"]))
    if not app.exists():
        raise FileNotFoundError(f"{app} not built (needs the reference sources)")
    tmp = None
    if workdir is None:
        tmp = tempfile.TemporaryDirectory()
        workdir = Path(tmp.name)
    if snapshot is not None:
        snap = workdir / f"given_{cfg['n']}.dat"
        write_snapshot(snap, snapshot)
    else:
        snap = workdir / f"plummer_{cfg['n']}_{seed}.dat"
        if not snap.exists():
            write_snapshot(snap, plummer(cfg["n"], seed))
    dtmax = 1.0 / cfg["dtmaxinv"]
    log_interval = max(dtmax, cfg["tend"] / 8)
    env = dict(os.environ)
    env["HERMITE_B200_PRECISION"] = "mixed" if impl == "gpu-mixed" else "fp64"
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    t0 = time.perf_counter()
    r = subprocess.run([str(app)], input=input_text(cfg, snap.name, log_interval), cwd=workdir,
                       env=env, capture_output=True, text=True)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError(f"{app.name} exited {r.returncode}:\n{r.stderr[-3000:]}")
    rows = re.findall(r"^## (\d+) (\S+) (\S+) (\S+) (\S+)\s*$", r.stdout, re.M)
    init = re.search(r"^## Init N square : (\S+) Gflops", r.stdout, re.M)
    de = re.findall(r"de\(local/global\) : (\S+) (\S+)", r.stderr)
    e0 = re.search(r",\s*e =\s*(\S+)", r.stderr)
    steps = re.findall(r"steps: (\d+) (\d+) (\d+) (\d+)", r.stderr)
    last = rows[-1] if rows else None
    out = {"config": config, "impl": impl, "order": cfg["order"], "n": cfg["n"],
           "eps": cfg["eps"], "eta": cfg["eta"], "eta_s": cfg["eta_s"], "dtmax": dtmax,
           "tend": cfg["tend"], "wall_s": wall,
           "init_n2_gflops": float(init.group(1)) if init else None,
           "e0": float(e0.group(1)) if e0 else None,
           "de_global": float(de[-1][1]) if de else None,
           "de_global_max_abs": max(abs(float(d[1])) for d in de) if de else None,
           "block_steps": int(steps[-1][2]) if steps else None,
           "particle_steps": int(steps[-1][3]) if steps else None}
    if last:
        out.update({"app_wtime_s": float(last[1]), "app_gflops": float(last[2]),
                    "us_per_block": float(last[3]), "nact_mean": float(last[4]),
                    "app_gint_s": float(last[2]) / {4: 60, 6: 97, 8: 144}[cfg["order"]]})
    if tmp:
        tmp.cleanup()
    return out


def run_device(config: str, precision: str = "fp64", tend: float | None = None,
               n: int | None = None, seed: int = 0, engine: str = "auto") -> dict:
    """The same configuration on the library's device-resident integrator
    (corrector and block-step scheduler on the GPU, hb_integrator_*): block
    and particle steps, wall time per block step, interactions per second
    (particle steps x N / wall) and the relative energy error at the end, with
    the reference's sign convention (E0 - E) / E0 (SRC/nbodysystem.h:948-951)."""
    from hermite_b200 import Gravity
    from hermite_b200.ic import plummer, records
    cfg = dict(CONFIGS[config])
    if tend is not None:
        cfg["tend"] = tend
    if n is not None:
        cfg["n"] = n
    order, nb = cfg["order"], cfg["n"]
    eps2 = cfg["eps"] ** 2
    with Gravity(order, nb, precision) as g:
        g.set_engine(engine)
        used = g.engine()
        g.set_jp_records(records(plummer(nb, seed), order))
        t0 = time.perf_counter()
        g.integrator_init(0.0, eps2, cfg["eta"], cfg["eta_s"], 1.0 / cfg["dtmaxinv"])
        init_s = time.perf_counter() - t0
        ke0, pe0 = g.energy(eps2)
        t0 = time.perf_counter()
        g.integrator_run(cfg["tend"])
        wall = time.perf_counter() - t0
        ps, bs, t = g.integrator_stats()
        ke, pe = g.energy(eps2)
    e0 = ke0 + pe0
    return {"config": config, "impl": f"device-{precision}", "engine": used[0],
            "order": order, "n": nb, "eps": cfg["eps"], "eta": cfg["eta"], "eta_s": cfg["eta_s"],
            "dtmax": 1.0 / cfg["dtmaxinv"], "tend": cfg["tend"], "t": t, "init_s": init_s,
            "wall_s": wall, "block_steps": bs, "particle_steps": ps,
            "nact_mean": ps / max(bs, 1), "us_per_block": wall / max(bs, 1) * 1e6,
            "app_gint_s": ps * nb / wall * 1e-9, "e0": e0, "de_global": (e0 - (ke + pe)) / e0}


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--config", default="c1", choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="gpu", choices=sorted(APP) + ["device", "device-mixed"])
    ap.add_argument("--tend", type=float, default=None)
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--threads", type=int, default=None)
    a = ap.parse_args()
    if a.impl.startswith("device"):
        prec = "mixed" if a.impl == "device-mixed" else "fp64"
        print(json.dumps(run_device(a.config, prec, a.tend, a.n)))
        return
    print(json.dumps(run(a.config, a.impl, a.tend, a.n, threads=a.threads)))


if __name__ == "__main__":
    main()
