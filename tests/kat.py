"""The block-step `nact` fingerprint of the reference's published runs.

The reference's integrator prints, per dump interval, a row
    ## nbody wtime Gflops wtime/block nact
(SRC/nbodysystem.h:146-150).  nact, the mean number of active particles per
block step, depends on every power-of-two timestep choice and so on the last
bits of every force: it is a known-answer test of the whole FP64 path.
Inputs: gen-plum N/1024 (RUN/gen-plum.c, seed 19640916) with the run
parameters of RUN/inp.{4,6,8}th.  Values: RUN/gpu-{4,6,8}th.log.
"""
from __future__ import annotations

import re
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
GEN_PLUM = ROOT / "oracle" / "_ref" / "gen-plum"

# (order, N) -> the two published nact values (t = 0..1, 1..2)
PUBLISHED_NACT = {
    (4, 1024): ("5.489229e+01", "5.392111e+01"),   # RUN/gpu-4th.log:2,4
    (4, 2048): ("7.706775e+01", "7.671722e+01"),   # RUN/gpu-4th.log:6,8
    (4, 4096): ("1.090551e+02", "1.164058e+02"),   # RUN/gpu-4th.log:10,12
    (6, 1024): ("7.783597e+01", "7.474305e+01"),   # RUN/gpu-6th.log:2,4
    (6, 2048): ("1.113227e+02", "1.103890e+02"),   # RUN/gpu-6th.log:6,8
    (6, 4096): ("1.651473e+02", "1.754420e+02"),   # RUN/gpu-6th.log:10,12
    (8, 1024): ("9.150482e+01", "8.746174e+01"),   # RUN/gpu-8th.log:3,5
    (8, 2048): ("1.307613e+02", "1.300743e+02"),   # RUN/gpu-8th.log:8,10
    (8, 4096): ("1.910739e+02", "2.016963e+02"),   # RUN/gpu-8th.log:13,15
}

# run parameters of RUN/inp.{4,6,8}th: (eta, eta_s)
ETA = {4: (0.1, 0.01), 6: (0.5, 0.1), 8: (0.75, 0.1)}


def input_text(order: int, snap: str) -> str:
    eta, eta_s = ETA[order]
    return (f"order {order}\neta {eta}\neta_s {eta_s}\nsnapin {snap}\ntend 2.0\n"
            "dtmaxinv 16\nkt_for_eps 1.0\nlog_interval 0.25\nsnap_interval 2.0\n"
            "dump_interval 1.0\n")


def make_snapshot(workdir: Path, nk: int) -> str:
    name = f"pl{nk}k.dat"
    if not (workdir / name).exists():
        subprocess.run([str(GEN_PLUM), str(nk)], cwd=workdir, check=True,
                       capture_output=True)
    return name


def run_app(app: Path, order: int, nk: int, workdir: Path, env=None, timeout=600):
    """Run an integrator binary; return (nact strings, stdout)."""
    nact, r = run_app_full(app, order, nk, workdir, env, timeout)
    return nact, r.stdout


def run_app_full(app: Path, order: int, nk: int, workdir: Path, env=None, timeout=600):
    """Run an integrator binary; return (nact strings, the CompletedProcess)."""
    snap = make_snapshot(workdir, nk)
    r = subprocess.run([str(app)], input=input_text(order, snap), cwd=workdir, env=env,
                       capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{app.name} failed ({r.returncode}):\n{r.stderr[-2000:]}")
    rows = re.findall(r"^## (\d+) (\S+) (\S+) (\S+) (\S+)\s*$", r.stdout, re.M)
    return [row[4] for row in rows], r


def energy_error(stderr: str) -> float:
    """The last global relative energy error the integrator printed
    (" de(local/global) : ..", SRC/nbodysystem.h:948-951)."""
    return float(re.findall(r"de\(local/global\) : \S+ (\S+)", stderr)[-1])
