"""How much force error the reference's Hermite integrator tolerates, and why
the mixed-precision pair arithmetic exceeds it at small eta and at 6th order.

The reference's own integrator (SRC/nbodysystem.h with the corrector and
Aarseth criterion of SRC/hermite{4,6}.h) runs on the CPU against
tests/noise/noise_gravity.inl: the oracle's FP64 forces, optionally with a
seeded relative perturbation of size s per derivative, or the mixed kernel's
pair arithmetic restated in C float.  The corrector forms the higher
derivatives from differences of consecutive forces of a particle, scaled by
dt^-2..dt^-3 (4th order, SRC/hermite4.h:118-153) or dt^-3..dt^-5 (6th order,
SRC/hermite6.h:136-184); white force noise of relative size s thus enters
the step criterion amplified by about (tau/dt)^3 or (tau/dt)^5, and once it
dominates, shorter steps amplify it further and the block steps collapse.

Measured (block steps to t = 1/8, gen-plum-like Plummer N = 1024, eps = 1/256;
6th order: N = 4096, eps = 1/4096, eta = 0.1, dtmax = 1/32, t = 1/32):
  4th order, eta = 0.01: FP64 and s = 1e-9 take the same steps; s = 1e-8 and
    the FP32 pair arithmetic blow up (> 10x), and so does FP64 arithmetic
    whose relative position alone is the hi/lo FP32 difference: one FP32
    rounding per pair already exceeds what the criterion tolerates.
  4th order, eta = 0.1 (the reference's RUN/inp.4th): s = 1e-6 and the FP32
    pair arithmetic take FP64's steps within 1%.
  6th order, eta = 0.1: s = 1e-11 is tolerated, s = 1e-10 is not.
FP32 pair arithmetic leaves s ~ 1e-8..1e-7 (tests/test_config_parity.py), so
6th/8th-order integrations and 4th-order ones at eta of about 0.02 or less
need the FP64 force; the mixed kernel integrates 4th order at the
reference's own eta.
"""
import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
NOISE = ROOT / "tests" / "noise"
BLOWUP = 3            # noise_gravity's exit code when HB_NOISE_MAX_CALLS is reached


@pytest.fixture(scope="module")
def apps():
    sys.path.insert(0, str(ROOT))
    from __graft_entry__ import reference_checkout
    ref = reference_checkout()
    if ref is None:
        pytest.skip("the reference checkout is needed to build its integrator")
    r = subprocess.run(["make", "-C", str(NOISE), f"REF={ref}"], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(f"building tests/noise failed:\n{r.stderr[-2000:]}")
    return NOISE / "_build"


def run(apps, tmp_path, order, n, eps, eta, eta_s, dtmax_inv, tend, env, max_calls=0):
    """Block steps and energy error of one run (None when it blew up)."""
    from hermite_b200.ic import plummer, write_snapshot
    snap = tmp_path / f"plummer_{n}.dat"
    if not snap.exists():
        write_snapshot(snap, plummer(n, 0))
    text = (f"order {order}\neta {eta!r}\neta_s {eta_s!r}\nsnapin {snap.name}\n"
            f"tend {tend!r}\ndtmaxinv {dtmax_inv}\neps {eps!r}\nlog_interval {tend!r}\n"
            f"snap_interval {2 * tend!r}\ndump_interval {tend!r}\n")
    e = dict(os.environ, OMP_NUM_THREADS=str(min(8, os.cpu_count() or 1)))
    e.update({k: str(v) for k, v in env.items()})
    if max_calls:
        e["HB_NOISE_MAX_CALLS"] = str(max_calls)
    r = subprocess.run([str(apps / f"noise-app-{order}")], input=text, cwd=tmp_path, env=e,
                       capture_output=True, text=True, timeout=600)
    if r.returncode == BLOWUP or "Assertion `dtlim" in r.stderr:
        return None
    assert r.returncode == 0, r.stderr[-2000:]
    steps = re.findall(r"steps: (\d+) (\d+) (\d+) (\d+)", r.stderr)
    de = re.findall(r"de\(local/global\) : (\S+) (\S+)", r.stderr)
    return int(steps[-1][2]), float(de[-1][1])


C1 = dict(order=4, n=1024, eps=1 / 256, dtmax_inv=8, tend=0.125)
C3S = dict(order=6, n=4096, eps=1 / 4096, eta=0.1, eta_s=0.02, dtmax_inv=32, tend=1 / 32)


def test_fourth_order_small_eta(apps, tmp_path):
    c1 = dict(C1, eta=0.01, eta_s=0.0025)
    bs64, de64 = run(apps, tmp_path, env={}, **c1)
    cap = 10 * bs64
    quiet = run(apps, tmp_path, env={"HB_NOISE_REL": 1e-9}, max_calls=cap, **c1)
    assert quiet is not None and quiet[0] <= 1.1 * bs64
    assert run(apps, tmp_path, env={"HB_NOISE_REL": 1e-8}, max_calls=cap, **c1) is None
    assert run(apps, tmp_path, env={"HB_NOISE_MODE": "fp32pair"}, max_calls=cap, **c1) is None
    # one FP32 rounding per pair, of the relative position, is enough
    assert run(apps, tmp_path, env={"HB_NOISE_MODE": "dr32"}, max_calls=cap, **c1) is None


def test_fourth_order_reference_eta(apps, tmp_path):
    c1 = dict(C1, eta=0.1, eta_s=0.01)
    bs64, de64 = run(apps, tmp_path, env={}, **c1)
    for env in ({"HB_NOISE_REL": 1e-6}, {"HB_NOISE_MODE": "fp32pair"}):
        bs, de = run(apps, tmp_path, env=env, max_calls=10 * bs64, **c1)
        assert abs(bs - bs64) <= 0.01 * bs64, (env, bs, bs64)
        assert abs(de) <= 2 * abs(de64) + 1e-12, (env, de, de64)


def test_sixth_order(apps, tmp_path):
    bs64, de64 = run(apps, tmp_path, env={}, **C3S)
    cap = 10 * bs64
    quiet = run(apps, tmp_path, env={"HB_NOISE_REL": 1e-11}, max_calls=cap, **C3S)
    assert quiet is not None and quiet[0] <= 1.1 * bs64
    assert run(apps, tmp_path, env={"HB_NOISE_REL": 1e-10}, max_calls=cap, **C3S) is None
    assert run(apps, tmp_path, env={"HB_NOISE_MODE": "fp32pair"}, max_calls=cap, **C3S) is None


def _fp32pair_lib():
    import ctypes
    r = subprocess.run(["make", "-C", str(NOISE), "lib"], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(f"building tests/noise lib failed:\n{r.stderr[-2000:]}")
    lib = ctypes.CDLL(str(NOISE / "_build" / "libfp32pair.so"))
    dp = ctypes.POINTER(ctypes.c_double)
    lib.fp32pair_force.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_int, dp]
    lib.fp32pair_force.restype = None
    return lib


def test_split_velocities_do_not_change_fp32_errors(oracle):
    """Hi/lo velocities and accelerations (formed like the hi/lo positions)
    leave the FP32 pair arithmetic's per-evaluation errors where they are:
    the rounding of the pair terms themselves dominates.  6th order, Plummer
    N = 4096 with acc/jrk/snp from the oracle's forces (the integrator's
    start-up), eps = 1/4096."""
    import ctypes
    import numpy as np
    from hermite_b200.ic import plummer, records
    lib = _fp32pair_lib()
    order, n, eps2 = 6, 4096, (1 / 4096) ** 2
    rec = records(plummer(n, 2), order)
    for _ in range(2):                      # acc, jrk; then snp with acc in the records
        f = oracle.predict_force(order, rec, 0.0, n, eps2)
        rec[:, 8:17] = f[:, 0:9]
    pred = np.ascontiguousarray(oracle.predict(order, rec, 0.0))
    ref = oracle.force(order, pred, n, eps2)
    dp = ctypes.POINTER(ctypes.c_double)
    err = {}
    for split in (0, 1):
        got = np.empty_like(ref)
        lib.fp32pair_force(order, n, pred.ctypes.data_as(dp), n, eps2, split,
                           got.ctypes.data_as(dp))
        e = np.linalg.norm((got - ref).reshape(n, 3, 3), axis=2) / \
            np.linalg.norm(ref.reshape(n, 3, 3), axis=2)
        err[split] = (np.median(e, axis=0), e.max(axis=0))
    for k in range(3):                      # acc, jrk, snp
        med0, med1 = err[0][0][k], err[1][0][k]
        assert abs(med1 - med0) <= 0.15 * med0, (k, med0, med1)
        assert err[1][1][k] >= 0.5 * err[0][1][k], (k, err[0][1][k], err[1][1][k])


def test_fp32_acceleration_error_follows_the_sum_condition(oracle):
    """The FP32 pair arithmetic's acceleration error at a particle is bounded
    by the condition number of its force sum, kappa = sum_j |t_j| / |sum_j t_j|
    (t_j the pair terms), times a few FP32 roundings: the errors above 5e-7
    sit at particles with kappa >= 5, where a close neighbour's pull is
    largely cancelled by the rest.  4th order, Plummer N = 16384,
    eps = 1/1024 (c2's softening)."""
    import ctypes
    import numpy as np
    from hermite_b200.ic import plummer, records
    lib = _fp32pair_lib()
    order, n, eps2 = 4, 16384, (1 / 1024) ** 2
    pred = np.ascontiguousarray(oracle.predict(order, records(plummer(n, 0), order), 0.0))
    ref = oracle.force(order, pred, n, eps2)
    got = np.empty_like(ref)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.fp32pair_force(order, n, pred.ctypes.data_as(dp), n, eps2, 0, got.ctypes.data_as(dp))
    anorm = np.linalg.norm(ref[:, :3], axis=1)
    err = np.linalg.norm(got[:, :3] - ref[:, :3], axis=1) / anorm
    assert np.median(err) < 5e-8
    worst = np.argsort(err)[::-1][:40]
    assert err[worst[0]] > 5e-7
    for i in worst:
        d = pred[:, :3] - pred[i, :3]
        r2 = (d * d).sum(1) + eps2
        kappa = (pred[:, 3] * np.sqrt((d * d).sum(1)) / r2 ** 1.5).sum() / anorm[i]
        assert err[i] <= 2e-7 * kappa, (i, err[i], kappa)
        if err[i] > 5e-7:
            assert kappa >= 5.0, (i, err[i], kappa)
