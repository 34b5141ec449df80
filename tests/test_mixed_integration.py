"""Mixed-precision forces inside 4th-order integrations at the reference's
own run parameters (RUN/inp.4th: eta = 0.1, eta_s = 0.01, dtmax = 1/16,
gen-plum N = 1k..4k, t = 0..2).

At this eta the 4th-order step criterion tolerates force noise of relative
size 1e-6 (tests/test_noise_tolerance.py), far above what the FP32 pair
arithmetic leaves (about 1e-7 at most), so the mixed path must take
essentially the FP64 block steps: the published mean active count per
interval (RUN/gpu-4th.log) within 1 %, and the energy error within 2x of
the reference's own FP64 integrator on the same snapshot.  (At eta = 0.01,
and at 6th/8th order, the tolerance is 1e-9 .. 1e-11 and integrations use
the FP64 path.)
"""
import os
import subprocess

import pytest

from kat import ETA, GEN_PLUM, PUBLISHED_NACT, ROOT, energy_error, input_text, run_app_full

pytestmark = pytest.mark.gpu
APP = ROOT / "hermite_b200" / "gravity" / "_build" / "hb-app-4"
REF_APP = ROOT / "oracle" / "_ref" / "avx2-4"


def _need(*paths):
    for p in (*paths, GEN_PLUM):
        if not p.exists():
            pytest.skip(f"{p.name} not built (needs the reference sources)")


def _reference_de(nk, tmp_path):
    _, r = run_app_full(REF_APP, 4, nk, tmp_path, env=dict(os.environ, OMP_NUM_THREADS="8"))
    return energy_error(r.stderr)


def _close(got, want, rel=0.01):
    return all(abs(float(g) / float(w) - 1.0) <= rel for g, w in zip(got, want))


@pytest.mark.parametrize("nk", [1, 2, 4])
def test_drop_in_mixed_fourth_order(nk, tmp_path):
    _need(APP, REF_APP)
    env = dict(os.environ, HERMITE_B200_PRECISION="mixed", OMP_NUM_THREADS="4")
    nact, r = run_app_full(APP, 4, nk, tmp_path, env=env)
    want = PUBLISHED_NACT[(4, nk * 1024)]
    assert len(nact) == 2 and _close(nact, want), (nact, want)
    de, ref_de = energy_error(r.stderr), _reference_de(nk, tmp_path)
    assert abs(de) <= 2.0 * abs(ref_de) + 1e-13, (de, ref_de)


@pytest.mark.parametrize("nk", [1, 2])
def test_device_integrator_mixed_fourth_order(nk, tmp_path):
    from hermite_b200 import Gravity
    from hermite_b200.ic import read_snapshot, records
    _need(REF_APP)
    subprocess.run([str(GEN_PLUM), str(nk)], cwd=tmp_path, check=True, capture_output=True)
    snap = read_snapshot(tmp_path / f"pl{nk}k.dat")
    n = snap.n
    eps = 4.0 / n                             # kt_for_eps 1.0 (set_thermal_eps)
    eta, eta_s = ETA[4]
    with Gravity(4, n, "mixed") as g:
        assert g.engine()[0] == "graph"       # the team engine integrates in FP64 only
        g.set_jp_records(records(snap, 4))
        g.integrator_init(0.0, eps * eps, eta, eta_s, 1.0 / 16)
        ke0, pe0 = g.energy(eps * eps)
        g.integrator_run(1.0)
        ps1, bs1, _ = g.integrator_stats()
        g.integrator_run(2.0)
        ps2, bs2, _ = g.integrator_stats()
        ke, pe = g.energy(eps * eps)
    got = (ps1 / bs1, (ps2 - ps1) / (bs2 - bs1))
    assert _close(got, PUBLISHED_NACT[(4, n)]), got
    e0 = ke0 + pe0
    de = (e0 - (ke + pe)) / e0
    ref_de = _reference_de(nk, tmp_path)
    assert abs(de) <= 2.0 * abs(ref_de) + 1e-13, (de, ref_de)
