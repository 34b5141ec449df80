"""The 8th order with double-double positions (precision "dd", the
reference's SRC/hermite8dd.h) on the GPU, through the C ABI, against the
oracle's order code 9 (pinned bit-exact to the reference's own DD Gravity in
tests/test_oracle.py).

* Force: predicted positions are posH + posL with the separation taken as
  (posHj - posHi) + (posLj - posLi); agreement with the oracle to
  summation-order rounding (1e-12), for every launch shape, fused and
  two-pass, all-active and partial nact, ragged N.
* Potential: the same separation, self pair skipped.
* The low part matters: positions far from the origin whose separations are
  below the double's resolution there come out right only with posL.
* Integration: the device integrator (both engines) on gen-plum 1k with the
  reference's 8th-order run parameters, against the reference's own DD
  integrator (oracle/_ref/generic-8dd): the same mean nact per interval and
  an energy error of the same size.
"""
import re
import subprocess

import numpy as np
import pytest

import hermite_b200 as hb
from inputs import make_records, rel_err
from kat import GEN_PLUM, ROOT

pytestmark = pytest.mark.gpu

EPS2 = (1.0 / 256) ** 2


def _force(rec, nact, variant=-1, jsplit=0):
    n = rec.shape[0]
    with hb.Gravity(8, n, "dd") as g:
        assert g.R == 29
        g.set_force_shape(variant, jsplit)
        g.set_jp_records(rec)
        g.predict_all(0.0)
        return g.calc_force_on_first_nact(nact, EPS2)


@pytest.mark.parametrize("n,nact", [(1, 1), (33, 33), (1000, 1000), (4097, 4097), (3000, 7),
                                    (3000, 300)])
def test_force_matches_oracle(n, nact, oracle):
    rec = make_records(9, n, seed=21 + n)
    ref = oracle.predict_force(9, rec, 0.0, nact, EPS2)
    got = _force(rec, nact)
    assert np.all(np.isfinite(got))
    assert rel_err(got, ref).max() <= 1e-12


@pytest.mark.parametrize("variant", list(range(20)))
def test_every_launch_shape(variant, oracle):
    rec = make_records(9, 2500, seed=5)
    ref = oracle.predict_force(9, rec, 0.0, 700, EPS2)
    got = _force(rec, 700, variant, 3)
    assert rel_err(got, ref).max() <= 1e-12, variant


def test_potential_matches_oracle(oracle):
    rec = make_records(9, 1500, seed=4)
    ref = oracle.potential(9, rec, EPS2)
    with hb.Gravity(8, 1500, "dd") as g:
        g.set_jp_records(rec)
        got = g.calc_potential(EPS2)
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=0)


def test_low_part_resolves_far_positions(oracle):
    """A cluster of size 1e-9 at distance 2^20 from the origin: a double
    resolves positions there to ~2e-10, so the separations live in posL."""
    n = 256
    rec = make_records(9, n, seed=8)
    rng = np.random.default_rng(3)
    rel = rng.normal(size=(n, 3)) * 1e-9
    big = 2.0 ** 20
    hi = big + rel
    rec[:, 0:3] = hi
    rec[:, 26:29] = rel - (hi - big)             # the part the double lost (hi - big is exact)
    rec[:, 4:7] *= 1e-9
    rec[:, 8:26] = 0.0
    rec[:, 7] = 0.0
    eps2 = 1e-24
    ref = oracle.predict_force(9, rec, 0.0, n, eps2)
    with hb.Gravity(8, n, "dd") as g:
        g.set_jp_records(rec)
        g.predict_all(0.0)
        got = g.calc_force_on_first_nact(n, eps2)
    assert rel_err(got[:, :3], ref[:, :3]).max() <= 1e-12


def test_precision_is_fixed():
    with hb.Gravity(8, 64, "dd") as g:
        assert g._lib.hb_get_precision(g._h) == hb.FP64_DD
        with pytest.raises(hb.HermiteError):
            g.set_precision("mixed")
    with pytest.raises(hb.HermiteError):
        hb.Gravity(6, 64, "dd")


@pytest.mark.parametrize("engine", ["graph", "team"])
def test_integration_agrees_with_reference_dd(engine, tmp_path):
    from hermite_b200.ic import read_snapshot, records
    app = ROOT / "oracle" / "_ref" / "generic-8dd"
    if not app.exists() or not GEN_PLUM.exists():
        pytest.skip("the reference's DD integrator is not built")
    subprocess.run([str(GEN_PLUM), "1"], cwd=tmp_path, check=True, capture_output=True)
    inp = ("order 8\neta 0.75\neta_s 0.1\nsnapin pl1k.dat\ntend 0.25\ndtmaxinv 16\n"
           "kt_for_eps 1.0\nlog_interval 0.125\nsnap_interval 100.0\ndump_interval 100.0\n")
    r = subprocess.run([str(app)], input=inp, cwd=tmp_path, capture_output=True, text=True,
                       timeout=600, env={"OMP_NUM_THREADS": "8", "PATH": "/usr/bin:/bin"})
    assert r.returncode == 0, r.stderr[-1000:]
    ref_nact = re.findall(r"nact : (\S+)", r.stderr)
    ref_de = [float(x) for x in re.findall(r"de\(local/global\) : \S+ (\S+)", r.stderr)]
    snap = read_snapshot(tmp_path / "pl1k.dat")
    n = snap.n
    eps2 = (4.0 / n) ** 2
    rec8 = records(snap, 8)
    rec = np.concatenate([rec8, np.zeros((n, 3))], axis=1)
    got = []
    with hb.Gravity(8, n, "dd") as g:
        g.set_engine(engine)
        g.set_jp_records(rec)
        g.integrator_init(0.0, eps2, 0.75, 0.1, 1.0 / 16)
        ke0, pe0 = g.energy(eps2)
        last = (0, 0)
        for t in (0.125, 0.25):
            g.integrator_run(t)
            ps, bs, _ = g.integrator_stats()
            got.append("%f" % ((ps - last[0]) / (bs - last[1])))
            last = (ps, bs)
        ke, pe = g.energy(eps2)
    assert got == ref_nact[:2]
    de = (ke0 + pe0 - ke - pe) / (ke0 + pe0)
    assert abs(de) <= 2.0 * abs(ref_de[-1]) + 1e-14, (de, ref_de)
