"""CUDA force / predictor / potential vs the FP64 oracle, through the C ABI.

FP64 path: agreement to summation-order rounding (relative 1e-12 per
particle per derivative; the oracle sums j in ascending order, the kernel in
tiles and slices).
Mixed path (hi/lo FP32 relative positions, FP32 pair terms, FP64 flushes):
per-particle relative error of acc <= 1e-6 (the stated target); the higher
derivatives suffer cancellation between pair terms and are bounded loosely
here (jrk 1e-5, snp 1e-4, crk 1e-2 at these small N) -- their measured
distributions are reported by bench.py.
"""
from pathlib import Path

import numpy as np
import pytest

from hermite_b200 import Gravity
from inputs import make_records, rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = {0: 1e-6, 1: 1e-5, 2: 1e-4, 3: 1e-2}
EPS2 = (1.0 / 256) ** 2
GOLDEN = Path(__file__).resolve().parent / "golden"


def _check(order, n, nact, precision, oracle, seed=1, eps2=EPS2, variant=-1, jsplit=0):
    rec = make_records(order, n, seed=seed)
    ref = oracle.predict_force(order, rec, 0.0, nact, eps2)
    with Gravity(order, n, precision) as g:
        g.set_force_shape(variant, jsplit)
        g.set_jp_records(rec)
        g.predict_all(0.0)
        got = g.calc_force_on_first_nact(nact, eps2)
    assert got.shape == ref.shape
    assert np.all(np.isfinite(got))
    err = rel_err(got, ref)
    for k in range(err.shape[1]):
        tol = FP64_TOL if precision == "fp64" else MIXED_TOL[k]
        assert err[:, k].max() <= tol, (order, n, nact, precision, k, err[:, k].max())


@pytest.mark.parametrize("order", [4, 6, 8])
@pytest.mark.parametrize("n", [1, 2, 3, 31, 33, 64, 65, 1000, 4097])
def test_fp64_all_active(order, n, oracle):
    _check(order, n, n, "fp64", oracle)


@pytest.mark.parametrize("order", [4, 6, 8])
@pytest.mark.parametrize("nact", [1, 7, 64, 1000])
def test_fp64_partial_nact(order, nact, oracle):
    _check(order, 3000, nact, "fp64", oracle, seed=5)


@pytest.mark.parametrize("order", [4, 6, 8])
@pytest.mark.parametrize("n", [1, 33, 1000, 4097])
def test_mixed_all_active(order, n, oracle):
    _check(order, n, n, "mixed", oracle)


@pytest.mark.parametrize("order", [4, 6, 8])
@pytest.mark.parametrize("nact", [1, 7, 300])
def test_mixed_partial_nact(order, nact, oracle):
    _check(order, 3000, nact, "mixed", oracle, seed=9)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("variant", list(range(20)))
@pytest.mark.parametrize("jsplit", [1, 3, 16])
def test_every_launch_shape(precision, variant, jsplit, oracle):
    _check(6, 2500, 700, precision, oracle, seed=11, variant=variant, jsplit=jsplit)


@pytest.mark.parametrize("order", [4, 6, 8])
def test_potential(order, oracle):
    n = 1500
    rec = make_records(order, n, seed=4)
    ref = oracle.potential(order, rec, EPS2)
    with Gravity(order, n) as g:
        g.set_jp_records(rec)
        got = g.calc_potential(EPS2)
    np.testing.assert_allclose(got, ref, rtol=1e-13, atol=0)


@pytest.mark.parametrize("order", [4, 6, 8])
@pytest.mark.parametrize("n", [1, 5, 33, 1000, 4097, 70000])
def test_fp64_small_blocks(order, n, oracle):
    """Block steps of at most 16 active particles take the lane-split kernel
    (lanes of a warp share an i-particle and split j): nact across every
    lane-group size and a few j-slice counts (set by N) against the oracle,
    and the first nact past it (the tiled kernel)."""
    for nact in sorted({1, 2, 3, 5, 8, 13, 16, 17} & set(range(1, n + 1))):
        _check(order, n, nact, "fp64", oracle, seed=31)


@pytest.mark.parametrize("order", [4, 6, 8])
def test_small_blocks_match_tiled_kernel(order):
    """The lane-split kernel and the tiled kernel (an explicit shape) agree
    to summation-order rounding, and the lane-split result is reproducible
    to the bit."""
    n = 20000
    rec = make_records(order, n, seed=41)
    for nact in (1, 2, 4, 11, 16):
        out = []
        for variant in (-1, -1, 0):
            with Gravity(order, n) as g:
                g.set_force_shape(variant, 0)
                g.set_jp_records(rec)
                g.predict_all(0.0)
                out.append(g.calc_force_on_first_nact(nact, EPS2))
        assert np.array_equal(out[0], out[1]), nact
        assert rel_err(out[0], out[2]).max() <= FP64_TOL, nact


@pytest.mark.parametrize("variant", [0, 2, 12, 13, -1])   # two-pass, fused, automatic shapes
def test_self_term_is_zero(variant):
    """One particle: the force on it is exactly zero in both precisions (the
    fused kernels predict i and j separately; the two states must agree to
    the bit).  The automatic shape is the lane-split kernel in FP64."""
    for order in (4, 6, 8):
        rec = make_records(order, 1, seed=2)
        for prec in ("fp64", "mixed"):
            with Gravity(order, 1, prec) as g:
                g.set_force_shape(variant, 0)
                g.set_jp_records(rec)
                g.predict_all(0.0)
                f = g.calc_force_on_first_nact(1, EPS2)
            assert np.all(f == 0.0), (order, prec, variant)


@pytest.mark.parametrize("order", [4, 6, 8])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_matches_two_pass(order, precision):
    """The fused predict+force shapes and the two-pass shapes (predictor
    kernel, then force) agree: to summation-order rounding in FP64, to the
    mixed tolerance otherwise."""
    n, nact = 3000, 777
    rec = make_records(order, n, seed=13)
    out = {}
    for v in (0, 12):
        with Gravity(order, n, precision) as g:
            g.set_force_shape(v, 4)
            g.set_jp_records(rec)
            g.predict_all(0.0)
            out[v] = g.calc_force_on_first_nact(nact, EPS2)
    err = rel_err(out[12], out[0])
    tol = [FP64_TOL] * 4 if precision == "fp64" else [MIXED_TOL[k] for k in range(4)]
    for k in range(err.shape[1]):
        assert err[:, k].max() <= tol[k], (k, err[:, k].max())


def test_upload_contract(oracle):
    """Only slots passed to set_jp since the last upload are re-sent, and a
    later update of a prefix (the integrator's pattern) is seen."""
    order, n = 4, 1200
    rec = make_records(order, n, seed=21)
    with Gravity(order, n) as g:
        g.set_jp_records(rec)
        g.predict_all(0.0)
        g.calc_force_on_first_nact(n, EPS2)
        rec2 = rec.copy()
        rec2[:50, 0:3] += 0.01
        for i in range(50):
            g.set_jp(i, rec2[i, 0:3], rec2[i, 3], rec2[i, 4:7], rec2[i, 7], rec2[i, 8:])
        g.predict_all(0.0)
        got = g.calc_force_on_first_nact(n, EPS2)
    ref = oracle.predict_force(order, rec2, 0.0, n, EPS2)
    assert rel_err(got, ref).max() <= FP64_TOL


def test_nact_zero_and_errors(oracle):
    from hermite_b200 import HermiteError
    rec = make_records(4, 100)
    with Gravity(4, 100) as g:
        with pytest.raises(HermiteError):
            g.calc_force_on_first_nact(10, EPS2)          # before any predict_all
        g.set_jp_records(rec)
        g.predict_all(0.0)
        assert g.calc_force_on_first_nact(0, EPS2).shape == (0, 6)
        with pytest.raises(HermiteError):
            g.calc_force_on_first_nact(101, EPS2)
        with pytest.raises(HermiteError):
            g.set_jp(100, [0, 0, 0], 1.0, [0, 0, 0], 0.0, np.zeros(6))


def test_deterministic(oracle):
    rec = make_records(6, 5000, seed=8)
    outs = []
    for _ in range(2):
        with Gravity(6, 5000, "mixed") as g:
            g.set_jp_records(rec)
            g.predict_all(0.0)
            outs.append(g.calc_force_on_first_nact(37, EPS2))
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_predictor_pass_on_its_own(precision):
    """An explicit predictor pass (hb_predict_pass) before a two-pass force
    leaves the forces unchanged to the bit; before any predict_all it is a
    state error."""
    from hermite_b200 import HermiteError
    order, n, nact = 6, 3000, 500
    rec = make_records(order, n, seed=17)
    out = []
    for explicit in (False, True):
        with Gravity(order, n, precision) as g:
            if explicit:
                with pytest.raises(HermiteError):
                    g.predict_pass()
            g.set_force_shape(0, 4)           # a two-pass shape
            g.set_jp_records(rec)
            g.predict_all(0.125)
            if explicit:
                g.predict_pass()
            out.append(g.calc_force_on_first_nact(nact, EPS2))
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("order", [4, 6, 8, 9])
def test_golden_fixtures(order):
    """The reference's own outputs stored in tests/golden (its generic
    Gravity, SRC/hermite{4,6,8}.h and SRC/hermite8dd.h, on 64 seeded slots):
    the FP64 device force and potential match them to summation order."""
    z = np.load(GOLDEN / f"ref_order{order}.npz")
    rec, nact, eps2, tsys = z["records"], int(z["nact"]), float(z["eps2"]), float(z["tsys"])
    with Gravity(8 if order == 9 else order, rec.shape[0], "dd" if order == 9 else "fp64") as g:
        g.set_jp_records(rec)
        g.predict_all(tsys)
        got = g.calc_force_on_first_nact(nact, eps2)
        pot = g.calc_potential(eps2)
    assert rel_err(got, z["force"]).max() <= FP64_TOL
    np.testing.assert_allclose(pot, z["potential"], rtol=1e-13, atol=0)
