"""The oracle (oracle/hermite_oracle.c) pinned against the reference itself.

* bit-exact against the reference's generic Gravity (SRC/hermite{4,6,8}.h),
  compiled from its sources into oracle/_ref/ (skipped when not built);
* within FP64 rounding of the reference's AVX Gravity (SRC/hermite*-avx.h);
* bit-exact against the committed golden vectors (tests/golden/, made by
  tests/golden/make_golden.py from the reference's own build);
* against closed-form two-body derivatives.
"""
import math

import numpy as np
import pytest

from inputs import make_records, rel_err
from oracle import RefGravity, ref_available

EPS2 = (1.0 / 256) ** 2
GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("order", [4, 6, 8, 9])
@pytest.mark.parametrize("n", [1, 2, 5, 64, 100])
def test_bit_exact_vs_reference_generic(order, n, oracle):
    if not ref_available("generic", order):
        pytest.skip("reference not built (make -C oracle ref)")
    rec = make_records(order, n, seed=3 + n)
    g = RefGravity(order, n, "generic")
    g.set_jp_all(rec)
    g.predict_all(0.0)
    nact = max(1, n - 1)
    assert np.array_equal(oracle.predict_force(order, rec, 0.0, nact, EPS2), g.force(nact, EPS2))
    assert np.array_equal(oracle.potential(order, rec, EPS2), g.potential(EPS2))


@pytest.mark.parametrize("order", [4, 6, 8])
def test_close_to_reference_avx(order, oracle):
    if not ref_available("avx", order):
        pytest.skip("reference not built (make -C oracle ref)")
    n = 256
    rec = make_records(order, n, seed=17)
    g = RefGravity(order, n, "avx")
    g.set_jp_all(rec)
    g.predict_all(0.0)
    assert rel_err(oracle.predict_force(order, rec, 0.0, n, EPS2), g.force(n, EPS2)).max() < 1e-13
    np.testing.assert_allclose(oracle.potential(order, rec, EPS2), g.potential(EPS2), rtol=1e-14)


@pytest.mark.parametrize("order", [4, 6, 8, 9])
def test_golden_vectors(order, oracle):
    z = np.load(GOLDEN / f"ref_order{order}.npz")
    rec, nact, eps2 = z["records"], int(z["nact"]), float(z["eps2"])
    f = oracle.predict_force(order, rec, float(z["tsys"]), nact, eps2)
    assert np.array_equal(f, z["force"])
    assert np.array_equal(oracle.potential(order, rec, eps2), z["potential"])
    if order == 9:          # double-double positions: the reference has no AVX backend
        return
    assert rel_err(f, z["force_avx"]).max() < 1e-13
    np.testing.assert_allclose(oracle.potential(order, rec, eps2), z["potential_avx"], rtol=1e-14)


def test_two_body_closed_form(oracle):
    """Two bodies on a line: acc, jerk, snap, crackle from differentiating
    a(t) = m d(t) / (d(t)^2 + eps2)^{3/2} along d(t) = d0 + v t + a t^2/2 + j t^3/6."""
    order, m, eps2 = 8, 0.3, 0.01
    d0, v, a, j = 0.7, -0.2, 0.05, 0.01
    rec = np.zeros((2, 26))
    rec[1, 0], rec[1, 3], rec[1, 4], rec[1, 8], rec[1, 11] = d0, m, v, a, j
    rec[0, 3] = 1.0
    f = oracle.predict_force(order, rec, 0.0, 1, eps2)[0]

    def acc_t(t):
        d = d0 + v * t + a * t * t / 2 + j * t ** 3 / 6
        return m * d / (d * d + eps2) ** 1.5

    h = 1e-2
    ts = np.arange(-4, 5) * h
    coef = np.polyfit(ts, [acc_t(t) for t in ts], 8)[::-1]
    derivs = [coef[k] * math.factorial(k) for k in range(4)]
    for k in range(4):
        assert f[3 * k + 1] == 0.0 and f[3 * k + 2] == 0.0
        assert abs(f[3 * k] - derivs[k]) <= 1e-6 * max(1.0, abs(derivs[k])), (k, f[3 * k], derivs[k])
