"""Size-independent properties at the benchmark sizes, where the oracle
would take too long (GPU, through the C ABI).

* Newton's third law: with every particle active, the pair terms of every
  derivative cancel in the mass-weighted sum, so |sum_i m_i F_i| is rounding
  only.  Against sum_i m_i |F_i| it is bounded by the largest per-particle
  relative error plus exact-arithmetic rounding: about 1e-15 in FP64
  (measured with the CPU oracle up to N = 16384), and the per-derivative
  mixed-precision tolerances of the parity tests.
* Rows do not depend on nact: the forces of a partial step equal the same
  rows of the all-active step to summation-order rounding (the two use
  different launch shapes).
"""
import numpy as np
import pytest

from hermite_b200 import Gravity
from hermite_b200.ic import plummer, records
from inputs import rel_err

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = (1e-6, 1e-5, 1e-4, 1e-2)
CASES = [(4, 65536, 1.0 / 1024), (6, 262144, 1.0 / 4096), (8, 131072, 1.0 / 8192)]


def _records(order, n, seed):
    rec = records(plummer(n, seed=seed), order)
    rng = np.random.default_rng(seed)
    rec[:, 8:] = rng.normal(0.0, 0.1, size=(n, rec.shape[1] - 8))
    rec[:, 7] = -rng.choice([0.0, 1 / 1024, 1 / 512, 1 / 256], size=n)
    return rec


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("order,n,eps", CASES)
def test_third_law_at_full_size(order, n, eps, precision):
    rec = _records(order, n, seed=order)
    with Gravity(order, n, precision) as g:
        g.set_jp_records(rec)
        g.predict_all(0.0)
        f = g.calc_force_on_first_nact(n, eps * eps)
    assert np.all(np.isfinite(f))
    m = rec[:, 3]
    F = f.reshape(n, -1, 3)
    residual = np.linalg.norm(np.einsum("i,idk->dk", m, F), axis=1)
    scale = np.einsum("i,id->d", m, np.linalg.norm(F, axis=2))
    for d in range(F.shape[1]):
        tol = FP64_TOL if precision == "fp64" else MIXED_TOL[d]
        assert residual[d] <= tol * scale[d], (d, residual[d] / scale[d])


@pytest.mark.parametrize("order,n,eps", CASES)
def test_rows_do_not_depend_on_nact(order, n, eps):
    rec = _records(order, n, seed=10 + order)
    with Gravity(order, n, "fp64") as g:
        g.set_jp_records(rec)
        g.predict_all(0.0)
        full = g.calc_force_on_first_nact(n, eps * eps)
        part = {k: g.calc_force_on_first_nact(k, eps * eps) for k in (1, 37, 1000, 5000)}
    for k, f in part.items():   # both within FP64_TOL of the exact sums
        assert rel_err(f, full[:k]).max() <= 2 * FP64_TOL, k
