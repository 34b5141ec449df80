"""Force parity against the FP64 oracle at the benchmark sizes, on realistic
states.

c3: 6th order, N = 262144, eps = 1/4096;  c4: 8th order, N = 2^20,
eps = 1/16384.  The states come from the FP64 device integrator after its
start-up and a short run (tests/states.py), so acc, jrk, snp [, crk] and the
spread of tlast are those of a real run.  A random sample of 4096 i-particles
is moved to the front; both precisions compute their forces against all N
j-particles, predicted to the integrator's time, and the C oracle
(oracle/hermite_oracle.c, a restatement of the reference's generic Gravity,
SRC/hermite6.h:332-360, SRC/hermite8.h:385-425) does the same on the CPU.

Bounds, per derivative (max over the sample of |f - f_oracle| / |f_oracle|):
FP64 1e-12 (summation order only); mixed precision at about three times the
maxima measured on a B200.
"""
import numpy as np
import pytest

import hermite_b200 as hb
from inputs import rel_err
from states import CONFIGS, integrator_state, sample_first

NSAMPLE = 4096
FP64_TOL = 1e-12
# acc, jrk, snp [, crk]
MIXED_TOL = {"c3": (1.5e-6, 3e-5, 1e-4), "c4": (1.5e-6, 3e-5, 1e-4, 1e-4)}
T_RUN = {"c3": 1.0 / 1024, "c4": 1.0 / 4096}

_cache = {}


def sampled_case(name, oracle):
    if name not in _cache:
        rec, t, eps2 = integrator_state(name, T_RUN[name])
        recp, _ = sample_first(rec, NSAMPLE, seed=1)
        order = CONFIGS[name][0]
        ref = oracle.predict_force(order, recp, t, NSAMPLE, eps2)
        _cache[name] = (order, recp, t, eps2, ref)
    return _cache[name]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", ["c3", "c4"])
def test_sample_against_oracle(name, precision, oracle):
    order, recp, t, eps2, ref = sampled_case(name, oracle)
    with hb.Gravity(order, recp.shape[0], precision) as g:
        g.set_jp_records(recp)
        g.predict_all(t)
        got = g.calc_force_on_first_nact(NSAMPLE, eps2)
    assert np.all(np.isfinite(got))
    err = rel_err(got, ref)
    print(f"{name} {precision}: max", " ".join(f"{e:.2e}" for e in err.max(axis=0)),
          "median", " ".join(f"{e:.2e}" for e in np.median(err, axis=0)))
    for k in range(err.shape[1]):
        tol = FP64_TOL if precision == "fp64" else MIXED_TOL[name][k]
        assert err[:, k].max() <= tol, (name, precision, k, err[:, k].max())
