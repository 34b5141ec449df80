"""Integrator states at the benchmark configurations, for force checks.

A seeded Plummer sphere of the configuration's N is handed to the device
integrator (FP64): its start-up (the reference's init_step,
SRC/nbodysystem.h:565-631: a bootstrap force pass at 6th/8th order, then the
forces and the first steps) fills acc, jrk [, snp, crk [, d4a, d5a]], and a
short run leaves the particles at different tlast.  Forces evaluated at the
integrator's current time then exercise every term of the pair algebra
(SRC/hermite6.h:332-360, SRC/hermite8.h:385-425) with realistic derivative
sizes, unlike records with zero derivatives.
"""
from __future__ import annotations

import numpy as np

# name -> (order, N, eps, eta, eta_s, dtmax); eta_s = eta/4 (c1) or eta/5
# (RUN/inp.6th's ratio) where the configuration does not give it.
CONFIGS = {
    "c1": (4, 1024, 1 / 256, 0.01, 0.0025, 1 / 8),
    "c2": (4, 65536, 1 / 1024, 0.01, 0.0025, 1 / 16),
    "c3": (6, 262144, 1 / 4096, 0.1, 0.02, 1 / 32),
    "c4": (8, 1 << 20, 1 / 16384, 0.2, 0.04, 1 / 64),
}


def integrator_state(name: str, t_run: float, seed: int = 0):
    """(records in slot order, current time, eps2) of the FP64 device
    integrator after start-up and a run to t_run."""
    from hermite_b200 import Gravity
    from hermite_b200.ic import plummer, records
    order, n, eps, eta, eta_s, dtmax = CONFIGS[name]
    with Gravity(order, n, "fp64") as g:
        g.set_jp_records(records(plummer(n, seed), order))
        g.integrator_init(0.0, eps * eps, eta, eta_s, dtmax)
        if t_run > 0:
            g.integrator_run(t_run)
        t = g.integrator_stats()[2]
        rec = g.get_records()
    return rec, t, eps * eps


def sample_first(rec: np.ndarray, nsample: int, seed: int = 0):
    """Records permuted so that a random sample of nsample slots comes first
    (the force entry points compute the first nact slots), and the sample."""
    rng = np.random.default_rng(seed)
    n = rec.shape[0]
    pick = rng.choice(n, size=nsample, replace=False)
    rest = np.setdiff1d(np.arange(n), pick)
    return np.ascontiguousarray(rec[np.concatenate([pick, rest])]), pick
