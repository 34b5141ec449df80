"""Seeded synthetic inputs shared by the tests (Plummer spheres, reference units)."""
from __future__ import annotations

import numpy as np

from hermite_b200.ic import plummer, records

DERIV_SCALES = (1.0, 3.0, 10.0, 30.0, 100.0, 300.0)   # acc, jrk, snp, crk, d4a, d5a


def make_records(order: int, n: int, seed: int = 1, masses=None) -> np.ndarray:
    """Records at tlast = -dt_i (dt_i a power of two up to 1/32, or 0), so that
    predicting to tsys = 0 exercises every term of the Taylor series.  Order
    code 9 (8th order, double-double positions): the 8th-order records with a
    low position part posL of the size of a double's rounding of pos."""
    if order == 9:
        rec = make_records(8, n, seed, masses)
        rng = np.random.default_rng(seed + 104729)
        posl = rec[:, 0:3] * rng.uniform(-2.0 ** -53, 2.0 ** -53, (n, 3))
        return np.ascontiguousarray(np.concatenate([rec, posl], axis=1))
    snap = plummer(n, seed, masses=masses)
    rng = np.random.default_rng(seed + 7919)
    nd = order - 2
    derivs = np.concatenate([rng.normal(0.0, s, (n, 3)) for s in DERIV_SCALES[:nd]], axis=1)
    rec = records(snap, order, derivs=derivs)
    rec[:, 7] = -rng.choice([0.0, 1 / 256, 1 / 128, 1 / 64, 1 / 32], size=n)
    return rec


def rel_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-particle relative error |a-b|/|b| of each 3-vector block (n, F/3)."""
    a = a.reshape(a.shape[0], -1, 3)
    b = b.reshape(b.shape[0], -1, 3)
    num = np.linalg.norm(a - b, axis=2)
    den = np.linalg.norm(b, axis=2)
    return num / np.where(den > 0, den, 1.0)
