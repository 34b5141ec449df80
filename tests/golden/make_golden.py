"""Regenerate tests/golden/*.npz from the reference's OWN force calculator.

Needs oracle/_ref/ (built from the reference sources by `make -C oracle ref`).
For each order, a seeded Plummer-like input of 64 slots (records with every
derivative populated, tlast spread over power-of-two offsets) is pushed
through the reference's generic Gravity (SRC/hermite{4,6,8}.h: set_jp,
predict_all, calc_force_on_first_nact, calc_potential) and the outputs are
stored next to the inputs:

    records (64, R)  tsys  eps2  nact  force (nact, F)  potential (64,)
    force_avx (nact, F) potential_avx (64,)   -- the AVX backend, same input

Order code 9 (the 8th order with double-double positions,
SRC/hermite8dd.h) has no AVX backend: its file holds the generic outputs
only, from records whose low position words are populated.

    python tests/golden/make_golden.py [order ...]     (default: 4 6 8 9)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path[:0] = [str(ROOT), str(ROOT / "tests")]

from inputs import make_records  # noqa: E402
from oracle import RefGravity  # noqa: E402

N = 64
EPS2 = (1.0 / 128) ** 2
NACT = {4: 64, 6: 40, 8: 17, 9: 23}


def main(orders=(4, 6, 8, 9)):
    for order in orders:
        rec = make_records(order, N, seed=100 + order)
        out = {"records": rec, "tsys": 0.0, "eps2": EPS2, "nact": NACT[order]}
        backends = (("generic", ""),) if order == 9 else (("generic", ""), ("avx", "_avx"))
        for backend, suffix in backends:
            g = RefGravity(order, N, backend)
            g.set_jp_all(rec)
            g.predict_all(0.0)
            out["force" + suffix] = g.force(NACT[order], EPS2)
            out["potential" + suffix] = g.potential(EPS2)
            g.close()
        np.savez_compressed(HERE / f"ref_order{order}.npz", **out)
        print(f"wrote ref_order{order}.npz")


if __name__ == "__main__":
    main(tuple(int(a) for a in sys.argv[1:]) or (4, 6, 8, 9))
