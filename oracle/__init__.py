"""TEST INFRASTRUCTURE ONLY -- CPU checkers for the CUDA force path.

Only tests/, __graft_entry__.smoke() and the CPU-baseline / reference legs of
bench.py may import this package.  It never stands in for the product: the
product path (hermite_b200) has no CPU fallback.

* `Oracle`      -- the scalar FP64 C restatement (oracle/hermite_oracle.c) of the
                   reference's generic Gravity (SRC/hermite{4,6,8}.h; order code
                   9: SRC/hermite8dd.h, double-double positions).
* `RefGravity`  -- the reference's OWN Gravity (generic or AVX backend),
                   compiled from its sources by oracle/Makefile into oracle/_ref/.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "liboracle.so"
REF_DIR = HERE / "_ref"


def record_words(order):
    return 8 + 3 * (order - 2)


def predicted_words(order):
    # order code 9: the 8th order with double-double positions (+ posL)
    return 7 + 3 * (order // 2 - 2) + (3 if order == 9 else 0)


def force_words(order):
    return 3 * (order // 2)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def build_oracle() -> Path:
    """Build the C restatement if missing (needs only gcc)."""
    if not ORACLE_LIB.exists():
        subprocess.run(["make", "-C", str(HERE), "oracle"], check=True, capture_output=True)
    return ORACLE_LIB


class Oracle:
    """Scalar FP64 restatement; j summed in ascending order."""

    def __init__(self):
        self.lib = ctypes.CDLL(str(build_oracle()))
        I, D = ctypes.c_int, ctypes.c_double
        dp = ctypes.POINTER(ctypes.c_double)
        self.lib.oracle_predict.argtypes = [I, I, dp, D, dp]
        self.lib.oracle_force.argtypes = [I, I, dp, I, D, dp]
        self.lib.oracle_potential.argtypes = [I, I, dp, D, dp]
        for f in ("oracle_predict", "oracle_force", "oracle_potential"):
            getattr(self.lib, f).restype = None

    def predict(self, order, rec, tsys):
        rec = np.ascontiguousarray(rec, dtype=np.float64).reshape(-1, record_words(order))
        out = np.empty((rec.shape[0], predicted_words(order)))
        self.lib.oracle_predict(order, rec.shape[0], _dp(rec), float(tsys), _dp(out))
        return out

    def force(self, order, pred, nact, eps2):
        pred = np.ascontiguousarray(pred, dtype=np.float64).reshape(-1, predicted_words(order))
        out = np.empty((int(nact), force_words(order)))
        self.lib.oracle_force(order, pred.shape[0], _dp(pred), int(nact), float(eps2), _dp(out))
        return out

    def predict_force(self, order, rec, tsys, nact, eps2):
        return self.force(order, self.predict(order, rec, tsys), nact, eps2)

    def potential(self, order, rec, eps2):
        rec = np.ascontiguousarray(rec, dtype=np.float64).reshape(-1, record_words(order))
        out = np.empty(rec.shape[0])
        self.lib.oracle_potential(order, rec.shape[0], _dp(rec), float(eps2), _dp(out))
        return out


def ref_available(backend: str = "generic", order: int = 4) -> bool:
    return (REF_DIR / f"libref_{backend}{order}.so").exists()


class RefGravity:
    """The reference's own Gravity (backend 'generic' or 'avx') via ctypes.

    The AVX backend works on groups of 4 slots: n must be a multiple of 4.
    """

    def __init__(self, order: int, n: int, backend: str = "generic"):
        path = REF_DIR / f"libref_{backend}{order}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} (build with `make -C oracle ref`)")
        self.lib = ctypes.CDLL(str(path))
        self.order, self.n = order, n
        P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        dp = ctypes.POINTER(ctypes.c_double)
        self.lib.ref_create.restype = P
        self.lib.ref_create.argtypes = [I]
        self.lib.ref_destroy.argtypes = [P]
        self.lib.ref_set_jp_all.argtypes = [P, I, dp]
        self.lib.ref_predict_all.argtypes = [P, D]
        self.lib.ref_force.argtypes = [P, I, D, dp]
        self.lib.ref_potential.argtypes = [P, D, dp]
        self.h = self.lib.ref_create(n)

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_jp_all(self, rec):
        rec = np.ascontiguousarray(rec, dtype=np.float64).reshape(-1, record_words(self.order))
        self.lib.ref_set_jp_all(self.h, rec.shape[0], _dp(rec))

    def predict_all(self, tsys):
        self.lib.ref_predict_all(self.h, float(tsys))

    def force(self, nact, eps2):
        out = np.empty((int(nact), force_words(self.order)))
        self.lib.ref_force(self.h, int(nact), float(eps2), _dp(out))
        return out

    def potential(self, eps2):
        out = np.empty(self.n)
        self.lib.ref_potential(self.h, float(eps2), _dp(out))
        return out
