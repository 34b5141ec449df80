"""hermite_b200 -- B200-native Hermite N-body force calculator.

Python mirror of the reference's force-calculator interface (`struct Gravity`
of SRC/hermite{4,6,8}-titan.h, driven by SRC/nbodysystem.h), over the C ABI of
libhermite_b200.so (include/hermite_b200.h):

    g = Gravity(order=6, nbody=N, precision="mixed")
    g.set_jp_records(records)               # or g.set_jp(addr, ...)
    g.predict_all(tsys)
    force = g.calc_force_on_first_nact(nact, eps2)     # (nact, 3*(order/2))
    pot = g.calc_potential(eps2)                        # (N,)

Record layouts are those of the reference's CUDA path:
  j-particle record (8 + 3*(order-2) doubles):
      pos[3] mass vel[3] tlast acc[3] jrk[3] [snp[3] crk[3]] [d4a[3] d5a[3]]
  force record (3*(order/2) doubles): acc[3] jrk[3] [snp[3]] [crk[3]]

There is no CPU fallback: if the CUDA library is missing or no sm_100 device
is present, constructing a Gravity raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

__all__ = ["Gravity", "Ensemble", "HermiteError", "record_words", "force_words", "FP64", "MIXED",
           "library_path", "load_library", "measure_fma_peak", "EXPORTED_SYMBOLS"]

FP64 = 0
MIXED = 1
FP64_DD = 2      # 8th order with double-double positions (records: 29 words)
_PREC = {"fp64": FP64, "mixed": MIXED, "dd": FP64_DD, FP64: FP64, MIXED: MIXED, FP64_DD: FP64_DD}

_PKG = Path(__file__).resolve().parent
_LIB_PATH = _PKG / "_lib" / "libhermite_b200.so"
_lib = None

# Every entry point declared in include/hermite_b200.h.
EXPORTED_SYMBOLS = (
    "hb_create", "hb_destroy", "hb_set_jp", "hb_set_jp_records", "hb_predict_all",
    "hb_force_first_nact", "hb_potential", "hb_set_precision", "hb_get_precision",
    "hb_last_error", "hb_status_string", "hb_set_stream", "hb_upload",
    "hb_predict_all_device", "hb_predict_pass", "hb_force_device", "hb_download_forces", "hb_device_forces",
    "hb_synchronize", "hb_launch_count", "hb_set_force_shape", "hb_set_wait_limit",
    "hb_force_variant_count",
    "hb_force_variant_info", "hb_measure_fma_peak", "hb_force_predicted_noalloc",
    "hb_integrator_init", "hb_integrator_run", "hb_integrator_stats", "hb_energy",
    "hb_integrator_set_engine", "hb_integrator_engine",
    "hb_get_records", "hb_ens_create", "hb_ens_destroy", "hb_ens_last_error",
    "hb_ens_set_cluster", "hb_ens_get_cluster", "hb_ens_cluster_offset", "hb_ens_init",
    "hb_ens_run", "hb_ens_stats", "hb_ens_energy", "hb_ens_set_engine", "hb_ens_cluster_engine",
    "hb_ens_cluster_stats", "hb_dump_write", "hb_dump_read_header", "hb_dump_read",
    "hb_integrator_dump", "hb_integrator_restore", "hb_snapshot_read_header", "hb_snapshot_read",
    "hb_snapshot_write",
)


ENGINES = {"auto": 0, "graph": 1, "team": 2, "persistent": 3}


def record_words(order: int) -> int:
    return 8 + 3 * (order - 2)


def force_words(order: int) -> int:
    return 3 * (order // 2)


AUX_WORDS = 6    # per particle: snp crk (4th), d4a d5a (6th), d6a d7a (8th)


def write_dump(path, order: int, records, aux, tsys: float, dumpid: int = 0,
               energies=(0.0, 0.0), steps=(0, 0), ids=None):
    """Write a checkpoint in the reference's dump format (host only)."""
    lib = load_library()
    rec = np.ascontiguousarray(records, dtype=np.float64).reshape(-1, record_words(order))
    ax = np.ascontiguousarray(aux, dtype=np.float64).reshape(rec.shape[0], AUX_WORDS)
    idp = None
    if ids is not None:
        idarr = np.ascontiguousarray(ids, dtype=np.int64)
        idp = idarr.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    st = lib.hb_dump_write(str(path).encode(), int(order), int(dumpid), rec.shape[0], float(tsys),
                           float(energies[0]), float(energies[1]), int(steps[0]), int(steps[1]),
                           idp, _dptr(rec), _dptr(ax))
    if st != 0:
        raise HermiteError(st, f"hb_dump_write {path}: " + lib.hb_status_string(st).decode())


def read_dump(path, dd: bool = False) -> dict:
    """Read a checkpoint in the reference's dump format (host only): header
    fields, ids, records (tlast = tsys) and the aux derivatives.  dd: the file
    holds double-double positions (the header says order 8 for both), read
    into 29-word records with order code 9."""
    lib = load_library()
    o, d, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    t, e0, e1 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    ps, bs = ctypes.c_longlong(), ctypes.c_longlong()
    st = lib.hb_dump_read_header(str(path).encode(), ctypes.byref(o), ctypes.byref(d),
                                 ctypes.byref(n), ctypes.byref(t), ctypes.byref(e0),
                                 ctypes.byref(e1), ctypes.byref(ps), ctypes.byref(bs))
    if st != 0:
        raise HermiteError(st, f"hb_dump_read_header {path}: " + lib.hb_status_string(st).decode())
    code = 9 if dd else o.value
    rec = np.empty((n.value, record_words(code)))
    aux = np.empty((n.value, AUX_WORDS))
    ids = np.empty(n.value, dtype=np.int64)
    st = lib.hb_dump_read(str(path).encode(), code, n.value,
                          ids.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), _dptr(rec), _dptr(aux))
    if st != 0:
        raise HermiteError(st, f"hb_dump_read {path}: " + lib.hb_status_string(st).decode())
    return {"order": code, "dumpid": d.value, "nbody": n.value, "tsys": t.value,
            "energies": (e0.value, e1.value), "steps": (ps.value, bs.value), "ids": ids,
            "records": rec, "aux": aux}


class HermiteError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


def library_path() -> Path:
    return Path(os.environ.get("HERMITE_B200_LIB", _LIB_PATH))


def load_library() -> ctypes.CDLL:
    """Load libhermite_b200.so (built by `python -m hermite_b200.build`)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not path.exists():
        raise RuntimeError(f"{path} is missing: build it with `python -m hermite_b200.build`")
    lib = ctypes.CDLL(str(path))
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    dp = ctypes.POINTER(ctypes.c_double)
    sig = {
        "hb_create": (I, [I, I, I, ctypes.POINTER(P)]),
        "hb_destroy": (I, [P]),
        "hb_set_jp": (I, [P, I, dp, D, dp, D, dp]),
        "hb_set_jp_records": (I, [P, I, I, dp]),
        "hb_predict_all": (I, [P, D]),
        "hb_force_first_nact": (I, [P, I, D, dp]),
        "hb_potential": (I, [P, D, dp]),
        "hb_set_precision": (I, [P, I]),
        "hb_get_precision": (I, [P]),
        "hb_last_error": (ctypes.c_char_p, [P]),
        "hb_status_string": (ctypes.c_char_p, [I]),
        "hb_set_stream": (I, [P, P]),
        "hb_upload": (I, [P]),
        "hb_predict_all_device": (I, [P, D]),
        "hb_predict_pass": (I, [P]),
        "hb_force_device": (I, [P, I, D]),
        "hb_download_forces": (I, [P, I, dp]),
        "hb_device_forces": (P, [P]),
        "hb_synchronize": (I, [P]),
        "hb_launch_count": (ctypes.c_longlong, [P]),
        "hb_set_force_shape": (I, [P, I, I]),
        "hb_set_wait_limit": (I, [P, ctypes.c_longlong]),
        "hb_force_variant_count": (I, [I, I]),
        "hb_force_variant_info": (I, [I, I, I, ctypes.POINTER(I), ctypes.POINTER(I),
                                      ctypes.POINTER(I)]),
        "hb_measure_fma_peak": (I, [I, dp]),
        "hb_force_predicted_noalloc": (I, [I, I, P, I, I, D, P, P]),
        "hb_integrator_init": (I, [P, D, D, D, D, D]),
        "hb_integrator_run": (I, [P, D, ctypes.c_longlong]),
        "hb_integrator_set_engine": (I, [P, I, I]),
        "hb_integrator_engine": (I, [P, ctypes.POINTER(I), ctypes.POINTER(I)]),
        "hb_integrator_stats": (I, [P, ctypes.POINTER(ctypes.c_longlong),
                                    ctypes.POINTER(ctypes.c_longlong), dp]),
        "hb_energy": (I, [P, D, dp, dp]),
        "hb_get_records": (I, [P, I, I, dp, dp]),
        "hb_ens_create": (I, [I, I, ctypes.POINTER(I), I, ctypes.POINTER(P)]),
        "hb_ens_destroy": (I, [P]),
        "hb_ens_last_error": (ctypes.c_char_p, [P]),
        "hb_ens_set_cluster": (I, [P, I, dp, D]),
        "hb_ens_get_cluster": (I, [P, I, dp, dp]),
        "hb_ens_cluster_offset": (I, [P, I]),
        "hb_ens_init": (I, [P, D, D, D, D]),
        "hb_ens_run": (I, [P, D, ctypes.c_longlong]),
        "hb_ens_stats": (I, [P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                             dp, dp]),
        "hb_ens_energy": (I, [P, dp, dp]),
        "hb_ens_set_engine": (I, [P, I, I]),
        "hb_ens_cluster_engine": (I, [P, I, ctypes.POINTER(I), ctypes.POINTER(I)]),
        "hb_ens_cluster_stats": (I, [P, I, ctypes.POINTER(ctypes.c_longlong),
                                     ctypes.POINTER(ctypes.c_longlong), dp]),
        "hb_dump_write": (I, [ctypes.c_char_p, I, I, I, D, D, D, ctypes.c_longlong,
                              ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong), dp, dp]),
        "hb_dump_read_header": (I, [ctypes.c_char_p, ctypes.POINTER(I), ctypes.POINTER(I),
                                    ctypes.POINTER(I), dp, dp, dp,
                                    ctypes.POINTER(ctypes.c_longlong),
                                    ctypes.POINTER(ctypes.c_longlong)]),
        "hb_dump_read": (I, [ctypes.c_char_p, I, I, ctypes.POINTER(ctypes.c_longlong), dp, dp]),
        "hb_integrator_dump": (I, [P, ctypes.c_char_p, I, D, D]),
        "hb_snapshot_read_header": (I, [ctypes.c_char_p, ctypes.POINTER(I), ctypes.POINTER(I), dp]),
        "hb_snapshot_read": (I, [ctypes.c_char_p, I, ctypes.POINTER(ctypes.c_longlong), dp, dp, dp,
                                 dp]),
        "hb_snapshot_write": (I, [ctypes.c_char_p, I, I, D, ctypes.POINTER(ctypes.c_longlong), dp,
                                  dp, dp, dp]),
        "hb_integrator_restore": (I, [P, ctypes.c_char_p, D, D, D, ctypes.POINTER(I), dp, dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    _lib = lib
    return lib


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _out_buffer(out, rows: int, cols: int | None = None) -> np.ndarray:
    """A caller's result array, checked before the library writes rows x
    cols doubles into it (a new array when out is None)."""
    shape = (max(int(rows), 0),) if cols is None else (max(int(rows), 0), int(cols))
    if out is None:
        return np.empty(shape, dtype=np.float64)
    if not isinstance(out, np.ndarray) or out.dtype != np.float64 or not out.flags.c_contiguous \
            or not out.flags.writeable:
        raise ValueError("out must be a writeable C-contiguous float64 array")
    if out.size < int(np.prod(shape)):
        raise ValueError(f"out holds {out.size} doubles, {int(np.prod(shape))} needed")
    return out


def measure_fma_peak(mode: int) -> float:
    """Measured FMA-pipe peak in GFLOP/s: mode 0 FP64, 1 FP32, 2 packed FP32."""
    lib = load_library()
    out = ctypes.c_double(0.0)
    st = lib.hb_measure_fma_peak(mode, ctypes.byref(out))
    if st != 0:
        raise HermiteError(st, lib.hb_status_string(st).decode())
    return out.value


class Gravity:
    """The reference's `struct Gravity`, one CUDA context-owned instance."""

    def __init__(self, order: int, nbody: int, precision="fp64"):
        """precision: "fp64", "mixed", or "dd" (order 8 only: double-double
        positions; records carry posL after the 8th-order fields, 29 words)."""
        self._lib = load_library()
        self.order, self.nbody = int(order), int(nbody)
        self.dd = _PREC[precision] == FP64_DD
        self.R, self.F = record_words(9 if self.dd else self.order), force_words(self.order)
        h = ctypes.c_void_p()
        st = self._lib.hb_create(self.order, self.nbody, _PREC[precision], ctypes.byref(h))
        if st != 0:
            raise HermiteError(st, f"hb_create(order={order}, nbody={nbody}): "
                                   + self._lib.hb_status_string(st).decode())
        self._h = h

    # -- plumbing ---------------------------------------------------------
    def _check(self, st: int, what: str):
        if st != 0:
            msg = self._lib.hb_last_error(self._h).decode() or self._lib.hb_status_string(st).decode()
            raise HermiteError(st, f"{what}: {msg}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.hb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return self._h.value

    # -- the reference interface -----------------------------------------
    def set_jp(self, addr: int, pos, mass: float, vel, tlast: float, derivs):
        pos = np.ascontiguousarray(pos, dtype=np.float64)
        vel = np.ascontiguousarray(vel, dtype=np.float64)
        derivs = np.ascontiguousarray(derivs, dtype=np.float64).reshape(-1)
        if derivs.size != self.R - 8:
            raise ValueError(f"derivs needs {self.R - 8} values")
        self._check(self._lib.hb_set_jp(self._h, int(addr), _dptr(pos), float(mass), _dptr(vel),
                                        float(tlast), _dptr(derivs)), "set_jp")

    def set_jp_records(self, records: np.ndarray, addr0: int = 0):
        rec = np.ascontiguousarray(records, dtype=np.float64).reshape(-1, self.R)
        self._check(self._lib.hb_set_jp_records(self._h, int(addr0), rec.shape[0], _dptr(rec)),
                    "set_jp_records")

    def predict_all(self, tsys: float):
        self._check(self._lib.hb_predict_all(self._h, float(tsys)), "predict_all")

    def calc_force_on_first_nact(self, nact: int, eps2: float, out: np.ndarray | None = None):
        out = _out_buffer(out, nact, self.F)
        self._check(self._lib.hb_force_first_nact(self._h, int(nact), float(eps2), _dptr(out)),
                    "calc_force_on_first_nact")
        return out

    def calc_potential(self, eps2: float, out: np.ndarray | None = None):
        out = _out_buffer(out, self.nbody)
        self._check(self._lib.hb_potential(self._h, float(eps2), _dptr(out)), "calc_potential")
        return out

    # -- extras ----------------------------------------------------------------
    def set_precision(self, precision):
        self._check(self._lib.hb_set_precision(self._h, _PREC[precision]), "set_precision")

    def set_stream(self, stream_handle: int | None):
        self._check(self._lib.hb_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)),
                    "set_stream")

    def upload(self):
        self._check(self._lib.hb_upload(self._h), "upload")

    def predict_all_device(self, tsys: float):
        self._check(self._lib.hb_predict_all_device(self._h, float(tsys)), "predict_all_device")

    def predict_pass(self):
        """Run the predictor pass now (normally it runs with the next
        two-pass force launch); for timing the predictor alone."""
        self._check(self._lib.hb_predict_pass(self._h), "predict_pass")

    def force_device(self, nact: int, eps2: float):
        self._check(self._lib.hb_force_device(self._h, int(nact), float(eps2)), "force_device")

    def download_forces(self, nact: int, out: np.ndarray | None = None):
        out = _out_buffer(out, nact, self.F)
        self._check(self._lib.hb_download_forces(self._h, int(nact), _dptr(out)), "download_forces")
        return out

    def synchronize(self):
        self._check(self._lib.hb_synchronize(self._h), "synchronize")

    def launch_count(self) -> int:
        return int(self._lib.hb_launch_count(self._h))

    def set_force_shape(self, variant: int = -1, jsplit: int = 0):
        self._check(self._lib.hb_set_force_shape(self._h, int(variant), int(jsplit)),
                    "set_force_shape")


    def set_wait_limit(self, polls: int = -1):
        """Test hook: poll limit of the force kernel's waits for incoming j
        tiles (0: give up at once; < 0: the default)."""
        self._check(self._lib.hb_set_wait_limit(self._h, int(polls)), "set_wait_limit")

    def device_forces_ptr(self) -> int:
        return int(self._lib.hb_device_forces(self._h) or 0)

    # -- device-resident integration (corrector + block-step scheduler) --------
    def integrator_init(self, tsys: float, eps2: float, eta: float, eta_s: float, dtmax: float):
        self._check(self._lib.hb_integrator_init(self._h, float(tsys), float(eps2), float(eta),
                                                 float(eta_s), float(dtmax)), "integrator_init")

    def integrator_run(self, tend: float, max_block_steps: int = 0):
        self._check(self._lib.hb_integrator_run(self._h, float(tend), int(max_block_steps)),
                     "integrator_run")

    def set_engine(self, engine: str = "auto", team_ctas: int = 0):
        """Integration engine: "auto", "graph" (multi-kernel, CUDA graph),
        "team" (one thread-block cluster, whole loop in one kernel) or
        "persistent" (one cooperative kernel over the whole GPU, grid
        barriers between the phases of a step)."""
        self._check(self._lib.hb_integrator_set_engine(self._h, ENGINES[engine], int(team_ctas)),
                    "set_engine")

    def engine(self):
        """(engine name, CTAs per team) that the next integrator_run uses."""
        e, c = ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.hb_integrator_engine(self._h, ctypes.byref(e), ctypes.byref(c)),
                    "engine")
        return {v: k for k, v in ENGINES.items()}[e.value], c.value

    def integrator_stats(self):
        ps, bs, t = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_double()
        self._check(self._lib.hb_integrator_stats(self._h, ctypes.byref(ps), ctypes.byref(bs),
                                                  ctypes.byref(t)), "integrator_stats")
        return ps.value, bs.value, t.value

    def integrator_dump(self, path, dumpid: int = 0, init_energy: float = 0.0,
                        prev_energy: float = 0.0):
        """Checkpoint the device integrator in the reference's dump format
        (every particle must be at the block time: a multiple of dtmax)."""
        self._check(self._lib.hb_integrator_dump(self._h, str(path).encode(), int(dumpid),
                                                 float(init_energy), float(prev_energy)),
                    "integrator_dump")

    def integrator_restore(self, path, eps2: float, eta: float, dtmax: float):
        """Restore a dump (ours or the reference's) and prepare the integrator
        as the reference's restore + reinitialize_steps; returns (dumpid,
        initial energy, previous energy)."""
        d, e0, e1 = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.hb_integrator_restore(self._h, str(path).encode(), float(eps2),
                                                    float(eta), float(dtmax), ctypes.byref(d),
                                                    ctypes.byref(e0), ctypes.byref(e1)),
                    "integrator_restore")
        return d.value, e0.value, e1.value

    def energy(self, eps2: float):
        ke, pe = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.hb_energy(self._h, float(eps2), ctypes.byref(ke), ctypes.byref(pe)),
                    "energy")
        return ke.value, pe.value

    def get_records(self, addr0: int = 0, count: int | None = None, with_dt: bool = False):
        count = self.nbody - addr0 if count is None else int(count)
        rec = np.empty((count, self.R))
        dt = np.empty(count) if with_dt else None
        self._check(self._lib.hb_get_records(self._h, int(addr0), count, _dptr(rec),
                                             _dptr(dt) if with_dt else None), "get_records")
        return (rec, dt) if with_dt else rec


class Ensemble:
    """Independent clusters integrated together on the device; each particle
    interacts only with its own cluster."""

    def __init__(self, order: int, sizes, precision="mixed"):
        self._lib = load_library()
        self.order = int(order)
        self.sizes = [int(n) for n in sizes]
        self.R, self.F = record_words(self.order), force_words(self.order)
        arr = (ctypes.c_int * len(self.sizes))(*self.sizes)
        h = ctypes.c_void_p()
        st = self._lib.hb_ens_create(self.order, len(self.sizes), arr, _PREC[precision],
                                     ctypes.byref(h))
        if st != 0:
            raise HermiteError(st, "hb_ens_create: " + self._lib.hb_status_string(st).decode())
        self._h = h

    def _check(self, st, what):
        if st != 0:
            msg = self._lib.hb_ens_last_error(self._h).decode() or self._lib.hb_status_string(st).decode()
            raise HermiteError(st, f"{what}: {msg}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.hb_ens_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_cluster(self, c: int, records: np.ndarray, eps2: float):
        rec = np.ascontiguousarray(records, dtype=np.float64).reshape(-1, self.R)
        if rec.shape[0] != self.sizes[c]:
            raise ValueError(f"cluster {c} has {self.sizes[c]} particles")
        self._check(self._lib.hb_ens_set_cluster(self._h, int(c), _dptr(rec), float(eps2)),
                    "set_cluster")

    def get_cluster(self, c: int, with_dt: bool = False):
        rec = np.empty((self.sizes[c], self.R))
        dt = np.empty(self.sizes[c]) if with_dt else None
        self._check(self._lib.hb_ens_get_cluster(self._h, int(c), _dptr(rec),
                                                 _dptr(dt) if with_dt else None), "get_cluster")
        return (rec, dt) if with_dt else rec

    def init(self, tsys: float, eta: float, eta_s: float, dtmax: float):
        self._check(self._lib.hb_ens_init(self._h, float(tsys), float(eta), float(eta_s),
                                          float(dtmax)), "init")

    def run(self, tend: float, max_block_steps: int = 0):
        self._check(self._lib.hb_ens_run(self._h, float(tend), int(max_block_steps)), "run")

    def set_engine(self, engine: str = "auto", team_ctas: int = 0):
        """"auto", "graph" (lockstep over the union of clusters) or "team"
        (each cluster on its own block steps, one thread-block cluster each)."""
        self._check(self._lib.hb_ens_set_engine(self._h, ENGINES[engine], int(team_ctas)),
                    "set_engine")

    def cluster_engine(self, c: int):
        """("team", CTAs) or ("graph", 0): how run() integrates cluster c."""
        e, k = ctypes.c_int(), ctypes.c_int()
        self._check(self._lib.hb_ens_cluster_engine(self._h, int(c), ctypes.byref(e),
                                                    ctypes.byref(k)), "cluster_engine")
        return {v: n for n, v in ENGINES.items()}[e.value], k.value

    def cluster_stats(self, c: int):
        """(particle steps, block steps, time) of cluster c."""
        ps, bs, t = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_double()
        self._check(self._lib.hb_ens_cluster_stats(self._h, int(c), ctypes.byref(ps),
                                                   ctypes.byref(bs), ctypes.byref(t)),
                    "cluster_stats")
        return ps.value, bs.value, t.value

    def stats(self):
        """Sums over clusters: (particle steps, block steps, earliest time,
        interactions)."""
        ps, bs = ctypes.c_longlong(), ctypes.c_longlong()
        t, inter = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.hb_ens_stats(self._h, ctypes.byref(ps), ctypes.byref(bs),
                                           ctypes.byref(t), ctypes.byref(inter)), "stats")
        return ps.value, bs.value, t.value, inter.value

    def energy(self):
        ke = np.empty(len(self.sizes))
        pe = np.empty(len(self.sizes))
        self._check(self._lib.hb_ens_energy(self._h, _dptr(ke), _dptr(pe)), "energy")
        return ke, pe
