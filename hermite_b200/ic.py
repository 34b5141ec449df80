"""Initial conditions and snapshot I/O in the reference's formats.

* `plummer(n, seed, ...)` -- Plummer sphere by the Aarseth-Henon-Wielen
  rejection method the reference's generator uses (RUN/gen-plum.c:116-181:
  radius from the inverted cumulative mass, isotropic direction, speed by
  rejection on q^2 (1-q^2)^(7/2)), scaled by conv = 3*pi/16 so that G = M = 1
  and E ~ -1/4 (RUN/gen-plum.c:104), centre-of-mass corrected
  (RUN/gen-plum.c:187-226).  Generalised: any n, a seeded numpy PCG64 stream
  instead of glibc rand(), an optional power-law mass function, and an
  optional exact rescale to E = -1/4 with virial ratio 1/2.
* `write_snapshot` / `read_snapshot` -- the hex-float text format read by
  NbodySystem::read_snapshot_masaki (SRC/nbodysystem.h:379-403) and written by
  write_snapshot_masaki (:359-378) and gen-plum (RUN/gen-plum.c:240-252),
  through the library's multi-threaded reader and writer
  (hb_snapshot_read / hb_snapshot_write).  `read_snapshot_py` and
  `write_snapshot_py` are plain-Python equivalents (no library needed).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Snapshot:
    snapid: int
    t: float
    ids: np.ndarray     # (n,) int64
    mass: np.ndarray    # (n,)
    pos: np.ndarray     # (n, 3)
    vel: np.ndarray     # (n, 3)
    pot: np.ndarray     # (n,)  (NaN when unknown)

    @property
    def n(self) -> int:
        return int(self.mass.shape[0])


def _plummer_unit(n: int, rng: np.random.Generator, rmax: float = 100.0):
    """Positions and velocities in the G = M = a = 1 Plummer model."""
    pos = np.empty((n, 3))
    vel = np.empty((n, 3))
    filled = 0
    while filled < n:
        m = (n - filled) * 11 // 10 + 16
        x1, x2, x3 = rng.random(m), rng.random(m), rng.random(m)
        with np.errstate(divide="ignore", invalid="ignore"):
            r = 1.0 / np.sqrt(x1 ** (-2.0 / 3.0) - 1.0)
        keep = np.isfinite(r) & (r < rmax)
        r, x2, x3 = r[keep], x2[keep], x3[keep]
        k = min(r.size, n - filled)
        r, x2, x3 = r[:k], x2[:k], x3[:k]
        z = (1.0 - 2.0 * x2) * r
        rho = np.sqrt(np.maximum(r * r - z * z, 0.0))
        pos[filled:filled + k, 0] = rho * np.cos(2.0 * math.pi * x3)
        pos[filled:filled + k, 1] = rho * np.sin(2.0 * math.pi * x3)
        pos[filled:filled + k, 2] = z
        ve = math.sqrt(2.0) * (1.0 + r * r) ** -0.25
        # speed fraction q by rejection: accept when 0.1*x5 < q^2 (1-q^2)^3.5
        q = np.empty(k)
        todo = np.arange(k)
        while todo.size:
            x4, x5 = rng.random(todo.size), rng.random(todo.size)
            ok = 0.1 * x5 < x4 * x4 * (1.0 - x4 * x4) ** 3.5
            q[todo[ok]] = x4[ok]
            todo = todo[~ok]
        v = ve * q
        x6, x7 = rng.random(k), rng.random(k)
        vz = (1.0 - 2.0 * x6) * v
        vr = np.sqrt(np.maximum(v * v - vz * vz, 0.0))
        vel[filled:filled + k, 0] = vr * np.cos(2.0 * math.pi * x7)
        vel[filled:filled + k, 1] = vr * np.sin(2.0 * math.pi * x7)
        vel[filled:filled + k, 2] = vz
        filled += k
    return pos, vel


def power_law_masses(n: int, rng: np.random.Generator, slope: float = -2.35,
                     mmin: float = 0.1, mmax: float = 100.0) -> np.ndarray:
    """dN/dm ~ m^slope on [mmin, mmax], normalised to total mass 1."""
    a = slope + 1.0
    u = rng.random(n)
    m = (mmin ** a + u * (mmax ** a - mmin ** a)) ** (1.0 / a)
    return m / m.sum()


def energies(mass, pos, vel, eps2: float = 0.0):
    """(kinetic, potential) by direct summation (small n only)."""
    ke = 0.5 * float(np.sum(mass * np.sum(vel * vel, axis=1)))
    pe = 0.0
    for i in range(mass.shape[0] - 1):
        d = pos[i + 1:] - pos[i]
        r = np.sqrt(np.sum(d * d, axis=1) + eps2)
        pe -= float(mass[i] * np.sum(mass[i + 1:] / r))
    return ke, pe


def plummer(n: int, seed: int = 0, masses: np.ndarray | None = None,
            exact_henon: bool = False, eps2_for_scaling: float = 0.0) -> Snapshot:
    rng = np.random.default_rng(seed)
    pos, vel = _plummer_unit(n, rng)
    conv = 3.0 * math.pi / 16.0
    pos *= conv
    vel /= math.sqrt(conv)
    mass = np.full(n, 1.0 / n) if masses is None else np.asarray(masses, dtype=np.float64)
    mtot = mass.sum()
    pos -= (mass[:, None] * pos).sum(axis=0) / mtot
    vel -= (mass[:, None] * vel).sum(axis=0) / mtot
    if exact_henon:
        ke, pe = energies(mass, pos, vel, eps2_for_scaling)
        # virial ratio 1/2 then E = -1/4 (G = M = 1)
        vel *= math.sqrt(-0.5 * pe / ke)
        scale = (0.5 * pe) / -0.25
        pos *= scale
        vel /= math.sqrt(scale)
    return Snapshot(0, 0.0, np.arange(n, dtype=np.int64), mass, pos, vel, np.full(n, np.nan))


def _hexf(x: float) -> str:
    return float(x).hex().upper() if math.isfinite(x) else ("NAN" if x != x else
                                                             ("INF" if x > 0 else "-INF"))


def write_snapshot_py(path, snap: Snapshot) -> None:
    with open(path, "w") as fp:
        fp.write(f"{snap.snapid}\n{snap.n}\n{snap.t:f}\n")
        for i in range(snap.n):
            p, v = snap.pos[i], snap.vel[i]
            fp.write(f"{int(snap.ids[i]):6d}    {_hexf(snap.mass[i])}    "
                     f"{_hexf(p[0])} {_hexf(p[1])} {_hexf(p[2])}    "
                     f"{_hexf(v[0])} {_hexf(v[1])} {_hexf(v[2])}    {_hexf(snap.pot[i])}\n")


def _parse(tok: str) -> float:
    t = tok.lower()
    if "0x" in t:
        return float.fromhex(t)
    return float(t)


def read_snapshot_py(path) -> Snapshot:
    with open(path) as fp:
        toks = fp.read().split()
    snapid, n, t = int(toks[0]), int(toks[1]), float(toks[2])
    body = toks[3:3 + 9 * n]
    if len(body) != 9 * n:
        raise ValueError(f"{path}: expected {n} particles")
    a = np.array([_parse(s) for s in body], dtype=np.float64).reshape(n, 9)
    return Snapshot(snapid, t, a[:, 0].astype(np.int64), a[:, 1].copy(), a[:, 2:5].copy(),
                    a[:, 5:8].copy(), a[:, 8].copy())


def _dp(a):
    import ctypes
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def write_snapshot(path, snap: Snapshot) -> None:
    import ctypes
    import hermite_b200 as hb
    lib = hb.load_library()
    ids = np.ascontiguousarray(snap.ids, dtype=np.int64)
    mass = np.ascontiguousarray(snap.mass, dtype=np.float64)
    pos = np.ascontiguousarray(snap.pos, dtype=np.float64)
    vel = np.ascontiguousarray(snap.vel, dtype=np.float64)
    pot = np.ascontiguousarray(snap.pot, dtype=np.float64)
    st = lib.hb_snapshot_write(str(path).encode(), int(snap.snapid), snap.n, float(snap.t),
                               ids.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), _dp(mass),
                               _dp(pos), _dp(vel), _dp(pot))
    if st != 0:
        raise hb.HermiteError(st, f"hb_snapshot_write {path}")


def read_snapshot(path) -> Snapshot:
    import ctypes
    import hermite_b200 as hb
    lib = hb.load_library()
    sid, n, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    st = lib.hb_snapshot_read_header(str(path).encode(), ctypes.byref(sid), ctypes.byref(n),
                                     ctypes.byref(t))
    if st != 0:
        raise hb.HermiteError(st, f"hb_snapshot_read_header {path}")
    ids = np.empty(n.value, dtype=np.int64)
    mass, pot = np.empty(n.value), np.empty(n.value)
    pos, vel = np.empty((n.value, 3)), np.empty((n.value, 3))
    st = lib.hb_snapshot_read(str(path).encode(), n.value,
                              ids.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong)), _dp(mass),
                              _dp(pos), _dp(vel), _dp(pot))
    if st != 0:
        raise hb.HermiteError(st, f"hb_snapshot_read {path}")
    return Snapshot(sid.value, t.value, ids, mass, pos, vel, pot)


def records(snap: Snapshot, order: int, tlast: float = 0.0,
            derivs: np.ndarray | None = None) -> np.ndarray:
    """j-particle records (n, 8 + 3*(order-2)) from a snapshot."""
    n = snap.n
    rec = np.zeros((n, 8 + 3 * (order - 2)))
    rec[:, 0:3] = snap.pos
    rec[:, 3] = snap.mass
    rec[:, 4:7] = snap.vel
    rec[:, 7] = tlast
    if derivs is not None:
        rec[:, 8:] = derivs.reshape(n, -1)
    return rec
