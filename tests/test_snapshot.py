"""Snapshots in the reference's text format (hb_snapshot_*; read_snapshot_masaki
/ write_snapshot_masaki, SRC/nbodysystem.h:359-403).  CPU only.

* The library's multi-threaded reader agrees with the plain-Python reader on
  files written by the reference's generator (RUN/gen-plum.c) and by the
  reference's integrator.
* A snapshot written by the reference's integrator is written back byte for
  byte (same %A formatting as the C library's printf).
* Round trips keep every bit, including signed zeros, tiny and huge values.
"""
import subprocess

import numpy as np
import pytest

from hermite_b200.ic import (Snapshot, plummer, read_snapshot, read_snapshot_py, write_snapshot,
                             write_snapshot_py)
from kat import GEN_PLUM, ROOT


def _same(a: Snapshot, b: Snapshot):
    assert (a.snapid, a.t, a.n) == (b.snapid, b.t, b.n)
    for f in ("ids", "mass", "pos", "vel"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    np.testing.assert_array_equal(np.nan_to_num(a.pot, nan=7.0), np.nan_to_num(b.pot, nan=7.0))


def _gen_plum(tmp_path, nk=1):
    if not GEN_PLUM.exists():
        pytest.skip("gen-plum not built (needs the reference sources)")
    subprocess.run([str(GEN_PLUM), str(nk)], cwd=tmp_path, check=True, capture_output=True)
    return tmp_path / f"pl{nk}k.dat"


def test_reader_matches_python_on_gen_plum(tmp_path):
    path = _gen_plum(tmp_path, 2)
    _same(read_snapshot(path), read_snapshot_py(path))


def test_reference_snapshot_rewritten_byte_for_byte(tmp_path):
    app = ROOT / "oracle" / "_ref" / "avx2-4"
    if not app.exists():
        pytest.skip("the reference's integrator is not built")
    _gen_plum(tmp_path)
    inp = ("order 4\neta 0.1\neta_s 0.01\nsnapin pl1k.dat\ntend 0.125\ndtmaxinv 16\n"
           "kt_for_eps 1.0\nlog_interval 0.125\nsnap_interval 0.125\nsnapout_base snap%d.dat\n"
           "dump_interval 100.0\n")
    r = subprocess.run([str(app)], input=inp, cwd=tmp_path, capture_output=True, text=True,
                       timeout=600, env={"OMP_NUM_THREADS": "4", "PATH": "/usr/bin:/bin"})
    assert r.returncode == 0, r.stderr[-1000:]
    src = tmp_path / "snap1.dat"
    snap = read_snapshot(src)
    _same(snap, read_snapshot_py(src))
    assert snap.n == 1024 and snap.t == 0.125 and np.all(np.isfinite(snap.pot))
    write_snapshot(tmp_path / "again.dat", snap)
    assert (tmp_path / "again.dat").read_bytes() == src.read_bytes()


def test_round_trip_every_bit(tmp_path):
    rng = np.random.default_rng(5)
    n = 20011
    s = plummer(n, 3)
    s.pos[0] = [0.0, -0.0, 5e-324]
    s.vel[1] = [1e300, -2.5e-310, 1.0]
    s.pot = rng.normal(size=n)
    s.ids = rng.permutation(n) * 7
    write_snapshot(tmp_path / "a.dat", s)
    got = read_snapshot(tmp_path / "a.dat")
    _same(got, s)
    assert np.signbit(got.pos[0, 1])
    _same(read_snapshot_py(tmp_path / "a.dat"), s)
    write_snapshot_py(tmp_path / "b.dat", s)         # Python's own %A spelling parses the same
    _same(read_snapshot(tmp_path / "b.dat"), s)


def test_read_errors(tmp_path):
    import hermite_b200 as hb
    with pytest.raises(hb.HermiteError):
        read_snapshot(tmp_path / "missing.dat")
    (tmp_path / "short.dat").write_text("0\n3\n0.000000\n1 0X1P+0 0 0 0 0 0 0 0\n")
    with pytest.raises(hb.HermiteError):
        read_snapshot(tmp_path / "short.dat")
