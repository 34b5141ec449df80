"""Checkpoints in the reference's dump format (hb_dump_*, hb_integrator_dump /
hb_integrator_restore; NbodySystem::dump / restore, SRC/nbodysystem.h:405-458).

* Host (CPU): the reader and writer round-trip records exactly, and a dump
  written by the reference's own integrator (oracle/_ref/avx2-{4,6,8}) is read
  and written back byte for byte.
* Device (GPU): a run restored from a dump takes the same block steps as the
  reference's integrator restored from the same file (the restore recomputes
  every dt with Particle::recalc_dt, so the continuation differs from the
  uninterrupted run; both sides must agree on it), for a dump written by the
  reference and for a dump written by the device integrator.
"""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import hermite_b200 as hb
from kat import GEN_PLUM, ROOT

HB_ERR_IO = 8
ETA = {4: (0.1, 0.01), 6: (0.5, 0.1), 8: (0.75, 0.1)}


def ref_app(order):
    # order code 9: the reference's integrator with double-double positions
    app = ROOT / "oracle" / "_ref" / ("generic-8dd" if order == 9 else f"avx2-{order}")
    if not app.exists() or not GEN_PLUM.exists():
        pytest.skip("the reference's integrator is not built (needs the reference sources)")
    return app


def run_ref(app, order, workdir, tend, start, dump_interval=None, dumpout=None):
    """Run the reference integrator from a snapshot (start = ("snap", name)) or
    a dump (("dump", name)); returns the mean-nact strings ("%f") it prints
    per log interval (NbodySystem::print_stat)."""
    eta, eta_s = ETA[min(order, 8)]
    lines = [f"order {min(order, 8)}", f"eta {eta}", f"eta_s {eta_s}", f"tend {tend!r}", "dtmaxinv 16",
             "kt_for_eps 1.0", "log_interval 0.125", "snap_interval 100.0",
             f"dump_interval {dump_interval or 100.0!r}"]
    lines.append(("snapin " if start[0] == "snap" else "dumpin ") + start[1])
    if dumpout:
        lines.append(f"dumpout_base {dumpout}")
    r = subprocess.run([str(app)], input="\n".join(lines) + "\n", cwd=workdir, capture_output=True,
                       text=True, timeout=600, env={"OMP_NUM_THREADS": "4", "PATH": "/usr/bin:/bin"})
    assert r.returncode == 0, r.stderr[-2000:]
    return re.findall(r"nact : (\S+)", r.stderr)


@pytest.mark.parametrize("order", [4, 6, 8, 9])
def test_host_round_trip(order, tmp_path):
    n, R = 37, hb.record_words(order)
    rng = np.random.default_rng(order)
    rec = rng.normal(size=(n, R)) * np.exp(rng.normal(size=(n, R)) * 20)
    rec[:, 7] = 0.375
    aux = rng.normal(size=(n, hb.AUX_WORDS))
    ids = rng.permutation(n) + 1000
    hb.write_dump(tmp_path / "d.dat", order, rec, aux, 0.375, dumpid=7, energies=(-0.25, -0.2501),
                  steps=(12345, 678), ids=ids)
    d = hb.read_dump(tmp_path / "d.dat", dd=order == 9)
    assert (d["order"], d["dumpid"], d["nbody"], d["tsys"]) == (order, 7, n, 0.375)
    assert d["energies"] == (-0.25, -0.2501) and d["steps"] == (12345, 678)
    np.testing.assert_array_equal(d["ids"], ids)
    np.testing.assert_array_equal(d["records"], rec)
    np.testing.assert_array_equal(d["aux"], aux)


@pytest.mark.parametrize("order", [4, 6, 8, 9])
def test_reference_dump_rewritten_byte_for_byte(order, tmp_path):
    app = ref_app(order)
    subprocess.run([str(GEN_PLUM), "1"], cwd=tmp_path, check=True, capture_output=True)
    run_ref(app, order, tmp_path, 0.125, ("snap", "pl1k.dat"), dump_interval=0.125,
            dumpout="dump%d.dat")
    src = tmp_path / "dump1.dat"
    d = hb.read_dump(src, dd=order == 9)
    assert d["order"] == order and d["nbody"] == 1024 and d["tsys"] == 0.125
    if order == 9:
        assert np.any(d["records"][:, 26:29] != 0.0)     # the low parts are in the file
    hb.write_dump(tmp_path / "again.dat", order, d["records"], d["aux"], d["tsys"],
                  dumpid=d["dumpid"], energies=d["energies"], steps=d["steps"], ids=d["ids"])
    assert (tmp_path / "again.dat").read_bytes() == src.read_bytes()


def test_read_errors(tmp_path):
    lib = hb.load_library()
    with pytest.raises(hb.HermiteError) as e:
        hb.read_dump(tmp_path / "missing.dat")
    assert e.value.status == HB_ERR_IO
    rec = np.zeros((3, hb.record_words(4)))
    hb.write_dump(tmp_path / "d4.dat", 4, rec, np.zeros((3, 6)), 0.0)
    out = np.empty((3, hb.record_words(6)))
    aux = np.empty((3, 6))
    # a 4th-order dump read as 6th order, or with the wrong N
    assert lib.hb_dump_read(str(tmp_path / "d4.dat").encode(), 6, 3, None,
                            out.ctypes.data_as(hb.ctypes.POINTER(hb.ctypes.c_double)),
                            aux.ctypes.data_as(hb.ctypes.POINTER(hb.ctypes.c_double))) == HB_ERR_IO
    out4 = np.empty((4, hb.record_words(4)))
    aux4 = np.empty((4, 6))
    assert lib.hb_dump_read(str(tmp_path / "d4.dat").encode(), 4, 4, None,
                            out4.ctypes.data_as(hb.ctypes.POINTER(hb.ctypes.c_double)),
                            aux4.ctypes.data_as(hb.ctypes.POINTER(hb.ctypes.c_double))) == HB_ERR_IO


def _restored_nact(order, path, engine, tend=0.25):
    d = hb.read_dump(path, dd=order == 9)
    n = d["nbody"]
    eps = 4.0 / n                            # kt_for_eps 1.0 (set_thermal_eps)
    eta, _ = ETA[min(order, 8)]
    with hb.Gravity(min(order, 8), n, "dd" if order == 9 else "fp64") as g:
        g.set_engine(engine)
        did, e0, e1 = g.integrator_restore(path, eps * eps, eta, 1.0 / 16)
        assert (did, e0, e1) == (d["dumpid"], *d["energies"])
        ps0, bs0, t0 = g.integrator_stats()
        assert (ps0, bs0, t0) == (*d["steps"], d["tsys"])
        g.integrator_run(tend)
        ps, bs, t = g.integrator_stats()
    assert t == tend
    return "%f" % ((ps - ps0) / (bs - bs0))


@pytest.mark.gpu
@pytest.mark.parametrize("engine", ["graph", "team"])
@pytest.mark.parametrize("order", [4, 6, 8, 9])
def test_restore_agrees_with_reference_restore(order, engine, tmp_path):
    app = ref_app(order)
    subprocess.run([str(GEN_PLUM), "1"], cwd=tmp_path, check=True, capture_output=True)
    run_ref(app, order, tmp_path, 0.125, ("snap", "pl1k.dat"), dump_interval=0.125,
            dumpout="dump%d.dat")
    ref_rows = run_ref(app, order, tmp_path, 0.25, ("dump", "dump1.dat"))
    assert _restored_nact(order, tmp_path / "dump1.dat", engine) == ref_rows[0]


@pytest.mark.gpu
@pytest.mark.parametrize("order", [4, 6, 8])
def test_device_dump_restores_in_reference(order, tmp_path):
    from hermite_b200.ic import read_snapshot, records
    app = ref_app(order)
    subprocess.run([str(GEN_PLUM), "1"], cwd=tmp_path, check=True, capture_output=True)
    snap = read_snapshot(tmp_path / "pl1k.dat")
    n = snap.n
    eps = 4.0 / n
    eta, eta_s = ETA[order]
    with hb.Gravity(order, n, "fp64") as g:
        g.set_jp_records(records(snap, order))
        g.integrator_init(0.0, eps * eps, eta, eta_s, 1.0 / 16)
        ke, pe = g.energy(eps * eps)
        g.integrator_run(0.125)
        g.integrator_dump(tmp_path / "ours.dat", 1, ke + pe, ke + pe)
        g.integrator_run(0.125 + 1.0 / 1024)      # a block time where not all particles are
        with pytest.raises(hb.HermiteError) as e:
            g.integrator_dump(tmp_path / "bad.dat", 2, 0.0, 0.0)
        assert e.value.status == 6                # HB_ERR_STATE
    # the reference's own dump at the same time has the same step counters
    run_ref(app, order, tmp_path, 0.125, ("snap", "pl1k.dat"), dump_interval=0.125,
            dumpout="ref%d.dat")
    ours, ref = hb.read_dump(tmp_path / "ours.dat"), hb.read_dump(tmp_path / "ref1.dat")
    assert ours["steps"] == ref["steps"] and ours["tsys"] == ref["tsys"] == 0.125
    ref_rows = run_ref(app, order, tmp_path, 0.25, ("dump", "ours.dat"))
    assert _restored_nact(order, tmp_path / "ours.dat", "auto") == ref_rows[0]
