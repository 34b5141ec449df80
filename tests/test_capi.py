"""C ABI checks that need no GPU: the library loads, exports every entry
point include/hermite_b200.h declares, and rejects bad arguments before it
touches a device."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import hermite_b200 as hb

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "hermite_b200.h"


def declared_entry_points():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(hb_[a-z_0-9]+)\s*\(", text)))


def test_header_and_python_binding_agree():
    assert declared_entry_points() == sorted(hb.EXPORTED_SYMBOLS)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(hb.library_path()))
    missing = [s for s in declared_entry_points() if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings():
    lib = hb.load_library()
    assert lib.hb_status_string(0) == b"ok"
    assert lib.hb_status_string(4) == b"device-side wait timed out"
    assert lib.hb_last_error(None) == b"null context"


@pytest.mark.parametrize("order,n,prec", [(5, 10, 0), (4, 0, 0), (4, 1 << 25, 0), (6, 10, 7)])
def test_create_rejects_bad_arguments(order, n, prec):
    lib = hb.load_library()
    h = ctypes.c_void_p()
    assert lib.hb_create(order, n, prec, ctypes.byref(h)) == 1   # HB_ERR_INVALID
    assert not h.value


def test_null_context_is_rejected():
    lib = hb.load_library()
    assert lib.hb_predict_all(None, 0.0) == 1
    assert lib.hb_force_first_nact(None, 1, 0.0, None) == 1
    assert lib.hb_destroy(None) == 0
    assert lib.hb_set_wait_limit(None, 0) == 1
    assert lib.hb_integrator_set_engine(None, 3, 0) == 1       # HB_ENGINE_PERSISTENT


def test_engine_names_match_the_header():
    """The Python engine names map to the header's HB_ENGINE_* values."""
    import re
    from pathlib import Path
    header = (Path(hb.__file__).resolve().parent.parent / "include" / "hermite_b200.h").read_text()
    enum = re.search(r"enum \{ HB_ENGINE_AUTO = 0,[^}]*\}", header).group(0)
    values = {m.group(1).lower(): int(m.group(2)) for m in re.finditer(r"HB_ENGINE_(\w+) = (\d+)", enum)}
    assert values == {k: v for k, v in hb.ENGINES.items()}


def test_no_device_is_reported(cuda_ok):
    if cuda_ok:
        pytest.skip("a CUDA device is present")
    with pytest.raises(hb.HermiteError) as e:
        hb.Gravity(4, 16)
    assert e.value.status == 5                                   # HB_ERR_NO_DEVICE


def test_variant_table():
    for order in (4, 6, 8):
        for prec in (0, 1):
            n = hb.load_library().hb_force_variant_count(order, prec)
            assert n >= 5
            for v in range(n):
                t, ni, wj = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
                assert hb.load_library().hb_force_variant_info(order, prec, v, ctypes.byref(t),
                                                               ctypes.byref(ni), ctypes.byref(wj)) == 0
                assert t.value % 32 == 0 and ni.value >= 1 and wj.value >= 1


def test_drop_in_headers_compile():
    """The C++ drop-in Gravity compiles against stand-ins for the reference's
    Particle/Force types (the full integrator build is in hermite_b200/gravity)."""
    import subprocess
    import tempfile
    src = r'''
#include <cstddef>
struct dvec3 { double x, y, z; };
struct Force { dvec3 acc, jrk, snp; };
struct Particle { long id; double mass, tlast, dt; dvec3 pos, vel, acc, jrk, snp, crk, d4a, d5a; };
#include "hermite6-titan.h"
int main() { return sizeof(Gravity::GParticle) == 160 && sizeof(Gravity::GPredictor) == 80 ? 0 : 1; }
'''
    with tempfile.TemporaryDirectory() as d:
        p = Path(d) / "t.cpp"
        p.write_text(src)
        r = subprocess.run(["g++", "-std=c++11", "-I", str(ROOT / "include"),
                            "-I", str(ROOT / "hermite_b200" / "gravity"), str(p),
                            "-L", str(ROOT / "hermite_b200" / "_lib"), "-lhermite_b200",
                            f"-Wl,-rpath,{ROOT / 'hermite_b200' / '_lib'}", "-o", str(Path(d) / "t")],
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert subprocess.run([str(Path(d) / "t")]).returncode == 0


def test_result_buffers_are_checked():
    """Caller-supplied result arrays are checked before the library writes
    into them: dtype, layout, writeability and size."""
    from hermite_b200 import _out_buffer
    assert _out_buffer(None, 5, 6).shape == (5, 6) and _out_buffer(None, -1, 6).shape == (0, 6)
    ok = np.empty((8, 6))
    assert _out_buffer(ok, 5, 6) is ok
    for bad in (np.empty((4, 6)), np.empty((5, 6), np.float32), np.empty((6, 10))[:, :6],
                [[0.0] * 6] * 5):
        with pytest.raises(ValueError):
            _out_buffer(bad, 5, 6)
    ro = np.empty(100)
    ro.flags.writeable = False
    with pytest.raises(ValueError):
        _out_buffer(ro, 100)


@pytest.mark.parametrize("order", ["FOURTH", "SIXTH", "EIGHTH"])
def test_fast_omp_sync_integrator_builds(order, tmp_path):
    """The reference's -DFAST_OMP_SYNC integrator loop (one OpenMP region
    per dtmax, SRC/nbodysystem.h:767-838) compiles and links against the
    drop-in, which adds the members only its CPU backends had."""
    import subprocess
    gdir = ROOT / "hermite_b200" / "gravity"
    ovl = gdir / "_build" / "overlay"
    if not (ovl / "compile.cpp").exists() or not (gdir / "_build" / "parameter.o").exists():
        pytest.skip("the reference integrator overlay is not built (needs the reference sources)")
    r = subprocess.run(["g++", "-O1", "-fopenmp", "-w", "-I", str(ROOT / "include"), "-I", str(gdir),
                        f"-D{order}", "-DCUDA_TITAN", "-DFAST_OMP_SYNC", "-I", str(ovl),
                        str(ovl / "compile.cpp"), str(gdir / "_build" / "parameter.o"),
                        "-L", str(ROOT / "hermite_b200" / "_lib"), "-lhermite_b200",
                        "-o", str(tmp_path / "app")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
