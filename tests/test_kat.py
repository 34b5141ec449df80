"""nact known-answer test (see tests/kat.py).

GPU: the reference's own integrator (SRC/compile.cpp + SRC/nbodysystem.h,
unmodified) built against the drop-in Gravity of hermite_b200/gravity,
FP64 path, must print the published nact values exactly.
CPU: the reference's AVX2 build (oracle/_ref/avx2-*) prints them too in this
environment -- the fingerprint is a property of the FP64 algorithm, not of
the hardware the logs came from.
"""
import os

import pytest

from kat import GEN_PLUM, PUBLISHED_NACT, ROOT, run_app

APP = ROOT / "hermite_b200" / "gravity" / "_build"
REF_APP = ROOT / "oracle" / "_ref"


def _need(path):
    if not path.exists() or not GEN_PLUM.exists():
        pytest.skip(f"{path.name} or gen-plum not built (needs the reference sources)")


@pytest.mark.gpu
@pytest.mark.parametrize("order,nk", sorted((o, n // 1024) for (o, n) in PUBLISHED_NACT))
def test_nact_fp64_drop_in(order, nk, tmp_path):
    app = APP / f"hb-app-{order}"
    _need(app)
    env = dict(os.environ, HERMITE_B200_PRECISION="fp64", OMP_NUM_THREADS="4")
    nact, out = run_app(app, order, nk, tmp_path, env=env)
    assert tuple(nact) == PUBLISHED_NACT[(order, nk * 1024)], out[-1500:]


@pytest.mark.parametrize("order", [4, 6, 8])
def test_nact_reference_avx2_cpu(order, tmp_path):
    app = REF_APP / f"avx2-{order}"
    _need(app)
    env = dict(os.environ, OMP_NUM_THREADS="4")
    nact, out = run_app(app, order, 1, tmp_path, env=env)
    assert tuple(nact) == PUBLISHED_NACT[(order, 1024)], out[-1500:]
