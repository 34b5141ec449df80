"""The force kernel's bounded waits, exercised on the GPU without a fault.

Every wait of the force kernel for an incoming j tile is bounded; when it gives
up, the kernel raises the context's error flag, waits (with the full bound) for
the bulk copies it has already issued, and returns, and the host call returns
HB_ERR_DEVICE_TIMEOUT.  hb_set_wait_limit(ctx, 0) makes those waits give up at
once, so the path runs on a small case here; the same context must then give
the oracle's forces with the default limit restored.  The reference's CUDA
path has no such path: it aborts (SRC/cuda_pointer.h:6-10).
"""
import pytest

import hermite_b200 as hb
from inputs import make_records, rel_err

EPS2 = (1.0 / 256) ** 2
HB_ERR_DEVICE_TIMEOUT = 4
TOL = {"fp64": 1e-12, "mixed": 1e-5}


@pytest.mark.gpu
@pytest.mark.parametrize("order,precision,variant,jsplit", [
    (4, "fp64", 0, 1),     # two-pass shape, one slice: no partials
    (6, "mixed", 1, 4),    # 2 i-chunks per warp, four j-slices
    (8, "fp64", 2, 8),     # four warps split every tile, eight j-slices
    (4, "fp64", 12, 2),    # fused predict + force: the i-record wait gives up
])
def test_wait_timeout_reported_and_context_recovers(order, precision, variant, jsplit, oracle):
    n, nact = 4096, 1000
    rec = make_records(order, n, seed=17 + order)
    ref = oracle.predict_force(order, rec, 0.0, nact, EPS2)
    with hb.Gravity(order, n, precision) as g:
        g.set_jp_records(rec)
        g.predict_all(0.0)
        g.set_force_shape(variant, jsplit)
        g.set_wait_limit(0)
        with pytest.raises(hb.HermiteError) as ei:
            g.calc_force_on_first_nact(nact, EPS2)
        assert ei.value.status == HB_ERR_DEVICE_TIMEOUT
        g.set_wait_limit(-1)
        got = g.calc_force_on_first_nact(nact, EPS2)
        again = g.calc_force_on_first_nact(nact, EPS2)
    err = rel_err(got, ref)
    assert err[:, 0].max() <= TOL[precision], err.max(axis=0)
    assert (got == again).all()


@pytest.mark.gpu
@pytest.mark.parametrize("order", [4, 6, 8])
def test_small_step_kernel_wait_timeout(order, oracle):
    """The small-step kernel (automatic shape, FP64, nact <= 16) waits on the
    bulk copies of each warp's raw chunks with the same bounded waits: with
    the limit at 0 the call reports HB_ERR_DEVICE_TIMEOUT, and the context
    then gives the oracle's forces."""
    n, nact = 20000, 3
    rec = make_records(order, n, seed=23 + order)
    ref = oracle.predict_force(order, rec, 0.0, nact, EPS2)
    with hb.Gravity(order, n, "fp64") as g:
        g.set_jp_records(rec)
        g.predict_all(0.0)
        g.set_wait_limit(0)
        with pytest.raises(hb.HermiteError) as ei:
            g.calc_force_on_first_nact(nact, EPS2)
        assert ei.value.status == HB_ERR_DEVICE_TIMEOUT
        g.set_wait_limit(-1)
        got = g.calc_force_on_first_nact(nact, EPS2)
    assert rel_err(got, ref).max() <= TOL["fp64"]
