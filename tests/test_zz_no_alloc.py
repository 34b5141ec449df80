"""The allocation-free force entry point, hb_force_predicted_noalloc.

It serves callers that cannot call cudaMalloc: code inside a host framework
that owns all device memory through its own pool (an allocation behind the
pool's back breaks its accounting or fails against its reservation), and
fixed-budget jobs on a shared GPU that must not grow their footprint.
They pass their own device buffers (predicted j-particles in, forces out) and
the entry point uses only its own static device scratch.

Checked here through the C ABI against the context path
(hb_create / set_jp / predict_all / calc_force_on_first_nact) on the same
particles, within the tolerances of tests/test_gpu_parity.py, over two calls
in a row with different shapes (the second call reuses the shared scratch the
first one left behind), plus a repeat of the first call.  This file is
collected last so that a run stopping at the first failure has run every
other test before it.
"""
import ctypes

import numpy as np
import pytest

import hermite_b200 as hb
from inputs import make_records, rel_err

FP64_TOL = 1e-12
MIXED_TOL = {0: 1e-6, 1: 1e-5, 2: 1e-4, 3: 1e-2}
EPS2 = (1.0 / 256) ** 2
HB_ERR_INVALID, HB_ERR_TOO_LARGE = 1, 7


def pack_predicted(order, precision, pred, nslots):
    """The library's AoSoA32 predicted layout from oracle-predicted states
    pos[3] mass vel[3] [acc[3]] [jrk[3]] (n rows); slots past n are
    zero-mass padding at distinct far-away positions."""
    n, p = pred.shape
    full = np.zeros((nslots, p))
    full[:n] = pred
    slots = np.arange(n, nslots)
    for k in range(3):
        full[n:, k] = 2.0 ** 40 + (slots * 3 + k)
    if precision == "fp64":
        comps = full
        dtype = np.float64
    else:
        hi = full[:, 0:3].astype(np.float32)
        lo = (full[:, 0:3] - hi.astype(np.float64)).astype(np.float32)
        comps = np.concatenate([hi, lo, full[:, 3:].astype(np.float32)], axis=1)
        dtype = np.float32
    nc = comps.shape[1]
    return np.ascontiguousarray(comps.reshape(nslots // 32, 32, nc).transpose(0, 2, 1),
                                dtype=dtype)


def test_rejects_sizes_beyond_capacity():
    lib = hb.load_library()
    dummy = ctypes.c_void_p(256)           # never dereferenced: the checks come first
    assert lib.hb_force_predicted_noalloc(4, 0, dummy, (1 << 20) + 256, 1, EPS2, dummy, None) \
        == HB_ERR_TOO_LARGE
    assert lib.hb_force_predicted_noalloc(4, 0, dummy, 1000, 1, EPS2, dummy, None) == HB_ERR_INVALID
    assert lib.hb_force_predicted_noalloc(5, 0, dummy, 1024, 1, EPS2, dummy, None) == HB_ERR_INVALID
    assert lib.hb_force_predicted_noalloc(4, 0, dummy, 1024, 2000, EPS2, dummy, None) == HB_ERR_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("order", [4, 6, 8])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_noalloc_matches_context_path(order, precision, oracle):
    import torch
    lib = hb.load_library()
    n, nslots = 3000, 3072
    rec = make_records(order, n, seed=31 + order)
    pred = oracle.predict(order, rec, 0.0)
    d_pred = torch.from_numpy(pack_predicted(order, precision, pred, nslots)).cuda()
    F = hb.force_words(order)
    prec_code = hb.FP64 if precision == "fp64" else hb.MIXED
    stream = torch.cuda.current_stream().cuda_stream

    def noalloc(nact):
        out = torch.full((nact, F), float("nan"), dtype=torch.float64, device="cuda")
        st = lib.hb_force_predicted_noalloc(order, prec_code, ctypes.c_void_p(d_pred.data_ptr()),
                                            nslots, nact, EPS2, ctypes.c_void_p(out.data_ptr()),
                                            ctypes.c_void_p(stream))
        assert st == 0, lib.hb_status_string(st)
        torch.cuda.synchronize()
        return out.cpu().numpy()

    with hb.Gravity(order, n, precision) as g:
        g.set_jp_records(rec)
        g.predict_all(0.0)
        ref = {nact: g.calc_force_on_first_nact(nact, EPS2) for nact in (7, 1000)}

    first = noalloc(7)          # small nact: j-split over many CTAs, uses the scratch
    second = noalloc(1000)      # second call in a row, different launch shape
    again = noalloc(7)
    for nact, got in ((7, first), (1000, second), (7, again)):
        assert np.all(np.isfinite(got))
        err = rel_err(got, ref[nact])
        for k in range(err.shape[1]):
            tol = FP64_TOL if precision == "fp64" else MIXED_TOL[k]
            assert err[:, k].max() <= tol, (order, precision, nact, k, err[:, k].max())
    assert np.array_equal(first, again)


@pytest.mark.gpu
@pytest.mark.parametrize("order,n,nacts", [
    # 8th order, nact 16384: the j-split wanted for occupancy (5 slices) needs
    # more than the 4 MiB of partials, so the call takes fewer slices
    (8, 65536, (16384, 5000)),
    # 4th order, nact = N = 2^18: enough i-tiles to fill the GPU, one slice
    # (no partials, no counters), then a split call after it
    (4, 262144, (262144, 64)),
])
def test_noalloc_large_shapes(order, n, nacts, oracle):
    import torch
    lib = hb.load_library()
    nslots = n
    rec = make_records(order, n, seed=7 + order)
    pred = oracle.predict(order, rec, 0.0)
    d_pred = torch.from_numpy(pack_predicted(order, "fp64", pred, nslots)).cuda()
    F = hb.force_words(order)
    stream = torch.cuda.current_stream().cuda_stream
    with hb.Gravity(order, n, "fp64") as g:
        g.set_jp_records(rec)
        g.predict_all(0.0)
        ref = {nact: g.calc_force_on_first_nact(nact, EPS2) for nact in nacts}
    for nact in nacts:          # two calls in a row on the shared scratch
        out = torch.full((nact, F), float("nan"), dtype=torch.float64, device="cuda")
        st = lib.hb_force_predicted_noalloc(order, hb.FP64, ctypes.c_void_p(d_pred.data_ptr()),
                                            nslots, nact, EPS2, ctypes.c_void_p(out.data_ptr()),
                                            ctypes.c_void_p(stream))
        assert st == 0, lib.hb_status_string(st)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_err(got, ref[nact]).max() <= FP64_TOL, (order, nact)
