"""The persistent engine against the graph engine.

The persistent engine runs the graph engine's four phases per block step (next
block time, active set, force work items, corrector) inside one cooperative
kernel, with grid barriers in place of kernel boundaries.  It takes the same
work items, so both engines must give the same block steps and the same
records bit for bit, over runs of more than one launch (4096 block steps per
launch), at every order (mixed precision at 4th order, where it integrates).  Its barrier waits are
bounded: with the wait limit lowered to zero they give up at once, the run
returns HB_ERR_DEVICE_TIMEOUT, and a re-initialised integrator on the same
context integrates correctly afterwards.
"""
import numpy as np
import pytest

import hermite_b200 as hb
from hermite_b200.ic import plummer, records

pytestmark = pytest.mark.gpu
HB_ERR_DEVICE_TIMEOUT = 4


def _run(order, n, precision, engine, eps, eta, eta_s, dtmax, tend, seed=0, max_steps=0):
    with hb.Gravity(order, n, precision) as g:
        g.set_engine(engine)
        assert g.engine()[0] == engine
        g.set_jp_records(records(plummer(n, seed), order))
        g.integrator_init(0.0, eps * eps, eta, eta_s, dtmax)
        g.integrator_run(tend, max_block_steps=max_steps)
        stats = g.integrator_stats()
        rec, dt = g.get_records(with_dt=True)
    return stats, rec, dt


def test_graph_engine_is_deterministic():
    """The premise of the comparisons below: two graph-engine runs from the
    same state agree bit for bit."""
    a = _run(4, 20000, "fp64", "graph", 4 / 20000, 0.02, 0.005, 1 / 16, 1 / 256)
    b = _run(4, 20000, "fp64", "graph", 4 / 20000, 0.02, 0.005, 1 / 16, 1 / 256)
    assert a[0] == b[0] and np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


@pytest.mark.parametrize("order,n,precision,eps,eta,eta_s,dtmax,tend", [
    (4, 1024, "fp64", 1 / 256, 0.01, 0.0025, 1 / 8, 1 / 8),        # c1 to 1/8: > 4096 steps
    (4, 20000, "fp64", 4 / 20000, 0.02, 0.005, 1 / 16, 1 / 256),
    (4, 4096, "mixed", 4 / 4096, 0.1, 0.01, 1 / 16, 1 / 8),
    (6, 5000, "fp64", 4 / 5000, 0.1, 0.02, 1 / 16, 1 / 64),
    (8, 3000, "fp64", 4 / 3000, 0.75, 0.1, 1 / 16, 1 / 64),      # RUN/inp.8th's eta
    (4, 8192, "mixed", 4 / 8192, 0.1, 0.01, 1 / 16, 1 / 16),     # large steps, mixed
])
def test_persistent_matches_graph(order, n, precision, eps, eta, eta_s, dtmax, tend):
    a = _run(order, n, precision, "graph", eps, eta, eta_s, dtmax, tend)
    b = _run(order, n, precision, "persistent", eps, eta, eta_s, dtmax, tend)
    assert a[0] == b[0]
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])


def test_persistent_runs_split_over_calls():
    """Runs cut by a block-step budget and resumed, also across engines,
    take the same steps as one uninterrupted run."""
    whole = _run(4, 1024, "fp64", "graph", 1 / 256, 0.01, 0.0025, 1 / 8, 1 / 16)
    with hb.Gravity(4, 1024, "fp64") as g:
        g.set_jp_records(records(plummer(1024, 0), 4))
        g.integrator_init(0.0, (1 / 256) ** 2, 0.01, 0.0025, 1 / 8)
        g.set_engine("persistent")
        with pytest.raises(hb.HermiteError):
            g.integrator_run(1 / 16, max_block_steps=700)      # stops at the budget
        g.set_engine("graph")
        g.integrator_run(1 / 32)
        g.set_engine("persistent")
        g.integrator_run(1 / 16)
        stats = g.integrator_stats()
        rec, dt = g.get_records(with_dt=True)
    assert stats == whole[0]
    assert np.array_equal(rec, whole[1]) and np.array_equal(dt, whole[2])


def test_persistent_barrier_timeout_recovers():
    n, eps2 = 2048, (4 / 2048) ** 2
    rec0 = records(plummer(n, 3), 6)
    ref = _run(6, n, "fp64", "graph", 4 / 2048, 0.1, 0.02, 1 / 16, 1 / 64, seed=3)
    with hb.Gravity(6, n, "fp64") as g:
        g.set_engine("persistent")
        g.set_jp_records(rec0)
        g.integrator_init(0.0, eps2, 0.1, 0.02, 1 / 16)
        g.set_wait_limit(0)
        with pytest.raises(hb.HermiteError) as ei:
            g.integrator_run(1 / 64)
        assert ei.value.status == HB_ERR_DEVICE_TIMEOUT
        g.set_wait_limit(-1)
        g.set_jp_records(rec0)
        g.integrator_init(0.0, eps2, 0.1, 0.02, 1 / 16)
        g.integrator_run(1 / 64)
        stats = g.integrator_stats()
        rec, dt = g.get_records(with_dt=True)
    assert stats == ref[0]
    assert np.array_equal(rec, ref[1]) and np.array_equal(dt, ref[2])
