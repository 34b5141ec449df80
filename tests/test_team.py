"""The team engine: one thread-block cluster runs the whole block-step loop.

It must integrate exactly the algorithm of the multi-kernel (graph) engine.
Only the order of the j summation differs (a j-split over the team's CTAs),
so forces agree to a few ulp and, over a short window, the block-step
sequence (every quantised timestep) is identical.  The known-answer test on
the published nact values runs on both engines in tests/test_integrator.py.

Cases: team sizes from 1 to 16 CTAs, N not a multiple of 32, teams with
more CTAs than 32-slot chunks (CTAs that own no slots), more active slots
than one force round holds (kTeamIMax = 256), and the engine selection
rules.
"""
import numpy as np
import pytest

import hermite_b200 as hb
from hermite_b200.ic import plummer, records

pytestmark = pytest.mark.gpu

HB_ERR_INVALID, HB_ERR_TOO_LARGE = 1, 7


def integrate(order, n, engine, ctas=0, tend=1.0 / 8, seed=3, eta=None):
    eps2 = (4.0 / n) ** 2
    eta = eta if eta is not None else {4: 0.1, 6: 0.5, 8: 0.75}[order]
    with hb.Gravity(order, n, "fp64") as g:
        g.set_engine(engine, ctas)
        g.set_jp_records(records(plummer(n, seed), order))
        g.integrator_init(0.0, eps2, eta, eta / 5, 1.0 / 16)
        g.integrator_run(tend)
        stats = g.integrator_stats()
        rec, dt = g.get_records(with_dt=True)
        used = g.engine()
    return stats, rec, dt, used


@pytest.mark.parametrize("order,n,ctas", [
    (4, 1000, 0), (4, 1000, 1), (4, 1000, 3), (4, 1000, 16),
    (6, 777, 0), (6, 777, 5), (8, 513, 0), (8, 513, 8),
    (4, 40, 4),            # 2 chunks over 4 CTAs: two CTAs own nothing
    (6, 33, 2),
    (4, 3000, 0),          # first steps have > 256 active slots: several rounds
    (6, 4500, 0),          # steps with > 4096 active slots: the graph engine's large-step kernel
    (8, 4200, 0),
    (4, 4000, 2),          # more slots per CTA than shared memory holds with their records:
    (6, 3000, 4),          # the records stay in global memory
    (8, 2000, 2),
])
def test_team_matches_graph_engine(order, n, ctas):
    s_g, rec_g, dt_g, used_g = integrate(order, n, "graph")
    s_t, rec_t, dt_t, used_t = integrate(order, n, "team", ctas)
    assert used_g == ("graph", 0)
    assert used_t[0] == "team" and (ctas == 0 or used_t[1] == ctas)
    assert s_t == s_g                                  # (particle steps, block steps, tsys)
    np.testing.assert_array_equal(dt_t, dt_g)
    scale = np.abs(rec_g).max(axis=0) + 1e-300
    err = np.abs(rec_t - rec_g) / scale
    assert err[:, 0:8].max() < 1e-10, err[:, 0:8].max()    # pos mass vel tlast
    assert np.all(rec_t[:, 7] == rec_g[:, 7])


def test_team_continues_across_calls_and_engines():
    """A run split over several calls, switching engines between them, ends
    in the same state as one uninterrupted team run."""
    order, n = 4, 1024
    s_one, rec_one, _, _ = integrate(order, n, "team", tend=0.25)
    eps2 = (4.0 / n) ** 2
    with hb.Gravity(order, n, "fp64") as g:
        g.set_jp_records(records(plummer(n, 3), order))
        g.integrator_init(0.0, eps2, 0.1, 0.02, 1.0 / 16)
        for k, eng in enumerate(["team", "graph", "team", "team"]):
            g.set_engine(eng)
            g.integrator_run(0.0625 * (k + 1))
        stats = g.integrator_stats()
        rec = g.get_records()
    assert stats == s_one
    assert np.abs(rec[:, 0:7] - rec_one[:, 0:7]).max() < 1e-10


def test_team_block_step_limit():
    order, n = 4, 512
    with hb.Gravity(order, n, "fp64") as g:
        g.set_engine("team")
        g.set_jp_records(records(plummer(n, 1), order))
        g.integrator_init(0.0, (4.0 / n) ** 2, 0.1, 0.02, 1.0 / 16)
        with pytest.raises(hb.HermiteError, match="limit"):
            g.integrator_run(1.0, max_block_steps=10)
        ps, bs, t = g.integrator_stats()
        assert bs == 10 and 0.0 < t < 1.0
        g.integrator_run(1.0)
        assert g.integrator_stats()[2] == 1.0


def test_engine_selection():
    lib = hb.load_library()
    import ctypes
    with hb.Gravity(4, 2048, "fp64") as g:
        assert g.engine()[0] == "team"
        assert 1 <= g.engine()[1] <= 16
        g.set_engine("graph")
        assert g.engine() == ("graph", 0)
    with hb.Gravity(4, 2048, "mixed") as g:
        assert g.engine() == ("graph", 0)
        g.set_engine("team")
        e, c = ctypes.c_int(), ctypes.c_int()
        assert lib.hb_integrator_engine(ctypes.c_void_p(g.handle), ctypes.byref(e),
                                        ctypes.byref(c)) == HB_ERR_INVALID
    with hb.Gravity(4, 4096, "fp64") as g:
        assert g.engine() == ("graph", 0)          # above the automatic crossover
    with hb.Gravity(4, 65536, "fp64") as g:
        assert g.engine() == ("graph", 0)
        g.set_engine("team", 2)
        e, c = ctypes.c_int(), ctypes.c_int()
        assert lib.hb_integrator_engine(ctypes.c_void_p(g.handle), ctypes.byref(e),
                                        ctypes.byref(c)) == HB_ERR_TOO_LARGE
