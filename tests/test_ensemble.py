"""Batched ensembles (hb_ens_*): independent clusters on one GPU.

Two engines: the lockstep engine (one global block-step loop over the union
of all clusters) and the team engine (each cluster on its own block steps,
one thread-block cluster per system); by default clusters that fit a team
use the team engine and the rest the lockstep engine.

* Two copies of the same gen-plum cluster must each reproduce the
  reference's published block-step fingerprint (per-cluster counters), on
  both engines.
* Clusters of different sizes, softenings and masses stay independent: a
  cluster integrated inside the ensemble matches the same cluster
  integrated alone to near rounding level after a short interval, and
  every cluster conserves energy.
* The engines agree cluster by cluster (block steps, particle steps,
  states), also when one run mixes them.
"""
import subprocess

import numpy as np
import pytest

from kat import ETA, GEN_PLUM, PUBLISHED_NACT

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("engine", ["graph", "team"])
def test_two_identical_clusters_reproduce_fingerprint(engine, tmp_path):
    from hermite_b200 import Ensemble
    from hermite_b200.ic import read_snapshot, records
    if not GEN_PLUM.exists():
        pytest.skip("gen-plum not built (needs the reference sources)")
    subprocess.run([str(GEN_PLUM), "1"], cwd=tmp_path, check=True, capture_output=True)
    snap = read_snapshot(tmp_path / "pl1k.dat")
    order, n = 4, snap.n
    eps2 = (4.0 / n) ** 2
    eta, eta_s = ETA[order]
    rec = records(snap, order)
    with Ensemble(order, [n, n], "fp64") as ens:
        ens.set_engine(engine)
        assert ens.cluster_engine(0)[0] == engine
        ens.set_cluster(0, rec, eps2)
        ens.set_cluster(1, rec, eps2)
        ens.init(0.0, eta, eta_s, 1.0 / 16)
        ens.run(1.0)
        per = [ens.cluster_stats(c) for c in range(2)]
        ps, bs, t, _ = ens.stats()
    assert per[0] == per[1]
    assert t == 1.0 and per[0][2] == 1.0
    assert (ps, bs) == (2 * per[0][0], 2 * per[0][1])
    assert "%e" % (per[0][0] / per[0][1]) == PUBLISHED_NACT[(order, n)][0]


@pytest.mark.parametrize("engine", ["graph", "team"])
def test_clusters_are_independent(engine):
    from hermite_b200 import Ensemble, Gravity
    from hermite_b200.ic import plummer, power_law_masses, records
    order, eta, eta_s, dtmax, tend = 6, 0.1, 0.02, 1.0 / 16, 1.0 / 16
    sizes = [700, 1500, 333]
    recs, eps2s = [], []
    for c, n in enumerate(sizes):
        rng = np.random.default_rng(c)
        snap = plummer(n, seed=c, masses=power_law_masses(n, rng))
        recs.append(records(snap, order))
        eps2s.append((4.0 / n) ** 2)
    with Ensemble(order, sizes, "fp64") as ens:
        ens.set_engine(engine)
        for c in range(len(sizes)):
            ens.set_cluster(c, recs[c], eps2s[c])
        ens.init(0.0, eta, eta_s, dtmax)
        ke0, pe0 = ens.energy()
        ens.run(tend)
        ke1, pe1 = ens.energy()
        out = [ens.get_cluster(c) for c in range(len(sizes))]
    de = np.abs((ke1 + pe1 - ke0 - pe0) / (ke0 + pe0))
    assert np.all(de < 1e-7), de
    # cluster 1 alone
    with Gravity(order, sizes[1], "fp64") as g:
        g.set_jp_records(recs[1])
        g.integrator_init(0.0, eps2s[1], eta, eta_s, dtmax)
        g.integrator_run(tend)
        alone = g.get_records()
    assert np.max(np.abs(out[1][:, 0:3] - alone[:, 0:3])) < 1e-9


def _ensemble(order, sizes, engine, team_ctas=0, tend=1.0 / 16, eta=0.1):
    from hermite_b200 import Ensemble
    from hermite_b200.ic import plummer, power_law_masses, records
    with Ensemble(order, sizes, "fp64") as ens:
        ens.set_engine(engine, team_ctas)
        for c, n in enumerate(sizes):
            rng = np.random.default_rng(10 + c)
            snap = plummer(n, seed=10 + c, masses=power_law_masses(n, rng))
            ens.set_cluster(c, records(snap, order), (4.0 / n) ** 2)
        ens.init(0.0, eta, eta / 5, 1.0 / 16)
        ens.run(tend / 2)
        ens.run(tend)
        used = [ens.cluster_engine(c) for c in range(len(sizes))]
        stats = [ens.cluster_stats(c) for c in range(len(sizes))]
        out = [ens.get_cluster(c, with_dt=True) for c in range(len(sizes))]
        tot = ens.stats()
    return used, stats, out, tot


@pytest.mark.parametrize("order", [4, 6, 8])
def test_engines_agree_cluster_by_cluster(order):
    sizes = [1500, 64, 700, 2100, 333, 2]
    used_g, st_g, out_g, tot_g = _ensemble(order, sizes, "graph")
    # team size 2 holds at most 2 x (slots per CTA) particles: at 8th order
    # the 2100-particle cluster does not fit and goes to the lockstep engine
    used_a, st_a, out_a, tot_a = _ensemble(order, sizes, "team", team_ctas=2)
    assert all(u == ("graph", 0) for u in used_g)
    assert all(u[0] == "team" for n, u in zip(sizes, used_a) if n <= 1024)
    for c, (u, sa, sg) in enumerate(zip(used_a, st_a, st_g)):
        (ra, da), (rg, dg) = out_a[c], out_g[c]
        assert sa[2] == sg[2] == 1.0 / 16
        if u[0] == "graph":
            # the same engine in both runs: a cluster's result does not depend
            # on which other clusters share the lockstep loop
            assert sa == sg, c
            np.testing.assert_array_equal(ra, rg)
            np.testing.assert_array_equal(da, dg)
        else:
            # another engine sums in another order: at 8th order the
            # criterion's h^-5..h^-7 differences may move a step by one level
            assert abs(sa[0] - sg[0]) <= 1e-3 * sg[0], (c, sa, sg)
            scale = np.abs(rg[:, 0:7]).max(axis=0) + 1e-300
            assert (np.abs(ra[:, 0:7] - rg[:, 0:7]) / scale).max() < 1e-7, c
    assert tot_a[2] == tot_g[2] == 1.0 / 16


def test_engine_choice_per_cluster():
    from hermite_b200 import Ensemble
    with Ensemble(4, [100, 40000], "fp64") as ens:
        ens.set_engine("team", 1)          # the 40000-particle cluster fits no team of 1 CTA
        assert ens.cluster_engine(0) == ("team", 1)
        assert ens.cluster_engine(1) == ("graph", 0)
        ens.set_engine("auto", 1)          # not all fit: lockstep for all
        assert ens.cluster_engine(0) == ("graph", 0)
        ens.set_engine("auto")             # 40000 fits no team of up to 16 CTAs either
        assert ens.cluster_engine(0) == ("graph", 0)
    with Ensemble(4, [100, 2000], "fp64") as ens:
        assert ens.cluster_engine(0)[0] == "team" and ens.cluster_engine(1)[0] == "team"
    with Ensemble(4, [100, 200], "mixed") as ens:
        assert ens.cluster_engine(0) == ("graph", 0)
