"""Batched ensembles (hb_ens_*): independent clusters advanced by one
device-resident block-step loop.

* Two copies of the same gen-plum cluster must each reproduce the
  reference's published block-step fingerprint: the batch has the block
  steps of one copy and twice its particle steps.
* Clusters of different sizes, softenings and masses stay independent: a
  cluster integrated inside the ensemble matches the same cluster
  integrated alone to near rounding level after a short interval, and
  every cluster conserves energy.
"""
import subprocess

import numpy as np
import pytest

from kat import ETA, GEN_PLUM, PUBLISHED_NACT

pytestmark = pytest.mark.gpu


def test_two_identical_clusters_reproduce_fingerprint(tmp_path):
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
        ens.set_cluster(0, rec, eps2)
        ens.set_cluster(1, rec, eps2)
        ens.init(0.0, eta, eta_s, 1.0 / 16)
        ens.run(1.0)
        ps, bs, t, _ = ens.stats()
    assert t == 1.0
    assert ps % 2 == 0
    assert "%e" % (ps / 2 / bs) == PUBLISHED_NACT[(order, n)][0]


def test_clusters_are_independent():
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
