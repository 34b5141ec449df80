"""Seeded initial conditions (hermite_b200.ic, CPU): the Plummer generator
restates RUN/gen-plum.c:104-226 with a seeded stream, the power-law mass
function is the batched-ensemble configuration's, and records() lays out the
j-particle record the library takes."""
import math

import numpy as np
import pytest

from hermite_b200 import ic


def test_plummer_units_and_centre_of_mass():
    s = ic.plummer(4096, seed=3)
    assert s.n == 4096 and s.mass.sum() == pytest.approx(1.0, abs=1e-15)
    np.testing.assert_allclose((s.mass[:, None] * s.pos).sum(axis=0), 0.0, atol=1e-15)
    np.testing.assert_allclose((s.mass[:, None] * s.vel).sum(axis=0), 0.0, atol=1e-15)
    ke, pe = ic.energies(s.mass, s.pos, s.vel)
    # gen-plum's scaling (conv = 3 pi / 16) gives E ~ -1/4 and a virial
    # ratio ~ 1/2 up to sampling noise (E0 = -0.2623 at N = 1k there)
    assert ke + pe == pytest.approx(-0.25, rel=0.08)
    assert ke / -pe == pytest.approx(0.5, rel=0.08)


def test_plummer_is_seeded():
    a, b, c = ic.plummer(500, seed=1), ic.plummer(500, seed=1), ic.plummer(500, seed=2)
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.vel, b.vel)
    assert not np.array_equal(a.pos, c.pos)


def test_plummer_exact_henon_scaling():
    s = ic.plummer(800, seed=5, exact_henon=True)
    ke, pe = ic.energies(s.mass, s.pos, s.vel)
    assert ke + pe == pytest.approx(-0.25, abs=1e-12)
    assert ke / -pe == pytest.approx(0.5, abs=1e-12)


def test_power_law_masses():
    rng = np.random.default_rng(7)
    m = ic.power_law_masses(200_000, rng)
    assert m.sum() == pytest.approx(1.0, abs=1e-12) and np.all(m > 0)
    ratio = m / m.min()
    assert ratio.max() <= 1000.0 * (1 + 1e-9)
    # median of dN/dm ~ m^-2.35 on [0.1, 100], relative to the lower bound
    a = -1.35
    m_med = (0.1 ** a + 0.5 * (100.0 ** a - 0.1 ** a)) ** (1 / a)
    assert np.median(ratio) == pytest.approx(m_med / 0.1, rel=0.01)


def test_plummer_with_masses():
    rng = np.random.default_rng(0)
    m = ic.power_law_masses(1000, rng)
    s = ic.plummer(1000, seed=0, masses=m)
    assert np.array_equal(s.mass, m)
    np.testing.assert_allclose((s.mass[:, None] * s.pos).sum(axis=0), 0.0, atol=1e-14)


@pytest.mark.parametrize("order,words", [(4, 14), (6, 20), (8, 26), (9, 29)])
def test_record_layout(order, words):
    s = ic.plummer(37, seed=1)
    rec = ic.records(s, order, tlast=0.5)
    assert rec.shape == (37, words)
    np.testing.assert_array_equal(rec[:, 0:3], s.pos)
    np.testing.assert_array_equal(rec[:, 3], s.mass)
    np.testing.assert_array_equal(rec[:, 4:7], s.vel)
    assert np.all(rec[:, 7] == 0.5) and np.all(rec[:, 8:] == 0.0)
    d = np.arange(37 * (words - 8), dtype=float).reshape(37, words - 8)
    np.testing.assert_array_equal(ic.records(s, order, derivs=d)[:, 8:], d)


def test_energies_two_body():
    mass = np.array([0.25, 0.75])
    pos = np.array([[0.0, 0.0, 0.0], [0.0, 3.0, 4.0]])
    vel = np.array([[1.0, 0.0, 0.0], [0.0, 0.0, 2.0]])
    ke, pe = ic.energies(mass, pos, vel, eps2=0.0)
    assert ke == pytest.approx(0.5 * (0.25 * 1.0 + 0.75 * 4.0))
    assert pe == pytest.approx(-0.25 * 0.75 / 5.0)
    _, pe_soft = ic.energies(mass, pos, vel, eps2=11.0)
    assert pe_soft == pytest.approx(-0.25 * 0.75 / math.sqrt(36.0))
