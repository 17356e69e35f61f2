"""Seeded initial conditions (CPU): Plummer spheres in N-body units and the
Salpeter mass function, checked with the oracle's potential."""
import numpy as np


def test_plummer_units_and_virial(oracle):
    from starlab_b200 import ics
    n = 4096
    m, x, v = ics.plummer(n, 42)
    assert np.allclose(m.sum(), 1.0)
    assert np.allclose((m[:, None] * x).sum(0), 0, atol=1e-12)
    assert np.allclose((m[:, None] * v).sum(0), 0, atol=1e-12)
    _, _, pot, _, _ = oracle.force(x, v, m, np.arange(n), x, v, 0.0)
    w = 0.5 * np.sum(m * pot)
    t = 0.5 * np.sum(m * np.sum(v * v, axis=1))
    assert abs(t / -w - 0.5) < 0.05          # virial equilibrium
    assert abs((t + w) - (-0.25)) < 0.02     # E = -1/4 in N-body units


def test_plummer_is_seeded():
    from starlab_b200 import ics
    a = ics.plummer(100, 7)
    b = ics.plummer(100, 7)
    c = ics.plummer(100, 8)
    assert all(np.array_equal(p, q) for p, q in zip(a, b))
    assert not np.array_equal(a[1], c[1])


def test_salpeter_masses():
    from starlab_b200 import ics
    m = ics.salpeter_masses(200000, 3)
    assert np.isclose(m.sum(), 1.0)
    ratio = m.max() / m.min()
    assert 100 < ratio <= 1000 * (1 + 1e-9)
    # dN/dm ~ m^-2.35: the fraction below 2 m_min is 1 - 2^-1.35
    frac = np.mean(m < 2 * m.min())
    assert abs(frac - (1 - 2 ** -1.35)) < 0.01


def test_scale_to_energy(oracle):
    from starlab_b200 import ics
    n = 1000
    m, x, v = ics.plummer(n, 9)
    _, _, pot, _, _ = oracle.force(x, v, m, np.arange(n), x, v, 0.0)
    x2, v2 = ics.scale_to_energy(m, x, v, pot, e_target=-0.25, q_vir=0.5)
    _, _, pot2, _, _ = oracle.force(x2, v2, m, np.arange(n), x2, v2, 0.0)
    w = 0.5 * np.sum(m * pot2)
    t = 0.5 * np.sum(m * np.sum(v2 * v2, axis=1))
    assert np.isclose(t + w, -0.25, rtol=1e-10)
    assert np.isclose(t / -w, 0.5, rtol=1e-10)
