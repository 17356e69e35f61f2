"""Seeded initial conditions in N-body units (G = M = 1, E = -1/4).

* ``plummer``  -- the Plummer sphere sampled as in Aarseth, Henon & Wielen
  (1974, A&A 37, 183): radius from the inverted cumulative mass
  m(r) = r^3 (1 + r^2)^(-3/2) (truncated at a mass fraction of 0.999, the
  default cut of Starlab's makeplummer), isotropic directions, speed
  q v_esc with q drawn from g(q) ~ q^2 (1 - q^2)^(7/2) by rejection, then
  lengths scaled by 3 pi / 16 and velocities by sqrt(16 / (3 pi)) so that the
  virial-equilibrium energy is -1/4; the centre of mass is moved to rest at
  the origin.
* ``salpeter_masses`` -- a power-law mass function dN/dm ~ m^-2.35 between
  m_lo and m_hi, normalised to total mass 1 (as makemass -f 1 -x -2.35).

Inputs are synthetic stand-ins for the reference generators' output
(makeplummer / makemass), drawn from a numpy Generator seeded explicitly.
"""
import numpy as np


def plummer(n, seed, mfrac=0.999, masses=None):
    """Return (mass[n], pos[n,3], vel[n,3]) for an n-body Plummer sphere."""
    rng = np.random.default_rng(seed)
    if masses is None:
        m = np.full(n, 1.0 / n)
    else:
        m = np.asarray(masses, dtype=np.float64)
        m = m / m.sum()
    x1 = rng.uniform(0.0, mfrac, n)
    x1 = np.maximum(x1, 1e-300)
    r = 1.0 / np.sqrt(x1 ** (-2.0 / 3.0) - 1.0)
    pos = r[:, None] * _iso(rng, n)
    # speeds: rejection sampling of q in [0,1) from q^2 (1-q^2)^3.5
    q = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        qq = rng.uniform(0.0, 1.0, todo.size)
        yy = rng.uniform(0.0, 0.1, todo.size)
        ok = yy < qq * qq * (1.0 - qq * qq) ** 3.5
        q[todo[ok]] = qq[ok]
        todo = todo[~ok]
    vesc = np.sqrt(2.0) * (1.0 + r * r) ** -0.25
    vel = (q * vesc)[:, None] * _iso(rng, n)
    pos *= 3.0 * np.pi / 16.0
    vel *= np.sqrt(16.0 / (3.0 * np.pi))
    pos -= (m[:, None] * pos).sum(0) / m.sum()
    vel -= (m[:, None] * vel).sum(0) / m.sum()
    return m, np.ascontiguousarray(pos), np.ascontiguousarray(vel)


def _iso(rng, n):
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    s = np.sqrt(1.0 - z * z)
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)


def salpeter_masses(n, seed, slope=-2.35, m_lo=0.1, m_hi=100.0):
    """Masses from dN/dm ~ m^slope on [m_lo, m_hi], normalised to sum 1."""
    rng = np.random.default_rng(seed)
    a = slope + 1.0
    u = rng.uniform(0.0, 1.0, n)
    m = (m_lo ** a + u * (m_hi ** a - m_lo ** a)) ** (1.0 / a)
    return m / m.sum()


def scale_to_energy(m, pos, vel, pot, e_target=-0.25, q_vir=0.5):
    """Rescale positions/velocities to total energy e_target and virial
    ratio q_vir (= T/|W|), given the potential pot[i] = sum_j -m_j/r_ij of
    the current positions (as Starlab's scale -e -q does)."""
    w = 0.5 * float(np.sum(m * pot))
    t = 0.5 * float(np.sum(m * np.sum(vel * vel, axis=1)))
    # scale velocities to the virial ratio, then lengths to the energy
    vfac = np.sqrt(q_vir * -w / t)
    vel = vel * vfac
    e = w * (1.0 - q_vir)
    rfac = e / e_target
    return pos * rfac, vel / np.sqrt(rfac)
