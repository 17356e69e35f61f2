"""Potential-only calls and device-side energies, through the C ABI.

The reference's energy path (grape6_calculate_energies,
src/node/dyn/hdyn/evolve/hdyn_grape6.C:1403-1546) needs only the potential
of every particle and forms epot = sum 1/2 m_i pot_i and ekin = sum 1/2 m_i
v_i^2 on the host.  g6b200_calc_pot runs a potential-only kernel and
g6b200_energies forms both sums on the device.  Checked against the FP64
oracle (FP64 mode <= 1e-12; mixed mode <= 1e-6), and the mixed mode's
potential-only kernel against the full kernel's pot (the same rounding
sequence: bit-identical except where the full call's refinement recomputed
a particle in FP64).
"""
import numpy as np
import pytest

from helpers import oracle_forces, snapshot

pytestmark = pytest.mark.gpu

EPS2 = 1e-6
TOL = {"fp64": 1e-12, "mixed": 1e-6}


def _engine(mode, cid, npipes=8192):
    from starlab_b200 import G6Engine
    return G6Engine(cluster_id=cid, precision=mode, npipes=npipes)


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_potential_only_matches_oracle_and_full_kernel(mode, oracle, monkeypatch):
    # the mixed mode's full calls below 2^25 interactions run in FP64;
    # here every full call stays mixed, to compare the two mixed kernels
    monkeypatch.setenv("G6B200_MIXED_MIN_WORK", "0")
    n = 8192
    m, x, v, a, j = snapshot(n, 41)
    ti = 1.0 / 128
    eng = _engine(mode, 5100 if mode == "fp64" else 5101)
    eng.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    eng.set_ti(ti)
    xp, vp = oracle.predict(ti, 0.0, x, v, 0.5 * a, j / 6.0)
    for ni, i0 in ((8192, 0), (300, 1000), (1, 77)):
        idx = np.arange(i0, i0 + ni, dtype=np.int32)
        pot = eng.potential(n, idx, xp[idx], EPS2)
        ref = oracle.force(xp, vp, m, idx, xp[idx], vp[idx], EPS2)[2]
        err = np.abs(pot - ref) / np.abs(ref)
        assert err.max() <= TOL[mode], (ni, float(err.max()))
        full = eng.force(n, idx, xp[idx], vp[idx], EPS2)[2]
        if mode == "mixed":
            # the same rounding sequence; the full call's refinement replaces
            # its ill-conditioned particles (about 1%) by FP64 values
            same = pot.view(np.uint64) == full.view(np.uint64)
            assert same.mean() >= 0.95, (ni, float(same.mean()))
            assert (np.abs(pot - full) / np.abs(full)).max() <= 1e-6
        else:
            assert np.abs(pot - full).max() <= 1e-13 * np.abs(full).max()
    st = eng.stats()
    eng.close()
    assert st["launches"] > 0


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_energies_on_the_device(mode, oracle):
    n = 6000  # not a multiple of the tile
    m, x, v, a, j = snapshot(n, 43)
    eng = _engine(mode, 5110 if mode == "fp64" else 5111)
    # unpredicted (ti = tj = 0), as the reference's energy call sends them
    eng.set_j_particles(0.0, m, j / 6.0, 0.5 * a, v, x)
    eng.set_ti(0.0)
    ep, ek, pot = eng.energies(n, EPS2, want_pot=True)
    ref_pot = oracle_forces(m, x, v, EPS2)[2]
    assert np.abs(pot - ref_pot).max() / np.abs(ref_pot).max() <= TOL[mode]
    ep_ref = 0.5 * np.sum(m * ref_pot)
    ek_ref = 0.5 * np.sum(m * np.sum(v * v, axis=1))
    assert abs(ep - ep_ref) <= TOL[mode] * abs(ep_ref), (ep, ep_ref)
    assert abs(ek - ek_ref) <= 1e-13 * ek_ref, (ek, ek_ref)
    # predicted to a block time: velocities are the predicted ones
    ti = 1.0 / 256
    eng.set_ti(ti)
    ep2, ek2 = eng.energies(n, EPS2)
    xp, vp = oracle.predict(ti, 0.0, x, v, 0.5 * a, j / 6.0)
    ref_pot2 = oracle_forces(m, xp, vp, EPS2)[2]
    ep2_ref = 0.5 * np.sum(m * ref_pot2)
    ek2_ref = 0.5 * np.sum(m * np.sum(vp * vp, axis=1))
    assert abs(ep2 - ep2_ref) <= TOL[mode] * abs(ep2_ref)
    assert abs(ek2 - ek2_ref) <= 1e-13 * ek2_ref
    # repeatable: a fixed summation order
    assert eng.energies(n, EPS2) == (ep2, ek2)
    eng.close()
