"""NVE integrator pieces on the CPU: the Maxwell-Boltzmann start and the
oracle's velocity-Verlet loop against the reference's own NVESimulation
(tests/golden/md_nve_si64_tersoff.npz, 64 Si atoms, Tersoff, 20 steps)."""
import numpy as np
import pytest

import oracle
from conftest import TERSOFF_SI, golden

from akitsushima_b200 import md


def test_mb_velocities_match_reference_draw():
    g = golden("md_nve_si64_tersoff")
    m = md.masses_for(list(g["atom_types"]))
    v = md.init_velocities_mb(float(g["temperature"]), m, np.random.default_rng(int(g["seed"])))
    np.testing.assert_allclose(v, g["velocities0"], rtol=0, atol=1e-15)
    vo = oracle.init_velocities_mb(float(g["temperature"]), m, np.random.default_rng(int(g["seed"])))
    np.testing.assert_array_equal(v, vo)
    assert np.abs((m[:, None] * v).sum(0)).max() < 1e-12


def test_oracle_nve_matches_reference_trajectory():
    g = golden("md_nve_si64_tersoff")
    lat = g["lattice"]
    m = md.masses_for(list(g["atom_types"]))

    def force(r):
        i, j, _, _ = oracle.nl_build(lat, r, 3.0, 0.3)
        e, f, _ = oracle.tersoff_single(TERSOFF_SI, lat, r, (i, j))
        return e, f

    traj = oracle.nve(force, lat, g["positions"], m, g["velocities0"], float(g["dt"]), int(g["n_steps"]))
    r, v, _, _ = traj[-1]
    np.testing.assert_allclose(r, g["positions_final"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(v, g["velocities_final"], rtol=0, atol=1e-11)
    th = g["thermo"]  # step, time, e_pot, e_kin, e_tot, T, P, drift (6 decimals)
    for k, (_, _, e, ek) in enumerate(traj, start=1):
        assert abs(e - th[k, 2]) < 1e-6 and abs(ek - th[k, 3]) < 1e-6


def test_masses_and_arguments():
    assert md.masses_for(["Si", "C"]).tolist() == [28.086, 12.011]
    assert md.masses_for(["X"], {"X": 10.0}).tolist() == [10.0]
    with pytest.raises(ValueError):
        md.masses_for(["Xx"])
    with pytest.raises(ValueError):
        md.masses_for(["Si"], [-1.0])
    assert md.init_velocities_mb(300.0, [], np.random.default_rng(0)).shape == (0, 3)
