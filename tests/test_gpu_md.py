"""Device NVE against the reference's trajectory and the oracle (GPU).

Trajectories are compared only over a few tens of steps (before chaotic
divergence); longer runs are checked by energy conservation and by force
parity at identical positions."""
import numpy as np
import pytest

import oracle
from conftest import DIAMOND, FCC, SW_SI, TERSOFF_SI, cubic, golden

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")
from akitsushima_b200 import md  # noqa: E402


@pytest.mark.parametrize("graph", [True, False])
@pytest.mark.parametrize("rebuild_every", [None, 5])
def test_tersoff_nve_matches_reference_trajectory(cuda_device, graph, rebuild_every):
    g = golden("md_nve_si64_tersoff")
    pot = ak.TersoffPotential(TERSOFF_SI, species=["Si"])
    sim = md.NVE(pot, g["lattice"], g["positions"], list(g["atom_types"]), velocities=g["velocities0"],
                 dt=float(g["dt"]), rebuild_every=rebuild_every, skin=0.3)
    sim.run(int(g["n_steps"]), graph=graph)
    res = sim.results()
    np.testing.assert_allclose(sim.positions, g["positions_final"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(sim.velocities, g["velocities_final"], rtol=0, atol=1e-10)
    th = g["thermo"]
    np.testing.assert_allclose(res["e_pot"], th[1:, 2], rtol=0, atol=2e-6)
    np.testing.assert_allclose(res["e_kin"], th[1:, 3], rtol=0, atol=2e-6)
    np.testing.assert_allclose(res["temperature"], th[1:, 5], rtol=0, atol=0.02)
    assert len(res["skin_displacement"]) == (20 if rebuild_every is None else 4)


def test_mb_start_on_device_equals_reference_draw(cuda_device):
    g = golden("md_nve_si64_tersoff")
    pot = ak.TersoffPotential(TERSOFF_SI, species=["Si"])
    sim = md.NVE(pot, g["lattice"], g["positions"], list(g["atom_types"]), temperature=300.0,
                 seed=int(g["seed"]))
    np.testing.assert_allclose(sim.velocities, g["velocities0"], rtol=0, atol=1e-15)
    assert abs(sim.e_kin0 - g["thermo"][0, 3]) < 1e-6


def _oracle_run(kind, lat, pos, types, v0, steps, rc, params=None):
    m = md.masses_for(types)

    def force(r):
        i, j, _, _ = oracle.nl_build(lat, r, rc, 0.3)
        if kind == "sw":
            e, f, _ = oracle.sw_single(SW_SI, lat, r, (i, j))
        else:
            e, f, _ = oracle.eam(params, lat, r, types, (i, j))
        return e, f

    return oracle.nve(force, lat, pos, m, v0, 1.0, steps)


def test_sw_nve_fp64_matches_oracle(cuda_device):
    lat, pos, types = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.1, seed=4)
    pot = ak.StillingerWeberPotential(SW_SI, species=["Si"])
    v0 = md.init_velocities_mb(600.0, md.masses_for(types), np.random.default_rng(1))
    sim = md.NVE(pot, lat, pos, types, velocities=v0)
    sim.run(30)
    ref = _oracle_run("sw", lat, pos, types, v0, 30, pot.r_cut)
    np.testing.assert_allclose(sim.positions, ref[-1][0], rtol=0, atol=1e-8)
    res = sim.results()
    np.testing.assert_allclose(res["e_pot"], [x[2] for x in ref], rtol=0, atol=1e-8)
    np.testing.assert_allclose(res["e_kin"], [x[3] for x in ref], rtol=0, atol=1e-8)


def test_eam_nve_fp64_matches_oracle(cuda_device):
    lat, pos, _ = cubic(FCC, 3.58, 4, ["Cu"] * 4, rattle=0.05, seed=3)
    types = [str(t) for t in np.random.default_rng(4).choice(["Cu", "Ni"], len(pos))]
    pot = ak.zhou_eam({s: ak.ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    spec = oracle.zhou_spec({s: ak.ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    v0 = md.init_velocities_mb(300.0, md.masses_for(types), np.random.default_rng(2))
    sim = md.NVE(pot, lat, pos, types, velocities=v0)
    sim.run(20)
    ref = _oracle_run("eam", lat, pos, types, v0, 20, spec.r_cut, spec)
    np.testing.assert_allclose(sim.positions, ref[-1][0], rtol=0, atol=1e-8)
    np.testing.assert_allclose(sim.results()["e_pot"], [x[2] for x in ref], rtol=0, atol=1e-8)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_energy_conservation_and_force_parity(cuda_device, precision):
    """Velocity Verlet's energy error is O(dt^2): at dt = 1 fs this hot
    (sigma = 0.1 A) SW silicon drifts about 5e-4 eV/atom in the oracle too.
    The device run must match the oracle's drift envelope, shrink about 4x
    at dt / 2, and give oracle forces at its final positions."""
    lat, pos, types = cubic(DIAMOND, 5.431, 4, ["Si"] * 8, rattle=0.1, seed=0)
    n = len(pos)
    m = md.masses_for(types)
    v0 = md.init_velocities_mb(300.0, m, np.random.default_rng(0))
    env = {}
    for dt in (1.0, 0.5):
        pot = ak.StillingerWeberPotential(SW_SI, species=["Si"], precision=precision)
        sim = md.NVE(pot, lat, pos, types, velocities=v0, dt=dt)
        sim.run(int(200 / dt))
        res = sim.results()
        env[dt] = np.abs(res["drift"]).max() / n
        assert res["rebuilds"] > 0 and len(res["skin_displacement"]) == int(200 / dt)
    ref = _oracle_run("sw", lat, pos, types, v0, 200, SW_SI["a"] * SW_SI["sigma"])
    e_ref = np.array([x[2] + x[3] for x in ref])
    env_ref = np.abs(e_ref - (sim_e0(lat, pos, m, v0))).max() / n
    assert 0.7 * env_ref < env[1.0] < 1.3 * env_ref, (env, env_ref)
    assert 0.15 < env[0.5] / env[1.0] < 0.4, env
    # forces at the final (identical) positions against the oracle
    r = sim.positions
    i, j, _, _ = oracle.nl_build(lat, r, pot.r_cut, 0.3)
    e0, f0, _ = oracle.sw_single(SW_SI, lat, r, (i, j))
    tol = 1e-8 if precision == "fp64" else 1e-5
    assert np.abs(sim.forces - f0).max() < tol
    assert abs(sim.results()["e_pot"][-1] - e0) / n < (1e-10 if precision == "fp64" else 1e-6)


def sim_e0(lat, pos, m, v0):
    i, j, _, _ = oracle.nl_build(lat, pos, SW_SI["a"] * SW_SI["sigma"], 0.3)
    e, _, _ = oracle.sw_single(SW_SI, lat, pos, (i, j))
    return e + 0.5 * float(np.sum(m[:, None] * v0 ** 2)) / md.EV_ANG_TO_AMU_ANG_FS2


def test_skin_criterion_violation_is_reported(cuda_device):
    lat, pos, types = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.1, seed=0)
    pot = ak.StillingerWeberPotential(SW_SI, species=["Si"])
    sim = md.NVE(pot, lat, pos, types, temperature=3000.0, seed=0, rebuild_every=40, skin=0.02)
    sim.run(80)
    with pytest.raises(RuntimeError, match="criterion"):
        sim.results()


def test_criterion_graph_equals_eager(cuda_device):
    lat, pos, types = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.1, seed=5)
    runs = []
    for graph in (True, False):
        pot = ak.StillingerWeberPotential(SW_SI, species=["Si"])
        sim = md.NVE(pot, lat, pos, types, temperature=1500.0, seed=3, skin=0.2, autotune=False)
        sim.run(60, graph=graph)
        runs.append((sim.positions, sim.results()))
    (p1, r1), (p2, r2) = runs
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(r1["e_tot"], r2["e_tot"])
    assert r1["rebuilds"] == r2["rebuilds"] > 0
    d = r1["skin_displacement"]
    # a rebuild resets the displacement: it never stays above the trigger
    assert np.all(2 * d < 0.2 + 2 * 0.1)


@pytest.mark.parametrize("graph", [True, False])
def test_fused_kicks_equal_separate_launches(cuda_device, graph):
    """A block of steps (the second half kick of each step but the last
    fused with the first half kick, drift and check of the next) gives the
    bits of the same steps run one by one as separate launches."""
    lat, pos, types = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.1, seed=41)
    pot = ak.StillingerWeberPotential(SW_SI, species=["Si"], precision="fp64")
    args = dict(temperature=900.0, seed=5, skin=0.3, autotune=False)
    blocked = md.NVE(pot, lat, pos, types, steps_per_graph=12, **args)
    single = md.NVE(pot, lat, pos, types, steps_per_graph=100, **args)
    blocked.run(24, graph=graph)    # two whole blocks
    single.run(24, graph=graph)     # no whole block: 24 single steps
    np.testing.assert_array_equal(blocked.positions, single.positions)
    np.testing.assert_array_equal(blocked.velocities, single.velocities)
    rb, rs = blocked.results(), single.results()
    for key in ("e_pot", "e_kin", "skin_displacement"):
        np.testing.assert_array_equal(rb[key], rs[key])
    assert rb["rebuilds"] == rs["rebuilds"]


def drift_per_ps(e_tot, n_atoms, dt_fs=1.0):
    """Least-squares slope of the total energy per atom against time, eV /
    atom / ps (the NVE drift measure of the reference's GPU plan)."""
    t_ps = np.arange(1, len(e_tot) + 1) * dt_fs * 1e-3
    return float(np.polyfit(t_ps, np.asarray(e_tot) / n_atoms, 1)[0])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nve_drift_over_10_ps(cuda_device, precision):
    """Mixed-precision NVE conserves energy to the reference's bar for a GPU
    path: drift <= 1e-5 eV/atom/ps over 10 ps (docs/adr/0016-gpu-support.md
    :115-123 of the reference).  Stillinger-Weber Si, 8^3 cells (4096 atoms),
    displacements 0.1 A, 300 K, dt 1 fs, 10,000 steps with the criterion
    rebuilds; float64 alongside for comparison."""
    lat, pos, types = cubic(DIAMOND, 5.431, 8, ["Si"] * 8, rattle=0.1, seed=3)
    pot = ak.StillingerWeberPotential(SW_SI, species=["Si"], precision=precision)
    sim = md.NVE(pot, lat, pos, types, temperature=300.0, seed=0, steps_per_graph=50)
    sim.run(10_000)
    res = sim.results()
    assert len(res["e_tot"]) == 10_000
    slope = drift_per_ps(res["e_tot"], len(pos))
    assert abs(slope) <= 1e-5, slope
