"""Phonon displacement and elastic strain sets as one batch (GPU): equal to
the reference's one-call-per-configuration arithmetic, restated with the
oracle's force calls."""
import numpy as np
import pytest

import oracle
from conftest import DIAMOND, FCC, SW_SI, TERSOFF_SI, cubic

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")
from akitsushima_b200 import sets  # noqa: E402


def _oracle_forces(lat, pos):
    i, j, _, _ = oracle.nl_build(lat, pos, 3.0, 0.3)
    return oracle.tersoff_single(TERSOFF_SI, lat, pos, (i, j))


def test_ifc_columns_equal_per_call_central_differences(cuda_device):
    lat, pos, types = cubic(DIAMOND, 5.431, 2, ["Si"] * 8, rattle=0.0, seed=0)
    fn = ak.force_fn_from_config({"type": "Tersoff", "species": ["Si"], "params": TERSOFF_SI})
    tasks = [(j, b) for j in (0, 4) for b in range(3)]
    cols = sets.ifc_columns(fn, lat, pos, types, tasks, delta=0.01)
    for t, (j, b) in enumerate(tasks):
        p, m = pos.copy(), pos.copy()
        p[j, b] += 0.01
        m[j, b] -= 0.01
        ref = -(_oracle_forces(lat, p)[1] - _oracle_forces(lat, m)[1]) / 0.02
        assert np.abs(cols[t] - ref).max() < 1e-6
    # acoustic sum rule of a column: sum over atoms of -dF/dr_j = 0
    assert np.abs(cols.sum(axis=1)).max() < 1e-8


def test_displaced_forces_and_engine_of_two(cuda_device):
    lat, pos, types = cubic(DIAMOND, 5.431, 2, ["Si"] * 8, rattle=0.02, seed=1)
    eng = ak.PotentialEngine().add(ak.TersoffPotential(TERSOFF_SI, species=["Si"])) \
        .add(ak.StillingerWeberPotential(SW_SI, species=["Si"]))
    disp = [(3, (0.01, 0.0, -0.02)), (10, (0.0, 0.015, 0.0))]
    F = sets.displaced_forces(eng, lat, pos, types, disp)
    for (j, d), f in zip(disp, F):
        p = pos.copy()
        p[j] += d
        i_, j_, _, _ = oracle.nl_build(lat, p, 3.77118, 0.3)
        ref = oracle.tersoff_single(TERSOFF_SI, lat, p, (i_, j_))[1] + oracle.sw_single(SW_SI, lat, p, (i_, j_))[1]
        assert np.abs(f - ref).max() < 1e-8


def test_clamped_elastic_constants_match_per_point_calls(cuda_device):
    lat, pos, types = cubic(DIAMOND, 5.431, 2, ["Si"] * 8, rattle=0.0, seed=0)
    fn = ak.force_fn_from_config({"type": "SW", "species": ["Si"], "params": SW_SI})
    C0, sig, pts = sets.clamped_elastic_constants(fn, lat, pos, types, strains=(0.005,))
    frac = pos @ np.linalg.inv(lat)
    for (j, s), st in zip(pts, sig):
        L = lat if j is None else lat @ (np.eye(3) + sets.strain_matrix(j, s))
        P = frac @ L
        i_, j_, _, _ = oracle.nl_build(L, P, 3.77118, 0.3)
        assert np.abs(st - oracle.sw_single(SW_SI, L, P, (i_, j_))[2]).max() < 1e-8
    # cubic symmetry of diamond silicon: C11 = C22 = C33, C12 = C13 = C23
    assert C0[0, 0] == pytest.approx(C0[1, 1], rel=1e-6) == pytest.approx(C0[2, 2], rel=1e-6)
    assert C0[0, 1] == pytest.approx(C0[0, 2], rel=1e-6)
    assert 100.0 < C0[0, 0] < 200.0     # SW silicon, clamped ions: ~151 GPa


def test_evaluate_many_equals_single_calls(cuda_device):
    structs = []
    for k, n in enumerate((4, 5)):
        lat, pos, types = cubic(FCC, 3.58, n, ["Cu"] * 4, rattle=0.05, seed=k)
        types = [str(t) for t in np.random.default_rng(k).choice(["Cu", "Ni"], len(pos))]
        structs.append((lat, pos, types))
    fn = ak.force_fn_from_config({"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"]})
    res = sets.evaluate_many(fn, structs)
    for (lat, pos, types), (e, f, s) in zip(structs, res):
        e0, f0, s0 = fn(lat, pos, types)
        assert abs(e - e0) < 1e-9 and np.abs(f - f0).max() < 1e-10 and np.abs(s - s0).max() < 1e-12
