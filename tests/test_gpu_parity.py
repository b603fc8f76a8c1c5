"""CUDA path against the oracle and the reference's golden outputs.

Every call goes through libmbforce.so's C ABI (ctypes).  Tolerances
(docs/adr/0016-gpu-support.md:115-123 of the reference, and the target of
this build): FP64 energy 1e-10 eV/atom, forces 1e-8 eV/A, stress 1e-8
eV/A^3 -- and 1e-10 relative to the largest force against the oracle run on
the same candidate pairs; mixed precision forces 1e-5 eV/A, energy 1e-6
eV/atom, stress 1e-5 eV/A^3 against the FP64 oracle.
"""
import numpy as np
import pytest

import oracle
from conftest import (DIAMOND, FCC, SW_GESN, SW_SI, TERSOFF_SI, TERSOFF_XY, cubic, golden,
                      nested_records, strained)

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")

FP64_E, FP64_F, FP64_S = 1e-10, 1e-8, 1e-8
MIX_E, MIX_F, MIX_S = 1e-6, 1e-5, 1e-5


@pytest.fixture(autouse=True)
def _need_cuda(cuda_device):
    yield


# ---------------------------------------------------------------- neighbour list

@pytest.mark.parametrize("name", ["nl_si512_cubic", "nl_si216_triclinic",
                                  "nl_hcp216_hexagonal", "nl_fcc500"])
def test_nl_pairs_bit_exact(name):
    g = golden(name)
    nl = ak.NeighbourList(float(g["r_cut"]), skin_width=float(g["skin"]))
    nl.build(g["lattice"], g["positions"])
    i, j = nl.get_candidate_pairs()
    np.testing.assert_array_equal(i, g["pair_i"])
    np.testing.assert_array_equal(j, g["pair_j"])


def test_nl_csr_structure():
    g = golden("nl_fcc500")
    nl = ak.NeighbourList(float(g["r_cut"]), skin_width=float(g["skin"]))
    nl.build(g["lattice"], g["positions"])
    d = nl.device_list
    ro = d.row_off.cpu().numpy()
    nbr = d.nbr[:d.n_slots].cpu().numpy()
    rev = d.rev[:d.n_slots].cpu().numpy()
    assert ro[-1] == d.n_slots == 2 * len(g["pair_i"])
    for a in range(len(ro) - 1):
        row = nbr[ro[a]:ro[a + 1]]
        assert np.all(np.diff(row) > 0)
    src = np.repeat(np.arange(len(ro) - 1), np.diff(ro))
    np.testing.assert_array_equal(nbr[rev], src)
    np.testing.assert_array_equal(rev[rev], np.arange(d.n_slots))


def test_nl_large_matches_oracle():
    lat, pos, _ = cubic(FCC, 3.58, 12, ["Cu"] * 4, rattle=0.08, seed=5)
    rc = 5.805810750600001
    nl = ak.NeighbourList(rc, skin_width=0.3)
    nl.build(lat, pos)
    i, j = nl.get_candidate_pairs()
    oi, oj, _, _ = oracle.nl_build(lat, pos, rc, 0.3)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(j, oj)


@pytest.mark.parametrize("rc", [6.75, 8.7])
def test_nl_long_rows_match_oracle(rc):
    """Rows near and above 128 entries, where the register sort gives way
    to the shared-memory one (fcc Cu, r_list 7.05 A: a mean row of 128;
    9.0 A: ~266): the oracle's pairs, rows ascending, the upper offsets,
    rev an involution onto the row owners."""
    lat, pos, _ = cubic(FCC, 3.58, 8, ["Cu"] * 4, rattle=0.08, seed=6)
    nl = ak.NeighbourList(rc, skin_width=0.3)
    nl.build(lat, pos)
    i, j = nl.get_candidate_pairs()
    oi, oj, _, _ = oracle.nl_build(lat, pos, rc, 0.3)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(j, oj)
    d = nl.device_list
    ro = d.row_off.cpu().numpy()
    nbr = d.nbr[:d.n_slots].cpu().numpy()
    rev = d.rev[:d.n_slots].cpu().numpy()
    up = d.upper[:len(ro) - 1].cpu().numpy()
    lens = np.diff(ro)
    assert lens.max() > 128
    for a in range(len(ro) - 1):
        row = nbr[ro[a]:ro[a + 1]]
        assert np.all(np.diff(row) > 0)
        assert up[a] - ro[a] == np.count_nonzero(row < a)
    src = np.repeat(np.arange(len(ro) - 1), lens)
    np.testing.assert_array_equal(nbr[rev], src)
    np.testing.assert_array_equal(rev[rev], np.arange(d.n_slots))


def test_nl_refuses_thin_cell():
    lat, pos, _ = cubic(DIAMOND, 5.431, 1, ["Si"] * 8)
    with pytest.raises(ValueError):
        ak.NeighbourList(3.0, 0.3).build(lat, pos)


def test_nl_check_and_rebuild_criterion():
    lat, pos, _ = cubic(DIAMOND, 5.431, 4, ["Si"] * 8, rattle=0.05, seed=1)
    nl = ak.NeighbourList(3.0, skin_width=0.5)
    assert nl.check_and_rebuild(lat, pos) is True
    moved = pos.copy()
    moved[0] += [0.1, 0.0, 0.0]          # 2 d_max = 0.2 < skin 0.5
    assert nl.check_and_rebuild(lat, moved) is False
    moved[0] += [0.2, 0.0, 0.0]          # d_max 0.3 -> 0.6 >= 0.5
    assert nl.check_and_rebuild(lat, moved) is True
    assert nl.rebuild_count == 2 and nl.step_count == 3
    # a periodic wrap of one atom is not motion (minimum image)
    wrapped = moved.copy()
    wrapped[5] += lat[0]
    assert nl.check_and_rebuild(lat, wrapped) is False


# ---------------------------------------------------------------- potentials

def _fn(cfg, precision="fp64"):
    return ak.force_fn_from_config(cfg, precision=precision)


def _run(cfg, g, precision="fp64", types=None):
    fn = _fn(cfg, precision)
    nl = ak.NeighbourList(float(fn.r_cut), skin_width=float(g["skin"]))
    nl.build(g["lattice"], g["positions"])
    t = list(g["atom_types"]) if types is None else types
    return fn(g["lattice"], g["positions"], t, nl), nl


def _assert_close(res, ref, n, tol_e, tol_f, tol_s):
    e, f, s = res
    e0, f0, s0 = ref
    assert abs(e - e0) / n < tol_e, (e, e0)
    assert np.abs(f - f0).max() < tol_f, np.abs(f - f0).max()
    assert np.abs(s - s0).max() < tol_s, np.abs(s - s0).max()


def _assert_rel(res, ref, rel=1e-10):
    e, f, s = res
    e0, f0, s0 = ref
    assert abs(e - e0) <= rel * max(1.0, abs(e0))
    assert np.abs(f - f0).max() <= rel * max(1.0, np.abs(f0).max())
    assert np.abs(s - s0).max() <= rel * max(1e-3, np.abs(s0).max())


CASES = {
    "tersoff_si512": ({"type": "Tersoff", "species": ["Si"], "params": TERSOFF_SI},
                      lambda g, p: oracle.tersoff_single(TERSOFF_SI, g["lattice"], g["positions"], p)),
    "tersoff_si216_triclinic": ({"type": "Tersoff", "species": ["Si"], "params": TERSOFF_SI},
                                lambda g, p: oracle.tersoff_single(TERSOFF_SI, g["lattice"],
                                                                   g["positions"], p)),
    "tersoff_xy512": ({"type": "Tersoff", "species": ["X", "Y"], "params": TERSOFF_XY},
                      lambda g, p: oracle.tersoff_multi(nested_records(TERSOFF_XY), ["X", "Y"],
                                                        g["lattice"], g["positions"],
                                                        list(g["atom_types"]), p)),
    "sw_si512": ({"type": "SW", "species": ["Si"], "params": SW_SI},
                 lambda g, p: oracle.sw_single(SW_SI, g["lattice"], g["positions"], p)),
    "sw_si216_triclinic": ({"type": "SW", "species": ["Si"], "params": SW_SI},
                           lambda g, p: oracle.sw_single(SW_SI, g["lattice"], g["positions"], p)),
    "sw_gesn512": ({"type": "SW", "species": ["Ge", "Sn"], "params": SW_GESN},
                   lambda g, p: oracle.sw_multi(nested_records(SW_GESN), ["Ge", "Sn"], g["lattice"],
                                                g["positions"], list(g["atom_types"]), p)),
    "eam_cuni500": ({"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"],
                     "species": ["Cu", "Ni"]},
                    lambda g, p: oracle.eam(oracle.zhou_spec(
                        {s: ak.ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"]),
                        g["lattice"], g["positions"], list(g["atom_types"]), p)),
    "eam_ni500": ({"type": "EAM", "form": "zhou2004", "elements": ["Ni"], "species": ["Ni"]},
                  lambda g, p: oracle.eam(oracle.zhou_spec({"Ni": ak.ZHOU_2004["Ni"]}, ["Ni"]),
                                          g["lattice"], g["positions"], list(g["atom_types"]), p)),
}


def _sic_cfg():
    el = ak.TERSOFF_1989["elements"]
    return {"type": "Tersoff", "species": ["Si", "C"],
            "params": {"mixing": "tersoff1989", "elements": {s: dict(el[s]) for s in ("Si", "C")},
                       "chi": {"C-Si": ak.TERSOFF_1989["chi"]["C-Si"]}}}


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_matches_reference_golden(name):
    cfg, _ = CASES[name]
    g = golden(name)
    res, _ = _run(cfg, g)
    _assert_close(res, (g["energy"], g["forces"], g["stress"]), len(g["positions"]),
                  FP64_E, FP64_F, FP64_S)


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_matches_oracle_same_pairs(name):
    cfg, orc = CASES[name]
    g = golden(name)
    res, nl = _run(cfg, g)
    ref = orc(g, nl.get_candidate_pairs())
    _assert_rel(res, ref, 1e-10)


@pytest.mark.parametrize("name", ["tersoff_si512", "tersoff_xy512", "sw_si512", "sw_gesn512"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_lane_group_width_matches_oracle(name, precision):
    """Each lanes-per-atom tile shape the autotuner may pick (4, 8 and 16
    lanes per centre) gives the oracle's result on the same pairs."""
    cfg, orc = CASES[name]
    g = golden(name)
    fn = _fn(cfg, precision)
    pot = fn.engine.potentials[0]
    nl = ak.NeighbourList(float(fn.r_cut), skin_width=float(g["skin"]))
    nl.build(g["lattice"], g["positions"])
    ref = orc(g, nl.get_candidate_pairs())
    assert tuple(pot.lane_choices) == (4, 8, 16)
    for lpa in pot.lane_choices:
        pot.lanes_per_atom = lpa
        res = fn(g["lattice"], g["positions"], list(g["atom_types"]), nl)
        if precision == "fp64":
            _assert_rel(res, ref, 1e-10)
        else:
            _assert_close(res, ref, len(g["positions"]), MIX_E, MIX_F, MIX_S)


@pytest.mark.parametrize("name", ["tersoff1989_sic64", "tersoff1989_sic216"])
def test_fp64_tersoff1989_sic(name):
    g = golden(name)
    res, nl = _run(_sic_cfg(), g)
    _assert_close(res, (g["energy"], g["forces"], g["stress"]), len(g["positions"]),
                  FP64_E, FP64_F, FP64_S)
    el = ak.TERSOFF_1989["elements"]
    rec = oracle.tersoff1989_to_triplets({s: el[s] for s in ("Si", "C")},
                                         {"C-Si": ak.TERSOFF_1989["chi"]["C-Si"]}, ["Si", "C"])
    ref = oracle.tersoff_multi(rec, ["Si", "C"], g["lattice"], g["positions"],
                               list(g["atom_types"]), nl.get_candidate_pairs())
    _assert_rel(res, ref, 1e-10)


def test_fp64_eam_setfl_spline():
    g = golden("eam_setfl_cuni500")
    specs = {"rho": {}, "F": {}}
    for s in ("Cu", "Ni"):
        specs["rho"][s] = ("spline", g[f"rho_{s}_x"], g[f"rho_{s}_c"])
        specs["F"][s] = ("spline", g[f"F_{s}_x"], g[f"F_{s}_c"])
    from akitsushima_b200.eam import SpecFunction
    phi = {frozenset(("Cu",)): SpecFunction(("spline_over_r", g["rphi_CuCu_x"], g["rphi_CuCu_c"])),
           frozenset(("Cu", "Ni")): SpecFunction(("spline_over_r", g["rphi_NiCu_x"], g["rphi_NiCu_c"])),
           frozenset(("Ni",)): SpecFunction(("spline_over_r", g["rphi_NiNi_x"], g["rphi_NiNi_c"]))}
    pot = ak.EAMPotential({s: SpecFunction(v) for s, v in specs["F"].items()},
                          {s: SpecFunction(v) for s, v in specs["rho"].items()}, phi,
                          r_cut=float(g["r_cut"]), species=["Cu", "Ni"])
    fn = ak.make_force_fn(pot)
    nl = ak.NeighbourList(float(g["r_cut"]), skin_width=0.3)
    nl.build(g["lattice"], g["positions"])
    res = fn(g["lattice"], g["positions"], list(g["atom_types"]), nl)
    _assert_close(res, (g["energy"], g["forces"], g["stress"]), 500, FP64_E, FP64_F, FP64_S)


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_within_tolerance(name):
    cfg, orc = CASES[name]
    g = golden(name)
    res, nl = _run(cfg, g, precision="mixed")
    ref = orc(g, nl.get_candidate_pairs())
    _assert_close(res, ref, len(g["positions"]), MIX_E, MIX_F, MIX_S)


# ---------------------------------------------------------------- API edges

def test_owned_list_and_null_list_paths():
    g = golden("tersoff_si512")
    fn = _fn(CASES["tersoff_si512"][0])
    assert fn.uses_neighbour_list is False
    e1, f1, s1 = fn(g["lattice"], g["positions"], list(g["atom_types"]))
    e2, f2, s2 = fn(g["lattice"], g["positions"], list(g["atom_types"]),
                    ak.NullNeighbourList(fn.r_cut))
    assert abs(e1 - e2) < 1e-12 and np.abs(f1 - f2).max() < 1e-12
    _assert_close((e1, f1, s1), (g["energy"], g["forces"], g["stress"]), 512, FP64_E, FP64_F, FP64_S)


def test_foreign_cpu_list_is_used():
    class CpuList:
        def __init__(self, i, j, r_list):
            self.i, self.j, self.r_list = i, j, r_list
            self.rebuild_count = 1

        def get_candidate_pairs(self):
            return self.i, self.j

    g = golden("eam_cuni500")
    cfg = CASES["eam_cuni500"][0]
    fn = _fn(cfg)
    res = fn(g["lattice"], g["positions"], list(g["atom_types"]),
             CpuList(g["pair_i"], g["pair_j"], float(g["r_cut"]) + 0.3))
    _assert_close(res, (g["energy"], g["forces"], g["stress"]), 500, FP64_E, FP64_F, FP64_S)


def test_need_stress_false_returns_none():
    g = golden("sw_si512")
    fn = _fn(CASES["sw_si512"][0])
    e, f, s = ak.call_force_fn(fn, g["lattice"], g["positions"], list(g["atom_types"]),
                               need_stress=False)
    assert s is None and f.shape == (512, 3)


def test_no_pairs_gives_zero():
    lat = np.eye(3) * 30.0
    pos = np.array([[0.0, 0.0, 0.0], [10.0, 10.0, 10.0]])
    fn = _fn(CASES["eam_ni500"][0])
    e, f, s = fn(lat, pos, ["Ni", "Ni"])
    assert e == 0.0
    assert np.abs(f).max() == 0.0


def test_translation_invariance_and_momentum():
    lat, pos, types = cubic(DIAMOND, 5.431, 4, ["Si"] * 8, rattle=0.1, seed=9)
    for cfg in (CASES["tersoff_si512"][0], CASES["sw_si512"][0]):
        fn = _fn(cfg)
        e, f, s = fn(lat, pos, types)
        e2, f2, s2 = fn(lat, pos + np.array([0.37, -1.2, 2.5]), types)
        assert abs(e - e2) < 1e-9
        assert np.abs(f.sum(0)).max() < 1e-9


def test_batch_of_structures_matches_single_calls():
    structs = []
    for n, seed in ((2, 1), (3, 2), (4, 3)):
        lat, pos, types = cubic(DIAMOND, 5.431, n, ["Si"] * 8, rattle=0.1, seed=seed)
        lat, pos = strained(lat, pos, 0.03, seed + 10)
        structs.append((lat, pos, np.zeros(len(pos), np.int32)))
    pot = ak.TersoffPotential(TERSOFF_SI, species=["Si"])
    batch = ak.Batch([s[0] for s in structs], [s[1] for s in structs], [s[2] for s in structs])
    dl = ak.DeviceNeighbourList(pot.r_cut + 0.3).build(batch)
    res = pot.evaluate(batch, dl)
    e = res.energy.cpu().numpy()
    f = res.forces.cpu().numpy()
    off = batch.offsets
    for k, (lat, pos, t) in enumerate(structs):
        e0, f0, s0 = pot.compute(lat, pos, ["Si"] * len(pos))
        assert abs(e[k] - e0) < 1e-9
        assert np.abs(f[off[k]:off[k + 1]] - f0).max() < 1e-10


def test_exp_clamp_beyond_500_matches_oracle():
    """The Tersoff zeta exponential exp(lambda3^3 (r_ij - r_ik)^3) driven past
    both clamps of the reference's _nb_exp (engine/_numba_common.py:12-33:
    x > 500 -> exp(500), x < -500 -> 0): lambda3 = 40 on a rattled Si cell
    gives arguments of both signs beyond 500; the float64 GPU path equals
    the oracle, which restates the clamp, on the same pairs."""
    lat, pos, types = cubic(DIAMOND, 5.431, 4, ["Si"] * 8, rattle=0.1, seed=11)
    p = dict(TERSOFF_SI, lambda3=40.0)
    nl = ak.NeighbourList(p["R"] + p["D"], skin_width=0.3)
    nl.build(lat, pos)
    i, j = nl.get_candidate_pairs()
    d = pos[j] - pos[i]
    s = d @ np.linalg.inv(lat)
    s -= np.round(s)
    r = np.linalg.norm(s @ lat, axis=1)
    inside = r < p["R"] + p["D"]
    rows = {}
    for a, b, rr in zip(i[inside], j[inside], r[inside]):
        rows.setdefault(a, []).append(rr)
        rows.setdefault(b, []).append(rr)
    spread = max(max(v) - min(v) for v in rows.values())
    assert (40.0 * spread) ** 3 > 500.0   # both signs occur: (r_ij - r_ik) and (r_ik - r_ij)
    fn = ak.force_fn_from_config({"type": "Tersoff", "species": ["Si"], "params": p})
    res = fn(lat, pos, types, nl)
    ref = oracle.tersoff_single(p, lat, pos, (i, j))
    assert np.all(np.isfinite(res[1]))
    _assert_rel(res, ref, 1e-10)
