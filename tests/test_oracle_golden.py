"""The CPU oracle against the reference's own outputs (CPU only).

Golden fixtures in tests/golden/ were written by tests/golden/make_golden.py,
which runs the reference; the ledger energies are the reference's own
benchmark records (benchmarks/adr0047.jsonl:2,4,12).  These tests pin the
oracle before it is trusted as the checker of the CUDA path.
"""
import numpy as np
import pytest

import oracle
from akitsushima_b200.published_parameters import TERSOFF_1989, ZHOU_2004
from conftest import (DIAMOND, FCC, SW_SI, TERSOFF_SI, TERSOFF_XY, SW_GESN,
                      cubic, golden, nested_records)


@pytest.mark.parametrize("name", ["nl_si512_cubic", "nl_si216_triclinic",
                                  "nl_hcp216_hexagonal", "nl_fcc500"])
def test_oracle_nl_bit_exact_to_reference(name):
    g = golden(name)
    i, j, _, _ = oracle.nl_build(g["lattice"], g["positions"], float(g["r_cut"]),
                                 float(g["skin"]))
    np.testing.assert_array_equal(i, g["pair_i"])
    np.testing.assert_array_equal(j, g["pair_j"])


@pytest.mark.parametrize("name", ["nl_si512_cubic", "nl_fcc500", "nl_hcp216_hexagonal"])
def test_oracle_nl_equals_brute_force(name):
    g = golden(name)
    rl = float(g["r_cut"]) + float(g["skin"])
    i, j, _, _ = oracle.nl_build(g["lattice"], g["positions"], float(g["r_cut"]),
                                 float(g["skin"]))
    bi, bj = oracle.brute_force_pairs(g["lattice"], g["positions"], rl)
    assert set(zip(i.tolist(), j.tolist())) == set(zip(bi.tolist(), bj.tolist()))


def test_oracle_nl_refuses_thin_cell():
    lat, pos, _ = cubic(DIAMOND, 5.431, 1, ["Si"] * 8)
    with pytest.raises(ValueError):
        oracle.nl_build(lat, pos, 3.0, 0.3)


def _check(e, f, s, g, rtol=1e-11):
    n = len(g["positions"])
    assert abs(e - float(g["energy"])) / n < 1e-10
    fs = max(1.0, float(np.abs(g["forces"]).max()))
    assert float(np.abs(f - g["forces"]).max()) / fs < rtol * 10
    ss = max(1e-3, float(np.abs(g["stress"]).max()))
    assert float(np.abs(s - g["stress"]).max()) / ss < rtol * 10


def _pairs(g):
    return g["pair_i"], g["pair_j"]


@pytest.mark.parametrize("name", ["tersoff_si512", "tersoff_si216_triclinic"])
def test_oracle_tersoff_single(name):
    g = golden(name)
    e, f, s = oracle.tersoff_single(TERSOFF_SI, g["lattice"], g["positions"], _pairs(g))
    _check(e, f, s, g)


def test_oracle_tersoff_multi():
    g = golden("tersoff_xy512")
    rec = nested_records(TERSOFF_XY)
    e, f, s = oracle.tersoff_multi(rec, ["X", "Y"], g["lattice"], g["positions"],
                                   list(g["atom_types"]), _pairs(g))
    _check(e, f, s, g)


@pytest.mark.parametrize("name", ["tersoff1989_sic64", "tersoff1989_sic216"])
def test_oracle_tersoff1989(name):
    g = golden(name)
    el = TERSOFF_1989["elements"]
    rec = oracle.tersoff1989_to_triplets({s: el[s] for s in ("Si", "C")},
                                         {"C-Si": TERSOFF_1989["chi"]["C-Si"]},
                                         ["Si", "C"])
    e, f, s = oracle.tersoff_multi(rec, ["Si", "C"], g["lattice"], g["positions"],
                                   list(g["atom_types"]), _pairs(g))
    _check(e, f, s, g)


@pytest.mark.parametrize("name", ["sw_si512", "sw_si216_triclinic"])
def test_oracle_sw_single(name):
    g = golden(name)
    e, f, s = oracle.sw_single(SW_SI, g["lattice"], g["positions"], _pairs(g))
    _check(e, f, s, g)


def test_oracle_sw_multi():
    g = golden("sw_gesn512")
    rec = nested_records(SW_GESN)
    e, f, s = oracle.sw_multi(rec, ["Ge", "Sn"], g["lattice"], g["positions"],
                              list(g["atom_types"]), _pairs(g))
    _check(e, f, s, g)


@pytest.mark.parametrize("name,els", [("eam_cuni500", ["Cu", "Ni"]), ("eam_ni500", ["Ni"])])
def test_oracle_eam_zhou(name, els):
    g = golden(name)
    spec = oracle.zhou_spec({s: ZHOU_2004[s] for s in els}, els)
    assert abs(spec.r_cut - float(g["r_cut"])) < 1e-12
    e, f, s = oracle.eam(spec, g["lattice"], g["positions"], list(g["atom_types"]),
                         _pairs(g))
    _check(e, f, s, g)


def test_oracle_eam_setfl_spline():
    g = golden("eam_setfl_cuni500")
    specs = [("spline", g["rho_Cu_x"], g["rho_Cu_c"]), ("spline", g["rho_Ni_x"], g["rho_Ni_c"]),
             ("spline", g["F_Cu_x"], g["F_Cu_c"]), ("spline", g["F_Ni_x"], g["F_Ni_c"]),
             ("spline_over_r", g["rphi_CuCu_x"], g["rphi_CuCu_c"]),
             ("spline_over_r", g["rphi_NiCu_x"], g["rphi_NiCu_c"]),
             ("spline_over_r", g["rphi_NiNi_x"], g["rphi_NiNi_c"])]
    phi = np.array([[4, 5], [5, 6]])
    spec = oracle.EAMSpec(["Cu", "Ni"], specs, [0, 1], [2, 3], phi, float(g["r_cut"]))
    e, f, s = oracle.eam(spec, g["lattice"], g["positions"], list(g["atom_types"]),
                         _pairs(g))
    _check(e, f, s, g)


# ---- the reference's own ledger (benchmarks/adr0047.jsonl) ----------------

def test_oracle_ledger_tersoff_si4096():
    lat, pos, types = cubic(DIAMOND, 5.431, 8, ["Si"] * 8)
    i, j, _, _ = oracle.nl_build(lat, pos, 3.0, 0.5)
    e, f, _ = oracle.tersoff_single(TERSOFF_SI, lat, pos, (i, j))
    assert abs(e / 4096 - (-4.570619398287601)) < 1e-12
    assert float(np.abs(f.sum(0)).max()) < 1e-9


def test_oracle_ledger_sw_si4096():
    lat, pos, types = cubic(DIAMOND, 5.431, 8, ["Si"] * 8)
    i, j, _, _ = oracle.nl_build(lat, pos, 2.0951 * 1.80, 0.5)
    e, f, _ = oracle.sw_single(SW_SI, lat, pos, (i, j))
    assert abs(e / 4096 - (-4.270680168516988)) < 1e-12


def test_oracle_ledger_eam_cuni4000():
    # species draw order of benchmarks/bench_force.py:214-231 (default sizes)
    rng = np.random.default_rng(1)
    for n in (4, 8):
        rng.choice(["Ge", "Sn"], 8 * n ** 3, p=[0.875, 0.125])
    rng.choice(["Cu", "Ni"], 4 * 5 ** 3)
    lat, pos, types = cubic(FCC, 3.58, 10, ["Cu"] * 4)
    types = [str(x) for x in rng.choice(["Cu", "Ni"], len(types))]
    spec = oracle.zhou_spec({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    i, j, _, _ = oracle.nl_build(lat, pos, spec.r_cut, 0.5)
    e, _, _ = oracle.eam(spec, lat, pos, types, (i, j))
    assert abs(e / 4000 - (-3.951219863199116)) < 1e-12
