"""CPU-only checks of the boundary and the host logic (no GPU calls).

* libmbforce.so loads and exports every function include/mbforce.h
  declares, and only calls that need no device are made;
* species tables, cell grids, thin-cell replication, Zhou parameter set-up
  and the config factory agree with the oracle / the reference's rules.
"""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from conftest import DIAMOND, FCC, SW_GESN, SW_SI, TERSOFF_XY, cubic, nested_records

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "mbforce.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mbf_\w+)\s*\(", txt)))


def test_library_exports_every_header_symbol():
    from akitsushima_b200 import _lib
    L = _lib.lib()
    names = _header_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(_lib.EXPORTED)


def test_library_cpu_safe_calls():
    from akitsushima_b200 import _lib
    L = _lib.lib()
    assert L.mbf_version() >= 10000
    assert L.mbf_error_string(-3).decode().startswith("neighbour capacity")
    assert L.mbf_nl_workspace_bytes(1000, 64) > 1000 * 4
    assert L.mbf_eval_workspace_bytes(1000, 80000, 1) > 80000 * 8 * 3


def test_library_is_sm100a():
    from akitsushima_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def test_species_ids():
    from akitsushima_b200.system import species_ids
    ids = species_ids(["Ni", "Cu", "Ni"], ["Cu", "Ni"])
    assert ids.tolist() == [1, 0, 1]
    assert species_ids(np.array([1, 0]), ["Cu", "Ni"]).tolist() == [1, 0]
    with pytest.raises(ValueError):
        species_ids(["Fe"], ["Cu", "Ni"])


def test_cell_grid_and_min_image():
    from akitsushima_b200.system import cell_grid, check_min_image
    lat = np.eye(3) * 143.2
    nc, w = cell_grid(lat, 6.1058)
    assert nc.tolist() == [23, 23, 23] and w.tolist() == [3, 3, 3]
    nc, w = cell_grid(np.eye(3) * 10.862, 3.3)
    assert nc.tolist() == [3, 3, 3]
    with pytest.raises(ValueError):
        check_min_image(np.eye(3) * 5.431, 3.3)
    with pytest.raises(ValueError):
        check_min_image(np.zeros((3, 3)), 1.0)


def test_replicate_thin_is_exact_periodic_supercell():
    from akitsushima_b200.system import replicate_thin
    lat, pos, _ = cubic(DIAMOND, 5.431, 1, ["Si"] * 8, rattle=0.1)
    big_lat, big_pos, big_t, reps = replicate_thin(lat, pos, np.zeros(8, np.int32), 3.3)
    assert reps.tolist() == [2, 2, 2]
    assert big_pos.shape == (64, 3)
    np.testing.assert_allclose(big_lat, lat * 2)
    e, f, _ = oracle.tersoff_single({"A": 1830.8, "B": 471.18, "lambda1": 2.4799,
                                     "lambda2": 1.7322, "lambda3": 0.0, "beta": 1.1e-6,
                                     "n": 0.78734, "c": 100390.0, "d": 16.217, "h": -0.59825,
                                     "R": 2.85, "D": 0.15}, big_lat, big_pos)
    lat3, pos3, _, reps3 = replicate_thin(lat, pos, np.zeros(8, np.int32), 8.0)
    assert reps3.tolist() == [3, 3, 3]
    e3, f3, _ = oracle.tersoff_single({"A": 1830.8, "B": 471.18, "lambda1": 2.4799,
                                       "lambda2": 1.7322, "lambda3": 0.0, "beta": 1.1e-6,
                                       "n": 0.78734, "c": 100390.0, "d": 16.217, "h": -0.59825,
                                       "R": 2.85, "D": 0.15}, lat3, pos3)
    assert abs(e / 64 - e3 / len(pos3)) < 1e-10
    np.testing.assert_allclose(f[:8], f3[:8], atol=1e-10)


def test_tersoff_tables_match_oracle():
    from akitsushima_b200 import TersoffPotential
    rec = nested_records(TERSOFF_XY)
    pot = TersoffPotential(rec, species=["X", "Y"])
    tb, tri = pot.host_tables()
    T = oracle.tersoff_tables(rec, ["X", "Y"])
    np.testing.assert_array_equal(tb[:, 0], T["tb_valid"].reshape(-1))
    for col, key in ((1, "A"), (2, "B"), (3, "lambda1"), (4, "lambda2"), (5, "R"), (6, "D"),
                     (7, "beta"), (8, "n")):
        np.testing.assert_array_equal(tb[:, col], T["tb_" + key].reshape(-1))
    for col, key in ((0, "valid"), (1, "c"), (2, "d"), (3, "h"), (4, "lambda3"), (5, "m"),
                     (6, "gamma")):
        np.testing.assert_array_equal(tri[:, col], T["tri_" + key].reshape(-1).astype(float))


def test_sw_tables_match_oracle():
    from akitsushima_b200 import StillingerWeberPotential
    rec = nested_records(SW_GESN)
    pot = StillingerWeberPotential(rec, species=["Ge", "Sn"])
    tb, leg, tri, rc = pot.host_tables()
    T = oracle.sw_tables(rec, ["Ge", "Sn"])
    np.testing.assert_array_equal(tb[:, 0], T["tb_valid"].reshape(-1))
    np.testing.assert_array_equal(leg[:, 2], T["leg_gam"].reshape(-1))
    np.testing.assert_array_equal(tri[:, 0], T["tri_valid"].reshape(-1))
    np.testing.assert_allclose(tri[:, 1], (T["tri_eps"] * T["tri_lam"] * 0.5).reshape(-1))
    assert abs(rc - oracle.sw_r_cut(rec)) < 1e-15


def test_sw_two_body_symmetry_refused():
    from akitsushima_b200 import StillingerWeberPotential
    rec = nested_records(SW_GESN)
    rec[("Ge", "Sn", "Sn")] = dict(rec[("Ge", "Sn", "Sn")], A=rec[("Ge", "Sn", "Sn")]["A"] * 1.2)
    with pytest.raises(ValueError):
        StillingerWeberPotential(rec, species=["Ge", "Sn"])


def test_zhou_setup_matches_oracle():
    from akitsushima_b200 import ZHOU_2004, continuous, zhou_cutoff, zhou_eam
    for el in ("Cu", "Ni", "Al"):
        a = continuous(ZHOU_2004[el])
        b = oracle.zhou_continuous(ZHOU_2004[el])
        assert all(abs(a[k] - b[k]) < 1e-15 for k in a)
        assert zhou_cutoff(a) == oracle.zhou_cutoff(b)
    pot = zhou_eam({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    assert abs(pot.r_cut - 5.805810750600001) < 1e-12
    t = pot.function_table()
    assert t["fused"]
    spec = oracle.zhou_spec({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    np.testing.assert_array_equal(t["codes"], spec.codes)
    np.testing.assert_array_equal(t["P"], spec.P)


def test_eam_host_functions_match_oracle_kernel_forms():
    from akitsushima_b200 import ZHOU_2004, zhou_eam
    pot = zhou_eam({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    r = np.linspace(2.0, 5.9, 50)
    v = pot._phi[frozenset(("Cu", "Ni"))](r)
    assert np.all(np.isfinite(v))
    assert abs(pot._phi[frozenset(("Cu", "Ni"))](np.array([5.9]))[0]) == 0.0


def test_force_fn_from_config_shapes_and_errors():
    import akitsushima_b200 as ak
    fn = ak.force_fn_from_config({"type": "SW", "species": ["Si"], "params": SW_SI})
    assert abs(fn.r_cut - 1.8 * 2.0951) < 1e-12 and fn.kind == "engine"
    assert fn.uses_neighbour_list is False and ak.accepts_need_stress(fn)
    fn = ak.force_fn_from_config({"type": "Tersoff", "species": ["X", "Y"], "params": TERSOFF_XY},
                                 precision="mixed")
    assert fn.precision == "mixed" and abs(fn.r_cut - 3.0) < 1e-12
    fn = ak.force_fn_from_config({"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"],
                                  "compute": {"device": "cuda", "precision": "mixed"}})
    assert fn.precision == "mixed"
    with pytest.raises(ValueError):
        ak.force_fn_from_config({"type": "EAM", "params": {}})
    with pytest.raises(ValueError):
        ak.force_fn_from_config({"type": "LJ"})
    with pytest.raises(ValueError):
        ak.force_fn_from_config({"type": "SW", "params": SW_SI}, precision="fp16")
    with pytest.raises(ValueError):
        ak.force_fn_from_config({"type": "SW", "params": SW_SI, "device": "cpu"})


def test_tersoff1989_expansion_matches_oracle():
    import akitsushima_b200 as ak
    el = ak.TERSOFF_1989["elements"]
    a = ak.tersoff1989_to_triplets({s: el[s] for s in ("Si", "C")}, {"C-Si": 0.9776}, ["Si", "C"])
    b = oracle.tersoff1989_to_triplets({s: el[s] for s in ("Si", "C")}, {"C-Si": 0.9776},
                                       ["Si", "C"])
    assert a == b
    with pytest.raises(ValueError):
        ak.tersoff1989_to_triplets({s: el[s] for s in ("C", "Ge")}, {}, ["C", "Ge"])


def test_neighbour_list_api_rejects_cpu_backends():
    import akitsushima_b200 as ak
    with pytest.raises(ValueError):
        ak.NeighbourList(3.0, backend="kdtree")
    with pytest.raises(ValueError):
        ak.NeighbourList(-1.0)
    assert ak.NeighbourList(3.0, 0.3).r_list == pytest.approx(3.3)


_ = (ctypes, FCC)


def test_batch_view_carries_host_cells():
    """The C view's optional host copy of the cells holds the rows uploaded
    to the device array, before and after a lattice change."""
    import torch
    from akitsushima_b200.system import Batch
    lat, pos, _ = cubic(FCC, 3.58, 3, ["Cu"] * 4, rattle=0.05, seed=2)
    b = Batch([lat], [pos], [np.zeros(len(pos), np.int32)], device=torch.device("cpu"))

    def host_rows():
        sysd = b.mbf_system()
        assert sysd.cells_host
        return np.ctypeslib.as_array((ctypes.c_double * (18 * b.n_struct)).from_address(sysd.cells_host))

    np.testing.assert_array_equal(host_rows(), b.cells.numpy().reshape(-1))
    b.set_lattice(0, np.asarray(lat) * 1.01)
    np.testing.assert_array_equal(host_rows(), b.cells.numpy().reshape(-1))
    np.testing.assert_array_equal(host_rows()[:9], (np.asarray(lat) * 1.01).reshape(-1))
