"""Zhou EAM fitting pieces on the CPU: ZhouEAMParameterSet against the
reference's (variables, x0, bounds, cutoff, decode), the differentiable
table against the potential's own function table, and the oracle's loss
against the reference's loss value."""
import numpy as np
import pytest
import torch

import oracle
from conftest import golden

from akitsushima_b200 import fit
from akitsushima_b200.eam import ZHOU_KEYS, continuous
from akitsushima_b200.published_parameters import ZHOU_2004

SPECIES = ["Al", "Ni"]
WEIGHTS = {"energy": 1.0, "forces": 1.0, "stress": 1.0, "r0": 0.1, "eps0": 0.01}


def structures():
    g = golden("fit_alni_zhou")
    out = []
    for q in range(int(g["n_structures"])):
        P = g[f"positions{q}"]
        out.append({"lattice": g[f"lattice{q}"], "positions": P, "atom_types": [str(t) for t in g[f"atom_types{q}"]],
                    "natoms": len(P), "ref_energy": float(g[f"ref_energy{q}"]), "ref_forces": g[f"ref_forces{q}"],
                    "ref_stress": g[f"ref_stress{q}"]})
    return out


def param_sets():
    el0 = {s: dict(ZHOU_2004[s]) for s in SPECIES}
    return {"zhou": fit.ZhouEAMParameterSet(el0, SPECIES),
            "zhou_chi": fit.ZhouEAMParameterSet(el0, SPECIES, fit_keys=["A", "B", "F2", "eta", "chi"])}


@pytest.mark.parametrize("tag", ["zhou", "zhou_chi"])
def test_parameter_set_mirrors_reference(tag):
    g = golden("fit_alni_zhou")
    ps = param_sets()[tag]
    assert ps.variable_names == [str(n) for n in g[f"{tag}_names"]]
    np.testing.assert_allclose(ps.x0, g[f"{tag}_x0"], rtol=0, atol=1e-15)
    np.testing.assert_allclose([b[0] for b in ps.bounds], g[f"{tag}_lo"], rtol=1e-15)
    np.testing.assert_allclose([b[1] for b in ps.bounds], g[f"{tag}_hi"], rtol=1e-15)
    assert ps.r_cut == float(g[f"{tag}_r_cut"])
    dec = ps.decode(g[f"{tag}_x_test"])["eam"]
    keys = [str(k) for k in g[f"{tag}_decoded_keys"]]
    mine = np.array([[dec["elements"][s][k] for k in keys] for s in SPECIES])
    np.testing.assert_allclose(mine, g[f"{tag}_decoded"], rtol=1e-14)
    assert dec["chi"]["Al-Ni"] == pytest.approx(float(g[f"{tag}_decoded_chi"]), rel=1e-15)
    assert dec["form"] == "zhou2004" and dec["r_cut"] == ps.r_cut


def test_parameter_set_refuses_derived_and_unknown_keys():
    el0 = {s: dict(ZHOU_2004[s]) for s in SPECIES}
    ps = fit.ZhouEAMParameterSet(el0, SPECIES)
    assert len(ps.x0) == 18 and ps.r_cut == pytest.approx(6.6904, abs=1e-3)
    with pytest.raises(ValueError, match="continuity"):
        fit.ZhouEAMParameterSet(el0, SPECIES, fit_keys=["F0"])
    with pytest.raises(ValueError, match="unknown"):
        fit.ZhouEAMParameterSet(el0, SPECIES, fit_keys=["zeta"])
    with pytest.raises(ValueError, match="no parameters"):
        fit.ZhouEAMParameterSet(el0, ["Al", "Xx"])
    assert fit.ZhouEAMParameterSet(el0, SPECIES, fit_keys=["chi"]).variable_names == ["chi:Al-Ni"]


def test_continuous_torch_equals_continuous():
    el = {s: dict(ZHOU_2004[s]) for s in ("Cu", "Ni", "Al", "Ag")}
    t = torch.tensor([[el[s][k] for k in ZHOU_KEYS] for s in el], dtype=torch.float64)
    mine = fit.continuous_torch(t).numpy()
    ref = np.array([[continuous(el[s])[k] for k in ZHOU_KEYS] for s in el])
    np.testing.assert_allclose(mine, ref, rtol=1e-14, atol=1e-15)


@pytest.mark.parametrize("tag", ["zhou", "zhou_chi"])
def test_table_torch_is_the_function_table(tag):
    """table_torch(x) holds the same rows as the EAMPotential of decode(x)
    builds for the device, and its x-gradient matches central differences."""
    g = golden("fit_alni_zhou")
    ps = param_sets()[tag]
    x = g[f"{tag}_x_test"]
    P = ps.table_torch(torch.tensor(x)).numpy()
    tab = ps.potential(x).function_table()
    assert tab["fused"]
    np.testing.assert_allclose(P, tab["P"], rtol=1e-14, atol=1e-15)
    w = torch.from_numpy(np.random.default_rng(5).normal(size=P.shape))
    xt = torch.tensor(x, requires_grad=True)
    (gx,) = torch.autograd.grad((ps.table_torch(xt) * w).sum(), xt)
    for q in range(len(x)):
        h = 1e-6
        xp, xm = np.array(x, float), np.array(x, float)
        xp[q] += h
        xm[q] -= h
        fd = float(((ps.table_torch(torch.tensor(xp)) - ps.table_torch(torch.tensor(xm))) * w).sum()) / (2 * h)
        assert float(gx[q]) == pytest.approx(fd, rel=1e-6, abs=1e-8)


@pytest.mark.parametrize("tag", ["zhou", "zhou_chi"])
def test_oracle_loss_matches_reference(tag):
    """The oracle's Zhou EAM loss at x0 and at the test point equals the
    reference's generic_loss_function value (the pin of the oracle's EAM
    loss)."""
    g = golden("fit_alni_zhou")
    ps = param_sets()[tag]
    st = structures()
    for x, key in ((ps.x0, "loss0"), (g[f"{tag}_x_test"], "loss_test")):
        d = ps.decode(x)["eam"]
        force = oracle.zhou_force(d["elements"], SPECIES, d["r_cut"], d["chi"])
        got = oracle.fit_loss(None, SPECIES, st, WEIGHTS, force=force)
        assert got == pytest.approx(float(g[f"{tag}_{key}"]), rel=1e-10)


@pytest.mark.parametrize("tag", ["zhou", "zhou_chi"])
def test_table_jacobian_equals_autograd(tag):
    """The complex-step table and x-Jacobian (the fused fit step's) equal
    table_torch and its autograd vector-Jacobian product."""
    g = golden("fit_alni_zhou")
    ps = param_sets()[tag]
    x = g[f"{tag}_x_test"]
    (P,), (J,) = ps.table_jacobian(x)
    xt = torch.tensor(x, requires_grad=True)
    Pt = ps.table_torch(xt)
    w = np.random.default_rng(4).normal(size=P.shape)
    (gt,) = torch.autograd.grad((Pt * torch.from_numpy(w)).sum(), xt)
    np.testing.assert_allclose(P, Pt.detach().numpy(), rtol=1e-14, atol=1e-15)
    gn = np.tensordot(J, w, axes=2)
    np.testing.assert_allclose(gn, gt.numpy(), rtol=1e-12, atol=1e-12 * np.abs(gn).max())
    np.testing.assert_allclose(ps.tables_np(x)[0], P, rtol=0, atol=0)
