"""Fitting pieces on the CPU: the parameter sets against the reference's
(variables, x0, bounds, decode), the differentiable decode, the tables, the
oracle's loss against the reference's loss value, and the sharding and
summation of the loss over two gloo ranks."""
import os

import numpy as np
import pytest
import torch

import oracle
from conftest import golden

from akitsushima_b200 import fit
from akitsushima_b200.published_parameters import TERSOFF_1989
from akitsushima_b200.tersoff import TersoffPotential, tersoff1989_to_triplets

SPECIES = ["Si", "C"]
KEYS = ("A", "B", "lambda1", "lambda2", "R", "D", "beta", "n", "c", "d", "h", "lambda3", "m", "gamma")


def structures():
    g = golden("fit_sic_t1989")
    out = []
    for q in range(int(g["n_structures"])):
        P = g[f"positions{q}"]
        out.append({"lattice": g[f"lattice{q}"], "positions": P, "atom_types": [str(t) for t in g[f"atom_types{q}"]],
                    "natoms": len(P), "ref_energy": float(g[f"ref_energy{q}"]), "ref_forces": g[f"ref_forces{q}"],
                    "ref_stress": g[f"ref_stress{q}"]})
    return out


def param_sets():
    el0 = {s: dict(TERSOFF_1989["elements"][s]) for s in SPECIES}
    chi0 = {"Si-C": TERSOFF_1989["chi"]["C-Si"]}
    return {"t1989": fit.Tersoff1989ParameterSet(el0, chi0, SPECIES),
            "multi": fit.MultiSpeciesTersoffParameterSet(tersoff1989_to_triplets(el0, chi0, SPECIES), SPECIES)}


@pytest.mark.parametrize("tag", ["t1989", "multi"])
def test_parameter_set_mirrors_reference(tag):
    g = golden("fit_sic_t1989")
    ps = param_sets()[tag]
    assert ps.variable_names == [str(n) for n in g[f"{tag}_names"]]
    np.testing.assert_allclose(ps.x0, g[f"{tag}_x0"], rtol=0, atol=1e-15)
    np.testing.assert_allclose([b[0] for b in ps.bounds], g[f"{tag}_lo"], rtol=1e-15)
    np.testing.assert_allclose([b[1] for b in ps.bounds], g[f"{tag}_hi"], rtol=1e-15)
    tab = ps.decode(g[f"{tag}_x_test"])["tersoff"]
    keys = [tuple(k.split("|")) for k in g[f"{tag}_decoded_keys"]]
    assert sorted(tab) == keys
    mine = np.array([[float(tab[k].get(n, np.nan)) for n in KEYS] for k in keys])
    np.testing.assert_allclose(mine, g[f"{tag}_decoded"], rtol=1e-14, equal_nan=True)


@pytest.mark.parametrize("tag", ["t1989", "multi"])
def test_decode_torch_equals_decode_and_tables(tag):
    g = golden("fit_sic_t1989")
    ps = param_sets()[tag]
    x = g[f"{tag}_x_test"]
    a = ps.decode(x)["tersoff"]
    b = ps.decode_torch(torch.tensor(x, dtype=torch.float64))["tersoff"]
    for k in a:
        for n, v in a[k].items():
            assert float(b[k][n]) == pytest.approx(v, rel=1e-14, abs=1e-300)
    tb, tri = fit.tables_from_records(b, SPECIES, "cpu")
    htb, htri = TersoffPotential(a, species=SPECIES).host_tables()
    np.testing.assert_allclose(tb.numpy(), htb, rtol=1e-14)
    np.testing.assert_allclose(tri.numpy(), htri, rtol=1e-14)
    assert fit.table_cutoff(tb) == pytest.approx(TersoffPotential(a, species=SPECIES).r_cut, rel=1e-15)


@pytest.mark.parametrize("tag", ["t1989", "multi"])
def test_vectorised_tables_equal_record_tables(tag):
    g = golden("fit_sic_t1989")
    ps = param_sets()[tag]
    x = torch.tensor(g[f"{tag}_x_test"], dtype=torch.float64, requires_grad=True)
    tb, tri = ps.tables_torch(x)
    tb2, tri2 = fit.tables_from_records(ps.decode_torch(x)["tersoff"], SPECIES, "cpu")
    np.testing.assert_allclose(tb.detach().numpy(), tb2.detach().numpy(), rtol=1e-14, atol=0)
    np.testing.assert_allclose(tri.detach().numpy(), tri2.detach().numpy(), rtol=1e-14, atol=0)
    w1, w2 = torch.randn_like(tb), torch.randn_like(tri)
    (ga,) = torch.autograd.grad((tb * w1).sum() + (tri * w2).sum(), x)
    (gb,) = torch.autograd.grad((tb2 * w1).sum() + (tri2 * w2).sum(), x)
    np.testing.assert_allclose(ga.numpy(), gb.numpy(), rtol=1e-12, atol=1e-12 * float(gb.abs().max()))


@pytest.mark.parametrize("tag", ["t1989", "multi"])
def test_oracle_loss_matches_reference(tag):
    g = golden("fit_sic_t1989")
    ps = param_sets()[tag]
    st = structures()
    w = {"energy": 1.0, "forces": 1.0, "stress": 0.1}
    for x, ref in ((g[f"{tag}_x0"], g[f"{tag}_loss0"]), (g[f"{tag}_x_test"], g[f"{tag}_loss_test"])):
        val = oracle.fit_loss(ps.decode(x)["tersoff"], SPECIES, st, w)
        assert val == pytest.approx(float(ref), rel=1e-11)


def test_shard_balance():
    n = [64, 64, 216, 216, 512, 8, 8]
    parts = fit.shard_structures(n, 3)
    assert sorted(sum(parts, [])) == list(range(len(n)))
    loads = [sum(n[q] for q in p) for p in parts]
    assert max(loads) - min(loads) <= max(n)
    assert parts == fit.shard_structures(n, 3)
    assert fit.shard_structures(n, 1) == [list(range(len(n)))]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = golden("fit_sic_t1989")
        ps = param_sets()["t1989"]
        st = structures()
        mine = fit.shard_structures([s["natoms"] for s in st], world)[rank]
        rec = ps.decode(g["t1989_x0"])["tersoff"]
        local = oracle.fit_loss(rec, SPECIES, [st[k] for k in mine], {"energy": 1.0, "forces": 1.0, "stress": 0.1})
        vec = fit.allreduce_sum(torch.tensor([local, float(len(mine))], dtype=torch.float64), world)
        q.put((rank, float(vec[0]), float(vec[1])))
    finally:
        dist.destroy_process_group()


def test_two_rank_loss_sum_equals_whole_set():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g = golden("fit_sic_t1989")
    for _, total, count in res:
        assert count == 4
        assert total == pytest.approx(float(g["t1989_loss0"]), rel=1e-11)


@pytest.mark.parametrize("tag", ["t1989", "multi"])
def test_table_jacobian_equals_autograd(tag):
    """The complex-step tables and x-Jacobians (the fused fit step's) equal
    tables_torch and its autograd vector-Jacobian product."""
    g = golden("fit_sic_t1989")
    ps = param_sets()[tag]
    x = g[f"{tag}_x_test"]
    tabs, jac = ps.table_jacobian(x)
    xt = torch.tensor(x, requires_grad=True)
    tt = ps.tables_torch(xt)
    rng = np.random.default_rng(3)
    ws = [rng.normal(size=a.shape) for a in tabs]
    (gt,) = torch.autograd.grad(sum((b * torch.from_numpy(w)).sum() for b, w in zip(tt, ws)), xt)
    gn = sum(np.tensordot(J, w, axes=w.ndim) for J, w in zip(jac, ws))
    for a, b in zip(tabs, tt):
        np.testing.assert_allclose(a, b.detach().numpy(), rtol=1e-15, atol=1e-15)
    np.testing.assert_allclose(gn, gt.numpy(), rtol=1e-13, atol=1e-13 * np.abs(gn).max())
