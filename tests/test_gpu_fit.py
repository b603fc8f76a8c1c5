"""The Tersoff adjoint and the fit gradient on the GPU, against central
finite differences (h = 1e-6 relative) and the reference's own loss value
and forward-difference fit gradient (tests/golden/fit_sic_t1989.npz)."""
import numpy as np
import pytest
import torch

from conftest import DIAMOND, TERSOFF_SI, cubic, golden, strained

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")
from akitsushima_b200 import fit  # noqa: E402
from test_fit_cpu import SPECIES, param_sets, structures  # noqa: E402

W = {"energy": 1.0, "forces": 1.0, "stress": 0.1}


def _batch(structs, species, device):
    from akitsushima_b200.system import species_ids
    return ak.Batch([s["lattice"] for s in structs], [s["positions"] for s in structs],
                    [species_ids(s["atom_types"], species) for s in structs], device=device)


def _vjp_case(device, records, species, structs, seed):
    ev = fit._TableEval(_batch(structs, species, device), skin=0.3)
    tb, tri = fit.tables_from_records(records, species, device)
    E, F, Wv = ev.evaluate(tb, tri)
    rng = np.random.default_rng(seed)
    gE = torch.as_tensor(rng.normal(size=E.shape), device=device)
    gF = torch.as_tensor(rng.normal(size=F.shape), device=device)
    gW = torch.as_tensor(rng.normal(size=Wv.shape), device=device)
    d_tb, d_tri = ev.adjoint(tb, tri, gE, gF, gW)

    def scalar(tb_, tri_):
        e, f, w = ev.evaluate(tb_.contiguous(), tri_.contiguous())
        return float((gE * e).sum() + (gF * f).sum() + (gW * w).sum())

    checks = []
    for tab, grad, cols, other in ((tb, d_tb, range(1, 9), "tb"), (tri, d_tri, (1, 2, 3, 4, 6), "tri")):
        for row in range(tab.shape[0]):
            if float(tab[row, 0]) == 0.0:
                continue
            for col in cols:
                v = float(tab[row, col])
                h = 1e-6 * abs(v) if v != 0.0 else 1e-6
                tp, tm = tab.clone(), tab.clone()
                tp[row, col] += h
                tm[row, col] -= h
                if other == "tb":
                    fd = (scalar(tp, tri) - scalar(tm, tri)) / (2 * h)
                else:
                    fd = (scalar(tb, tp) - scalar(tb, tm)) / (2 * h)
                checks.append((other, row, col, float(grad[row, col]), fd))
    return checks


@pytest.mark.parametrize("case", ["si", "sic"])
def test_adjoint_matches_central_differences(cuda_device, case):
    if case == "si":
        lat, pos, types = cubic(DIAMOND, 5.431, 2, ["Si"] * 8, rattle=0.1, seed=3)
        lat, pos = strained(lat, pos, 0.02, 4)
        structs = [{"lattice": lat, "positions": pos, "atom_types": types}]
        p = dict(TERSOFF_SI, lambda3=1.3, m=3.0)
        records, species = {("Si", "Si", "Si"): p}, ["Si"]
    else:
        g = golden("fit_sic_t1989")
        ps = param_sets()["multi"]
        records = ps.decode(g["multi_x_test"])["tersoff"]
        records = {k: dict(v, lambda3=0.7, gamma=1.1) for k, v in records.items()}
        structs, species = structures()[:2], SPECIES
    checks = _vjp_case(cuda_device, records, species, structs, seed=5)
    scale = max(abs(fd) for *_, fd in checks)
    bad = [c for c in checks if abs(c[3] - c[4]) > 1e-6 * max(abs(c[4]), 1e-3 * scale)]
    assert not bad, bad[:5]


@pytest.mark.parametrize("tag", ["t1989", "multi"])
def test_loss_matches_reference(cuda_device, tag):
    g = golden("fit_sic_t1989")
    ps = param_sets()[tag]
    f = fit.TersoffFit(ps, structures(), W, device=cuda_device)
    for x, ref in ((g[f"{tag}_x0"], g[f"{tag}_loss0"]), (g[f"{tag}_x_test"], g[f"{tag}_loss_test"])):
        assert f.loss(x) == pytest.approx(float(ref), rel=1e-10)
    assert fit.generic_loss_function(g[f"{tag}_x0"], ps, structures(), W, 3.5, None) == \
        pytest.approx(float(g[f"{tag}_loss0"]), rel=1e-10)


@pytest.mark.parametrize("tag", ["t1989", "multi"])
def test_gradient_matches_central_differences_and_reference(cuda_device, tag):
    g = golden("fit_sic_t1989")
    ps = param_sets()[tag]
    f = fit.TersoffFit(ps, structures(), W, device=cuda_device)
    x0 = g[f"{tag}_x0"]
    loss, grad = f.loss_and_grad(x0)
    assert loss == pytest.approx(float(g[f"{tag}_loss0"]), rel=1e-10)
    fd = np.empty_like(grad)
    for q in range(len(x0)):
        h = 1e-6 * max(abs(x0[q]), 1.0)
        xp, xm = x0.copy(), x0.copy()
        xp[q] += h
        xm[q] -= h
        fd[q] = (f.loss(xp) - f.loss(xm)) / (2 * h)
    scale = np.abs(fd).max()
    np.testing.assert_allclose(grad, fd, rtol=1e-6, atol=1e-6 * scale)
    # the reference's forward differences (step 1e-7 max(1, |x|)) carry an
    # O(h) truncation error of their own
    ref = g[f"{tag}_grad_fd"]
    np.testing.assert_allclose(grad, ref, rtol=1e-3, atol=1e-4 * np.abs(ref).max())


def test_huber_and_weights(cuda_device):
    g = golden("fit_sic_t1989")
    ps = param_sets()["t1989"]
    st = structures()
    st[1] = dict(st[1], weight=0.5, scale=2.0, ref_stress=None)
    w = dict(W, huber_delta_energy=5.0, huber_delta_forces=1.0, huber_delta_stress=2.0)
    f = fit.TersoffFit(ps, st, w, loss_type="huber", device=cuda_device)
    x0 = g["t1989_x0"]
    loss, grad = f.loss_and_grad(x0)
    fd = np.empty_like(grad)
    for q in range(len(x0)):
        h = 1e-6 * max(abs(x0[q]), 1.0)
        xp, xm = x0.copy(), x0.copy()
        xp[q] += h
        xm[q] -= h
        fd[q] = (f.loss(xp) - f.loss(xm)) / (2 * h)
    np.testing.assert_allclose(grad, fd, rtol=1e-6, atol=1e-6 * np.abs(fd).max())
