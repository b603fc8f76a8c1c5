"""The Zhou EAM adjoint and the EAM fit gradient on the GPU, against central
finite differences (h = 1e-6 relative) and the reference's own loss value
and forward-difference fit gradient (tests/golden/fit_alni_zhou.npz)."""
import numpy as np
import pytest
import torch

from conftest import FCC, cubic, golden, strained

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")
from akitsushima_b200 import fit  # noqa: E402
from akitsushima_b200.published_parameters import ZHOU_2004  # noqa: E402
from test_fit_eam_cpu import SPECIES, WEIGHTS, param_sets, structures  # noqa: E402

# columns each row kind reads (density, embedding, like pair, cross pair)
COLS = {3: (0, 1, 5, 9), 6: (2, 3) + tuple(range(10, 20)), 4: (0, 4, 5, 6, 7, 8, 9),
        5: (0, 1, 4, 5, 6, 7, 8, 9, 20, 21, 24, 25, 26, 27, 28, 29, 42)}


def _batch(structs, species, device):
    from akitsushima_b200.system import species_ids
    return ak.Batch([s["lattice"] for s in structs], [s["positions"] for s in structs],
                    [species_ids(s["atom_types"], species) for s in structs], device=device)


def _case(name):
    """(param set, x, structures): Al-Ni on the golden cells plus an expanded
    and a compressed cell (every branch of the embedding function), or a
    three-element Cu-Ni-Al random alloy with distinct cross factors."""
    if name == "alni":
        g = golden("fit_alni_zhou")
        ps = param_sets()["zhou_chi"]
        x = g["zhou_chi_x_test"]
        st = structures()
        for a, n, seed in ((3.57 * 1.12, 4, 71), (3.57 * 0.93, 5, 72)):
            L, P, T = cubic(FCC, a, n, ["Al", "Ni", "Ni", "Ni"], rattle=0.05, seed=seed)
            st.append({"lattice": L, "positions": P, "atom_types": T})
        return ps, x, st, SPECIES
    sp = ["Cu", "Ni", "Al"]
    ps = fit.ZhouEAMParameterSet({s: dict(ZHOU_2004[s]) for s in sp}, sp,
                                 chi={"Cu-Ni": 0.97, "Cu-Al": 1.05, "Ni-Al": 1.1},
                                 fit_keys=["A", "B", "alpha", "beta", "F2", "eta", "chi"])
    rng = np.random.default_rng(9)
    L, P, _ = cubic(FCC, 3.6, 5, ["Cu"] * 4, rattle=0.07, seed=8)
    L, P = strained(L, P, 0.02, 10)
    T = [sp[k] for k in rng.integers(0, 3, len(P))]
    return ps, ps.x0, [{"lattice": L, "positions": P, "atom_types": T}], sp


@pytest.mark.parametrize("name", ["alni", "cunial"])
def test_eam_adjoint_matches_central_differences(cuda_device, name):
    ps, x, st, sp = _case(name)
    skel = ps.potential(x).function_table()
    ev = fit._EamTableEval(_batch(st, sp, cuda_device), 0.3, skel, ps.r_cut)
    ev.fused = 0   # the generic evaluation reads each row as the adjoint differentiates it
    P = ps.table_torch(torch.as_tensor(x)).to(cuda_device)
    E, F, Wv = ev.evaluate(P)
    rng = np.random.default_rng(5)
    gE = torch.as_tensor(rng.normal(size=E.shape), device=cuda_device)
    gF = torch.as_tensor(rng.normal(size=F.shape), device=cuda_device)
    gW = torch.as_tensor(rng.normal(size=Wv.shape), device=cuda_device)
    d_P = ev.adjoint(P, gE, gF, gW)
    d_P2 = ev.adjoint(P, gE, gF, gW)
    assert torch.equal(d_P, d_P2)   # deterministic

    def scalar(P_):
        e, f, w = ev.evaluate(P_.contiguous())
        return float((gE * e).sum() + (gF * f).sum() + (gW * w).sum())

    codes = skel["codes"]
    checks, zero = [], []
    for row in range(P.shape[0]):
        cols = COLS[int(codes[row])]
        for col in range(P.shape[1]):
            if col not in cols:
                zero.append(float(d_P[row, col]))
                continue
            v = float(P[row, col])
            h = 1e-6 * abs(v) if v != 0.0 else 1e-6
            Pp, Pm = P.clone(), P.clone()
            Pp[row, col] += h
            Pm[row, col] -= h
            checks.append((row, col, float(d_P[row, col]), (scalar(Pp) - scalar(Pm)) / (2 * h)))
    assert not any(zero)
    scale = max(abs(c[3]) for c in checks)
    bad = [c for c in checks if abs(c[2] - c[3]) > 1e-6 * max(abs(c[3]), 1e-3 * scale)]
    assert not bad, bad[:5]


@pytest.mark.parametrize("tag", ["zhou", "zhou_chi"])
def test_eam_loss_matches_reference(cuda_device, tag):
    g = golden("fit_alni_zhou")
    ps = param_sets()[tag]
    f = fit.PotentialFit(ps, structures(), WEIGHTS, device=cuda_device)
    for x, ref in ((g[f"{tag}_x0"], g[f"{tag}_loss0"]), (g[f"{tag}_x_test"], g[f"{tag}_loss_test"])):
        assert f.loss(x) == pytest.approx(float(ref), rel=1e-10)
    assert fit.generic_loss_function(g[f"{tag}_x0"], ps, structures(), WEIGHTS, ps.r_cut, None) == \
        pytest.approx(float(g[f"{tag}_loss0"]), rel=1e-10)


@pytest.mark.parametrize("tag", ["zhou", "zhou_chi"])
def test_eam_gradient_matches_central_differences_and_reference(cuda_device, tag):
    g = golden("fit_alni_zhou")
    ps = param_sets()[tag]
    f = fit.PotentialFit(ps, structures(), WEIGHTS, device=cuda_device)
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


@pytest.mark.parametrize("which", ["zhou", "t1989"])
def test_fused_step_equals_autograd_path(cuda_device, which):
    """loss_and_grad (fused loss kernel, complex-step table Jacobian) equals
    the torch autograd composition (EamEFS / TersoffEFS under the torch
    loss), Huber weights and a structure without stress included."""
    if which == "zhou":
        g = golden("fit_alni_zhou")
        ps, st, x = param_sets()["zhou_chi"], structures(), g["zhou_chi_x_test"]
        w = dict(WEIGHTS, huber_delta_energy=3.0, huber_delta_forces=0.05, huber_delta_stress=1.0)
    else:
        import test_fit_cpu as tc
        g = golden("fit_sic_t1989")
        ps, st, x = tc.param_sets()["t1989"], tc.structures(), g["t1989_x_test"]
        w = {"energy": 1.0, "forces": 1.0, "stress": 0.1, "huber_delta_energy": 2.0,
             "huber_delta_forces": 0.5, "huber_delta_stress": 1.0}
    st[1] = dict(st[1], weight=0.5, scale=2.0, ref_stress=None)
    f = fit.PotentialFit(ps, st, w, loss_type="huber", device=cuda_device)
    loss, grad = f.loss_and_grad(x)
    xt = torch.tensor(x, requires_grad=True)
    lt = f._local_loss(xt)
    (gt,) = torch.autograd.grad(lt, xt)
    assert loss == pytest.approx(float(lt.detach()), rel=1e-12)
    np.testing.assert_allclose(grad, gt.numpy(), rtol=1e-10, atol=1e-12 * np.abs(gt.numpy()).max())
    assert f.loss(x) == pytest.approx(loss, rel=1e-14)
