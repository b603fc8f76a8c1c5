"""Batched evaluation of many uneven, strained structures (GPU).

Thin members (any axis of one diamond cell) are replicated to the smallest
supercell the minimum image admits; the reference refuses them
(engine/neighborlist.py:489-572), so the oracle evaluates the same
replicated supercells and the results are mapped back (energy / k, first N
forces, stress unchanged).  Tolerances as tests/test_gpu_parity.py.
"""
import numpy as np
import pytest

import oracle
from conftest import DIAMOND, SW_SI, TERSOFF_SI, cubic, strained

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")


def _structures(n, seed, amp=0.03, rattle=0.1):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        na, nb, nc = rng.integers(1, 5, size=3)   # {1..4} cells per axis, as the benchmark set
        cells = np.array([[i, j, l] for i in range(na) for j in range(nb) for l in range(nc)])
        frac = (np.asarray(DIAMOND, float)[None] + cells[:, None]).reshape(-1, 3)
        lat = np.diag([na, nb, nc]).astype(float) * 5.431
        pos = frac * 5.431 + rng.normal(0, rattle, frac.shape)
        lat, pos = strained(lat, pos, amp, seed * 1000 + k)
        out.append((lat, pos, ["Si"] * len(pos)))
    return out


def _oracle(kind, lat, pos, r_list):
    from akitsushima_b200.system import replicate_thin
    L2, P2, _, reps = replicate_thin(lat, pos, np.zeros(len(pos), np.int32), r_list)
    k = int(np.prod(reps))
    rc = r_list - 0.3
    i, j, _, _ = oracle.nl_build(L2, P2, rc, 0.3)
    if kind == "tersoff":
        e, f, s = oracle.tersoff_single(TERSOFF_SI, L2, P2, (i, j))
    else:
        e, f, s = oracle.sw_single(SW_SI, L2, P2, (i, j))
    return e / k, f[:len(pos)], s


@pytest.mark.parametrize("kind", ["tersoff", "sw"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_matches_oracle(cuda_device, kind, precision):
    structs = _structures(12, seed=3)
    pot = (ak.TersoffPotential(TERSOFF_SI, species=["Si"]) if kind == "tersoff"
           else ak.StillingerWeberPotential(SW_SI, species=["Si"]))
    ev = ak.BatchedEvaluator(pot, structs, skin=0.3, precision=precision)
    e, f, s = ev.results()
    tol_e, tol_f, tol_s = (1e-10, 1e-8, 1e-8) if precision == "fp64" else (1e-6, 1e-5, 1e-5)
    for k, (lat, pos, _) in enumerate(structs):
        e0, f0, s0 = _oracle(kind, lat, pos, pot.r_cut + 0.3)
        n = len(pos)
        assert abs(e[k] - e0) / n < tol_e, (k, e[k], e0)
        assert np.abs(f[k] - f0).max() < tol_f
        assert np.abs(s[k] - s0).max() < tol_s


def test_graph_replay_and_autotune_agree(cuda_device):
    structs = _structures(20, seed=5)
    pot = ak.StillingerWeberPotential(SW_SI, species=["Si"])
    ev = ak.BatchedEvaluator(pot, structs, skin=0.3)
    e1, f1, s1 = ev.results()
    tuned = ev.autotune(candidates=(4, 8, 16), reps=2)
    assert tuned["lanes_per_atom"] in (4, 8, 16)
    ev.capture()
    e2, f2, s2 = ev.results()
    e3, f3, s3 = ev.results()
    np.testing.assert_allclose(e2, e1, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(e3, e2, rtol=0, atol=0)
    for a, b in zip(f1, f2):
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-12)


def test_batch_of_one_equals_single_call(cuda_device):
    lat, pos, types = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.1, seed=2)
    pot = ak.TersoffPotential(TERSOFF_SI, species=["Si"])
    ev = ak.BatchedEvaluator(pot, [(lat, pos, types)])
    e, f, s = ev.results()
    e0, f0, s0 = pot.compute(lat, pos, types)
    assert abs(e[0] - e0) < 1e-9 and np.abs(f[0] - f0).max() < 1e-10
