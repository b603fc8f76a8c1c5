"""Force functions called concurrently from a thread pool, as the
reference's phonon and elastic solvers call them
(solvers/phonon.py:474-480, solvers/elastic.py:288-293): every thread
owns its list and workspace, so the results equal serial calls."""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from conftest import DIAMOND, FCC, TERSOFF_SI, cubic

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")


@pytest.mark.parametrize("case", ["tersoff", "eam"])
def test_concurrent_calls_equal_serial(cuda_device, case):
    if case == "tersoff":
        fn = ak.force_fn_from_config({"type": "Tersoff", "species": ["Si"], "params": TERSOFF_SI})
        lat, pos, types = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.05, seed=31)
    else:
        fn = ak.force_fn_from_config({"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"]},
                                     precision="fp64")
        lat, pos, types = cubic(FCC, 3.58, 4, ["Cu", "Ni", "Ni", "Cu"], rattle=0.05, seed=32)
    rng = np.random.default_rng(33)
    confs = [pos + rng.normal(0.0, 0.01, pos.shape) for _ in range(16)]
    serial = [fn(lat, p, list(types)) for p in confs]
    with ThreadPoolExecutor(max_workers=4) as ex:
        par = list(ex.map(lambda p: fn(lat, p, list(types)), confs))
    for (e0, f0, s0), (e1, f1, s1) in zip(serial, par):
        assert e1 == pytest.approx(e0, rel=1e-12, abs=1e-12)
        np.testing.assert_allclose(f1, f0, rtol=0, atol=1e-11)
        np.testing.assert_allclose(s1, s0, rtol=0, atol=1e-13)


def test_returned_forces_are_not_overwritten_by_later_calls(cuda_device):
    """The force arrays live in pinned host blocks that are recycled: a
    block is reused only when no array of it is alive, so results the caller
    keeps (or a view of them) survive later calls, and dropped ones give
    their blocks back."""
    fn = ak.force_fn_from_config({"type": "Tersoff", "species": ["Si"], "params": TERSOFF_SI})
    lat, pos, types = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.05, seed=34)
    rng = np.random.default_rng(35)
    confs = [pos + rng.normal(0.0, 0.01, pos.shape) for _ in range(7)]
    want = [fn(lat, p, list(types))[1].copy() for p in confs]
    kept = []
    for k, p in enumerate(confs):
        f = fn(lat, p, list(types))[1]
        kept.append(f[1:] if k % 2 else f)      # keep a view of some, the array of others
        for j, g in enumerate(kept):
            np.testing.assert_array_equal(g, want[j][1:] if j % 2 else want[j])
    kept.clear()
    for p, w in zip(confs, want):                # blocks recycled once dropped
        np.testing.assert_array_equal(fn(lat, p, list(types))[1], w)
