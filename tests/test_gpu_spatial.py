"""One structure evaluated as slabs (owned atoms + a two-list-radius halo,
the owned atoms' records summed), rank by rank on one GPU and combined:
the whole structure's energy, forces and virial.  No kernel waits on
another rank's, so the ranks run one after the other here."""
import numpy as np
import pytest

from conftest import DIAMOND, FCC, SW_SI, TERSOFF_SI, cubic

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")
from akitsushima_b200.spatial import SpatialForceFn, combine, evaluate_slab  # noqa: E402
from akitsushima_b200.system import species_ids  # noqa: E402


def _stack(lat, pos, types, reps):
    big = np.concatenate([pos + k * lat[2] for k in range(reps)])
    lat = lat.copy()
    lat[2] = lat[2] * reps
    return lat, big, list(types) * reps


def _case(kind, precision):
    if kind == "eam":
        pot = ak.zhou_eam({s: ak.ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"], precision=precision)
        lat, pos, types = cubic(FCC, 3.58, 4, ["Cu", "Ni", "Ni", "Cu"], rattle=0.06, seed=51)
        return pot, _stack(lat, pos, types, 5)
    lat, pos, types = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.08, seed=52)
    if kind == "tersoff":
        pot = ak.TersoffPotential(TERSOFF_SI, species=["Si"], precision=precision)
    else:
        pot = ak.StillingerWeberPotential(SW_SI, species=["Si"], precision=precision)
    return pot, _stack(lat, pos, types, 4)


def _whole(pot, lat, pos, types, dev):
    b = ak.Batch([lat], [pos], [species_ids(types, pot.species)], device=dev)
    dl = ak.DeviceNeighbourList(pot.r_cut + 0.3).build(b)
    r = pot.evaluate(b, dl)
    return float(r.energy[0].item()), r.forces.cpu().numpy(), r.virial[0].cpu().numpy()


@pytest.mark.parametrize("kind,precision", [("eam", "fp64"), ("eam", "mixed"), ("tersoff", "fp64"),
                                            ("sw", "fp64"), ("sw", "mixed")])
@pytest.mark.parametrize("world", [2, 3])
def test_slabs_combine_to_whole_structure(cuda_device, kind, precision, world):
    pot, (lat, pos, types) = _case(kind, precision)
    ids = species_ids(types, pot.species)
    e0, F0, w0 = _whole(pot, lat, pos, types, cuda_device)
    parts = [evaluate_slab(pot, lat, pos, ids, r, world, device=cuda_device) for r in range(world)]
    assert all(len(p[0]) < len(pos) for p in parts)
    e, F, w = combine(len(pos), parts)
    tol_f = 1e-10 if precision == "fp64" else 1e-5
    assert e == pytest.approx(e0, rel=1e-12 if precision == "fp64" else 1e-9)
    np.testing.assert_allclose(F, F0, rtol=0, atol=tol_f)
    np.testing.assert_allclose(w, w0, rtol=0, atol=1e-8 * max(1.0, np.abs(w0).max()))


def test_single_rank_spatial_force_fn_equals_force_fn(cuda_device):
    pot, (lat, pos, types) = _case("eam", "fp64")
    e, F, s = SpatialForceFn(pot)(lat, pos, types)
    e0, F0, w0 = _whole(pot, lat, pos, types, cuda_device)
    assert e == pytest.approx(e0, rel=1e-13)
    np.testing.assert_allclose(F, F0, rtol=0, atol=1e-12)
    np.testing.assert_allclose(s, w0.reshape(3, 3) / abs(np.linalg.det(lat)), rtol=0, atol=1e-14)
