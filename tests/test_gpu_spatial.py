"""One structure evaluated as slabs (owned atoms + a halo; the owned atoms'
records summed), rank by rank on one GPU and combined: the whole
structure's energy, forces and virial.  EAM slabs carry a halo of one list
radius and get the halo atoms' F'(rho-bar) from their owners between the
embedding and force passes; Tersoff and SW slabs a halo of two.  No kernel
waits on another rank's, so the ranks run one after the other here, or as
two processes sharing the GPU over gloo (the exchanges go through host
memory)."""
import os
import numpy as np
import pytest

from conftest import DIAMOND, FCC, SW_SI, TERSOFF_SI, cubic

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")
from akitsushima_b200.spatial import SpatialForceFn, combine, evaluate_slabs  # noqa: E402
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
    parts = evaluate_slabs(pot, lat, pos, ids, world, device=cuda_device)
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


def _spatial_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        pot, (lat, pos, types) = _case("eam", "fp64")
        fn = SpatialForceFn(pot, device="cuda:0")
        out = []
        rng = np.random.default_rng(5)
        moves = [0.0, 0.02, 0.4]   # the same slab twice, then past the skin: a rebuild
        p = pos.copy()
        for amp in moves:
            p = p + rng.normal(0.0, amp, p.shape) if amp else p
            e, F, s = fn(lat, p, types)
            out.append((p.copy(), e, F, s))
        q.put((rank, out, fn.rebuild_count))
    finally:
        dist.destroy_process_group()


def test_two_process_eam_spatial_force_fn(cuda_device):
    """Two ranks (processes sharing cuda:0, gloo): SpatialForceFn with the
    EAM halo of one list radius and the F' exchange gives every rank the
    whole structure's energy, forces and stress, on three calls -- the slab
    and its list kept for a small move, rebuilt past the skin."""
    import multiprocessing as mp
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_spatial_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    pot, (lat, _, types) = _case("eam", "fp64")
    for _, out, rebuilds in res:
        assert rebuilds == 2
        for p, e, F, s in out:
            e0, F0, w0 = _whole(pot, lat, p, types, cuda_device)
            assert e == pytest.approx(e0, rel=1e-12)
            np.testing.assert_allclose(F, F0, rtol=0, atol=1e-10)
            np.testing.assert_allclose(s, w0.reshape(3, 3) / abs(np.linalg.det(lat)), rtol=0, atol=1e-12)
