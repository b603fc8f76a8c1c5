"""Spatial decomposition of one structure (host side): the slab partition,
the halo's completeness against the oracle, and the two-rank exchange over
gloo.  The device evaluation of the slabs is in test_gpu_spatial.py."""
import os

import numpy as np
import pytest
import torch

import oracle
from conftest import DIAMOND, FCC, TERSOFF_SI, cubic

from akitsushima_b200 import ZHOU_2004
from akitsushima_b200.spatial import HALO_LISTS, combine, exchange, slab_partition


def _long_fcc(nz=20, seed=3):
    lat, pos, types = cubic(FCC, 3.58, 4, ["Cu", "Ni", "Ni", "Cu"], rattle=0.05, seed=seed)
    # 4 x 4 x nz cells: stack copies of the 4^3 block along z
    reps = nz // 4
    big = np.concatenate([pos + k * lat[2] for k in range(reps)])
    lat = lat.copy()
    lat[2] = lat[2] * reps
    return lat, big, types * reps


def _mic_dist(lat, a, b):
    d = (b - a) @ np.linalg.inv(lat)
    d -= np.rint(d)
    return np.linalg.norm(d @ lat, axis=-1)


@pytest.mark.parametrize("world", [1, 2, 3])
def test_partition_owns_each_atom_once_and_halo_is_complete(world):
    lat, pos, _ = _long_fcc()
    r_list = 6.1
    axis, parts = slab_partition(lat, pos, world, r_list)
    assert axis == 2
    owners = np.zeros(len(pos), int)
    for local, own in parts:
        assert np.all(np.diff(local) > 0)
        owners[local[own]] += 1
        missing = np.setdiff1d(np.arange(len(pos)), local)
        if len(missing) and own.any():
            d = np.min([_mic_dist(lat, pos[local[own]], pos[m]).min() for m in missing])
            assert d >= HALO_LISTS * r_list
    assert np.all(owners == 1)


def test_slab_forces_equal_whole_structure_oracle_eam():
    lat, pos, types = _long_fcc()
    spec = oracle.zhou_spec({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    rc = spec.r_cut
    i, j, _, _ = oracle.nl_build(lat, pos, rc, 0.3)
    _, F, _ = oracle.eam(spec, lat, pos, np.array(types), (i, j))
    _, parts = slab_partition(lat, pos, 2, rc + 0.3)
    for local, own in parts:
        assert len(local) < len(pos)          # a real halo, not the whole cell
        p = pos[local]
        il, jl, _, _ = oracle.nl_build(lat, p, rc, 0.3)
        _, f, _ = oracle.eam(spec, lat, p, np.array(types)[local], (il, jl))
        np.testing.assert_allclose(f[own], F[local[own]], rtol=0, atol=1e-11)


def test_slab_forces_equal_whole_structure_oracle_tersoff():
    lat, pos, _ = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.05, seed=4)
    big = np.concatenate([pos + k * lat[2] for k in range(4)])
    lat = lat.copy()
    lat[2] *= 4
    rc = TERSOFF_SI["R"] + TERSOFF_SI["D"]
    i, j, _, _ = oracle.nl_build(lat, big, rc, 0.3)
    _, F, _ = oracle.tersoff_single(TERSOFF_SI, lat, big, (i, j))
    _, parts = slab_partition(lat, big, 3, rc + 0.3)
    for local, own in parts:
        assert len(local) < len(big)
        il, jl, _, _ = oracle.nl_build(lat, big[local], rc, 0.3)
        _, f, _ = oracle.tersoff_single(TERSOFF_SI, lat, big[local], (il, jl))
        np.testing.assert_allclose(f[own], F[local[own]], rtol=0, atol=1e-11)


def test_combine_places_owned_forces():
    parts = [(np.array([0, 2]), np.ones((2, 3)), 1.5, np.arange(9.0)),
             (np.array([1]), 2 * np.ones((1, 3)), -0.5, np.ones(9))]
    e, F, w = combine(3, parts)
    assert e == 1.0
    np.testing.assert_array_equal(F[:, 0], [1, 2, 1])
    np.testing.assert_array_equal(w, np.arange(9.0) + 1)


def _exchange_rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        owned = [np.array([0, 3, 4]), np.array([1, 2])]
        f = np.full((len(owned[rank]), 3), 10.0 * (rank + 1)) + np.arange(len(owned[rank]))[:, None]
        e, F, w = exchange(5, owned, f, 1.0 + rank, np.full(9, rank + 0.5))
        q.put((rank, e, F, w))
    finally:
        dist.destroy_process_group()


def test_two_rank_exchange_gives_every_rank_the_whole_result():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_exchange_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = np.array([[10, 10, 10], [20, 20, 20], [21, 21, 21], [11, 11, 11], [12, 12, 12]], float)
    for _, e, F, w in res:
        assert e == 3.0
        np.testing.assert_array_equal(F, want)
        np.testing.assert_array_equal(w, np.full(9, 2.0))
