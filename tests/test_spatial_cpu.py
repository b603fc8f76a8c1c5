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


# ---- EAM with a one-list-radius halo and the F'(rho-bar) exchange ----------

def _eam_phases(pot, lat, pos, types):
    """The two halves of an EAM evaluation on the host (numpy, the package's
    host function forms): phase 1 -> (F, F') per atom; phase 2 (F') ->
    (forces, per-atom energy of the pairs each atom is the lower index of)."""
    from akitsushima_b200.eam import eval_spec
    sp = pot.species
    spc = np.array([sp.index(t) for t in types])
    i, j, _, _ = oracle.nl_build(lat, pos, pot.r_cut, 0.3)
    ii, jj, rij, r = oracle.mic_mask(lat, pos, i, j, pot.r_cut)
    n = len(pos)

    def phase1():
        rho = np.zeros(n)
        for k, s in enumerate(sp):
            v = eval_spec(pot.rho_spec[s], r)[0]
            np.add.at(rho, ii, np.where(spc[jj] == k, v, 0.0))
            np.add.at(rho, jj, np.where(spc[ii] == k, v, 0.0))
        rb = np.maximum(rho, 0.0)
        F, dF = np.zeros(n), np.zeros(n)
        for k, s in enumerate(sp):
            m = spc == k
            F[m], dF[m] = eval_spec(pot.F_spec[s], rb[m])
        return F, dF

    def phase2(dF):
        c = np.zeros(len(r))
        e_pair = np.zeros(len(r))
        for a, sa in enumerate(sp):
            for b, sb in enumerate(sp):
                m = (spc[ii] == a) & (spc[jj] == b)
                if not m.any():
                    continue
                phi, dphi = eval_spec(pot.phi_spec[frozenset((sa, sb))], r[m])
                drho_b = eval_spec(pot.rho_spec[sb], r[m])[1]
                drho_a = eval_spec(pot.rho_spec[sa], r[m])[1]
                c[m] = dphi + dF[ii[m]] * drho_b + dF[jj[m]] * drho_a
                e_pair[m] = phi
        f = (c / r)[:, None] * rij
        forces = np.zeros((n, 3))
        np.add.at(forces, ii, f)
        np.add.at(forces, jj, -f)
        e_low = np.zeros(n)
        np.add.at(e_low, np.minimum(ii, jj), e_pair)
        return forces, e_low

    return phase1, phase2


def _eam_case():
    from akitsushima_b200 import zhou_eam
    lat, pos, types = _long_fcc(nz=24, seed=8)
    return zhou_eam({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"]), lat, pos, list(types)


def test_host_eam_phases_equal_oracle():
    pot, lat, pos, types = _eam_case()
    p1, p2 = _eam_phases(pot, lat, pos, types)
    F, dF = p1()
    forces, e_low = p2(dF)
    spec = oracle.zhou_spec({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    i, j, _, _ = oracle.nl_build(lat, pos, spec.r_cut, 0.3)
    e0, f0, _ = oracle.eam(spec, lat, pos, np.array(types), (i, j))
    assert abs(F.sum() + e_low.sum() - e0) < 1e-9 * abs(e0)
    np.testing.assert_allclose(forces, f0, rtol=0, atol=1e-10)


def test_fprime_plan_covers_every_halo_atom():
    from akitsushima_b200.spatial import EAM_HALO_LISTS, fprime_plan
    lat, pos, _ = _long_fcc()
    _, parts = slab_partition(lat, pos, 3, 6.1, halo_lists=EAM_HALO_LISTS)
    plans = fprime_plan(parts)
    for r, ((local, own), plan) in enumerate(zip(parts, plans)):
        hpos, src, spos = plan["fill"]
        assert np.array_equal(np.sort(hpos), np.flatnonzero(~own))
        for k, q, p in zip(hpos, src, spos):
            qlocal, qown = parts[q]
            g = qlocal[plans[q]["send"][p]]
            assert g == local[k] and qown[plans[q]["send"][p]]
        assert len(plan["send"]) <= plan["width"]


def _eam_rank(rank, world, port, q):
    import torch.distributed as dist
    from akitsushima_b200.spatial import EAM_HALO_LISTS, exchange_fprime, fprime_plan
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pot, lat, pos, types = _eam_case()
        _, parts = slab_partition(lat, pos, world, pot.r_cut + 0.3, halo_lists=EAM_HALO_LISTS)
        plan = fprime_plan(parts)[rank]
        local, own = parts[rank]
        p1, p2 = _eam_phases(pot, lat, pos[local], [types[k] for k in local])
        F, dF = p1()
        dF = exchange_fprime(torch.as_tensor(dF), plan).numpy()
        forces, e_low = p2(dF)
        e = float(F[own].sum() + e_low[own].sum())
        ew = torch.tensor([e], dtype=torch.float64)
        dist.all_reduce(ew)
        q.put((rank, local[own], forces[own], float(ew[0]), len(local)))
    finally:
        dist.destroy_process_group()


def test_two_rank_eam_fprime_exchange_equals_whole_structure():
    """Two gloo ranks, a halo of one list radius each: the owned atoms'
    F'(rho-bar) is exact, the halo atoms' comes from their owners through
    exchange_fprime, and the owned forces and the summed energy equal the
    whole structure's oracle."""
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_eam_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pot, lat, pos, types = _eam_case()
    spec = oracle.zhou_spec({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    i, j, _, _ = oracle.nl_build(lat, pos, spec.r_cut, 0.3)
    e0, f0, _ = oracle.eam(spec, lat, pos, np.array(types), (i, j))
    seen = np.zeros(len(pos), int)
    for _, idx, f, e, n_local in res:
        assert n_local < len(pos)
        np.testing.assert_allclose(f, f0[idx], rtol=0, atol=1e-10)
        assert abs(e - e0) < 1e-9 * abs(e0)
        seen[idx] += 1
    assert np.all(seen == 1)
