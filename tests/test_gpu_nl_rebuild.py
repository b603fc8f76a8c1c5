"""The in-place list rebuild of device MD (mbf_nl_rebuild_async), through
the C ABI: with the staged workspace (one search: rows kept at the row
bound's stride, then sorted into the CSR) and with the plain one (count,
then fill) it gives exactly the general build's rows, reverse slots and
upper offsets; a row bound below the longest row is reported, with every
row left empty.  The general build (mbf_nl_build) gives one list with
and without staging rows, whatever their stride."""
import numpy as np
import pytest
import torch

from conftest import DIAMOND, FCC, cubic, strained

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")
from akitsushima_b200 import _lib  # noqa: E402
from akitsushima_b200.neighbourlist import DeviceNeighbourList  # noqa: E402

STATUS_ROW_TOO_LONG = 1


def _cases():
    lat, pos, _ = cubic(DIAMOND, 5.431, 4, ["Si"] * 8, rattle=0.1, seed=21)
    one = ([lat], [pos], 4.07)
    l2, p2, _ = cubic(FCC, 3.58, 5, ["Cu"] * 4, rattle=0.08, seed=22)
    l2, p2 = strained(l2, p2, 0.03, 23)
    l3, p3, _ = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.1, seed=24)
    many = ([l2, l3], [p2, p3], 6.1)
    l4, p4, _ = cubic(FCC, 3.58, 8, ["Cu"] * 4, rattle=0.08, seed=25)
    long_rows = ([l4], [p4], 9.0)   # ~266 entries a row: the shared-memory sort
    return {"si512": one, "batch_fcc_si": many, "fcc_long_rows": long_rows}


def _rebuild(batch, ref, limit, staged):
    L = _lib.lib()
    dev = batch.device
    grids, n_cells = ref._grid_table(batch)
    grids_t = torch.as_tensor(grids, device=dev)
    N = batch.n_atoms
    plain = int(L.mbf_nl_workspace_bytes(N, n_cells))
    need = int(L.mbf_nl_rebuild_workspace_bytes(N, n_cells, limit)) if staged else plain
    assert need > plain if staged else True
    ws = torch.empty(need, dtype=torch.uint8, device=dev)
    cap = ref.n_slots + 1024
    row_off = torch.full((N + 1,), -7, dtype=torch.int32, device=dev)
    upper = torch.full((N,), -7, dtype=torch.int32, device=dev)
    nbr = torch.full((cap,), -7, dtype=torch.int32, device=dev)
    rev = torch.full((cap,), -7, dtype=torch.int32, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    st = torch.cuda.current_stream(dev).cuda_stream
    _lib.check(L.mbf_nl_rebuild_async(batch.mbf_system(), _lib.ptr(grids_t), n_cells, ref.r_list, _lib.ptr(ws), need,
                                      _lib.ptr(row_off), _lib.ptr(nbr), _lib.ptr(rev), _lib.ptr(upper), cap, limit,
                                      _lib.ptr(status), st), "mbf_nl_rebuild_async")
    torch.cuda.synchronize(dev)
    return row_off.cpu().numpy(), upper.cpu().numpy(), nbr.cpu().numpy(), rev.cpu().numpy(), int(status.item())


@pytest.mark.parametrize("case", ["si512", "batch_fcc_si", "fcc_long_rows"])
@pytest.mark.parametrize("staged", [True, False])
def test_rebuild_equals_general_build(cuda_device, case, staged):
    lats, poss, r_list = _cases()[case]
    ids = [np.zeros(len(p), np.int32) for p in poss]
    batch = ak.Batch(lats, poss, ids, device=cuda_device)
    ref = DeviceNeighbourList(r_list).build(batch)
    N, ns = batch.n_atoms, ref.n_slots
    want = (ref.row_off[:N + 1].cpu().numpy(), ref.upper[:N].cpu().numpy(), ref.nbr[:ns].cpu().numpy(),
            ref.rev[:ns].cpu().numpy())
    limit = ref.max_row + 3
    for _ in range(2):   # the second call reuses the same workspace contents
        row_off, upper, nbr, rev, status = _rebuild(batch, ref, limit, staged)
        assert status == 0
        np.testing.assert_array_equal(row_off, want[0])
        np.testing.assert_array_equal(upper, want[1])
        np.testing.assert_array_equal(nbr[:ns], want[2])
        np.testing.assert_array_equal(rev[:ns], want[3])


@pytest.mark.parametrize("staged", [True, False])
def test_row_bound_too_small_is_reported(cuda_device, staged):
    lats, poss, r_list = _cases()["si512"]
    batch = ak.Batch(lats, poss, [np.zeros(len(poss[0]), np.int32)], device=cuda_device)
    ref = DeviceNeighbourList(r_list).build(batch)
    row_off, upper, _, _, status = _rebuild(batch, ref, ref.max_row - 2, staged)
    assert status & STATUS_ROW_TOO_LONG
    assert not row_off.any() and not upper.any()


def _build(batch, r_list, grids_t, n_cells, ws_bytes, cap):
    L = _lib.lib()
    dev = batch.device
    N = batch.n_atoms
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    row_off = torch.full((N + 1,), -7, dtype=torch.int32, device=dev)
    upper = torch.full((N,), -7, dtype=torch.int32, device=dev)
    nbr = torch.full((cap,), -7, dtype=torch.int32, device=dev)
    rev = torch.full((cap,), -7, dtype=torch.int32, device=dev)
    n_slots, max_row = _lib._ll(0), _lib._i(0)
    st = torch.cuda.current_stream(dev).cuda_stream
    _lib.check(L.mbf_nl_build(batch.mbf_system(), _lib.ptr(grids_t), n_cells, r_list, _lib.ptr(ws), ws_bytes,
                              _lib.ptr(row_off), _lib.ptr(nbr), _lib.ptr(rev), _lib.ptr(upper), cap, n_slots,
                              max_row, st), "mbf_nl_build")
    torch.cuda.synchronize(dev)
    ns = int(n_slots.value)
    return (row_off.cpu().numpy(), upper.cpu().numpy(), nbr[:ns].cpu().numpy(), rev[:ns].cpu().numpy(),
            int(max_row.value))


@pytest.mark.parametrize("case", ["si512", "batch_fcc_si", "fcc_long_rows"])
def test_build_staging_widths_agree(cuda_device, case):
    """mbf_nl_build with no staging rows (count, then fill), with a stride
    below the longest row (the staged search falls back to the fill) and
    with one above it (a single search) gives one list."""
    lats, poss, r_list = _cases()[case]
    batch = ak.Batch(lats, poss, [np.zeros(len(p), np.int32) for p in poss], device=cuda_device)
    ref = DeviceNeighbourList(r_list).build(batch)
    grids, n_cells = ref._grid_table(batch)
    grids_t = torch.as_tensor(grids, device=cuda_device)
    L = _lib.lib()
    N = batch.n_atoms
    plain = int(L.mbf_nl_workspace_bytes(N, n_cells))
    cap = ref.n_slots + 64
    outs = [_build(batch, r_list, grids_t, n_cells, plain, cap)]
    for stride in (ref.max_row - 5, ref.max_row, ref.max_row + 40):
        outs.append(_build(batch, r_list, grids_t, n_cells,
                           int(L.mbf_nl_rebuild_workspace_bytes(N, n_cells, stride)), cap))
    for o in outs:
        assert o[4] == ref.max_row
        for k in range(4):
            np.testing.assert_array_equal(o[k], outs[0][k])
    np.testing.assert_array_equal(outs[0][2], ref.nbr[:ref.n_slots].cpu().numpy())


def _criterion(lat0, ref, lat, pos, r_list, r_cut):
    """The reference's decision (engine/neighborlist.py:653-673), restated."""
    if np.allclose(lat, lat0, atol=1e-12):
        sigma_min, M = 1.0, np.eye(3)
    else:
        M = np.linalg.inv(lat0) @ lat
        sigma_min = float(np.linalg.svd(M, compute_uv=False)[-1])
    dr = pos - ref @ M
    frac = dr @ np.linalg.inv(lat)
    frac -= np.round(frac)
    d_max = float(np.max(np.linalg.norm(frac @ lat, axis=1)))
    return sigma_min * r_list - 2.0 * d_max <= r_cut


def test_check_and_rebuild_under_lattice_change(cuda_device):
    """The skin criterion with the cell deforming between builds
    (engine/neighborlist.py:653-668): sigma_min(inv(L_build) L_now) r_list
    - 2 max|MIC(r - r_ref M)| <= r_cut.  An affine strain that keeps
    sigma_min r_list above r_cut does not rebuild (the old rule rebuilt on
    any lattice change), a compression beyond it does, and a small strain
    plus a non-affine move crosses over where the restated criterion does;
    a move across the strained cell's face is not motion."""
    lat0, pos0, _ = cubic(DIAMOND, 5.431, 4, ["Si"] * 8, rattle=0.05, seed=2)
    r_cut, skin = 3.0, 0.5
    nl = ak.NeighbourList(r_cut, skin_width=skin)
    assert nl.check_and_rebuild(lat0, pos0) is True
    # 1 % affine strain: sigma_min ~ 0.99, 0.99 * 3.5 > 3: no rebuild
    M = np.eye(3) + np.array([[0.01, 0.004, 0.0], [0.004, -0.008, 0.002], [0.0, 0.002, 0.005]])
    lat1, pos1 = lat0 @ M, pos0 @ M
    assert _criterion(lat0, pos0, lat1, pos1, r_cut + skin, r_cut) is False
    assert nl.check_and_rebuild(lat1, pos1) is False
    # the same strain with one atom moved 0.1 A (2 d = 0.2 < 0.99*3.5 - 3): no
    # rebuild; 0.3 A: rebuild
    moved = pos1.copy()
    moved[7] += [0.1, 0.0, 0.0]
    assert _criterion(lat0, pos0, lat1, moved, 3.5, 3.0) is False
    assert nl.check_and_rebuild(lat1, moved) is False
    moved[7] += [0.2, 0.0, 0.0]
    assert _criterion(lat0, pos0, lat1, moved, 3.5, 3.0) is True
    assert nl.check_and_rebuild(lat1, moved) is True
    # after that rebuild the reference frame is lat1: a 15 % compression
    # (sigma_min 0.85, 0.85 * 3.5 < 3) rebuilds with no atom moving
    lat2, pos2 = lat1 * 0.85, moved * 0.85
    assert nl.check_and_rebuild(lat2, pos2) is True
    assert nl.rebuild_count == 3
    # random strains and moves: the device decision equals the restated one
    rng = np.random.default_rng(4)
    for _ in range(12):
        nl.build(lat0, pos0)
        e = rng.uniform(-0.04, 0.04, (3, 3))
        Mk = np.eye(3) + 0.5 * (e + e.T)
        pk = pos0 @ Mk + rng.normal(0.0, 0.03, pos0.shape)
        pk[rng.integers(len(pk))] += lat0[0] @ Mk   # a periodic image, not a move
        want = _criterion(lat0, pos0, lat0 @ Mk, pk, 3.5, 3.0)
        assert nl.needs_rebuild(lat0 @ Mk, pk) is want
