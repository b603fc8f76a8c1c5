"""Device-resident Verlet-skin cell list with the reference's NeighbourList API.

``NeighbourList(r_cut, skin_width, backend='cuda')`` mirrors the reference's
engine/neighborlist.py:390-814 (build, check_and_rebuild, mark_dirty,
get_candidate_pairs, get_pairs_arrays, get_pairs, rebuild_count,
step_count, active_backend, r_list) with the pair list held on the GPU as a
two-way CSR.  The build is libmbforce's ``mbf_nl_build``: cell binning by an
integer counting sort, count -> scan -> fill of the rows, rows sorted, and a
reverse-slot index.  The pair set equals the reference's bit for bit.
"""
import threading
from collections import OrderedDict

import numpy as np
import torch

from . import _lib
from .system import Batch, cell_grid, cell_widths, check_min_image, default_device

_BACKENDS = ("auto", "cuda")
NL_MAX_ROW = 1024   # the longest row the device row sort holds (mbf_nl.cu)


class DeviceNeighbourList:
    """Two-way CSR of every pair within ``r_list`` of a :class:`Batch`.

    Rows are sorted ascending; ``rev[slot(a->b)] = slot(b->a)``.  Buffers
    are reused across rebuilds and grown by 25 % when a build needs more.
    """

    def __init__(self, r_list):
        if not r_list > 0.0:
            raise ValueError(f"r_list must be positive, got {r_list}")
        self.r_list = float(r_list)
        self.n_atoms = 0
        self.n_slots = 0
        self.max_row = 0
        self.row_off = None
        self.nbr = None
        self.rev = None
        self.upper = None
        self._ws = None
        self._grids = None
        self.device = None

    def _grid_table(self, batch):
        rows, first = [], 0
        for s in range(batch.n_struct):
            widths = cell_widths(batch.lattices[s])
            check_min_image(batch.lattices[s], self.r_list, widths=widths)
            nc, w = cell_grid(batch.lattices[s], self.r_list, widths=widths)
            rows.append([nc[0], nc[1], nc[2], first, w[0], w[1], w[2], 0])
            first += int(nc[0] * nc[1] * nc[2])
        return np.array(rows, np.int32), first

    def expected_rows(self, batch):
        """(total slots, longest mean row) expected from each structure's
        number density and the sphere of radius r_list."""
        cnt = np.asarray(batch.counts, float)
        if not len(cnt):
            return 0.0, 0.0
        rows = cnt / np.asarray(batch.volumes, float) * (4.0 / 3.0 * np.pi * self.r_list ** 3)
        return float(np.sum(cnt * rows)), float(np.max(rows))

    def build(self, batch, capacity=None):
        """(Re)build from the batch's current positions and lattices.
        ``capacity``: slots to reserve in nbr / rev before the first build
        (grown as needed either way)."""
        dev = batch.device
        self.device = dev
        grids, n_cells = self._grid_table(batch)
        self._grids = torch.as_tensor(grids, device=dev)
        N = batch.n_atoms
        self.n_atoms = N
        L = _lib.lib()
        # the rows expected from each structure's number density: the slot
        # capacity 20 % over their sum, and the staging stride (the workspace
        # beyond mbf_nl_workspace_bytes) 30 % over the longest, so one
        # search usually suffices
        slots, longest = self.expected_rows(batch)
        est = int(1.2 * slots) + 1024
        stride = min(NL_MAX_ROW, int(1.3 * longest) + 16)
        need = int(L.mbf_nl_rebuild_workspace_bytes(N, n_cells, stride) if N else L.mbf_nl_workspace_bytes(N, n_cells))
        if self._ws is None or self._ws.numel() < need or self._ws.device != dev:
            self._ws = torch.empty(need, dtype=torch.uint8, device=dev)
        if self.row_off is None or self.row_off.numel() < N + 1 or self.row_off.device != dev:
            self.row_off = torch.empty(N + 1, dtype=torch.int32, device=dev)
            self.upper = torch.empty(max(N, 1), dtype=torch.int32, device=dev)
        if capacity is not None:
            est = max(est, int(capacity))
        if self.nbr is None or self.nbr.device != dev or self.nbr.numel() < est and capacity is not None:
            self.nbr = torch.empty(est, dtype=torch.int32, device=dev)
            self.rev = torch.empty(est, dtype=torch.int32, device=dev)
        sysd = batch.mbf_system()
        stream = torch.cuda.current_stream(dev).cuda_stream
        n_slots = _lib._ll(0)
        max_row = _lib._i(0)
        for _ in range(3):
            rc = L.mbf_nl_build(sysd, _lib.ptr(self._grids), n_cells, self.r_list, _lib.ptr(self._ws),
                                self._ws.numel(), _lib.ptr(self.row_off), _lib.ptr(self.nbr), _lib.ptr(self.rev),
                                _lib.ptr(self.upper), self.nbr.numel(), n_slots, max_row, stream)
            if rc == _lib.MBF_ERR_CAPACITY:
                cap = int(n_slots.value * 1.25) + 1024
                self.nbr = torch.empty(cap, dtype=torch.int32, device=dev)
                self.rev = torch.empty(cap, dtype=torch.int32, device=dev)
                continue
            _lib.check(rc, "mbf_nl_build")
            break
        else:
            raise RuntimeError("mbf_nl_build: capacity did not converge")
        self.n_slots = int(n_slots.value)
        self.max_row = int(max_row.value)
        return self

    def mbf_nlist(self):
        return _lib.MbfNlist(self.n_atoms, self.n_slots, self.max_row, _lib.ptr(self.row_off),
                             _lib.ptr(self.nbr), _lib.ptr(self.rev), _lib.ptr(self.upper))

    def half_pairs(self):
        """Canonical (i < j, sorted by (i, j)) pairs as device int32 tensors."""
        n_half = self.n_slots // 2
        dev = self.device
        pi = torch.empty(n_half, dtype=torch.int32, device=dev)
        pj = torch.empty(n_half, dtype=torch.int32, device=dev)
        if n_half == 0:
            return pi, pj
        L = _lib.lib()
        need = int(L.mbf_nl_half_workspace_bytes(self.n_atoms))
        ws = torch.empty(need, dtype=torch.uint8, device=dev)
        nl = self.mbf_nlist()
        _lib.check(L.mbf_nl_half_pairs(nl, _lib.ptr(pi), _lib.ptr(pj), _lib.ptr(ws), need,
                                       torch.cuda.current_stream(dev).cuda_stream),
                   "mbf_nl_half_pairs")
        return pi, pj

    @classmethod
    def from_pairs(cls, n_atoms, pair_i, pair_j, r_list, device):
        """Two-way CSR from half pairs (any order), e.g. a list built by the
        reference's CPU NeighbourList, using device sorts."""
        self = cls(r_list)
        self.device = device
        i = torch.as_tensor(np.asarray(pair_i), device=device).to(torch.int64)
        j = torch.as_tensor(np.asarray(pair_j), device=device).to(torch.int64)
        src = torch.cat([i, j])
        dst = torch.cat([j, i])
        key = src * n_atoms + dst
        skey, order = torch.sort(key)
        nbr = dst[order]
        cnt = torch.bincount(src, minlength=n_atoms)
        row_off = torch.zeros(n_atoms + 1, dtype=torch.int64, device=device)
        row_off[1:] = torch.cumsum(cnt, 0)
        rkey = nbr * n_atoms + (skey // n_atoms)
        rev = torch.searchsorted(skey, rkey)
        self.n_atoms = n_atoms
        self.n_slots = int(nbr.numel())
        self.max_row = int(cnt.max().item()) if n_atoms else 0
        self.row_off = row_off.to(torch.int32)
        self.nbr = nbr.to(torch.int32)
        self.rev = rev.to(torch.int32)
        lower = torch.zeros(n_atoms, dtype=torch.int64, device=device)
        lower.index_add_(0, src[order], (nbr < src[order]).to(torch.int64))
        self.upper = (row_off[:-1] + lower).to(torch.int32)
        return self


class NeighbourList:
    """Verlet-skin cell list on the GPU (reference engine/neighborlist.py:390).

    Parameters
    ----------
    r_cut, skin_width : as the reference; r_list = r_cut + skin_width.
    backend           : 'cuda' (or 'auto', which means 'cuda' here).
    use_numba, canonical_order : accepted for signature compatibility; the
                        device list is always in canonical order.
    device            : torch device (default: the current CUDA device).
    """

    def __init__(self, r_cut, skin_width=0.5, backend="cuda", use_numba=None,
                 canonical_order=True, device=None):
        if r_cut <= 0.0:
            raise ValueError(f"NeighbourList: r_cut must be positive, got {r_cut}.")
        if backend not in _BACKENDS:
            raise ValueError(f"NeighbourList: backend must be one of {_BACKENDS}, got "
                             f"{backend!r} (this package builds lists on the GPU only).")
        self.r_cut = float(r_cut)
        self.skin_width = float(skin_width)
        self.r_list = self.r_cut + self.skin_width
        self.backend = backend
        self.use_numba = use_numba
        self.canonical_order = True
        self._device = torch.device(device) if device is not None else None
        self._lattice = None
        self._ref_pos = None
        self._n_builds = 0
        self._n_steps = 0
        self._dirty = False
        self._dnl = DeviceNeighbourList(self.r_list)
        self._batch = None
        self._half = None

    @property
    def active_backend(self):
        return "cuda"

    @property
    def rebuild_count(self):
        return self._n_builds

    @property
    def step_count(self):
        return self._n_steps

    @property
    def device_list(self):
        return self._dnl

    @property
    def n_atoms(self):
        return self._dnl.n_atoms

    def _check_min_cell(self, lattice):
        widths = cell_widths(lattice)
        if self.r_list >= float(np.min(widths)) / 2.0:
            check_min_image(lattice, self.r_list, "NeighbourList: r_cut + skin_width")

    def build(self, lattice, positions):
        """Force-rebuild the list (engine/neighborlist.py:574-585)."""
        lattice = np.asarray(lattice, dtype=np.float64)
        self._check_min_cell(lattice)
        dev = self._device or default_device()
        if isinstance(positions, torch.Tensor):
            pos_t = positions.to(dev, torch.float64).reshape(-1, 3)
            n = pos_t.shape[0]
        else:
            pos_np = np.ascontiguousarray(positions, dtype=np.float64)
            n = len(pos_np)
        if self._batch is None or self._batch.n_atoms != n or self._batch.device != dev:
            self._batch = Batch.single(lattice, np.zeros((n, 3)), np.zeros(n, np.int32), device=dev)
        else:
            self._batch.set_lattice(0, lattice)
        self._batch.set_positions(pos_t if isinstance(positions, torch.Tensor) else pos_np)
        self._dnl.build(self._batch)
        self._lattice = lattice.copy()
        self._ref_pos = self._batch.pos.clone()
        self._half = None
        self._n_builds += 1

    def build_batch(self, batch):
        """Build from an existing device :class:`Batch` of one structure."""
        if batch.n_struct != 1:
            raise ValueError("NeighbourList.build_batch: one structure expected")
        self._check_min_cell(batch.lattices[0])
        self._batch = batch
        self._dnl.build(batch)
        self._lattice = batch.lattices[0].copy()
        self._ref_pos = batch.pos.clone()
        self._half = None
        self._n_builds += 1

    def mark_dirty(self):
        self._dirty = True

    def needs_rebuild(self, lattice, positions):
        """The reference's criterion (engine/neighborlist.py:653-673):
        rebuild iff sigma_min(M) r_list - 2 d_max <= r_cut, with M the lattice
        map since the build and d_max the largest minimum-imaged non-affine
        displacement (computed on the device)."""
        lattice = np.asarray(lattice, dtype=np.float64)
        if np.allclose(lattice, self._lattice, atol=1e-12):
            sigma_min = 1.0
            M = np.eye(3)
        else:
            M = np.linalg.inv(self._lattice) @ lattice
            sigma_min = float(np.linalg.svd(M, compute_uv=False)[-1])
        b = self._batch
        b.set_lattice(0, lattice)
        if isinstance(positions, torch.Tensor):
            b.set_positions(positions)
        else:
            b.set_positions(np.ascontiguousarray(positions, dtype=np.float64))
        dev = b.device
        maps = torch.as_tensor(np.ascontiguousarray(M.reshape(1, 9)), device=dev)
        dmax = torch.empty(1, dtype=torch.float64, device=dev)
        _lib.check(_lib.lib().mbf_nl_max_displacement(
            b.mbf_system(), _lib.ptr(self._ref_pos), _lib.ptr(maps), _lib.ptr(dmax),
            torch.cuda.current_stream(dev).cuda_stream), "mbf_nl_max_displacement")
        d_max = float(dmax.item())
        return sigma_min * self.r_list - 2.0 * d_max <= self.r_cut

    def check_and_rebuild(self, lattice, positions):
        """Rebuild if needed; True when rebuilt (engine/neighborlist.py:613)."""
        self._n_steps += 1
        if self._dirty or self._ref_pos is None:
            self.build(lattice, positions)
            self._dirty = False
            return True
        if self.needs_rebuild(lattice, positions):
            self.build(lattice, positions)
            return True
        return False

    def _half_pairs_host(self):
        if self._half is None:
            pi, pj = self._dnl.half_pairs()
            self._half = (pi.cpu().numpy(), pj.cpu().numpy())
        return self._half

    def get_candidate_pairs(self):
        """Every pair within r_list as of the last build, canonical order
        (engine/neighborlist.py:679-714): (i, j) int32 host arrays."""
        if self._ref_pos is None:
            return np.empty(0, np.int32), np.empty(0, np.int32)
        return self._half_pairs_host()

    def get_pairs_arrays(self):
        """Pairs within r_cut at the last build, with the build-time
        displacements (engine/neighborlist.py:716-794)."""
        i, j = self.get_candidate_pairs()
        if len(i) == 0:
            return i, j, np.empty((0, 3)), np.empty(0)
        pos = self._ref_pos.cpu().numpy()
        lat = self._lattice
        s = (pos[j] - pos[i]) @ np.linalg.inv(lat)
        s -= np.round(s)
        rij = s @ lat
        r = np.sqrt(np.einsum("pk,pk->p", rij, rij))
        m = r <= self.r_cut
        return i[m], j[m], rij[m], r[m]

    def get_pairs(self):
        i, j, rij, r = self.get_pairs_arrays()
        return list(zip(i.tolist(), j.tolist(), [rij[k] for k in range(len(r))], r.tolist()))


class NullNeighbourList:
    """Stand-in list for a force function that keeps its own
    (engine/neighborlist.py:1036-1069)."""

    def __init__(self, r_cut, skin_width=0.5):
        self.r_cut = r_cut
        self.skin_width = skin_width
        self.r_list = r_cut + skin_width
        self._n_builds = 0
        self._n_steps = 0

    def build(self, lattice, positions):
        self._n_builds += 1

    def mark_dirty(self):
        pass

    def check_and_rebuild(self, lattice, positions):
        self._n_steps += 1
        return False

    @property
    def rebuild_count(self):
        return self._n_builds

    @property
    def step_count(self):
        return self._n_steps


def uses_neighbour_list(force_fn):
    """engine/neighborlist.py:1027-1033."""
    return bool(getattr(force_fn, "uses_neighbour_list", True))


def neighbour_list_for(force_fn, r_cut, skin_width=0.5):
    """engine/neighborlist.py:1072-1076."""
    if uses_neighbour_list(force_fn):
        return NeighbourList(r_cut=r_cut, skin_width=skin_width)
    return NullNeighbourList(r_cut=r_cut, skin_width=skin_width)


# ---- lists kept for force functions called without one --------------------
# engine/neighborlist.py:1083-1163: skin 0.3 A, per-thread LRU of 4 lists
# keyed by (r_cut, N).  Below 100 atoms or in a cell too thin for the skin the
# reference enumerates all pairs within r_cut; the device list then uses no
# skin (r_list = r_cut), which yields the same pairs.

_OWNED_SKIN = 0.3
_OWNED_CACHE_SIZE = 4
_owned = threading.local()


def owned_neighbour_list(lattice, positions, r_cut, device=None):
    """A device list valid for ``positions``: built, or reused when
    ``check_and_rebuild`` finds the cached one still complete."""
    lattice = np.asarray(lattice, dtype=float)
    n = len(positions)
    widths = cell_widths(lattice)
    half = float(np.min(widths)) / 2.0
    if r_cut + _OWNED_SKIN < half:
        skin = _OWNED_SKIN
    else:
        check_min_image(lattice, r_cut, "force call")
        skin = 0.0
    cache = getattr(_owned, "lists", None)
    if cache is None:
        cache = _owned.lists = OrderedDict()
    key = (float(r_cut), n, skin, str(device))
    nl = cache.get(key)
    if nl is None:
        nl = NeighbourList(r_cut=float(r_cut), skin_width=skin, device=device)
        nl.build(lattice, positions)
        cache[key] = nl
        while len(cache) > _OWNED_CACHE_SIZE:
            cache.popitem(last=False)
    else:
        cache.move_to_end(key)
        nl.check_and_rebuild(lattice, positions)
    return nl


def clear_owned_neighbour_lists():
    _owned.lists = OrderedDict()
