"""Structures on the device: one or many periodic cells concatenated.

A :class:`Batch` holds the flattened atom arrays of ``n_struct`` structures
(positions, species ids, structure id per atom), the per-structure lattice and
inverse, and the per-structure reduction plan the kernels use to sum energy
and virial.  A single structure is a batch of one.  Torch supplies the device
memory and the stream; every computation runs in libmbforce.so.
"""
import numpy as np
import torch

from . import _lib

# Atoms per reduction chunk (the per-structure energy/virial sums, one
# block of the last kernel of an evaluation per chunk): enough chunks for
# about two blocks per SM of a B200, 32 to 512 atoms each.
REDUCE_CHUNK = 512
REDUCE_CHUNK_MIN = 32
REDUCE_TARGET_CHUNKS = 296


def reduce_chunk_size(n_atoms):
    size = REDUCE_CHUNK_MIN
    while size < REDUCE_CHUNK and size * REDUCE_TARGET_CHUNKS < n_atoms:
        size *= 2
    return size


def cell_metrics(lattice):
    """Perpendicular widths d_i = V / |a_j x a_k| and sigma_min of a lattice
    (rows are lattice vectors); the reference's engine/neighborlist.py:170-267.
    Raises ValueError for a degenerate cell."""
    lat = np.asarray(lattice, dtype=float)
    return cell_widths(lat), float(np.linalg.svd(lat, compute_uv=False)[-1])


def cell_widths(lattice):
    """The perpendicular widths of :func:`cell_metrics` alone."""
    lat = np.asarray(lattice, dtype=float)
    if lat.shape != (3, 3):
        raise ValueError(f"NeighbourList: lattice must have shape (3, 3), got {lat.shape}.")
    volume = abs(float(np.linalg.det(lat)))
    cross = np.array([np.linalg.norm(np.cross(lat[(i + 1) % 3], lat[(i + 2) % 3]))
                      for i in range(3)])
    if volume <= 0.0 or not np.all(cross > 0.0) or not np.isfinite(volume):
        raise ValueError(
            f"NeighbourList: degenerate (singular) lattice with volume {volume:.6g} A^3 -- "
            "the three lattice vectors must be linearly independent for a minimum-image "
            "convention to exist.")
    return volume / cross


def check_min_image(lattice, r_list, caller="NeighbourList", widths=None):
    """Refuse r_list >= half the smallest perpendicular width
    (engine/neighborlist.py:98-132 and :489-572); ``widths`` are the
    lattice's from :func:`cell_widths` when the caller has them."""
    if widths is None:
        widths = cell_widths(lattice)
    if r_list >= float(np.min(widths)) / 2.0:
        lengths = np.linalg.norm(np.asarray(lattice, float), axis=1)
        raise ValueError(
            f"{caller}: cutoff radius ({r_list:.4f} A) must be < half the smallest "
            f"perpendicular cell width ({float(np.min(widths)) / 2.0:.4f} A) for the "
            f"minimum-image convention to be valid. Perpendicular widths are "
            f"[{widths[0]:.4f}, {widths[1]:.4f}, {widths[2]:.4f}] A for lattice vector "
            f"lengths [{lengths[0]:.4f}, {lengths[1]:.4f}, {lengths[2]:.4f}] A.")


def cell_grid(lattice, r_list, widths=None):
    """Sub-cell counts nc_i = max(1, floor(d_i / r_list))
    (engine/neighborlist.py:976-978) and the stencil width per axis."""
    if widths is None:
        widths = cell_widths(lattice)
    nc = np.maximum(1, np.floor(widths / r_list).astype(int))
    w = np.where(nc == 1, 1, np.where(nc == 2, 2, 3))
    return nc, w


def capture_graph(fn, device, warm=True):
    """A CUDA graph of fn()'s launches, captured on a side stream (after one
    eager call there when ``warm``).  capture_begin / capture_end directly:
    torch.cuda.graph() would also run the garbage collector and empty the
    allocator's cache, costing more than a small capture."""
    side = torch.cuda.Stream(device)
    side.wait_stream(torch.cuda.current_stream(device))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        if warm:
            fn()
        g.capture_begin()
        try:
            fn()
        finally:
            g.capture_end()
    torch.cuda.current_stream(device).wait_stream(side)
    return g


def default_device():
    if not torch.cuda.is_available():
        raise RuntimeError("akitsushima_b200 needs a CUDA device (B200); none is visible.")
    return torch.device("cuda", torch.cuda.current_device())


_IDS_CACHE = {}


def species_ids(atom_types, species):
    """Species index of every atom.  ``atom_types`` is a list / array of
    symbols, or an integer array of indices into ``species``.  A list of
    symbols equal to the previous call's (the solvers pass the same list
    every step) reuses its ids: comparing two lists of the same string
    objects is much cheaper than converting one."""
    if isinstance(atom_types, list) and atom_types and isinstance(atom_types[0], str):
        key = tuple(species)
        hit = _IDS_CACHE.get(key)
        if hit is not None and len(hit[0]) == len(atom_types) and hit[0] == atom_types:
            return hit[1]
    a = np.asarray(atom_types)
    if a.dtype.kind in "iu":
        ids = a.astype(np.int32, copy=False)
        if len(ids) and (ids.min() < 0 or ids.max() >= len(species)):
            raise ValueError("atom type index out of range of the potential's species")
        return ids
    if len(a) == 0:
        return np.zeros(0, np.int32)
    a = a.astype(str)
    ids = np.full(len(a), -1, np.int32)
    for k, sp in enumerate(species):
        ids[a == sp] = k
    if (ids < 0).any():
        bad = a[np.argmax(ids < 0)]
        raise ValueError(f"atom type {str(bad)!r} is not among the potential's species {list(species)}")
    ids.setflags(write=False)
    if isinstance(atom_types, list):
        _IDS_CACHE.clear()
        _IDS_CACHE[tuple(species)] = (list(atom_types), ids)
    return ids


def _runs(mask, a0, a1):
    """Maximal runs [r0, r1) of True in mask[a0:a1] (absolute indices)."""
    m = np.concatenate([[False], mask[a0:a1], [False]]).astype(np.int8)
    d = np.flatnonzero(np.diff(m))
    return [(a0 + int(d[k]), a0 + int(d[k + 1])) for k in range(0, len(d), 2)]


class Batch:
    """``n_struct`` periodic structures flattened on one device.

    Parameters
    ----------
    lattices  : sequence of (3, 3) row-vector lattices [A].
    positions : sequence of (N_s, 3) Cartesian positions [A] (numpy or torch).
    type_ids  : sequence of (N_s,) integer species ids.
    owned     : optional (n_atoms,) bool mask: the per-structure energy and
                virial sum only the records of these atoms (the others are
                halo atoms of a spatial slab, evaluated so that the owned
                atoms' neighbourhoods are complete).  Default: every atom.
    """

    def __init__(self, lattices, positions, type_ids, device=None, owned=None):
        self.device = torch.device(device) if device is not None else default_device()
        lats = [np.asarray(l, dtype=np.float64).reshape(3, 3) for l in lattices]
        if len(lats) == 0:
            raise ValueError("Batch: no structures")
        if not (len(lats) == len(positions) == len(type_ids)):
            raise ValueError("Batch: lattices, positions and type_ids differ in length")
        counts = [int(len(p)) for p in positions]
        self.n_struct = len(lats)
        self.n_atoms = int(sum(counts))
        self.counts = np.array(counts, np.int64)
        off = np.zeros(self.n_struct + 1, np.int64)
        off[1:] = np.cumsum(counts)
        self.offsets = off
        self.lattices = np.stack(lats)
        for lat in lats:
            cell_widths(lat)
        self.volumes = np.abs(np.linalg.det(self.lattices))
        invs = np.linalg.inv(self.lattices)
        cells = np.concatenate([self.lattices.reshape(-1, 9), invs.reshape(-1, 9)], axis=1)
        dev = self.device
        self._cells_np = np.ascontiguousarray(cells)   # the host copy the C view points to
        self.cells = torch.as_tensor(self._cells_np, device=dev)
        self.struct_off = torch.as_tensor(off.astype(np.int32), device=dev)
        self.atom_struct = torch.as_tensor(
            np.repeat(np.arange(self.n_struct, dtype=np.int32), counts), device=dev)
        self.pos = torch.empty((self.n_atoms, 3), dtype=torch.float64, device=dev)
        self.types = torch.empty(self.n_atoms, dtype=torch.int32, device=dev)
        self._types_host = None
        self.set_positions(positions)
        self.set_types(type_ids)
        # reduction plan: chunks of reduce_chunk_size atoms inside one
        # structure, over the runs of owned atoms (all atoms by default)
        if owned is not None:
            owned = np.asarray(owned, bool).reshape(-1)
            if owned.shape != (self.n_atoms,):
                raise ValueError("Batch: owned must have one entry per atom")
        size = reduce_chunk_size(self.n_atoms if owned is None else int(owned.sum()))
        chunk, first = [], [0]
        for s in range(self.n_struct):
            a0, a1 = int(off[s]), int(off[s + 1])
            n0 = len(chunk)
            for r0, r1 in ([(a0, a1)] if owned is None else _runs(owned, a0, a1)):
                for c0 in range(r0, r1, size):
                    chunk.append((s, c0, min(r1, c0 + size)))
            if len(chunk) == n0:
                chunk.append((s, a0, a0))
            first.append(len(chunk))
        self.chunk = torch.as_tensor(np.array(chunk, np.int32).reshape(-1, 3), device=dev)
        self.chunk_first = torch.as_tensor(np.array(first, np.int32), device=dev)

    @classmethod
    def single(cls, lattice, positions, type_ids, device=None):
        return cls([lattice], [positions], [type_ids], device=device)

    def set_positions(self, positions, check=True):
        """Copy new positions in place: one (N, 3) array or tensor for the
        whole batch, or a sequence of (N_s, 3) arrays, one per structure.
        Host arrays go through a page-locked staging buffer kept by the
        batch: torch's threaded host copy fills it (0.02 ms for 6 MB on a
        B200 host) and the upload is asynchronous on the current stream, so
        the caller's next launches queue behind it instead of the host
        waiting for a pageable copy (0.35 ms for the same 6 MB).  The buffer
        is refilled only after the previous upload from it has finished.
        check: refuse NaN / inf in host arrays (no kernel depends on it -- a
        non-finite coordinate only gives non-finite results)."""
        if isinstance(positions, torch.Tensor):
            src = positions.reshape(-1, 3)
            if tuple(src.shape) != (self.n_atoms, 3):
                raise ValueError(f"positions have shape {tuple(src.shape)}, expected ({self.n_atoms}, 3)")
            self.pos.copy_(src.to(torch.float64), non_blocking=src.device.type != "cpu")
            return
        if isinstance(positions, np.ndarray) and positions.ndim == 2:
            arr = positions
        else:
            arr = np.concatenate([np.asarray(p, np.float64).reshape(-1, 3) for p in positions]) \
                if len(positions) else np.zeros((0, 3))
        if arr.shape != (self.n_atoms, 3):
            raise ValueError(f"positions have shape {arr.shape}, expected ({self.n_atoms}, 3)")
        if check and not np.isfinite(np.add.reduce(arr, axis=None)):  # NaN and inf survive a sum
            raise ValueError("positions contain NaN or inf")
        src = torch.from_numpy(np.ascontiguousarray(arr, np.float64))
        if self.device.type != "cuda":
            self.pos.copy_(src)
            return
        stage = getattr(self, "_stage", None)
        if stage is None or stage.shape != src.shape:
            stage = self._stage = torch.empty(src.shape, dtype=torch.float64, pin_memory=True)
            self._stage_done = torch.cuda.Event()
        else:
            self._stage_done.synchronize()
        stage.copy_(src)
        self.pos.copy_(stage, non_blocking=True)
        self._stage_done.record(torch.cuda.current_stream(self.device))

    def forces_to_host(self, forces):
        """Device (N, 3) forces to a new host numpy array: a pinned block of
        torch's caching host allocator, copied into directly (no second host
        copy); the block returns to the cache when the caller drops it."""
        if self.device.type != "cuda":
            return forces.cpu().numpy()
        out = torch.empty((self.n_atoms, 3), dtype=torch.float64, pin_memory=True)
        out.copy_(forces, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        return out.numpy()

    def types_unchanged(self, type_ids, n_species):
        """True if type_ids is an integer array equal to the ids last
        uploaded from the host, all of them below n_species."""
        return (isinstance(type_ids, np.ndarray) and type_ids.dtype.kind in "iu" and self._types_host is not None
                and self._types_max < n_species and type_ids.shape == self._types_host.shape
                and np.array_equal(type_ids, self._types_host))

    def set_types(self, type_ids):
        """Species ids (torch tensor, or host arrays; an unchanged host array
        is not uploaded again)."""
        if isinstance(type_ids, torch.Tensor):
            self.types.copy_(type_ids.to(torch.int32), non_blocking=type_ids.device.type != "cpu")
            self._types_host = None
            return
        if isinstance(type_ids, np.ndarray) and type_ids.ndim == 1:
            arr = type_ids.astype(np.int32, copy=False)
        else:
            arr = np.concatenate([np.asarray(t, np.int32).reshape(-1) for t in type_ids]) \
                if len(type_ids) else np.zeros(0, np.int32)
        if arr.shape != (self.n_atoms,):
            raise ValueError("type_ids do not match the atom count")
        if self._types_host is not None and np.array_equal(arr, self._types_host):
            return
        host = np.ascontiguousarray(arr)
        self.types.copy_(torch.from_numpy(host if host.flags.writeable else host.copy()))
        self._types_host = arr.copy()
        self._types_max = int(arr.max()) if len(arr) else -1

    def set_lattice(self, s, lattice):
        lat = np.asarray(lattice, np.float64).reshape(3, 3)
        if np.array_equal(lat, self.lattices[s]):
            return
        cell_widths(lat)
        self._sysd = None
        self.lattices[s] = lat
        self.volumes[s] = abs(np.linalg.det(lat))
        row = np.concatenate([lat.reshape(9), np.linalg.inv(lat).reshape(9)])
        self._cells_np[s] = row
        self.cells[s].copy_(torch.from_numpy(row))

    def mbf_system(self):
        """The C ABI's view of the batch (device pointers, the diagonal
        cell flag and a host copy of the cells), built once and again only
        after a lattice change: the device arrays keep their addresses."""
        sysd = getattr(self, "_sysd", None)
        if sysd is None:
            off = self.lattices - np.einsum("sij,ij->sij", self.lattices, np.eye(3))
            ortho = 1 if not np.any(off) else 0
            sysd = _lib.MbfSystem(self.n_atoms, self.n_struct, _lib.ptr(self.pos), _lib.ptr(self.types),
                                  _lib.ptr(self.atom_struct), _lib.ptr(self.struct_off),
                                  _lib.ptr(self.cells), ortho)
            sysd.cells_host = self._cells_np.ctypes.data   # the rows uploaded to self.cells
            self._sysd = sysd
        return sysd

    def reduce_plan(self):
        plan = getattr(self, "_plan", None)
        if plan is None:
            plan = self._plan = _lib.MbfReducePlan(int(self.chunk.shape[0]), _lib.ptr(self.chunk),
                                                   _lib.ptr(self.chunk_first))
        return plan

    @property
    def n_chunks(self):
        return int(self.chunk.shape[0])


def replicate_thin(lattice, positions, type_ids, r_list):
    """Replicate a cell along every axis whose perpendicular width is below
    2 r_list, so the minimum image holds; returns (lattice, positions, types,
    reps).  Energy of the original = supercell energy / prod(reps); the
    forces of the first N atoms and the stress are unchanged (exact periodic
    physics)."""
    lat = np.asarray(lattice, float)
    widths = cell_widths(lat)
    reps = np.ones(3, int)
    for k in range(3):
        while widths[k] * reps[k] / 2.0 <= r_list:
            reps[k] += 1
    if np.all(reps == 1):
        return lat, np.asarray(positions, float), np.asarray(type_ids, np.int32), reps
    shifts = np.array([[a, b, c] for a in range(reps[0]) for b in range(reps[1])
                       for c in range(reps[2])], float)
    pos = np.asarray(positions, float)
    big = (pos[None, :, :] + (shifts @ lat)[:, None, :]).reshape(-1, 3)
    types = np.tile(np.asarray(type_ids, np.int32), len(shifts))
    return lat * reps[:, None], big, types, reps


__all__ = ["Batch", "capture_graph", "cell_metrics", "cell_widths", "check_min_image", "cell_grid", "species_ids",
           "replicate_thin", "default_device"]
