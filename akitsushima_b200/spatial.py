"""One structure split over ranks: slabs along its widest axis with a halo.

The reference evaluates a structure in one process; its multi-rank path
shards whole structures (fitting/loss.py:190-248).  Here one large
structure is split into ``world`` slabs of equal fractional width along the
lattice vector with the largest perpendicular width.  Each rank evaluates
the atoms of its slab plus a halo of every atom within 2 r_list of it, in
the global lattice and in global atom order, with the usual kernels:

- the forces of the slab's atoms are exact: every neighbour within r_list
  of an owned atom is present, and so is every neighbour of those
  neighbours (which the many-body terms need: EAM's F'(rho-bar), Tersoff's
  zeta and the Stillinger-Weber angles reach two cutoffs);
- every kernel puts each energy and virial term on one atom whose
  neighbourhood it completes (the centre of a three-body term, the lower
  index of an EAM pair, lower in global order because the local order is
  the global one), so summing the owned atoms' records over all ranks
  counts each term once.  The reduction plan of the rank's Batch covers only
  its owned atoms.

The exchange is one all-reduce of (energy, virial) and one all-gather of
the owned forces; the positions are the caller's on every rank, as in the
reference's force call.  A slab whose owned atoms have no pair inside the
cutoff contributes energy 0 (the reference's no-pair rule, applied per
slab).
"""
import numpy as np
import torch

from .neighbourlist import DeviceNeighbourList
from .system import Batch, cell_widths, default_device, species_ids

HALO_LISTS = 2.0   # halo width in list radii


def slab_partition(lattice, positions, world, r_list, axis=None):
    """(axis, [(local, owned), ...] per rank): ``local`` the ascending global
    indices a rank evaluates, ``owned`` the bool mask of its slab's atoms
    among them.  Slab r holds the atoms whose wrapped fractional coordinate
    along ``axis`` lies in [r / world, (r + 1) / world)."""
    lat = np.asarray(lattice, float).reshape(3, 3)
    pos = np.asarray(positions, float).reshape(-1, 3)
    widths = cell_widths(lat)
    if axis is None:
        axis = int(np.argmax(widths))
    world = int(world)
    if world < 1:
        raise ValueError("slab_partition: world must be >= 1")
    f = (pos @ np.linalg.inv(lat))[:, axis]
    f = f - np.floor(f)
    f[f >= 1.0] = 0.0
    slab = np.minimum((f * world).astype(np.int64), world - 1)
    h = HALO_LISTS * float(r_list) / float(widths[axis])
    out = []
    for r in range(world):
        own = slab == r
        if 2.0 * h + 1.0 / world >= 1.0:
            near = np.ones(len(pos), bool)
        else:
            lo, hi = r / world, (r + 1) / world
            below = np.mod(lo - f, 1.0)   # distance below the slab
            above = np.mod(f - hi, 1.0)   # distance above it
            near = own | (below < h) | (above < h)
        local = np.flatnonzero(near)
        out.append((local, own[local]))
    return axis, out


def evaluate_slab(potential, lattice, positions, type_ids, rank, world, skin=0.3, device=None):
    """One rank's share: (owned global indices, their forces (host), energy,
    virial (9,)) of the owned atoms' records."""
    dev = torch.device(device) if device is not None else default_device()
    r_list = float(potential.r_cut) + float(skin)
    _, parts = slab_partition(lattice, positions, world, r_list)
    local, owned = parts[rank]
    pos = np.asarray(positions, float).reshape(-1, 3)
    ids = np.asarray(type_ids, np.int32)
    batch = Batch([lattice], [pos[local]], [ids[local]], device=dev, owned=owned)
    dl = DeviceNeighbourList(r_list).build(batch)
    res = potential.evaluate(batch, dl)
    sel = torch.as_tensor(np.flatnonzero(owned), device=dev)
    f = res.forces.index_select(0, sel).cpu().numpy()
    return local[owned], f, float(res.energy[0].item()), res.virial[0].cpu().numpy()


def combine(n_atoms, parts):
    """Whole-structure (energy, forces (n_atoms, 3), virial (9,)) from every
    rank's evaluate_slab output, on one host (tests, single-process runs)."""
    F = np.zeros((n_atoms, 3))
    e, w = 0.0, np.zeros(9)
    for idx, f, ei, wi in parts:
        F[idx] = f
        e += ei
        w += wi
    return e, F, w


def exchange(n_atoms, owned, f, e, w, group=None, device="cpu"):
    """The whole result on every rank of ``group``: all ranks' owned forces
    (``owned`` = every rank's owned global indices, known to all since the
    partition is computed identically everywhere) gathered as equal-sized
    padded blocks, and (energy, virial) summed by one all-reduce."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    m = max(len(o) for o in owned)
    send = torch.zeros((m, 3), dtype=torch.float64, device=device)
    send[:len(f)] = torch.as_tensor(np.asarray(f, float).reshape(-1, 3), device=device)
    recv = [torch.empty((m, 3), dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(recv, send, group=group)
    ew = torch.as_tensor(np.concatenate([[float(e)], np.asarray(w, float).reshape(9)]), device=device)
    dist.all_reduce(ew, group=group)
    F = np.zeros((n_atoms, 3))
    for o, blk in zip(owned, recv):
        F[o] = blk.cpu().numpy()[:len(o)]
    ew = ew.cpu().numpy()
    return float(ew[0]), F, ew[1:]


class SpatialForceFn:
    """force_fn(lattice, positions, atom_types) -> (energy, forces, stress)
    with the structure split over the ranks of ``group`` (torch.distributed,
    one GPU per rank; default: the default group if initialised, else one
    rank).  Every rank passes the same inputs and gets the whole result."""

    def __init__(self, potential, group=None, skin=0.3, device=None):
        self.pot = potential
        self.group = group
        self.skin = float(skin)
        self.device = device

    def _world(self):
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            return dist, dist.get_world_size(self.group), dist.get_rank(self.group)
        return None, 1, 0

    def __call__(self, lattice, positions, atom_types):
        lattice = np.asarray(lattice, float)
        pos = np.asarray(positions, float).reshape(-1, 3)
        ids = species_ids(atom_types, self.pot.species)
        dist, world, rank = self._world()
        dev = torch.device(self.device) if self.device is not None else default_device()
        idx, f, e, w = evaluate_slab(self.pot, lattice, pos, ids, rank, world, self.skin, dev)
        if dist is None or world == 1:
            e, F, w = combine(len(pos), [(idx, f, e, w)])
        else:
            _, parts = slab_partition(lattice, pos, world, float(self.pot.r_cut) + self.skin)
            e, F, w = exchange(len(pos), [loc[own] for loc, own in parts], f, e, w, self.group, dev)
        vol = abs(float(np.linalg.det(lattice)))
        return e, F, w.reshape(3, 3) / vol
