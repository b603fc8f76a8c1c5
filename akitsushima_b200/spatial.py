"""One structure split over ranks: slabs along its widest axis with a halo.

The reference evaluates a structure in one process; its multi-rank path
shards whole structures (fitting/loss.py:190-248).  Here one large
structure is split into ``world`` slabs of equal fractional width along the
lattice vector with the largest perpendicular width.  Each rank evaluates
the atoms of its slab (its owned atoms) plus a halo, in the global lattice
and in global atom order, with the usual kernels:

- EAM: a halo of one list radius.  The owned atoms' densities are then
  complete, so their F'(rho-bar) is exact; a halo atom's is not, and one
  exchange gives each halo atom the F' its owner computed
  (mbf_eam_embedding, the exchange, then mbf_eam_forces).  Every pair of an
  owned atom then has both atoms' F', so the owned forces are exact.
- Tersoff and Stillinger-Weber: a halo of two list radii, since zeta and
  the angles of a neighbour's terms reach two cutoffs; no exchange inside
  the evaluation.

Every kernel puts each energy and virial term on one atom whose
neighbourhood it completes (the centre of a three-body term, the lower
index of an EAM pair, lower in global order because the local order is the
global one), so summing the owned atoms' records over all ranks counts each
term once: the reduction plan of a rank's Batch covers only its owned atoms.

Ownership and the list are fixed between rebuilds, as in the reference's
Verlet list (engine/neighborlist.py:613-673): while no atom has moved more
than half the skin since the build, every pair now inside the cutoff of an
owned atom was inside the list radius then, so the halo built with the list
still holds it.  The inputs are the caller's on every rank, as in a force
call; the result is gathered to every rank (one all-gather of the owned
forces and one all-reduce of energy and virial).  A slab whose owned atoms
have no pair inside the cutoff contributes energy 0 (the reference's
no-pair rule, applied per slab).
"""
import numpy as np
import torch

from . import _lib
from .neighbourlist import DeviceNeighbourList
from .system import Batch, cell_widths, default_device, species_ids

HALO_LISTS = 2.0       # three-body potentials: halo width in list radii
EAM_HALO_LISTS = 1.0   # EAM: the halo's F'(rho-bar) comes from the owners


def halo_lists_for(potential):
    return EAM_HALO_LISTS if hasattr(potential, "embedding") else HALO_LISTS


def _fractions(lattice, positions, axis):
    lat = np.asarray(lattice, float).reshape(3, 3)
    f = (np.asarray(positions, float).reshape(-1, 3) @ np.linalg.inv(lat))[:, axis]
    f = f - np.floor(f)
    f[f >= 1.0] = 0.0
    return f


def slab_partition(lattice, positions, world, r_list, axis=None, halo_lists=HALO_LISTS):
    """(axis, [(local, owned), ...] per rank): ``local`` the ascending global
    indices a rank evaluates, ``owned`` the bool mask of its slab's atoms
    among them.  Slab r holds the atoms whose wrapped fractional coordinate
    along ``axis`` lies in [r / world, (r + 1) / world); the halo, every
    atom within halo_lists list radii of the slab."""
    lat = np.asarray(lattice, float).reshape(3, 3)
    widths = cell_widths(lat)
    if axis is None:
        axis = int(np.argmax(widths))
    world = int(world)
    if world < 1:
        raise ValueError("slab_partition: world must be >= 1")
    f = _fractions(lat, positions, axis)
    slab = np.minimum((f * world).astype(np.int64), world - 1)
    h = float(halo_lists) * float(r_list) / float(widths[axis])
    out = []
    for r in range(world):
        own = slab == r
        if 2.0 * h + 1.0 / world >= 1.0:
            near = np.ones(len(f), bool)
        else:
            lo, hi = r / world, (r + 1) / world
            below = np.mod(lo - f, 1.0)   # distance below the slab
            above = np.mod(f - hi, 1.0)   # distance above it
            near = own | (below < h) | (above < h)
        local = np.flatnonzero(near)
        out.append((local, own[local]))
    return axis, out


def fprime_plan(parts):
    """The F'(rho-bar) exchange of an EAM split, computed identically on
    every rank from the partition.  For rank r: ``send`` the positions in
    r's local arrays of its owned atoms that lie in another rank's halo
    (ascending global order); ``fill`` = (positions of r's halo atoms in its
    local arrays, their owner ranks, their positions in the owners' send
    lists); ``width`` the longest send list (the exchange's block size)."""
    world = len(parts)
    n = max((int(loc.max()) + 1 for loc, _ in parts if len(loc)), default=0)
    owner = np.full(n, -1, np.int64)
    for r, (local, own) in enumerate(parts):
        owner[local[own]] = r
    wanted = [[] for _ in range(world)]
    for local, own in parts:
        halo = local[~own]
        for q in range(world):
            wanted[q].append(halo[owner[halo] == q])
    boundary = [np.unique(np.concatenate(w)) if w else np.zeros(0, np.int64) for w in wanted]
    plans = []
    for r, (local, own) in enumerate(parts):
        send = np.searchsorted(local, boundary[r])
        hpos = np.flatnonzero(~own)
        halo = local[hpos]
        src = owner[halo]
        spos = np.zeros(len(halo), np.int64)
        for q in range(world):
            m = src == q
            spos[m] = np.searchsorted(boundary[q], halo[m])
        plans.append({"send": send, "fill": (hpos, src, spos)})
    width = max((len(b) for b in boundary), default=0)
    for p in plans:
        p["width"] = width
    return plans


def exchange_fprime(fprime, plan, group=None):
    """Replace the halo atoms' entries of this rank's fprime (device tensor)
    by their owners' values: one all-gather of every rank's send block
    (padded to the plan's width).  Through NCCL the blocks stay on the
    device; other backends (gloo) move them through host memory."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    on_device = dist.get_backend(group) == "nccl"
    dev = fprime.device if on_device else torch.device("cpu")
    m = max(int(plan["width"]), 1)
    send = torch.zeros(m, dtype=torch.float64, device=dev)
    idx = torch.as_tensor(plan["send"], device=fprime.device)
    send[:len(plan["send"])] = fprime.index_select(0, idx).to(dev)
    recv = [torch.empty(m, dtype=torch.float64, device=dev) for _ in range(world)]
    dist.all_gather(recv, send, group=group)
    table = torch.stack(recv).to(fprime.device)
    hpos, src, spos = (torch.as_tensor(a, device=fprime.device) for a in plan["fill"])
    if len(hpos):
        fprime[hpos] = table[src, spos]
    return fprime


def combine(n_atoms, parts):
    """Whole-structure (energy, forces (n_atoms, 3), virial (9,)) from every
    rank's (owned global indices, owned forces, energy, virial), on one host
    (tests, single-process runs)."""
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


class SlabState:
    """One rank's slab between rebuilds: its local atoms (owned + halo), the
    device Batch (reduction plan over the owned atoms), the device list and
    workspace, the positions at the build, and for EAM the F' exchange
    plan."""

    def __init__(self, potential, lattice, positions, type_ids, rank, world, skin, device):
        self.pot = potential
        self.world, self.rank = int(world), int(rank)
        self.skin = float(skin)
        self.r_list = float(potential.r_cut) + self.skin
        self.lattice = np.array(lattice, float).reshape(3, 3)
        pos = np.asarray(positions, float).reshape(-1, 3)
        self.n_atoms = len(pos)
        self.ref = pos.copy()
        _, self.parts = slab_partition(self.lattice, pos, self.world, self.r_list,
                                       halo_lists=halo_lists_for(potential))
        self.local, self.owned = self.parts[self.rank]
        self.owned_global = [loc[own] for loc, own in self.parts]
        self.plan = fprime_plan(self.parts)[self.rank] if hasattr(potential, "embedding") else None
        ids = np.asarray(type_ids, np.int32)
        self.batch = Batch([self.lattice], [pos[self.local]], [ids[self.local]], device=device,
                           owned=self.owned)
        self.dlist = DeviceNeighbourList(self.r_list).build(self.batch)
        self._sel = torch.as_tensor(np.flatnonzero(self.owned), device=device)
        # a workspace of its own: the embedding pass leaves rho-bar, F and
        # the records there for the force pass
        nbytes = int(_lib.lib().mbf_eval_workspace_bytes(self.batch.n_atoms, self.dlist.n_slots,
                                                         self.batch.n_chunks))
        self.ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=device)

    def valid_for(self, lattice, positions, world, rank):
        """The reference's criterion with the lattice fixed: 2 max|MIC(r -
        r_build)| < skin (engine/neighborlist.py:653-673), over every atom,
        so that every rank reaches the same decision."""
        pos = np.asarray(positions, float).reshape(-1, 3)
        if (world != self.world or rank != self.rank or len(pos) != self.n_atoms
                or not np.array_equal(np.asarray(lattice, float).reshape(3, 3), self.lattice)):
            return False
        d = (pos - self.ref) @ np.linalg.inv(self.lattice)
        d -= np.rint(d)
        d_max = float(np.sqrt(np.max(np.einsum("ij,ij->i", d @ self.lattice, d @ self.lattice)))) \
            if len(pos) else 0.0
        return 2.0 * d_max < self.skin

    def evaluate(self, positions, type_ids, group=None, exchange_fn=None):
        """This rank's share: (owned global indices, owned forces (host),
        energy, virial (9,)) of the owned atoms' records.  ``exchange_fn``
        (EAM) completes the halo's F' between the two phases (default: the
        all-gather of exchange_fprime over ``group``)."""
        b = self.batch
        pos = np.asarray(positions, float).reshape(-1, 3)
        b.set_positions(pos[self.local], check=False)
        b.set_types(np.asarray(type_ids, np.int32)[self.local])
        if hasattr(self.pot, "embedding"):
            fp = self.pot.embedding(b, self.dlist, ws=self.ws)
            if exchange_fn is not None:
                fp = exchange_fn(self, fp)
            elif self.world > 1:
                fp = exchange_fprime(fp, self.plan, group)
            res = self.pot.forces_from_embedding(b, self.dlist, fp, ws=self.ws)
        else:
            res = self.pot.evaluate(b, self.dlist, ws=self.ws)
        f = res.forces.index_select(0, self._sel).cpu().numpy()
        return (self.local[self.owned], f, float(res.energy[0].item()), res.virial[0].cpu().numpy())


def evaluate_slabs(potential, lattice, positions, type_ids, world, skin=0.3, device=None):
    """Every rank's share of a split, the ranks one after another in this
    process on one device (no kernel of one rank waits on another's), with
    the EAM F' exchange done in memory; returns the list of shares for
    :func:`combine`.  The multi-process path is SpatialForceFn."""
    dev = torch.device(device) if device is not None else default_device()
    states = [SlabState(potential, lattice, positions, type_ids, r, world, skin, dev) for r in range(world)]
    if not hasattr(potential, "embedding"):
        return [s.evaluate(positions, type_ids) for s in states]
    pos = np.asarray(positions, float).reshape(-1, 3)
    fps = []
    for s in states:
        s.batch.set_positions(pos[s.local], check=False)
        fps.append(potential.embedding(s.batch, s.dlist, ws=s.ws))
    m = max(int(states[0].plan["width"]), 1)
    table = torch.zeros((world, m), dtype=torch.float64, device=dev)
    for r, (s, fp) in enumerate(zip(states, fps)):
        table[r, :len(s.plan["send"])] = fp[torch.as_tensor(s.plan["send"], device=dev)]
    shares = []
    for s, fp in zip(states, fps):
        hpos, src, spos = (torch.as_tensor(a, device=dev) for a in s.plan["fill"])
        if len(hpos):
            fp[hpos] = table[src, spos]
        res = potential.forces_from_embedding(s.batch, s.dlist, fp, ws=s.ws)
        f = res.forces.index_select(0, s._sel).cpu().numpy()
        shares.append((s.local[s.owned], f, float(res.energy[0].item()), res.virial[0].cpu().numpy()))
    return shares


class SpatialForceFn:
    """force_fn(lattice, positions, atom_types) -> (energy, forces, stress)
    with the structure split over the ranks of ``group`` (torch.distributed,
    one GPU per rank; default: the default group if initialised, else one
    rank).  Every rank passes the same inputs and gets the whole result.
    Each rank keeps its slab (ownership, halo, device list) between calls
    and rebuilds it when the skin criterion fires."""

    def __init__(self, potential, group=None, skin=0.3, device=None):
        self.pot = potential
        self.group = group
        self.skin = float(skin)
        self.device = device
        self.r_cut = float(potential.r_cut)
        self.rebuild_count = 0
        self._state = None

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
        st = self._state
        if st is None or not st.valid_for(lattice, pos, world, rank):
            st = self._state = SlabState(self.pot, lattice, pos, ids, rank, world, self.skin, dev)
            self.rebuild_count += 1
        if dist is None or world == 1:
            e, F, w = combine(len(pos), [st.evaluate(pos, ids)])
        else:
            idx, f, e, w = st.evaluate(pos, ids, group=self.group)
            xdev = dev if dist.get_backend(self.group) == "nccl" else "cpu"
            e, F, w = exchange(len(pos), st.owned_global, f, e, w, self.group, xdev)
        vol = abs(float(np.linalg.det(lattice)))
        return e, F, w.reshape(3, 3) / vol
