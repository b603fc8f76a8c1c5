"""Many structures of uneven size evaluated together.

The fit training sets, phonon displacement sets and elastic strain sets of
the reference are loops of single-structure force calls
(fitting/loss.py:190-242, solvers/phonon.py:469-480,
solvers/elastic.py:288-293).  Here they are one batch: the atoms of every
structure concatenated behind a structure offset table, one neighbour-list
build and one launch sequence for the whole set, per-structure energy and
virial from segmented reductions.  Repeated evaluations replay a CUDA graph.

Cells thinner than twice the list radius cannot be handled with the minimum
image (the reference refuses them, engine/neighborlist.py:489-572).  With
``replicate_thin`` such a cell is replaced by the smallest supercell that
can, which is exact periodic physics: energy / k, the forces of the first N
atoms and the stress are those of the original cell.
"""
import numpy as np
import torch

from .neighbourlist import DeviceNeighbourList
from . import _lib
from .potential import EvalResult
from .system import Batch, capture_graph, default_device, species_ids
from .system import replicate_thin as _replicate


class BatchedEvaluator:
    """Evaluate ``potential`` on a list of (lattice, positions, atom_types).

    Parameters
    ----------
    potential      : a TersoffPotential, StillingerWeberPotential or
                     EAMPotential of this package.
    structures     : sequence of (lattice (3, 3), positions (N, 3), types).
    skin           : list skin [A] (the list is built once).
    replicate_thin : replicate cells too thin for the minimum image.
    precision      : 'fp64' or 'mixed' (default: the potential's).
    """

    def __init__(self, potential, structures, skin=0.3, replicate_thin=True, precision=None,
                 device=None):
        self.pot = potential
        self.precision = precision or potential.precision
        self.device = torch.device(device) if device is not None else default_device()
        self.r_list = float(potential.r_cut) + float(skin)
        lats, poss, ids, self.reps, self.n_orig = [], [], [], [], []
        for lat, pos, types in structures:
            t = species_ids(types, potential.species)
            if replicate_thin:
                L2, P2, T2, reps = _replicate(lat, pos, t, self.r_list)
            else:
                L2, P2, T2, reps = np.asarray(lat, float), np.asarray(pos, float), t, np.ones(3, int)
            lats.append(L2)
            poss.append(P2)
            ids.append(T2)
            self.reps.append(int(np.prod(reps)))
            self.n_orig.append(len(pos))
        self.batch = Batch(lats, poss, ids, device=self.device)
        self.dlist = DeviceNeighbourList(self.r_list).build(self.batch)
        off = self.batch.offsets
        idx = np.concatenate([np.arange(off[s], off[s] + n) for s, n in enumerate(self.n_orig)]) \
            if self.n_orig else np.zeros(0, np.int64)
        self._orig_index = torch.as_tensor(idx, device=self.device)
        self._inv_reps = torch.as_tensor(1.0 / np.array(self.reps, float), device=self.device)
        ends = np.cumsum(self.n_orig)
        self._slices = [slice(int(b - n), int(b)) for b, n in zip(ends, self.n_orig)]
        self._vol = torch.as_tensor(self.batch.volumes, device=self.device)
        dev = self.device
        self.out = EvalResult(torch.empty(self.batch.n_struct, dtype=torch.float64, device=dev),
                              torch.empty((self.batch.n_atoms, 3), dtype=torch.float64, device=dev),
                              torch.empty((self.batch.n_struct, 9), dtype=torch.float64, device=dev))
        nbytes = int(_lib.lib().mbf_eval_workspace_bytes(self.batch.n_atoms, self.dlist.n_slots,
                                                         self.batch.n_chunks))
        self._ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
        # results() reads one block: energies / reps (S), virials / volume
        # (S, 9), the original atoms' forces (n0, 3)
        S, n0 = self.batch.n_struct, int(sum(self.n_orig))
        self._packed = torch.empty(10 * S + 3 * n0, dtype=torch.float64, device=dev)
        self._graph = None

    def _eval(self):
        return self.pot.evaluate(self.batch, self.dlist, precision=self.precision, out=self.out,
                                 ws=self._ws)

    def _pack(self):
        S, n0, out, p = self.batch.n_struct, int(sum(self.n_orig)), self.out, self._packed
        torch.mul(out.energy, self._inv_reps, out=p[:S])
        torch.div(out.virial, self._vol[:, None], out=p[S:10 * S].view(S, 9))
        torch.index_select(out.forces, 0, self._orig_index, out=p[10 * S:].view(n0, 3))

    def _eval_and_pack(self):
        self._eval()
        self._pack()

    @property
    def n_structures(self):
        return self.batch.n_struct

    @property
    def n_atoms(self):
        """Atoms of the original structures (replicas not counted)."""
        return int(sum(self.n_orig))

    def run(self):
        """One evaluation of every structure (device, asynchronous)."""
        if self._graph is not None:
            self._graph.replay()
        else:
            self._eval()
        return self.out

    def capture(self):
        """Capture one evaluation in a CUDA graph; later run() calls replay
        it (positions, lattices and species are read from the batch's device
        arrays, so updating those in place keeps the graph valid).  The graph
        also packs the per-structure results into the block results() copies
        to the host."""
        self._eval_and_pack()
        self._graph = capture_graph(self._eval_and_pack, self.device)
        torch.cuda.synchronize(self.device)
        return self

    def results(self):
        """Per-structure (energies (S,), forces list of (N_s, 3), stresses
        (S, 3, 3)) of the ORIGINAL structures, on the host: the results packed
        into one device block (inside the captured graph, if any) and one
        copy into a fresh pinned block (the arrays returned are views of it,
        which the caller's references keep)."""
        self.run()
        if self._graph is None:
            self._pack()
        S, n0 = self.batch.n_struct, int(sum(self.n_orig))
        host = torch.empty(self._packed.numel(), dtype=torch.float64, pin_memory=True)
        host.copy_(self._packed, non_blocking=True)
        torch.cuda.current_stream(self.device).synchronize()
        h = host.numpy()
        e = h[:S]
        s = h[S:10 * S].reshape(-1, 3, 3)
        f = h[10 * S:10 * S + 3 * n0].reshape(-1, 3)
        return e, [f[sl] for sl in self._slices], s

    def autotune(self, candidates=None, reps=5):
        """Time every lanes-per-atom candidate on this batch and keep the
        fastest (CUDA events; the graph, if any, is recaptured)."""
        had_graph = self._graph is not None
        self._graph = None
        self.tuned = self.pot.autotune_lanes(self.batch, self.dlist, candidates, reps, ws=self._ws, out=self.out)
        if had_graph:
            self.capture()
        return self.tuned
