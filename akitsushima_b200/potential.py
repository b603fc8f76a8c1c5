"""Common machinery of the device potentials.

Every potential exposes the reference's protocol
``compute(lattice, positions, atom_types, neigh_list=None, use_numba=False)
-> (energy, forces (N, 3), stress (3, 3))`` (engine/potential_engine.py:76-105,
engine/tersoff.py:1208, engine/stillinger_weber.py:900, engine/eam.py:174)
and a device-level ``evaluate(batch, dlist)`` returning torch tensors, which
the batched, MD and benchmark paths use without host round trips.

Stress is compressive-positive and divided by the volume, as the reference
returns it (engine/tersoff.py:1512).
"""
import threading
import weakref

import numpy as np
import torch

from . import _lib
from .neighbourlist import DeviceNeighbourList, NeighbourList, owned_neighbour_list
from .system import Batch, capture_graph, species_ids

PRECISIONS = {"fp64": _lib.MBF_FP64, "mixed": _lib.MBF_MIXED}

_ws_local = threading.local()


def _set_last_ws(pot, ws):
    """The workspace of this thread's last evaluation with `pot` (its status
    words are read back after the call); held weakly."""
    _ws_local.__dict__.setdefault("last", {})[id(pot)] = weakref.ref(ws)


def _get_last_ws(pot):
    ref = getattr(_ws_local, "last", {}).get(id(pot))
    return ref() if ref is not None else None


def workspace(device, nbytes):
    """Per-thread, per-device scratch buffer (grown on demand), so
    concurrent callers on different threads never share one."""
    d = getattr(_ws_local, "bufs", None)
    if d is None:
        d = _ws_local.bufs = {}
    key = str(device)
    buf = d.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=device)
        d[key] = buf
    return buf


def precision_code(precision):
    try:
        return PRECISIONS[str(precision).lower()]
    except KeyError:
        raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision!r}") from None


class EvalResult:
    """Device-side result of one evaluation of a batch."""

    __slots__ = ("energy", "forces", "virial")

    def __init__(self, energy, forces, virial):
        self.energy = energy    # (n_struct,) eV
        self.forces = forces    # (n_atoms, 3) eV/A
        self.virial = virial    # (n_struct, 9): sum of -f (x) r, eV (not / V)


class DevicePotential:
    """Base class: subclasses set ``species``, ``r_cut``, ``precision`` and
    implement ``_device_tables(device)`` and ``_call(...)``."""

    species = None
    r_cut = None
    precision = "fp64"

    def __init__(self):
        self._tabs = {}
        self._foreign = {}

    # -- subclass hooks ------------------------------------------------------
    def _device_tables(self, device):
        raise NotImplementedError

    def _call(self, L, sysd, nld, tabs, plan, prec, ws, nbytes, forces, energy, virial, stream):
        raise NotImplementedError

    def tables(self, device):
        key = str(device)
        t = self._tabs.get(key)
        if t is None:
            t = self._tabs[key] = self._device_tables(device)
        return t

    # -- device-level evaluation -----------------------------------------------
    def evaluate(self, batch, dlist, precision=None, out=None, ws=None):
        """Energy, forces and virial of every structure of ``batch`` with the
        device list ``dlist`` (a DeviceNeighbourList).  Returns EvalResult.
        ``ws`` is a caller-owned uint8 workspace (default: the thread's shared
        one, which a later, larger call may replace)."""
        prec = precision_code(precision or self.precision)
        dev = batch.device
        L = _lib.lib()
        nbytes = int(L.mbf_eval_workspace_bytes(batch.n_atoms, dlist.n_slots, batch.n_chunks))
        if ws is None:
            ws = workspace(dev, nbytes)
        elif ws.numel() < nbytes:
            raise ValueError(f"evaluate: workspace of {ws.numel()} bytes, {nbytes} needed")
        if out is None:
            out = EvalResult(torch.empty(batch.n_struct, dtype=torch.float64, device=dev),
                             torch.empty((batch.n_atoms, 3), dtype=torch.float64, device=dev),
                             torch.empty((batch.n_struct, 9), dtype=torch.float64, device=dev))
        tabs = self.tables(dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = self._call(L, batch.mbf_system(), dlist.mbf_nlist(), tabs, batch.reduce_plan(), prec,
                        _lib.ptr(ws), ws.numel(), _lib.ptr(out.forces), _lib.ptr(out.energy),
                        _lib.ptr(out.virial), stream)
        _lib.check(rc, type(self).__name__ + ".evaluate")
        _set_last_ws(self, ws)
        return out

    def evaluate_sites(self, batch, dlist, precision=None):
        """evaluate() plus the site-energy decomposition (heat flux): returns
        (EvalResult, site_e (N,), dU/dv (n_slots, 3), v (n_slots, 3)) on the
        device; slots beyond the cutoff have dU/dv = 0."""
        prec = precision_code(precision or self.precision)
        dev = batch.device
        L = _lib.lib()
        nbytes = int(L.mbf_eval_workspace_bytes(batch.n_atoms, dlist.n_slots, batch.n_chunks))
        ws = workspace(dev, nbytes)
        f64 = dict(dtype=torch.float64, device=dev)
        out = EvalResult(torch.empty(batch.n_struct, **f64), torch.empty((batch.n_atoms, 3), **f64),
                         torch.empty((batch.n_struct, 9), **f64))
        e = torch.empty(batch.n_atoms, **f64)
        dudv = torch.zeros((max(int(dlist.n_slots), 1), 3), **f64)
        vec = torch.zeros((max(int(dlist.n_slots), 1), 3), **f64)
        tabs = self.tables(dev)
        rc = getattr(L, self.sites_entry)(batch.mbf_system(), dlist.mbf_nlist(), tabs[0], batch.reduce_plan(), prec,
                                          int(self.lanes_per_atom), _lib.ptr(ws), ws.numel(), _lib.ptr(out.forces),
                                          _lib.ptr(out.energy), _lib.ptr(out.virial), _lib.ptr(e), _lib.ptr(dudv),
                                          _lib.ptr(vec), torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(rc, type(self).__name__ + ".evaluate_sites")
        _set_last_ws(self, ws)
        return out, e, dudv, vec

    def autotune_lanes(self, batch, dlist, candidates=None, reps=3, ws=None, out=None):
        """Time every lanes-per-atom candidate on this batch (CUDA events,
        after one untimed call each), keep the fastest and return
        {"lanes_per_atom": best, "ms": {candidate: ms}}.  With ``out`` and
        ``ws`` given, each candidate is captured in a CUDA graph and the
        replays are timed, so the host's launch cost (which can exceed a
        small batch's device time) does not decide the choice."""
        cands = tuple(candidates or self.lane_choices)
        timings = {}
        dev = batch.device
        for c in cands:
            self.lanes_per_atom = c
            self.evaluate(batch, dlist, out=out, ws=ws)
            run = lambda: self.evaluate(batch, dlist, out=out, ws=ws)  # noqa: E731
            graph = None
            if out is not None and ws is not None:
                graph = capture_graph(run, dev)
                graph.replay()
                run = graph.replay
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                run()
            b.record()
            b.synchronize()
            timings[c] = a.elapsed_time(b) / reps
            del graph
        best = min(cands, key=lambda c: (timings[c], c))
        self.lanes_per_atom = best
        return {"lanes_per_atom": best, "ms": timings}

    def status(self, device=None):
        """Device status words of the last evaluation (synchronises): raises
        if a kernel reported a bad index or an over-long row."""
        ws = _get_last_ws(self)
        if ws is None:
            return
        words = (_lib._i * 4)()
        _lib.check(_lib.lib().mbf_eval_status(_lib.ptr(ws), words,
                                              torch.cuda.current_stream(ws.device).cuda_stream),
                   "mbf_eval_status")
        self._raise_status(list(words))

    def _raise_status(self, words):
        if words[0] or words[1]:
            raise RuntimeError(f"{type(self).__name__}: device check failed (bits {words[0]}, "
                               f"site {words[1]}, index {words[2]})")

    # -- reference protocol ------------------------------------------------------
    def _resolve_list(self, lattice, positions, neigh_list, device):
        if isinstance(neigh_list, NeighbourList):
            if neigh_list._batch is None:
                neigh_list.build(lattice, positions)
            return neigh_list, neigh_list._batch, neigh_list.device_list
        if neigh_list is not None and hasattr(neigh_list, "get_candidate_pairs"):
            # a CPU list (e.g. the reference's own): its candidates on the device
            key = id(neigh_list)
            stamp = (getattr(neigh_list, "rebuild_count", None), len(positions))
            hit = self._foreign.get(key)
            if hit is None or hit[0] != stamp:
                i, j = neigh_list.get_candidate_pairs()
                dl = DeviceNeighbourList.from_pairs(len(positions), i, j,
                                                    float(getattr(neigh_list, "r_list", self.r_cut)),
                                                    device)
                b = Batch.single(lattice, positions, np.zeros(len(positions), np.int32), device=device)
                hit = (stamp, b, dl)
                self._foreign = {key: hit}
            return None, hit[1], hit[2]
        nl = owned_neighbour_list(lattice, positions, self.r_cut, device=device)
        return nl, nl._batch, nl.device_list

    def compute(self, lattice, positions, atom_types, neigh_list=None, use_numba=False,
                need_stress=True, device=None):
        """(energy, forces (N, 3), stress (3, 3) or None) on the host, like the
        reference; the evaluation itself runs on the GPU."""
        lattice = np.asarray(lattice, dtype=np.float64)
        is_t = isinstance(positions, torch.Tensor)
        pos = positions if is_t else np.ascontiguousarray(positions, dtype=np.float64)
        n = int(pos.shape[0])
        if n == 0:
            return 0.0, np.zeros((0, 3)), (np.zeros((3, 3)) if need_stress else None)
        dev = torch.device(device) if device is not None else None
        if dev is None:
            from .system import default_device
            dev = default_device()
        nl, batch, dl = self._resolve_list(lattice, pos, neigh_list, dev)
        batch.set_lattice(0, lattice)
        batch.set_positions(pos, check=False)   # as the reference: no scan of the input
        # an integer id array equal to the one on the device was validated
        # and uploaded before: one comparison instead of a range check and
        # a comparison
        if not batch.types_unchanged(atom_types, len(self.species)):
            batch.set_types(species_ids(atom_types, self.species))
        res = self.evaluate(batch, dl)
        # energy, virial and the device status words (the first 16 bytes of
        # the workspace, carried as two doubles) in one copy
        words = _get_last_ws(self)[:16].view(torch.float64)
        ev = torch.cat([res.energy[:1], res.virial[0], words]).to("cpu", non_blocking=True)
        f = batch.forces_to_host(res.forces)   # synchronises the stream
        ev = ev.numpy()
        self._raise_status(np.frombuffer(ev[10:12].tobytes(), dtype=np.int32))
        e = float(ev[0])
        if not need_stress:
            return e, f, None
        vol = abs(float(np.linalg.det(lattice)))
        s = ev[1:10].reshape(3, 3) / vol
        return e, f, s


def nested_records(params):
    """{(i, j, k): rec} from a list of {i, j, k, ...} records or a dict."""
    if isinstance(params, dict):
        return {tuple(k): dict(v) for k, v in params.items()}
    out = {}
    for rec in params:
        rec = dict(rec)
        out[(rec.pop("i"), rec.pop("j"), rec.pop("k"))] = rec
    return out
