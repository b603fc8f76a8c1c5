"""Velocity-Verlet NVE molecular dynamics with the whole step on the device.

The integrator of the reference's NVESimulation.run
(solvers/molecular_dynamics.py:1969-2000): half kick, drift, wrap into the
cell, force call, half kick; Maxwell-Boltzmann start as _init_velocities_mb
(:195-221); kinetic energy and temperature as :239-244 and :939-941 with
n_dof = max(3N - 3, 1) (nothing fixed).

Positions, velocities and forces stay in HBM for the whole run.  The
neighbour list is rebuilt in place with no host synchronisation
(mbf_nl_rebuild_async) when the reference's
displacement criterion (engine/neighborlist.py:613-673, lattice fixed:
rebuild iff r_list - 2 max|dr| <= r_cut), evaluated on the device every
step, fires:
in a captured graph the rebuild is an IF branch on that decision.  With a
fixed interval instead, the criterion is asserted at each rebuild.  A block
of steps is captured as one CUDA graph and replayed.
"""
import ctypes
import weakref

import numpy as np
import torch

from . import _lib
from .neighbourlist import DeviceNeighbourList
from .potential import EvalResult
from .system import Batch, capture_graph, default_device, species_ids

# solvers/../constants.py:8-20 of the reference (CODATA values it uses).
EV_ANG_TO_AMU_ANG_FS2 = (1.60217663e-19 / 1.0e-10) / (1.66053906660e-27) * 1.0e-20
K_B = 1.380649e-23 * 6.241509074e18

# Standard atomic weights [amu] of the elements the potentials of this
# package are parameterised for, rounded as the reference's table
# (constants.py:92-113).
ATOMIC_MASS = {
    "C": 12.011, "Mg": 24.305, "Al": 26.982, "Si": 28.086, "Ti": 47.867, "Fe": 55.845,
    "Co": 58.933, "Ni": 58.693, "Cu": 63.546, "Ge": 72.630, "Zr": 91.224, "Mo": 95.96,
    "Pd": 106.42, "Ag": 107.87, "Sn": 118.71, "Ta": 180.95, "W": 183.84, "Pt": 195.08,
    "Au": 196.97, "Pb": 207.2,
}


def init_velocities_mb(T, masses, rng):
    """Maxwell-Boltzmann velocities [A/fs] at T [K]: N(0, sqrt(k_B T conv /
    m)) per component, centre-of-mass momentum removed, rescaled to exactly
    T with n_dof = max(3N - 3, 1) (solvers/molecular_dynamics.py:195-221;
    the same draws from the same generator give the same velocities)."""
    masses = np.asarray(masses, float)
    N = len(masses)
    if N == 0:
        return np.empty((0, 3))
    sigma = np.sqrt(K_B * T * EV_ANG_TO_AMU_ANG_FS2 / masses)
    v = rng.standard_normal((N, 3)) * sigma[:, None]
    v -= np.sum(masses[:, None] * v, axis=0) / masses.sum()
    e_kin = 0.5 * float(np.sum(masses[:, None] * v ** 2)) / EV_ANG_TO_AMU_ANG_FS2
    n_dof = max(3 * N - 3, 1)
    t_act = 2.0 * e_kin / (n_dof * K_B)
    if t_act > 1e-12:
        v *= np.sqrt(T / t_act)
    return v


def masses_for(atom_types, masses=None):
    """Per-atom masses [amu] from a {species: mass} override or the table."""
    table = dict(ATOMIC_MASS)
    if masses is not None and not isinstance(masses, dict) and not np.ndim(masses):
        raise ValueError("masses: give a per-atom array or a {species: mass} dict")
    if isinstance(masses, dict):
        table.update(masses)
    elif masses is not None:
        m = np.asarray(masses, float)
        if m.shape != (len(atom_types),) or not np.all(m > 0):
            raise ValueError("masses: expected positive (N,) amu")
        return m
    try:
        return np.array([table[str(t)] for t in atom_types], float)
    except KeyError as exc:
        raise ValueError(f"no atomic mass for species {exc.args[0]!r}; pass masses=") from None


class _FixedList:
    """A device list seen with its buffer capacity as the slot count and a
    fixed row bound, so evaluation launches keep their arguments (and a
    captured graph stays valid) across in-place rebuilds."""

    def __init__(self, dlist, capacity, max_row):
        self.d = dlist
        self.n_slots = int(capacity)
        self.max_row = int(max_row)
        self._nl = None   # the C view, built once (the buffers never move)

    def mbf_nlist(self):
        if self._nl is None:
            d = self.d
            self._nl = _lib.MbfNlist(d.n_atoms, self.n_slots, self.max_row, _lib.ptr(d.row_off),
                                     _lib.ptr(d.nbr), _lib.ptr(d.rev), _lib.ptr(d.upper))
        return self._nl


def _row_bound(max_row):
    need = int(max_row * 1.25) + 4
    for b in (32, 64, 128):
        if need <= b:
            return b
    return max(need, 128)


# lanes-per-atom choices per potential (weakly held) and system shape
_TUNED = weakref.WeakKeyDictionary()


class NVE:
    """Velocity-Verlet NVE of one structure on the GPU.

    Parameters
    ----------
    potential     : a TersoffPotential, StillingerWeberPotential or
                    EAMPotential of this package.
    lattice, positions, atom_types : the structure (A; species names).
    temperature   : Maxwell-Boltzmann start [K] (ignored with velocities=).
    dt            : time step [fs].
    seed          : numpy default_rng seed of the velocity draw.
    skin          : list skin [A].
    rebuild_every : None (default): the reference's policy, the displacement
                    criterion evaluated on the device every step and the
                    list rebuilt when it fires (a graph IF branch); an int k:
                    rebuild every k steps, with the criterion asserted at
                    each rebuild (results() raises if it had fired).
    steps_per_graph : MD steps captured in one CUDA graph (criterion
                    policy; a fixed interval captures k steps).
    masses        : per-atom amu or {species: amu} (default: the table).
    precision     : 'fp64' or 'mixed' (default: the potential's).
    autotune      : time the potential's lanes-per-atom tile shapes on this
                    structure once and keep the fastest (remembered for
                    later NVEs of the same potential, atom count, row bound
                    and precision).
    """

    def __init__(self, potential, lattice, positions, atom_types, temperature=300.0, dt=1.0, seed=None,
                 skin=0.3, rebuild_every=None, steps_per_graph=10, masses=None, velocities=None,
                 precision=None, device=None, thermo_rows=1 << 16, autotune=True):
        if not dt > 0:
            raise ValueError("dt must be positive")
        if rebuild_every is not None and int(rebuild_every) < 1:
            raise ValueError("rebuild_every must be None or >= 1")
        if int(steps_per_graph) < 1:
            raise ValueError("steps_per_graph must be >= 1")
        self.pot = potential
        self.dt = float(dt)
        self.skin = float(skin)
        self.rebuild_every = None if rebuild_every is None else int(rebuild_every)
        self.block = self.rebuild_every or int(steps_per_graph)
        self.precision = precision or potential.precision
        self.device = torch.device(device) if device is not None else default_device()
        dev = self.device
        pos = np.asarray(positions, float)
        self.n_atoms = len(pos)
        self.masses = masses_for(atom_types, masses)
        ids = species_ids(atom_types, potential.species)
        self.batch = Batch.single(lattice, pos, ids, device=dev)
        # list buffers with room for the rows to grow: 1.5 x the slots, from
        # the density's estimate first and, if the list came out larger,
        # from its own count (then built once more)
        self.dlist = DeviceNeighbourList(float(potential.r_cut) + self.skin)
        self.dlist.build(self.batch, capacity=int(1.5 * self.dlist.expected_rows(self.batch)[0]) + 4096)
        cap = int(self.dlist.n_slots * 1.5) + 4096
        if self.dlist.nbr.numel() < cap:
            self.dlist.nbr = torch.empty(cap, dtype=torch.int32, device=dev)
            self.dlist.rev = torch.empty(cap, dtype=torch.int32, device=dev)
            self.dlist.build(self.batch)
        cap = self.dlist.nbr.numel()
        self.view = _FixedList(self.dlist, cap, _row_bound(self.dlist.max_row))
        L = _lib.lib()
        nbytes = int(L.mbf_eval_workspace_bytes(self.n_atoms, cap, self.batch.n_chunks))
        self._ws = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=dev)
        self._n_cells = self.dlist._grid_table(self.batch)[1]
        nl_bytes = int(L.mbf_nl_rebuild_workspace_bytes(self.n_atoms, self._n_cells, self.view.max_row))
        self._nl_ws = torch.empty(max(nl_bytes, 256), dtype=torch.uint8, device=dev)
        if velocities is None:
            rng = np.random.default_rng(seed)
            velocities = init_velocities_mb(temperature, self.masses, rng)
        v = np.asarray(velocities, float)
        if v.shape != pos.shape:
            raise ValueError("velocities: expected (N, 3) A/fs")
        self.vel = torch.as_tensor(np.ascontiguousarray(v), device=dev)
        self.inv_mass = torch.as_tensor(EV_ANG_TO_AMU_ANG_FS2 / self.masses, device=dev)
        self.out = EvalResult(torch.empty(1, dtype=torch.float64, device=dev),
                              torch.empty((self.n_atoms, 3), dtype=torch.float64, device=dev),
                              torch.empty((1, 9), dtype=torch.float64, device=dev))
        self.thermo_rows = int(thermo_rows)
        self.thermo = torch.zeros((self.thermo_rows, 1, 2), dtype=torch.float64, device=dev)
        self.skin_log = torch.zeros((self.thermo_rows, 1), dtype=torch.float64, device=dev)
        # device words: thermo row, skin row, status, rebuilds, rebuild gate,
        # and the completion counters of the two fused kick launches
        self._counters = torch.zeros(8, dtype=torch.int32, device=dev)
        self._partial = torch.empty(int(L.mbf_md_partial_count(self.n_atoms)), dtype=torch.float64, device=dev)
        self._dscratch = torch.empty(1, dtype=torch.float64, device=dev)
        self._dmax = torch.zeros(1, dtype=torch.int64, device=dev)   # left at 0 by every check
        self._ref = self.batch.pos.clone()
        self._body = torch.cuda.Stream(dev)
        self._graph = None
        self.steps_done = 0
        if autotune:
            # one tuning per potential, atom count, row bound and precision:
            # a later NVE of the same system shape reuses the choice
            key = (self.n_atoms, self.view.max_row, self.precision, str(dev))
            cache = _TUNED.setdefault(self.pot, {})
            if key in cache:
                self.tuned = cache[key]
                self.pot.lanes_per_atom = self.tuned["lanes_per_atom"]
            else:
                saved_precision = self.pot.precision
                self.pot.precision = self.precision
                self.tuned = self.pot.autotune_lanes(self.batch, self.view, ws=self._ws, out=self.out)
                self.pot.precision = saved_precision
                cache[key] = self.tuned
        self._eval()
        self.e_pot0 = float(self.out.energy[0].item())
        self.e_kin0 = self.kinetic_energy()
        self._warm()

    def _warm(self):
        """One eager step and one rebuild, then the state put back: every
        kernel is loaded before a graph capture needs it."""
        d = self.dlist
        state = (self.batch.pos, self.vel, self.out.forces, self.out.energy, self._ref, d.row_off, d.upper,
                 d.nbr, d.rev)
        saved = [t.clone() for t in state]
        st = torch.cuda.current_stream(self.device).cuda_stream
        self._step(0, capturing=False)
        self._kick_kick(st)
        self._skin_check(st, assert_only=False)
        self._rebuild(st)
        for dst, src in zip(state, saved):
            dst.copy_(src)
        self._counters.zero_()
        self.thermo.zero_()
        self.skin_log.zero_()
        torch.cuda.synchronize(self.device)

    # -- launch pieces --------------------------------------------------------
    def _word(self, k):
        return self._counters.data_ptr() + 4 * k

    def _eval(self):
        return self.pot.evaluate(self.batch, self.view, precision=self.precision, out=self.out, ws=self._ws)

    def _rebuild(self, stream):
        L = _lib.lib()
        d = self.dlist
        sysd = self.batch.mbf_system()
        _lib.check(L.mbf_nl_rebuild_async(sysd, _lib.ptr(d._grids), self._n_cells, d.r_list, _lib.ptr(self._nl_ws),
                                          self._nl_ws.numel(), _lib.ptr(d.row_off), _lib.ptr(d.nbr), _lib.ptr(d.rev),
                                          _lib.ptr(d.upper), self.view.n_slots, self.view.max_row, self._word(2),
                                          stream), "mbf_nl_rebuild_async")
        _lib.check(L.mbf_md_rebuild_done(sysd, _lib.ptr(self._ref), self._word(3), stream), "mbf_md_rebuild_done")

    def _skin_check(self, stream, assert_only, cond=0):
        _lib.check(_lib.lib().mbf_md_skin_check(self.batch.mbf_system(), _lib.ptr(self._ref), self.dlist.r_list,
                                                float(self.pot.r_cut), _lib.ptr(self._dscratch),
                                                _lib.ptr(self.skin_log), self.thermo_rows,
                                                self._word(1), self._word(4), self._word(2) if assert_only else None,
                                                cond, stream), "mbf_md_skin_check")

    def _kick_drift_check(self, stream, cond=0):
        """First half kick, drift and the criterion check in one launch."""
        _lib.check(_lib.lib().mbf_md_kick_drift_check(
            self.batch.mbf_system(), _lib.ptr(self.batch.pos), _lib.ptr(self.vel), _lib.ptr(self.out.forces),
            _lib.ptr(self.inv_mass), self.dt, _lib.ptr(self._ref), self.dlist.r_list, float(self.pot.r_cut),
            _lib.ptr(self._dmax), self._word(5), _lib.ptr(self.skin_log), self.thermo_rows, self._word(1),
            self._word(4), cond, stream), "mbf_md_kick_drift_check")

    def _kick_kick(self, stream, cond=0):
        """The second half kick (and thermo row) of a step and the first
        half kick, drift and criterion check of the next in one launch."""
        _lib.check(_lib.lib().mbf_md_kick_kick_drift_check(
            self.batch.mbf_system(), _lib.ptr(self.batch.pos), _lib.ptr(self.vel), _lib.ptr(self.out.forces),
            _lib.ptr(self.inv_mass), self.dt, _lib.ptr(self.out.energy), _lib.ptr(self._partial),
            _lib.ptr(self.thermo), self.thermo_rows, self._word(0), _lib.ptr(self._ref), self.dlist.r_list,
            float(self.pot.r_cut), _lib.ptr(self._dmax), _lib.ptr(self.skin_log), self.thermo_rows, self._word(1),
            self._word(4), cond, self._word(5), stream), "mbf_md_kick_kick_drift_check")

    def _check_then_rebuild(self, launch, capturing):
        """`launch` (a kick ending in the criterion check), then the list
        rebuild it asks for: an IF branch in a capture, else decided on the
        host from the gate word."""
        st = torch.cuda.current_stream(self.device).cuda_stream
        if capturing:
            L = _lib.lib()
            h = ctypes.c_ulonglong(0)
            _lib.check(L.mbf_capture_cond_create(st, ctypes.byref(h)), "mbf_capture_cond_create")
            launch(st, cond=h.value)
            body = self._body.cuda_stream
            _lib.check(L.mbf_capture_if_begin(st, body, h.value), "mbf_capture_if_begin")
            try:
                self._rebuild(body)
            finally:
                _lib.check(L.mbf_capture_if_end(body), "mbf_capture_if_end")
        else:
            launch(st)
            if int(self._counters[4].item()):
                self._rebuild(st)

    def _step(self, k, capturing):
        """MD step number k of a block (k counts from 0)."""
        L = _lib.lib()
        st = torch.cuda.current_stream(self.device).cuda_stream
        sysd = self.batch.mbf_system()
        if self.rebuild_every is not None:
            _lib.check(L.mbf_md_kick_drift(sysd, _lib.ptr(self.batch.pos), _lib.ptr(self.vel),
                                           _lib.ptr(self.out.forces), _lib.ptr(self.inv_mass), self.dt, st),
                       "mbf_md_kick_drift")
            if k % self.rebuild_every == 0:
                self._skin_check(st, assert_only=True)
                self._rebuild(st)
        else:
            self._check_then_rebuild(self._kick_drift_check, capturing)
        self._eval()
        self._kick(st)

    def _kick(self, stream):
        """Second half kick and the thermo row of the step."""
        L = _lib.lib()
        _lib.check(L.mbf_md_kick(self.batch.mbf_system(), _lib.ptr(self.vel), _lib.ptr(self.out.forces),
                                 _lib.ptr(self.inv_mass), self.dt, _lib.ptr(self.out.energy),
                                 _lib.ptr(self._partial), _lib.ptr(self.thermo), self.thermo_rows, self._word(0),
                                 self._word(6), stream), "mbf_md_kick")

    def _run_block(self, capturing=False):
        """A block of MD steps.  Under the criterion policy the second half
        kick of every step but the last shares a launch with the first half
        kick, drift and check of the next (the same arithmetic); the block
        still ends on a whole step, so positions, velocities and thermo
        between blocks are those of separate launches."""
        if self.rebuild_every is not None:
            for k in range(self.block):
                self._step(k, capturing)
            return
        self._check_then_rebuild(self._kick_drift_check, capturing)
        for k in range(self.block):
            self._eval()
            if k + 1 < self.block:
                self._check_then_rebuild(self._kick_kick, capturing)
            else:
                self._kick(torch.cuda.current_stream(self.device).cuda_stream)

    # -- public ---------------------------------------------------------------
    def capture(self):
        """Capture one block of MD steps (criterion checks and the gated
        rebuild branches included) as a CUDA graph; run() replays it."""
        torch.cuda.synchronize(self.device)
        self._graph = capture_graph(lambda: self._run_block(capturing=True), self.device, warm=False)
        torch.cuda.synchronize(self.device)
        return self

    def run(self, n_steps, graph=True):
        """Advance n_steps (asynchronous; results() reads them).  Whole
        blocks replay the captured graph; a remainder runs as eager launches
        (which synchronise once per step under the criterion policy)."""
        n_steps = int(n_steps)
        blocks, rem = divmod(n_steps, self.block)
        if graph and blocks and self._graph is None:
            self.capture()
        for _ in range(blocks):
            if graph:
                self._graph.replay()
            else:
                self._run_block()
        for k in range(rem):
            self._step(k, capturing=False)
        self.steps_done += n_steps
        return self

    @property
    def rebuilds(self):
        """List rebuilds since construction (the initial build not counted)."""
        return int(self._counters[3].item())

    def status(self):
        """Raise if a rebuild overflowed its buffers or a row outgrew its
        bound, or (fixed interval) the criterion had fired at a rebuild."""
        st = int(self._counters[2].item())
        if st & _lib.MBF_STATUS_SKIN:
            n = min(int(self._counters[1].item()), self.thermo_rows)
            d = self.skin_log[:n, 0].max().item() if n else float("nan")
            raise RuntimeError(f"NVE: an atom moved {d:.4f} A between rebuilds; 2 d >= skin "
                               f"{self.skin}: the reference's criterion would have rebuilt earlier; "
                               "lower rebuild_every, raise skin, or use rebuild_every=None")
        if st & (_lib.MBF_STATUS_CAPACITY | _lib.MBF_STATUS_ROW_TOO_LONG):
            raise RuntimeError(f"NVE: the neighbour list outgrew its buffers (status {st}); forces after "
                               "that rebuild are void")
        if st:
            raise RuntimeError(f"NVE: device status {st}")
        self.pot.status(self.device)

    def results(self):
        """Thermo rows of the steps run so far (up to thermo_rows, oldest
        first): dict of e_pot, e_kin, e_tot, temperature (K) arrays, the
        displacement the criterion saw at each check, the rebuild count, and
        the drift e_tot - e_tot(step 0), the reference's drift column
        (solvers/molecular_dynamics.py:1996)."""
        self.status()

        def rows_of(buf, n):
            m = min(n, self.thermo_rows)
            t = buf.cpu().numpy()
            if n > self.thermo_rows:
                t = np.roll(t, -(n % self.thermo_rows), axis=0)
            return t[:m]

        t = rows_of(self.thermo, int(self._counters[0].item()))[:, 0, :]
        e_pot, e_kin = t[:, 0].copy(), t[:, 1].copy()
        n_dof = max(3 * self.n_atoms - 3, 1)
        e_tot = e_pot + e_kin
        e0 = self.e_pot0 + self.e_kin0
        return {"e_pot": e_pot, "e_kin": e_kin, "e_tot": e_tot,
                "temperature": 2.0 * e_kin / (n_dof * K_B),
                "skin_displacement": rows_of(self.skin_log, int(self._counters[1].item()))[:, 0],
                "rebuilds": self.rebuilds, "drift": e_tot - e0, "e_tot0": e0}

    @property
    def positions(self):
        return self.batch.pos.cpu().numpy()

    @property
    def velocities(self):
        return self.vel.cpu().numpy()

    @property
    def forces(self):
        return self.out.forces.cpu().numpy()

    def kinetic_energy(self):
        v = self.vel.cpu().numpy()
        return 0.5 * float(np.sum(self.masses[:, None] * v ** 2)) / EV_ANG_TO_AMU_ANG_FS2
