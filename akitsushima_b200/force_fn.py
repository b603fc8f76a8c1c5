"""The force-function boundary: PotentialEngine, make_force_fn and
force_fn_from_config, mirroring the reference's
engine/potential_engine.py:40-105, fitting/force_fn.py:273-333, :386-419 and
solvers/config_bridge.py:148-166 with fitting/registry.py:572-799.

A force function is ``fn(lattice, positions, atom_types, neigh_list=None,
need_stress=True) -> (energy, forces (N, 3), stress (3, 3) | None)`` with
``.r_cut``, ``.kind = "engine"``, ``.engine`` and
``.uses_neighbour_list = False``: solvers then hand it a NullNeighbourList
and it keeps a device-resident list of its own (it also accepts a
NeighbourList of this package, or any list with get_candidate_pairs()).
"""
import inspect
import weakref

import numpy as np

from .eam import EAMPotential, read_setfl, zhou_eam
from .neighbourlist import NeighbourList
from .potential import precision_code
from .published_parameters import ZHOU_2004
from .stillinger_weber import StillingerWeberPotential
from .tersoff import TersoffPotential, tersoff1989_to_triplets


class PotentialEngine:
    """Sum of potentials (engine/potential_engine.py:40-105)."""

    def __init__(self):
        self.potentials = []

    def add(self, pot):
        self.potentials.append(pot)
        return self

    @property
    def r_cut(self):
        return max((float(p.r_cut) for p in self.potentials), default=0.0)

    @property
    def species(self):
        out = []
        for p in self.potentials:
            for s in p.species or []:
                if s not in out:
                    out.append(s)
        return out

    def set_precision(self, precision):
        precision_code(precision)
        for p in self.potentials:
            p.precision = precision
        return self

    def compute(self, lattice, positions, atom_types, neigh_list=None, use_numba=False,
                need_stress=True):
        N = len(positions)
        if not self.potentials:
            return 0.0, np.zeros((N, 3)), (np.zeros((3, 3)) if need_stress else None)
        e_tot = f_tot = s_tot = None
        for p in self.potentials:
            e, f, s = p.compute(lattice, positions, atom_types, neigh_list=neigh_list,
                                need_stress=need_stress)
            if f_tot is None:   # the first result is a new array: sum into it
                e_tot, f_tot, s_tot = e, f, s
                continue
            e_tot += e
            f_tot += f
            if need_stress:
                s_tot += s
        return e_tot, f_tot, s_tot

    def evaluate(self, batch, dlists, precision=None):
        """Device evaluation of a batch; ``dlists`` is one DeviceNeighbourList
        per potential (or one shared).  Returns (energy (S,), forces (N, 3),
        virial (S, 9)) torch tensors."""
        if not isinstance(dlists, (list, tuple)):
            dlists = [dlists] * len(self.potentials)
        e = f = v = None
        for p, dl in zip(self.potentials, dlists):
            r = p.evaluate(batch, dl, precision=precision)
            if e is None:
                e, f, v = r.energy, r.forces, r.virial
            else:
                e = e + r.energy
                f = f + r.forces
                v = v + r.virial
        return e, f, v


def make_force_fn(backend, r_cut=None, precision=None, device=None):
    """Force function of a PotentialEngine or a single potential
    (fitting/force_fn.py:273-333)."""
    eng = backend if isinstance(backend, PotentialEngine) else PotentialEngine().add(backend)
    if precision is not None:
        eng.set_precision(precision)
    rc = eng.r_cut if r_cut is None else float(r_cut)

    def _engine_fn(lattice, positions, atom_types, neigh_list=None, need_stress=True):
        if neigh_list is not None and not isinstance(neigh_list, NeighbourList) \
                and not hasattr(neigh_list, "get_candidate_pairs"):
            neigh_list = None          # a NullNeighbourList: use the owned device list
        if isinstance(neigh_list, NeighbourList) and abs(neigh_list.r_cut - rc) > 1e-12 \
                and neigh_list.r_list < eng.r_cut:
            raise ValueError(f"neighbour list r_list {neigh_list.r_list} is shorter than the "
                             f"potential cutoff {eng.r_cut}")
        e, f, s = eng.compute(lattice, positions, atom_types, neigh_list=neigh_list,
                              need_stress=need_stress)
        return e, f, (s if need_stress else None)

    _engine_fn.r_cut = rc
    _engine_fn.kind = "engine"
    _engine_fn.engine = eng
    _engine_fn.uses_neighbour_list = False
    _engine_fn.device = "cuda"
    return _engine_fn


_NEED_STRESS_CACHE = weakref.WeakKeyDictionary()


def accepts_need_stress(fn):
    """True when ``fn`` names a ``need_stress`` parameter
    (fitting/force_fn.py:386-410)."""
    try:
        return _NEED_STRESS_CACHE[fn]
    except (KeyError, TypeError):
        pass
    try:
        ok = "need_stress" in inspect.signature(fn).parameters
    except (TypeError, ValueError):
        ok = False
    try:
        _NEED_STRESS_CACHE[fn] = ok
    except TypeError:
        pass
    return ok


def call_force_fn(fn, lattice, positions, atom_types, need_stress=True, **kw):
    """fitting/force_fn.py:413-419."""
    if not need_stress and accepts_need_stress(fn):
        return fn(lattice, positions, atom_types, need_stress=False, **kw)
    return fn(lattice, positions, atom_types, **kw)


# ---- YAML / dict configuration (fitting/registry.py) ------------------------

def _compute_opts(cfg):
    comp = cfg.get("compute") or {}
    device = cfg.get("device", comp.get("device", "cuda"))
    precision = cfg.get("precision", comp.get("precision", "fp64"))
    if str(device).split(":")[0] != "cuda":
        raise ValueError(f"this package evaluates on 'cuda' only, got device {device!r}")
    precision_code(precision)
    return device, precision


def _records(params):
    nested = {}
    items = params if isinstance(params, list) else \
        [dict(i=t[0], j=t[1], k=t[2], **v) for t, v in params.items()]
    for rec in items:
        rec = dict(rec)
        nested[(rec.pop("i"), rec.pop("j"), rec.pop("k"))] = rec
    return nested


def _build_sw(cfg, precision):
    species = cfg.get("species", [])
    params = cfg.get("params", {})
    if isinstance(params, list):
        nested = _records(params)
        pot = StillingerWeberPotential(nested, species=species, precision=precision)
        r_cut = max(float(v["a"]) * float(v["sigma"]) for (i, j, k), v in nested.items() if j == k)
    else:
        pot = StillingerWeberPotential(params, species=species, precision=precision)
        r_cut = params.get("a", 1.80) * params.get("sigma", 2.0951)
    return pot, float(r_cut)


def _is_tersoff1989(p):
    return isinstance(p, dict) and str(p.get("mixing", "")).lower() == "tersoff1989"


def _build_tersoff(cfg, precision):
    species = cfg.get("species", [])
    params = cfg.get("params", {})
    if _is_tersoff1989(params):
        species = species or list(params["elements"])
        params = tersoff1989_to_triplets(params["elements"], params.get("chi", {}), species,
                                         params.get("omega"))
    if isinstance(params, list) or (isinstance(params, dict)
                                    and any(isinstance(k, tuple) for k in params)):
        nested = _records(params)
        pot = TersoffPotential(nested, species=species, precision=precision)
        r_cut = max(float(v["R"]) + float(v["D"]) for (i, j, k), v in nested.items() if j == k)
    else:
        pot = TersoffPotential(params, species=species, precision=precision)
        r_cut = float(params.get("R", 2.85)) + float(params.get("D", 0.15))
    return pot, float(r_cut)


def _zhou_elements(spec):
    if isinstance(spec, (list, tuple)):
        missing = [s for s in spec if s not in ZHOU_2004]
        if missing:
            raise ValueError(f"EAM zhou2004: {missing} not in Zhou et al. (2004) Table III")
        return {s: dict(ZHOU_2004[s]) for s in spec}
    return {s: dict(v) for s, v in spec.items()}


def _build_eam(cfg, precision):
    species = cfg.get("species")
    if "setfl" in cfg:
        pot = read_setfl(cfg["setfl"], species=species, precision=precision)
    elif str(cfg.get("form", "")).lower() == "zhou2004":
        el = _zhou_elements(cfg["elements"])
        species = species or list(el)
        pot = zhou_eam(el, species, r_cut=cfg.get("r_cut"), chi=cfg.get("chi"),
                       precision=precision)
    else:
        raise ValueError("an EAM potential needs 'setfl: <file>' or 'form: zhou2004' with "
                         "'elements:'.")
    return pot, float(pot.r_cut)


_BUILDERS = {"sw": _build_sw, "stillingerweber": _build_sw, "stillinger-weber": _build_sw,
             "tersoff": _build_tersoff, "t3": _build_tersoff, "eam": _build_eam}


def force_fn_from_config(potential, device=None, precision=None):
    """A force function from a ``potential:`` section
    (solvers/config_bridge.py:148-166), e.g. ``{"type": "Tersoff", "species":
    ["Si"], "params": {...}}`` or ``{"type": "EAM", "form": "zhou2004",
    "elements": ["Cu", "Ni"]}``.  Optional ``device`` / ``precision`` keys
    (or a ``compute: {device, precision}`` block) select the GPU path's
    arithmetic: 'fp64' (default) or 'mixed'."""
    cfg = dict(potential)
    if device is not None:
        cfg["device"] = device
    if precision is not None:
        cfg["precision"] = precision
    _, prec = _compute_opts(cfg)
    kind = str(cfg.get("type", "")).strip().lower()
    if kind not in _BUILDERS:
        raise ValueError(f"unsupported potential type {cfg.get('type')!r}: this package "
                         "implements SW, Tersoff and EAM")
    pot, r_cut = _BUILDERS[kind](cfg, prec)
    fn = make_force_fn(PotentialEngine().add(pot))
    fn.r_cut = float(r_cut)
    fn.precision = prec
    return fn

