"""Alloy EAM on the GPU (reference engine/eam.py, engine/eam_zhou.py,
engine/_eam_kernels.py).

E = sum_i F_{s_i}(rho_bar_i) + 1/2 sum_{i != j} phi_{s_i s_j}(r_ij),
rho_bar_i = max(0, sum_{j != i} rho_{s_j}(r_ij)) -- the density at an atom
comes from its NEIGHBOURS' species functions (DYNAMO / setfl alloy form).

The functions must have a form the device knows, the same restriction the
reference's compiled kernel has (engine/eam.py:119-157, ADR-0043):

* cubic splines (scipy CubicSpline / PPoly, or arrays on a grid, which are
  splined here exactly as the reference does);
* r*phi splines (setfl pair tables, phi = s(r) / r);
* the analytic Zhou, Johnson and Wadley (2004) forms with the C2 quintic
  switch (``zhou_eam``).

A function is described by a spec tuple: ("spline", x, c),
("spline_over_r", x, c), ("zhou_density", p, r_c, width),
("zhou_pair", p, r_c, width), ("zhou_cross", pa, pb, chi, r_c, width) or
("zhou_embedding", p) -- the reference's ``_ak_spec`` tuples, which are also
accepted on callables built by the reference.
"""
import math

import numpy as np
import torch

from . import _lib
from .potential import DevicePotential, EvalResult, _set_last_ws, precision_code, workspace

ZHOU_KEYS = ("r_e", "f_e", "rho_e", "rho_s", "alpha", "beta", "A", "B", "kappa", "lambda",
             "Fn0", "Fn1", "Fn2", "Fn3", "F0", "F1", "F2", "F3", "eta", "F_e")
_NZ = len(ZHOU_KEYS)
_NCOL = 2 * _NZ + 3
_CODES = {"spline": 1, "spline_over_r": 2, "zhou_density": 3, "zhou_pair": 4, "zhou_cross": 5,
          "zhou_embedding": 6}


# ---- host evaluation of the function forms (numpy) -------------------------

def _switch(r, r_c, width):
    s = np.clip((r - (r_c - width)) / width, 0.0, 1.0)
    return 1.0 - s ** 3 * (10.0 - 15.0 * s + 6.0 * s * s), -30.0 * s * s * (1.0 - s) ** 2 / width


def _decay(r, re, pre, expo, shift):
    x = r / re
    e = pre * np.exp(-expo * (x - 1.0))
    u = x - shift
    den = 1.0 + u ** 20
    return e / den, (-expo * e / den - e * 20.0 * u ** 19 / den ** 2) / re


def zhou_density(r, p):
    return _decay(r, p["r_e"], p["f_e"], p["beta"], p["lambda"])


def zhou_pair(r, p):
    a, da = _decay(r, p["r_e"], p["A"], p["alpha"], p["kappa"])
    b, db = _decay(r, p["r_e"], p["B"], p["beta"], p["lambda"])
    return a - b, da - db


def zhou_embedding(rho, p):
    """F(rho), dF/drho of Zhou et al. (2004) eqs. (A6)-(A8)."""
    rho = np.asarray(rho, float)
    rn, re, rs, eta = 0.85 * p["rho_e"], p["rho_e"], p["rho_s"], p["eta"]
    F = np.empty_like(rho)
    dF = np.empty_like(rho)
    lo = rho < rn
    hi = rho >= 1.15 * re
    mid = ~(lo | hi)
    z = rho[lo] / rn - 1.0
    F[lo] = p["Fn0"] + p["Fn1"] * z + p["Fn2"] * z ** 2 + p["Fn3"] * z ** 3
    dF[lo] = (p["Fn1"] + 2 * p["Fn2"] * z + 3 * p["Fn3"] * z ** 2) / rn
    z = rho[mid] / re - 1.0
    F[mid] = p["F0"] + p["F1"] * z + p["F2"] * z ** 2 + p["F3"] * z ** 3
    dF[mid] = (p["F1"] + 2 * p["F2"] * z + 3 * p["F3"] * z ** 2) / re
    t = rho[hi] / rs
    lt = np.log(t)
    F[hi] = p["F_e"] * (1.0 - eta * lt) * t ** eta
    dF[hi] = -p["F_e"] * eta * eta * lt * t ** (eta - 1.0) / rs
    return F, dF


def _ppoly(x, c, r):
    from scipy.interpolate import PPoly
    pp = PPoly(np.asarray(c, float), np.asarray(x, float), extrapolate=True)
    return pp(r), pp.derivative()(r)


def eval_spec(spec, r):
    """Value and derivative of a spec'd function at r (host, numpy)."""
    r = np.asarray(r, float)
    kind = spec[0]
    if kind == "spline":
        return _ppoly(spec[1], spec[2], r)
    if kind == "spline_over_r":
        s, ds = _ppoly(spec[1], spec[2], r)
        return s / r, (ds * r - s) / (r * r)
    if kind == "zhou_embedding":
        return zhou_embedding(r, spec[1])
    if kind == "zhou_density":
        v, dv = zhou_density(r, spec[1])
        rc, w = spec[2], spec[3]
    elif kind == "zhou_pair":
        v, dv = zhou_pair(r, spec[1])
        rc, w = spec[2], spec[3]
    elif kind == "zhou_cross":
        pa, pb, k, rc, w = spec[1], spec[2], spec[3], spec[4], spec[5]
        fa, dfa = zhou_density(r, pa)
        fb, dfb = zhou_density(r, pb)
        ua, dua = zhou_pair(r, pa)
        ub, dub = zhou_pair(r, pb)
        q = fb / fa
        dq = (dfb * fa - fb * dfa) / fa ** 2
        v = 0.5 * k * (q * ua + ub / q)
        dv = 0.5 * k * (dq * ua + q * dua + dub / q - ub * dq / q ** 2)
    else:
        raise ValueError(f"EAM: unknown function form {kind!r}")
    S, dS = _switch(r, rc, w)
    return v * S, dv * S + v * dS


class SpecFunction:
    """A callable EAM function (value only, numpy) carrying its spec."""

    def __init__(self, spec):
        self.spec = spec
        self._ak_spec = spec

    def __call__(self, r):
        return eval_spec(self.spec, r)[0]

    def derivative_at(self, r):
        return eval_spec(self.spec, r)[1]


def spec_of(fn, grid=None):
    """Spec of an EAM function given in any accepted form, or ValueError."""
    if isinstance(fn, tuple) and len(fn) == 2 and callable(fn[0]) and callable(fn[1]):
        fn = fn[0]
    sp = getattr(fn, "_ak_spec", None) or getattr(fn, "spec", None)
    if sp is not None:
        return tuple(sp)
    try:
        from scipy.interpolate import PPoly
    except ImportError:  # pragma: no cover
        PPoly = None
    if PPoly is not None and isinstance(fn, PPoly) and fn.c.shape[0] == 4 and fn.extrapolate:
        return ("spline", np.asarray(fn.x, float), np.asarray(fn.c, float))
    if not callable(fn):
        from scipy.interpolate import CubicSpline
        if grid is None:
            raise ValueError("EAM: a tabulated function needs its grid")
        cs = CubicSpline(np.asarray(grid, float), np.asarray(fn, float))
        return ("spline", np.asarray(cs.x, float), np.asarray(cs.c, float))
    raise ValueError("EAM: a bare Python callable has no form the GPU kernels can evaluate; "
                     "give a spline (array / CubicSpline / PPoly) or a Zhou (2004) form.")


class EAMPotential(DevicePotential):
    """Alloy EAM (reference engine/eam.py:18-157 signature).

    F_table, rho_table : {species: fn} or one fn (legacy single species);
    phi_table          : {frozenset({a, b}): fn} or one fn; fn is a spline,
                         a tabulated array on rho_grid / r_grid, a (f, df)
                         pair or a spec'd callable.
    """

    def __init__(self, F_table, rho_table, phi_table, rho_grid=None, r_grid=None, r_cut=6.0,
                 species=None, precision="fp64"):
        super().__init__()
        self.precision = precision
        self.r_cut = float(r_cut)
        self.species = list(species) if species else None
        if not isinstance(F_table, dict):
            sp0 = self.species[0] if self.species else "__X__"
            self.species = [sp0]
            F_table = {sp0: F_table}
            rho_table = {sp0: rho_table}
            phi_table = {frozenset({sp0}): phi_table}
        elif not self.species:
            raise ValueError("EAMPotential: 'species' is required for the multi-species "
                             "(dict) parameter format.")
        self.F_spec = {s: spec_of(F_table[s], rho_grid) for s in F_table}
        self.rho_spec = {s: spec_of(rho_table[s], r_grid) for s in rho_table}
        self.phi_spec = {frozenset(k): spec_of(v, r_grid) for k, v in phi_table.items()}
        for s in self.species:
            if s not in self.F_spec or s not in self.rho_spec:
                raise ValueError(f"EAMPotential: no F / rho function for species {s!r}")
            for t in self.species:
                if frozenset({s, t}) not in self.phi_spec:
                    raise ValueError(f"EAMPotential: no phi function for pair {s}-{t}")
        self._F = {s: SpecFunction(v) for s, v in self.F_spec.items()}
        self._rho = {s: SpecFunction(v) for s, v in self.rho_spec.items()}
        self._phi = {k: SpecFunction(v) for k, v in self.phi_spec.items()}

    def function_table(self):
        """Flat tables as the device reads them (mbforce.h, mbf_eam_tables):
        codes, P (nf, 43), spline offsets / sizes / knots / coefficients, the
        function ids per species, and whether the fused Zhou path applies."""
        sp = self.species
        ns = len(sp)
        specs, rho_f, F_f = [], [], []
        for s in sp:
            rho_f.append(len(specs))
            specs.append(self.rho_spec[s])
        for s in sp:
            F_f.append(len(specs))
            specs.append(self.F_spec[s])
        phi_f = np.zeros((ns, ns), np.int32)
        for a in range(ns):
            for b in range(a, ns):
                phi_f[a, b] = phi_f[b, a] = len(specs)
                specs.append(self.phi_spec[frozenset({sp[a], sp[b]})])
        nf = len(specs)
        codes = np.zeros(nf, np.int32)
        P = np.zeros((nf, _NCOL))
        xo = np.zeros(nf, np.int32)
        nx = np.zeros(nf, np.int32)
        Xs, Cs, off = [], [], 0
        switches = set()
        for f, spec in enumerate(specs):
            kind = spec[0]
            codes[f] = _CODES[kind]
            if kind in ("spline", "spline_over_r"):
                x, c = np.asarray(spec[1], float), np.asarray(spec[2], float)
                if c.shape[0] != 4:
                    raise ValueError("EAM: only cubic splines are supported")
                xo[f], nx[f] = off, len(x)
                h = (x[-1] - x[0]) / (len(x) - 1) if len(x) > 1 else 0.0
                if len(x) > 2 and h > 0 and np.allclose(np.diff(x), h, rtol=1e-9, atol=0.0):
                    P[f, 0], P[f, 1], P[f, 2] = 1.0, x[0], 1.0 / h   # uniform knots
                Xs.append(x)
                cc = np.zeros((4, len(x)))
                cc[:, :len(x) - 1] = c
                Cs.append(cc)
                off += len(x)
            elif kind == "zhou_embedding":
                P[f, :_NZ] = [spec[1][k] for k in ZHOU_KEYS]
            else:
                P[f, :_NZ] = [spec[1][k] for k in ZHOU_KEYS]
                if kind == "zhou_cross":
                    P[f, _NZ:2 * _NZ] = [spec[2][k] for k in ZHOU_KEYS]
                    P[f, 2 * _NZ + 2] = float(spec[3])
                    rc, w = spec[4], spec[5]
                else:
                    rc, w = spec[2], spec[3]
                P[f, 2 * _NZ] = rc
                P[f, 2 * _NZ + 1] = w
                switches.add((float(rc), float(w)))
        X = np.concatenate(Xs) if Xs else np.zeros(1)
        C = np.concatenate(Cs, axis=1) if Cs else np.zeros((4, 1))
        # the fused kernels take each element's parameters from its density
        # row, so every pair row must carry the same element parameters
        fused = (ns <= 8 and len(switches) == 1
                 and all(codes[rho_f[a]] == 3 and codes[F_f[a]] == 6 for a in range(ns))
                 and all(codes[phi_f[a, b]] == (4 if a == b else 5)
                         for a in range(ns) for b in range(ns))
                 and all(np.array_equal(P[phi_f[a, a], :_NZ], P[rho_f[a], :_NZ]) for a in range(ns))
                 and all(np.array_equal(P[phi_f[a, b], :_NZ], P[rho_f[a], :_NZ])
                         and np.array_equal(P[phi_f[a, b], _NZ:2 * _NZ], P[rho_f[b], :_NZ])
                         for a in range(ns) for b in range(a + 1, ns)))
        return dict(codes=codes, P=P, xo=xo, nx=nx, X=X, C=np.ascontiguousarray(C),
                    rho_f=np.array(rho_f, np.int32), F_f=np.array(F_f, np.int32),
                    phi_f=phi_f, fused=fused)

    def _device_tables(self, device):
        t = self.function_table()
        keep = {k: torch.as_tensor(np.ascontiguousarray(v), device=device)
                for k, v in t.items() if k != "fused"}
        # host copies of P, rho_f, phi_f: with them a one- or two-element
        # Zhou table runs with its constants as kernel arguments
        host = {k: np.ascontiguousarray(t[k], dtype=np.float64 if k == "P" else np.int32)
                for k in ("P", "rho_f", "phi_f")}
        keep.update({k + "_host": v for k, v in host.items()})
        st = _lib.MbfEamTables(len(self.species), int(len(t["codes"])), int(t["X"].shape[0]),
                               *[_lib.ptr(keep[k]) for k in ("codes", "P", "xo", "nx", "X", "C",
                                                             "rho_f", "F_f", "phi_f")],
                               self.r_cut, 1 if t["fused"] else 0,
                               *[host[k].ctypes.data for k in ("P", "rho_f", "phi_f")])
        return (st, keep)

    sites_entry = "mbf_eam_eval_sites"
    lane_choices = (1, 2, 4, 8)
    # lanes of one atom's group in the force pass: 4 measured fastest on B200 (256k Cu-Ni)
    lanes_per_atom = 4

    # ---- the evaluation in two halves (a structure split over ranks) --------
    def _split_ws(self, batch, dlist, ws):
        nbytes = int(_lib.lib().mbf_eval_workspace_bytes(batch.n_atoms, dlist.n_slots, batch.n_chunks))
        if ws is None:
            return workspace(batch.device, nbytes)
        if ws.numel() < nbytes:
            raise ValueError(f"workspace of {ws.numel()} bytes, {nbytes} needed")
        return ws

    def embedding(self, batch, dlist, precision=None, ws=None):
        """The density and embedding passes: F'(rho-bar) of every atom of
        ``batch`` (a new device float64 tensor).  The values of atoms whose
        neighbourhood lies inside the batch are exact; the caller replaces
        the others' (a spatial split's halo atoms) by their owners' before
        forces_from_embedding, which must get the same ``ws``
        (mbf_eam_embedding)."""
        prec = precision_code(precision or self.precision)
        ws = self._split_ws(batch, dlist, ws)
        fp = torch.empty(batch.n_atoms, dtype=torch.float64, device=batch.device)
        L = _lib.lib()
        rc = L.mbf_eam_embedding(batch.mbf_system(), dlist.mbf_nlist(), self.tables(batch.device)[0],
                                 batch.reduce_plan(), prec, int(self.lanes_per_atom), _lib.ptr(ws), ws.numel(),
                                 _lib.ptr(fp), torch.cuda.current_stream(batch.device).cuda_stream)
        _lib.check(rc, "EAMPotential.embedding")
        _set_last_ws(self, ws)
        return fp

    def forces_from_embedding(self, batch, dlist, fprime, precision=None, ws=None, out=None):
        """The force pass and the gather with the given F'(rho-bar) per atom
        (mbf_eam_forces); ``ws`` the workspace of the embedding call.
        Returns EvalResult; the energy and virial are the sums of the
        records the batch's reduction plan covers."""
        prec = precision_code(precision or self.precision)
        ws = self._split_ws(batch, dlist, ws)
        dev = batch.device
        if out is None:
            out = EvalResult(torch.empty(batch.n_struct, dtype=torch.float64, device=dev),
                             torch.empty((batch.n_atoms, 3), dtype=torch.float64, device=dev),
                             torch.empty((batch.n_struct, 9), dtype=torch.float64, device=dev))
        fp = fprime.to(device=dev, dtype=torch.float64).contiguous()
        L = _lib.lib()
        rc = L.mbf_eam_forces(batch.mbf_system(), dlist.mbf_nlist(), self.tables(dev)[0], batch.reduce_plan(), prec,
                              int(self.lanes_per_atom), _lib.ptr(ws), ws.numel(), _lib.ptr(fp),
                              _lib.ptr(out.forces), _lib.ptr(out.energy), _lib.ptr(out.virial),
                              torch.cuda.current_stream(dev).cuda_stream)
        _lib.check(rc, "EAMPotential.forces_from_embedding")
        _set_last_ws(self, ws)
        return out

    def _call(self, L, sysd, nld, tabs, plan, prec, ws, nbytes, forces, energy, virial, stream):
        return L.mbf_eam_eval(sysd, nld, tabs[0], plan, prec, int(self.lanes_per_atom), ws, nbytes,
                              forces, energy, virial, stream)


# ---- Zhou, Johnson & Wadley (2004) -------------------------------------------

def continuous(p):
    """Element parameters with Fn0, Fn1, F0, F_e re-derived so that F and
    dF/drho are continuous at rho_n = 0.85 rho_e and rho_0 = 1.15 rho_e
    (reference engine/eam_zhou.py:47-64)."""
    q = {k: float(v) for k, v in p.items()}
    re, rs, eta = q["rho_e"], q["rho_s"], q["eta"]
    F1, F2, F3 = q["F1"], q["F2"], q["F3"]
    y, x = 0.15, -0.15
    t0 = 1.15 * re / rs
    slope0 = (F1 + 2 * F2 * y + 3 * F3 * y * y) / re
    dg = -eta * eta * math.log(t0) * t0 ** (eta - 1.0) / rs
    if dg == 0.0:
        raise ValueError("Zhou EAM: rho_0 = rho_s (or eta = 0) leaves F_e undetermined")
    q["F_e"] = slope0 / dg
    q["F0"] = q["F_e"] * (1 - eta * math.log(t0)) * t0 ** eta - (F1 * y + F2 * y * y + F3 * y ** 3)
    q["Fn0"] = q["F0"] + F1 * x + F2 * x * x + F3 * x ** 3
    q["Fn1"] = 0.85 * (F1 + 2 * F2 * x + 3 * F3 * x * x)
    return q


def zhou_cutoff(p, tol=1e-6):
    """Distance beyond which |phi_aa| < tol max(A, B) and f < tol f_e, on the
    grid linspace(r_e, 5 r_e, 40001) (reference engine/eam_zhou.py:117-125)."""
    r = np.linspace(p["r_e"], 5.0 * p["r_e"], 40001)
    ok = ((np.abs(zhou_pair(r, p)[0]) < tol * max(p["A"], p["B"]))
          & (zhou_density(r, p)[0] < tol * p["f_e"]))
    bad = np.nonzero(~ok)[0]
    if len(bad) == len(r):
        raise ValueError("Zhou EAM: functions do not decay within 5 r_e")
    return float(r[bad[-1] + 1]) if len(bad) else float(r[0])


def zhou_eam(elements, species, r_cut=None, chi=None, width=0.5, tol=1e-6,
             enforce_continuity=True, precision="fp64"):
    """EAMPotential of Zhou (2004) element parameters (reference
    engine/eam_zhou.py:128-207): switched density and pair functions, the
    cross pair 1/2 k (f_b/f_a phi_aa + f_a/f_b phi_bb) formed from unswitched
    functions, r_cut by default the largest ``zhou_cutoff``."""
    KEYS = ZHOU_KEYS
    species = list(species)
    P = {}
    for s in species:
        if s not in elements:
            raise ValueError(f"Zhou EAM: no parameters for '{s}'")
        missing = [k for k in KEYS if k not in elements[s]]
        if missing:
            raise ValueError(f"Zhou EAM: '{s}' lacks {missing}")
        P[s] = continuous(elements[s]) if enforce_continuity else \
            {k: float(v) for k, v in elements[s].items()}
    if r_cut is None:
        r_cut = max(zhou_cutoff(P[s], tol) for s in species)
    chi = chi or {}

    def cfac(a, b):
        return float(chi.get(f"{a}-{b}", chi.get(f"{b}-{a}", 1.0))) if a != b else 1.0

    F_tab = {s: SpecFunction(("zhou_embedding", P[s])) for s in species}
    rho_tab = {s: SpecFunction(("zhou_density", P[s], r_cut, width)) for s in species}
    phi_tab = {}
    for i, a in enumerate(species):
        for b in species[i:]:
            spec = (("zhou_pair", P[a], r_cut, width) if a == b
                    else ("zhou_cross", P[a], P[b], cfac(a, b), r_cut, width))
            phi_tab[frozenset((a, b))] = SpecFunction(spec)
    pot = EAMPotential(F_tab, rho_tab, phi_tab, r_cut=r_cut, species=species,
                       precision=precision)
    pot.zhou_params = P
    pot.zhou_chi = {f"{a}-{b}": cfac(a, b) for i, a in enumerate(species) for b in species[i + 1:]}
    return pot


def tabulate(pot, n_r=2000, n_rho=2000, rho_max=None, precision=None):
    """The setfl form of an EAMPotential: F on a uniform rho grid, rho and
    r*phi on a uniform r grid up to r_cut, each a cubic spline (scipy
    CubicSpline) -- what writing the potential to an eam/alloy file and
    reading it back with read_setfl gives (reference engine/eam_zhou.py:
    258-315).  rho_max defaults to twice the largest rho-bar of a perfect
    lattice's worth of neighbours (50 x the largest rho(r) on the grid)."""
    from scipy.interpolate import CubicSpline
    r_g = np.linspace(0.0, pot.r_cut, n_r)
    r_pos = np.where(r_g > 0.0, r_g, r_g[1])
    if rho_max is None:
        rho_max = 50.0 * max(float(np.max(pot._rho[s](r_pos))) for s in pot.species)
    rho_g = np.linspace(0.0, rho_max, n_rho)

    def spline(x, y, kind):
        cs = CubicSpline(x, y)
        return SpecFunction((kind, np.asarray(cs.x, float), np.asarray(cs.c, float)))

    F_tab = {s: spline(rho_g, pot._F[s](rho_g), "spline") for s in pot.species}
    rho_tab = {s: spline(r_g, pot._rho[s](r_pos), "spline") for s in pot.species}
    phi_tab = {k: spline(r_g, r_g * f(r_pos), "spline_over_r") for k, f in pot._phi.items()}
    return EAMPotential(F_tab, rho_tab, phi_tab, r_cut=pot.r_cut, species=pot.species,
                        precision=precision or pot.precision)


def read_setfl(path, species=None, precision="fp64"):
    """A LAMMPS eam/alloy (setfl) file as an EAMPotential: every table a
    cubic spline (scipy CubicSpline), pair tables as r*phi
    (reference engine/eam_zhou.py:258-315)."""
    from scipy.interpolate import CubicSpline
    with open(path) as fh:
        lines = fh.read().splitlines()
    head = lines[3].split()
    n_el = int(head[0])
    names = head[1:1 + n_el]
    n_rho, drho, n_r, dr, r_cut = lines[4].split()[:5]
    n_rho, n_r = int(n_rho), int(n_r)
    drho, dr, r_cut = float(drho), float(dr), float(r_cut)
    pos = 5
    tables = {}

    def take(n):
        nonlocal pos
        out = []
        while len(out) < n:
            out.extend(float(v) for v in lines[pos].split())
            pos += 1
        return np.array(out[:n])

    for s in names:
        pos += 1
        tables[("F", s)] = take(n_rho)
        tables[("rho", s)] = take(n_r)
    for i, a in enumerate(names):
        for b in names[:i + 1]:
            tables[("rphi", a, b)] = take(n_r)
    rho_g = np.arange(n_rho) * drho
    r_g = np.arange(n_r) * dr

    def spline(x, y, kind):
        cs = CubicSpline(x, y)
        return SpecFunction((kind, np.asarray(cs.x, float), np.asarray(cs.c, float)))

    F_tab = {s: spline(rho_g, tables[("F", s)], "spline") for s in names}
    rho_tab = {s: spline(r_g, tables[("rho", s)], "spline") for s in names}
    phi_tab = {}
    for i, a in enumerate(names):
        for b in names[:i + 1]:
            phi_tab[frozenset((a, b))] = spline(r_g, tables[("rphi", a, b)], "spline_over_r")
    return EAMPotential(F_tab, rho_tab, phi_tab, r_cut=r_cut,
                        species=list(species) if species else names, precision=precision)
