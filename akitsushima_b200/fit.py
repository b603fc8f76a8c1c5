"""Tersoff and Zhou-EAM fitting on the GPU: the reference's weighted E/F/S
loss and its exact gradient with respect to the parameters.

The reference evaluates its fit loss structure by structure on the CPU
(fitting/loss.py:51-260) and gets gradients by forward differences, one
full loss evaluation per parameter (fitting/driver.py:802-816).  Here the
whole training set is one batch: one device neighbour list, one evaluation
launch sequence (mbf_tersoff_eval, float64), the loss in torch, and the
gradient from one adjoint call (mbf_tersoff_adjoint) behind a
torch.autograd.Function -- the vector-Jacobian product of (E, F, virial)
with respect to the dense parameter tables, which torch chains back
through the parameter decoding (log variables, Tersoff-1989 mixing rules,
tied records) to the optimisation vector x.

The Zhou (2004) EAM fit is the same construction over the analytic EAM
table: the rows P (nf, 43) built differentiably from the element
parameters (continuity of F included), one mbf_eam_eval and one
mbf_eam_adjoint call.

Parameter sets mirror the reference's (fitting/parameter_sets.py:1035-1400):
the same variables, names, x0, bounds, log-space keys and decode(); each
also builds its device tables differentiably in x.
"""
import math

import numpy as np
import torch

from . import _lib
from .force_fn import PotentialEngine
from .neighbourlist import DeviceNeighbourList
from .system import Batch, default_device, replicate_thin, species_ids
from .eam import ZHOU_KEYS, continuous, zhou_cutoff, zhou_eam
from .tersoff import TERSOFF1989_ELEMENT_KEYS, TersoffPotential, tersoff1989_to_triplets

_TB_KEYS = (("A", 0.0), ("B", 0.0), ("lambda1", 0.0), ("lambda2", 0.0), ("R", 1.0), ("D", 1.0),
            ("beta", 0.0), ("n", 1.0))


def _scalar(v, like):
    if torch.is_tensor(v):
        return v.to(dtype=torch.float64, device=like.device).reshape(())
    return torch.tensor(float(v), dtype=torch.float64, device=like.device)


def tables_from_records(records, species, device):
    """Dense tables (tb (ns*ns, 10), tri (ns^3, 8), float64 torch) of a
    {(i, j, k): record} table, laid out as TersoffPotential.host_tables
    builds them (engine/tersoff.py:1606-1653); entries given as 0-d tensors
    keep their autograd history."""
    ref = torch.zeros((), dtype=torch.float64, device=device)
    tb_rows, tri_rows = [], []
    for a in species:
        for b in species:
            rec = records.get((a, b, b))
            if rec is None:
                vals = [0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0, 1.0, 0.0]
            else:
                vals = [1.0] + [rec.get(k, d) for k, d in _TB_KEYS] + [0.0]
            tb_rows.append(torch.stack([_scalar(v, ref) for v in vals]))
    for a in species:
        for b in species:
            for c in species:
                rec = records.get((a, b, c))
                if rec is None:
                    vals = [0.0, 0.0, 1.0, 0.0, 0.0, 3.0, 1.0, 0.0]
                else:
                    vals = [1.0, rec["c"], rec["d"], rec["h"], rec.get("lambda3", 0.0), rec.get("m", 3.0),
                            rec.get("gamma", 1.0), 0.0]
                tri_rows.append(torch.stack([_scalar(v, ref) for v in vals]))
    return torch.stack(tb_rows).contiguous(), torch.stack(tri_rows).contiguous()


def table_cutoff(tb):
    """Largest R + D over the valid pair records (the list radius)."""
    t = tb.detach().cpu().numpy() if torch.is_tensor(tb) else np.asarray(tb)
    valid = t[:, 0] != 0.0
    return float(np.max(t[valid, 5] + t[valid, 6])) if valid.any() else 0.0


# ---- parameter sets ------------------------------------------------------------

class _Variables:
    """x <-> named variables (fitting/parameter_sets.py:1035-1065)."""

    _LOG_KEYS = frozenset()
    _BOUNDS = {}

    @property
    def x0(self):
        return self._x0.copy()

    @property
    def bounds(self):
        return self._bounds

    @property
    def variable_names(self):
        return [name for name, _, _ in self.variables]

    def _setup_vector(self, initial_values, owner):
        x0, bounds = [], []
        for (name, key, _), v in zip(self.variables, initial_values):
            lo, hi = self._BOUNDS[key]
            if not lo <= v <= hi:
                raise ValueError(f"{owner}: initial {name} = {v} lies outside its search range [{lo}, {hi}].")
            if key in self._LOG_KEYS:
                x0.append(math.log(v))
                bounds.append((math.log(lo), math.log(hi)))
            else:
                x0.append(v)
                bounds.append((lo, hi))
        self._x0 = np.array(x0)
        self._bounds = bounds

    def _value(self, key, xi):
        if torch.is_tensor(xi):
            return torch.exp(xi) if key in self._LOG_KEYS else xi
        return float(np.exp(xi)) if key in self._LOG_KEYS else float(xi)

    def build_engine(self, params):
        return PotentialEngine().add(TersoffPotential(params["tersoff"], species=self.species))

    def _vals_np(self, X):
        """Variable values of the rows of X (B, n_var), exp of the log keys."""
        logm = np.array([key in self._LOG_KEYS for _, key, _ in self.variables], bool)
        V = np.array(X, dtype=X.dtype, copy=True)
        V[:, logm] = np.exp(X[:, logm])
        return V

    def tables_np(self, x):
        """The device tables of decode(x) as float64 numpy arrays."""
        return [t[0].real.copy() for t in self._tables_np(np.asarray(x, float)[None].astype(complex))]

    def table_jacobian(self, x):
        """(tables at x, d tables / dx): every variable's derivative by the
        complex step (Squire and Trapp, SIAM Rev. 40, 110 (1998)) in one
        vectorised evaluation -- exact to rounding, as the table maps are
        analytic.  Jacobians have shape (n_var,) + table shape."""
        x = np.asarray(x, float)
        n = len(x)
        h = 1e-30
        X = np.repeat(x[None].astype(complex), n + 1, axis=0)
        X[1:] += 1j * h * np.eye(n)
        outs = self._tables_np(X)
        return [o[0].real.copy() for o in outs], [o[1:].imag / h for o in outs]


def _nested(records):
    if isinstance(records, dict) and all(isinstance(k, tuple) for k in records):
        return {tuple(k): dict(v) for k, v in records.items()}
    out = {}
    for rec in records:
        rec = dict(rec)
        out[(rec.pop("i"), rec.pop("j"), rec.pop("k"))] = rec
    return out


class MultiSpeciesTersoffParameterSet(_Variables):
    """The (i, j, k) record table as variables (reference
    fitting/parameter_sets.py:1068-1203): pair keys A, B, lambda1, lambda2
    (R, D) one variable per unordered pair, written to (i, j, j) and
    (j, i, i); beta, n one per diagonal record; c, d, h (lambda3, gamma) one
    per record, or per centre element with tie="centre".  Fixed by default:
    R, D, m, gamma, lambda3, beta, n."""

    _DEFAULT_FIX = ("R", "D", "m", "gamma", "lambda3", "beta", "n")
    _DEFAULT_FIT = ("A", "B", "lambda1", "lambda2", "c", "d", "h")
    _PAIR_KEYS = ("A", "B", "lambda1", "lambda2", "R", "D")
    _BOND_KEYS = ("beta", "n")
    _ANGLE_KEYS = ("c", "d", "h", "lambda3", "gamma")
    _LOG_KEYS = frozenset({"A", "B", "lambda1", "lambda2", "beta", "n", "c", "d", "gamma"})
    _BOUNDS = {"A": (1.0, 1e5), "B": (0.1, 1e4), "lambda1": (0.5, 10.0), "lambda2": (0.1, 8.0),
               "beta": (1e-10, 10.0), "n": (0.05, 10.0), "c": (1e-3, 1e7), "d": (1e-2, 1e4),
               "h": (-1.0, 1.0), "lambda3": (0.0, 5.0), "gamma": (1e-3, 100.0), "R": (1.0, 5.0),
               "D": (0.02, 0.5)}

    def __init__(self, initial_records, species, fix_params=None, fit_keys=None, tie="record"):
        if tie not in ("record", "centre"):
            raise ValueError("MultiSpeciesTersoffParameterSet: tie must be 'record' or 'centre'")
        self.species = list(species)
        self.records = _nested(initial_records)
        for sp in {e for t in self.records for e in t}:
            if sp not in self.species:
                raise ValueError(f"Tersoff record element '{sp}' is not among the species {self.species}")
        fixed = set(self._DEFAULT_FIX) | set(fix_params or ())
        keys = list(fit_keys) if fit_keys else list(self._DEFAULT_FIT)
        self.fit_keys = [k for k in keys if k not in fixed]
        unknown = [k for k in self.fit_keys if k not in self._BOUNDS]
        if unknown:
            raise ValueError(f"MultiSpeciesTersoffParameterSet: unknown fit key(s) {unknown}")
        self._check_pairs()
        self.variables = []
        seen_pairs, seen_centres = set(), set()
        for (i, j, k) in self.records:
            if j == k:
                pair = frozenset((i, j))
                if pair not in seen_pairs:
                    seen_pairs.add(pair)
                    tw = [(i, j, j)] + ([(j, i, i)] if i != j else [])
                    for key in self.fit_keys:
                        if key in self._PAIR_KEYS:
                            self.variables.append((f"{i}-{j}:{key}", key, [(t, key) for t in tw]))
                for key in self.fit_keys:
                    if key in self._BOND_KEYS:
                        self.variables.append((f"{i};{j}:{key}", key, [((i, j, j), key)]))
            for key in self.fit_keys:
                if key not in self._ANGLE_KEYS:
                    continue
                if tie == "centre":
                    if (i, key) in seen_centres:
                        continue
                    seen_centres.add((i, key))
                    tg = [(t, key) for t in self.records if t[0] == i]
                    self.variables.append((f"{i};*:{key}", key, tg))
                else:
                    self.variables.append((f"{i};{j},{k}:{key}", key, [((i, j, k), key)]))
        init = []
        for name, key, targets in self.variables:
            try:
                init.append(float(np.mean([self.records[t][kk] for t, kk in targets])))
            except KeyError:
                raise ValueError(f"MultiSpeciesTersoffParameterSet: a record of {name} has no '{key}'") from None
        self._setup_vector(init, "MultiSpeciesTersoffParameterSet")

    def _check_pairs(self):
        for (i, j, k), rec in self.records.items():
            if j != k or i == j:
                continue
            twin = self.records.get((j, i, i))
            if twin is None:
                raise ValueError(f"Tersoff record ({i},{j},{j}) has no partner ({j},{i},{i}); the {i}-{j} pair "
                                 "is read from whichever belongs to the lower-indexed atom, so both are required.")
            for key in self._PAIR_KEYS:
                a, b = rec.get(key), twin.get(key)
                if (a is None) != (b is None) or (a is not None and not np.isclose(a, b, rtol=1e-12, atol=0.0)):
                    raise ValueError(f"Tersoff records ({i},{j},{j}) and ({j},{i},{i}) disagree on '{key}' "
                                     f"({a} vs {b}); the engine would read one or the other depending on atom "
                                     "order.")

    def _decode(self, x):
        out = {t: dict(p) for t, p in self.records.items()}
        for xi, (_, key, targets) in zip(x, self.variables):
            v = self._value(key, xi)
            for triple, kk in targets:
                out[triple][kk] = v
        return {"tersoff": out}

    def decode(self, x):
        """{'tersoff': {(i, j, k): full parameter dict}} (floats)."""
        return self._decode(np.asarray(x, float))

    def decode_torch(self, x):
        """The same with 0-d tensor entries carrying x's autograd history."""
        return self._decode(list(x.unbind(0)))

    _TB_COL = {"A": 1, "B": 2, "lambda1": 3, "lambda2": 4, "R": 5, "D": 6, "beta": 7, "n": 8}
    _TRI_COL = {"c": 1, "d": 2, "h": 3, "lambda3": 4, "m": 5, "gamma": 6}

    def tables_torch(self, x):
        """(tb, tri) of decode(x) built directly: the tables of the initial
        records with every variable's targets overwritten -- a few tensor
        operations, differentiable in x."""
        if not hasattr(self, "_plan"):
            tb0, tri0 = tables_from_records(self.records, self.species, "cpu")
            idx = {s: a for a, s in enumerate(self.species)}
            ns = len(self.species)
            tbp, trip = ([], [], []), ([], [], [])
            for v, (_, key, targets) in enumerate(self.variables):
                for (i, j, k), kk in targets:
                    if kk in self._TB_COL:     # pair and bond keys live on diagonal records
                        tbp[0].append(v)
                        tbp[1].append(idx[i] * ns + idx[j])
                        tbp[2].append(self._TB_COL[kk])
                    else:
                        trip[0].append(v)
                        trip[1].append((idx[i] * ns + idx[j]) * ns + idx[k])
                        trip[2].append(self._TRI_COL[kk])
            logm = torch.tensor([key in self._LOG_KEYS for _, key, _ in self.variables])
            self._plan = (tb0, tri0, [torch.tensor(a, dtype=torch.long) for a in tbp],
                          [torch.tensor(a, dtype=torch.long) for a in trip], logm)
        tb0, tri0, tbp, trip, logm = self._plan
        vals = torch.where(logm, torch.exp(x), x)
        tb = tb0.clone().index_put((tbp[1], tbp[2]), vals[tbp[0]])
        tri = tri0.clone().index_put((trip[1], trip[2]), vals[trip[0]])
        return tb, tri

    def _tables_np(self, X):
        """tables_torch over the rows of X (B, n_var): (tb (B, ns^2, 10),
        tri (B, ns^3, 8)) in X's dtype."""
        if not hasattr(self, "_plan"):
            self.tables_torch(torch.as_tensor(self.x0))
        tb0, tri0, tbp, trip, _ = self._plan
        V = self._vals_np(X)
        B = X.shape[0]
        tb = np.repeat(tb0.numpy()[None].astype(X.dtype), B, axis=0)
        tri = np.repeat(tri0.numpy()[None].astype(X.dtype), B, axis=0)
        tb[:, tbp[1].numpy(), tbp[2].numpy()] = V[:, tbp[0].numpy()]
        tri[:, trip[1].numpy(), trip[2].numpy()] = V[:, trip[0].numpy()]
        return tb, tri


def _mix_1989(el, chi, species, omega):
    """Tersoff (1989) mixing rules (PRB 39, 5566, eqs. 1a-1e) on values that
    may be 0-d tensors: the expansion of tersoff1989_to_triplets written
    with torch operations so it can be differentiated."""
    def sq(v):
        return torch.sqrt(v) if torch.is_tensor(v) else math.sqrt(v)

    def pair(table, a, b, default):
        for k in (f"{a}-{b}", f"{b}-{a}"):
            if k in table:
                return table[k]
        return default

    out = {}
    for i in species:
        pi = el[i]
        for j in species:
            pj = el[j]
            x = 1.0 if i == j else pair(chi, i, j, None)
            r_ij = sq(pi["R"] * pj["R"])
            s_ij = sq(pi["S"] * pj["S"])
            for k in species:
                rec = {"c": pi["c"], "d": pi["d"], "h": pi["h"], "lambda3": 0.0, "m": 3.0,
                       "gamma": float(pair(omega, i, k, 1.0))}
                if j == k:
                    rec.update(A=sq(pi["A"] * pj["A"]), B=x * sq(pi["B"] * pj["B"]),
                               lambda1=0.5 * (pi["lambda"] + pj["lambda"]), lambda2=0.5 * (pi["mu"] + pj["mu"]),
                               R=0.5 * (r_ij + s_ij), D=0.5 * (s_ij - r_ij), beta=pi["beta"], n=pi["n"])
                out[(i, j, k)] = rec
    return out


class Tersoff1989ParameterSet(_Variables):
    """Per-element Tersoff (1989) parameters and one chi per pair of
    distinct elements (reference fitting/parameter_sets.py:1206-1296).
    Default variables: A, B, lambda, mu, c, d, h of every element and every
    chi; R, S, beta, n fixed."""

    _DEFAULT_FIX = ("R", "S", "beta", "n")
    _DEFAULT_FIT = ("A", "B", "lambda", "mu", "c", "d", "h", "chi")
    _LOG_KEYS = frozenset({"A", "B", "lambda", "mu", "beta", "n", "c", "d", "chi", "R", "S"})
    _BOUNDS = {"A": (1.0, 1e5), "B": (0.1, 1e4), "lambda": (0.5, 10.0), "mu": (0.1, 8.0),
               "beta": (1e-10, 10.0), "n": (0.05, 10.0), "c": (1e-3, 1e7), "d": (1e-2, 1e4),
               "h": (-1.0, 1.0), "chi": (0.3, 3.0), "R": (1.0, 5.0), "S": (1.0, 5.5)}

    def __init__(self, elements, chi, species, fix_params=None, fit_keys=None, omega=None):
        self.species = list(species)
        self.elements = {s: {k: float(v) for k, v in elements[s].items()} for s in self.species if s in elements}
        self.omega = dict(omega or {})
        self.chi = {}
        for a_i, a in enumerate(self.species):
            for b in self.species[a_i + 1:]:
                v = chi.get(f"{a}-{b}", chi.get(f"{b}-{a}"))
                if v is None:
                    raise ValueError(f"Tersoff1989ParameterSet: chi for {a}-{b} is not given")
                self.chi[f"{a}-{b}"] = float(v)
        tersoff1989_to_triplets(self.elements, self.chi, self.species, self.omega)
        fixed = set(self._DEFAULT_FIX) | set(fix_params or ())
        keys = list(fit_keys) if fit_keys else list(self._DEFAULT_FIT)
        self.fit_keys = [k for k in keys if k not in fixed]
        unknown = [k for k in self.fit_keys if k not in TERSOFF1989_ELEMENT_KEYS and k != "chi"]
        if unknown:
            raise ValueError(f"Tersoff1989ParameterSet: unknown fit key(s) {unknown}")
        self.variables, init = [], []
        for s in self.species:
            for key in self.fit_keys:
                if key != "chi":
                    self.variables.append((f"{s}:{key}", key, (s, key)))
                    init.append(self.elements[s][key])
        if "chi" in self.fit_keys:
            for pair, v in self.chi.items():
                self.variables.append((f"chi:{pair}", "chi", pair))
                init.append(v)
        self._setup_vector(init, "Tersoff1989ParameterSet")

    def _decode(self, x, torch_mode):
        el = {s: dict(p) for s, p in self.elements.items()}
        chi = dict(self.chi)
        for xi, (_, key, target) in zip(x, self.variables):
            v = self._value(key, xi)
            if key == "chi":
                chi[target] = v
            else:
                el[target[0]][key] = v
        table = _mix_1989(el, chi, self.species, self.omega) if torch_mode else \
            tersoff1989_to_triplets(el, chi, self.species, self.omega)
        return {"tersoff": table, "tersoff1989": {"elements": el, "chi": chi, "omega": dict(self.omega)}}

    def decode(self, x):
        """{'tersoff': (i, j, k) table, 'tersoff1989': {elements, chi, omega}}."""
        return self._decode(np.asarray(x, float), False)

    def decode_torch(self, x):
        return self._decode(list(x.unbind(0)), True)

    _EL_KEYS = ("A", "B", "lambda", "mu", "beta", "n", "c", "d", "h", "R", "S")

    def tables_torch(self, x):
        """(tb, tri) of decode(x) from the mixing rules applied to whole
        per-element vectors (PRB 39, 5566, eqs. 1a-1e; the same expressions
        as tersoff1989_to_triplets), differentiable in x."""
        ns = len(self.species)
        if not hasattr(self, "_plan"):
            el0 = torch.tensor([[self.elements[s][k] for k in self._EL_KEYS] for s in self.species],
                               dtype=torch.float64)
            chi0 = torch.ones((ns, ns), dtype=torch.float64)
            for a, sa in enumerate(self.species):
                for b, sb in enumerate(self.species):
                    if a != b:
                        chi0[a, b] = self.chi.get(f"{sa}-{sb}", self.chi.get(f"{sb}-{sa}"))
            om = torch.ones((ns, ns), dtype=torch.float64)
            for a, sa in enumerate(self.species):
                for b, sb in enumerate(self.species):
                    om[a, b] = float(self.omega.get(f"{sa}-{sb}", self.omega.get(f"{sb}-{sa}", 1.0)))
            ev, er, ec, cv, cr = [], [], [], [], []
            idx = {s: a for a, s in enumerate(self.species)}
            for v, (_, key, target) in enumerate(self.variables):
                if key == "chi":
                    a, b = (idx[t] for t in target.split("-"))
                    cv += [v, v]
                    cr += [(a, b), (b, a)]
                else:
                    ev.append(v)
                    er.append(idx[target[0]])
                    ec.append(self._EL_KEYS.index(key))
            logm = torch.tensor([key in self._LOG_KEYS for _, key, _ in self.variables])
            self._plan = (el0, chi0, om, torch.tensor(ev, dtype=torch.long), torch.tensor(er, dtype=torch.long),
                          torch.tensor(ec, dtype=torch.long), torch.tensor(cv, dtype=torch.long),
                          torch.tensor([c[0] for c in cr], dtype=torch.long),
                          torch.tensor([c[1] for c in cr], dtype=torch.long), logm)
        el0, chi0, om, ev, er, ec, cv, c0, c1, logm = self._plan
        vals = torch.where(logm, torch.exp(x), x)
        el = el0.clone().index_put((er, ec), vals[ev]) if len(ev) else el0
        chi = chi0.clone().index_put((c0, c1), vals[cv]) if len(cv) else chi0
        A, B, lam, mu, beta, n, c, d, h, R, S = el.unbind(1)
        r = torch.sqrt(R[:, None] * R[None, :])
        sx = torch.sqrt(S[:, None] * S[None, :])
        one = torch.ones((ns, ns), dtype=torch.float64)
        tb = torch.stack([one, torch.sqrt(A[:, None] * A[None, :]), chi * torch.sqrt(B[:, None] * B[None, :]),
                          0.5 * (lam[:, None] + lam[None, :]), 0.5 * (mu[:, None] + mu[None, :]),
                          0.5 * (r + sx), 0.5 * (sx - r), beta[:, None] * one, n[:, None] * one, 0.0 * one],
                         dim=-1).reshape(ns * ns, 10)
        one3 = torch.ones((ns, ns, ns), dtype=torch.float64)
        tri = torch.stack([one3, c[:, None, None] * one3, d[:, None, None] * one3, h[:, None, None] * one3,
                           0.0 * one3, 3.0 * one3, om[:, None, :] * one3, 0.0 * one3], dim=-1).reshape(ns ** 3, 8)
        return tb, tri

    def _tables_np(self, X):
        """tables_torch over the rows of X (B, n_var), in X's dtype."""
        ns = len(self.species)
        if not hasattr(self, "_plan"):
            self.tables_torch(torch.as_tensor(self.x0))
        el0, chi0, om, ev, er, ec, cv, c0, c1, _ = [t.numpy() if torch.is_tensor(t) else t for t in self._plan]
        V = self._vals_np(X)
        B = X.shape[0]
        el = np.repeat(el0[None].astype(X.dtype), B, axis=0)
        chi = np.repeat(chi0[None].astype(X.dtype), B, axis=0)
        if len(ev):
            el[:, er, ec] = V[:, ev]
        if len(cv):
            chi[:, c0, c1] = V[:, cv]
        A, Bb, lam, mu, beta, n, c, d, h, R, S = np.moveaxis(el, -1, 0)
        r = np.sqrt(R[:, :, None] * R[:, None, :])
        sx = np.sqrt(S[:, :, None] * S[:, None, :])
        one = np.ones((B, ns, ns), X.dtype)
        tb = np.stack([one, np.sqrt(A[:, :, None] * A[:, None, :]), chi * np.sqrt(Bb[:, :, None] * Bb[:, None, :]),
                       0.5 * (lam[:, :, None] + lam[:, None, :]), 0.5 * (mu[:, :, None] + mu[:, None, :]),
                       0.5 * (r + sx), 0.5 * (sx - r), beta[:, :, None] * one, n[:, :, None] * one, 0.0 * one],
                      axis=-1).reshape(B, ns * ns, 10)
        one3 = np.ones((B, ns, ns, ns), X.dtype)
        tri = np.stack([one3, c[:, :, None, None] * one3, d[:, :, None, None] * one3, h[:, :, None, None] * one3,
                        0.0 * one3, 3.0 * one3, om[None, :, None, :] * one3, 0.0 * one3],
                       axis=-1).reshape(B, ns ** 3, 8)
        return tb, tri


# ---- Zhou (2004) EAM -------------------------------------------------------------

_ZCOL = {k: c for c, k in enumerate(ZHOU_KEYS)}
ZHOU_DERIVED = ("Fn0", "Fn1", "F0", "F_e")


def continuous_torch(el):
    """continuous() (F and dF/drho continuous at rho_n = 0.85 rho_e and
    rho_0 = 1.15 rho_e, engine/eam_zhou.py:47-64) on every row of a (ns, 20)
    tensor of element parameters in ZHOU_KEYS order, differentiable."""
    c = _ZCOL
    re, rs, eta = el[:, c["rho_e"]], el[:, c["rho_s"]], el[:, c["eta"]]
    F1, F2, F3 = el[:, c["F1"]], el[:, c["F2"]], el[:, c["F3"]]
    y, x = 0.15, -0.15
    t0 = 1.15 * re / rs
    lt0 = torch.log(t0)
    slope0 = (F1 + 2 * F2 * y + 3 * F3 * y * y) / re
    dg = -eta * eta * lt0 * t0 ** (eta - 1.0) / rs
    if bool((dg == 0.0).any()):
        raise ValueError("Zhou EAM: rho_0 = rho_s (or eta = 0) leaves F_e undetermined")
    Fe = slope0 / dg
    F0 = Fe * (1 - eta * lt0) * t0 ** eta - (F1 * y + F2 * y * y + F3 * y ** 3)
    cols = list(el.unbind(1))
    cols[c["F_e"]] = Fe
    cols[c["F0"]] = F0
    cols[c["Fn0"]] = F0 + F1 * x + F2 * x * x + F3 * x ** 3
    cols[c["Fn1"]] = 0.85 * (F1 + 2 * F2 * x + 3 * F3 * x * x)
    return torch.stack(cols, 1)


def zhou_table_torch(el, chi, r_cut, width=0.5):
    """The rows P (nf, 43) of zhou_eam's function table (EAMPotential.
    function_table: a density row per species, an embedding row per
    species, a pair row per a <= b) from element rows el (ns, 20, ZHOU_KEYS
    order, already continuous) and the cross factors chi (ns, ns);
    differentiable in both."""
    ns = el.shape[0]
    f64 = dict(dtype=el.dtype, device=el.device)
    sw = torch.tensor([float(r_cut), float(width)], **f64)
    z20 = torch.zeros(20, **f64)
    z1 = torch.zeros(1, **f64)
    rows = [torch.cat([el[a], z20, sw, z1]) for a in range(ns)]
    rows += [torch.cat([el[a], z20, torch.zeros(3, **f64)]) for a in range(ns)]
    for a in range(ns):
        for b in range(a, ns):
            rows.append(torch.cat([el[a], z20, sw, z1]) if a == b else
                        torch.cat([el[a], el[b], sw, chi[a, b].reshape(1)]))
    return torch.stack(rows)


def continuous_np(el):
    """continuous_torch on a numpy array (..., 20), real or complex."""
    c = _ZCOL
    re, rs, eta = el[..., c["rho_e"]], el[..., c["rho_s"]], el[..., c["eta"]]
    F1, F2, F3 = el[..., c["F1"]], el[..., c["F2"]], el[..., c["F3"]]
    y, x = 0.15, -0.15
    t0 = 1.15 * re / rs
    lt0 = np.log(t0)
    slope0 = (F1 + 2 * F2 * y + 3 * F3 * y * y) / re
    dg = -eta * eta * lt0 * np.exp((eta - 1.0) * lt0) / rs
    if np.any(np.real(dg) == 0.0):
        raise ValueError("Zhou EAM: rho_0 = rho_s (or eta = 0) leaves F_e undetermined")
    Fe = slope0 / dg
    F0 = Fe * (1 - eta * lt0) * np.exp(eta * lt0) - (F1 * y + F2 * y * y + F3 * y ** 3)
    out = np.array(el, copy=True)
    out[..., c["F_e"]] = Fe
    out[..., c["F0"]] = F0
    out[..., c["Fn0"]] = F0 + F1 * x + F2 * x * x + F3 * x ** 3
    out[..., c["Fn1"]] = 0.85 * (F1 + 2 * F2 * x + 3 * F3 * x * x)
    return out


class ZhouEAMParameterSet(_Variables):
    """Alloy EAM in the analytic form of Zhou, Johnson and Wadley, PRB 69,
    144113 (2004) (reference fitting/parameter_sets.py:1306-1400).

    Variables (default, per element): A, B, alpha, beta, Fn2, Fn3, F2, F3,
    eta; Fn0, Fn1, F0, F_e follow from the continuity of F and are never
    variables; r_e, f_e, rho_e, rho_s, kappa, lambda, F1 fixed by default;
    "chi" in fit_keys adds one cross factor per pair of distinct elements.
    The cutoff is fixed for the whole fit (r_cut, default the largest
    zhou_cutoff of the start parameters)."""

    _DEFAULT_FIX = ("r_e", "f_e", "rho_e", "rho_s", "kappa", "lambda", "F1")
    _DEFAULT_FIT = ("A", "B", "alpha", "beta", "Fn2", "Fn3", "F2", "F3", "eta")
    _LOG_KEYS = frozenset({"A", "B", "alpha", "beta", "chi", "r_e", "f_e", "rho_e", "rho_s"})
    _BOUNDS = {"A": (1e-3, 10.0), "B": (1e-3, 10.0), "alpha": (1.0, 30.0), "beta": (0.5, 20.0),
               "Fn2": (-20.0, 20.0), "Fn3": (-20.0, 20.0), "F2": (-20.0, 20.0), "F3": (-20.0, 20.0),
               "eta": (-3.0, 3.0), "F1": (-20.0, 20.0), "chi": (0.2, 5.0), "r_e": (1.5, 5.0),
               "f_e": (0.05, 20.0), "rho_e": (0.5, 100.0), "rho_s": (0.5, 100.0), "kappa": (0.05, 2.0),
               "lambda": (0.05, 2.0)}
    width = 0.5

    def __init__(self, elements, species, chi=None, fix_params=None, fit_keys=None, r_cut=None):
        self.species = list(species)
        self.elements = {}
        for s in self.species:
            if s not in elements:
                raise ValueError(f"ZhouEAMParameterSet: no parameters for '{s}'")
            self.elements[s] = continuous(elements[s])
        self.chi = {}
        for a_i, a in enumerate(self.species):
            for b in self.species[a_i + 1:]:
                v = (chi or {}).get(f"{a}-{b}", (chi or {}).get(f"{b}-{a}", 1.0))
                self.chi[f"{a}-{b}"] = float(v)
        self.r_cut = float(r_cut) if r_cut else max(zhou_cutoff(self.elements[s]) for s in self.species)
        fixed = set(self._DEFAULT_FIX) | set(fix_params or ())
        keys = list(fit_keys) if fit_keys else list(self._DEFAULT_FIT)
        bad = [k for k in keys if k in ZHOU_DERIVED]
        if bad:
            raise ValueError(f"ZhouEAMParameterSet: {bad} follow from the continuity of F and cannot be fitted")
        self.fit_keys = [k for k in keys if k not in fixed]
        unknown = [k for k in self.fit_keys if k not in ZHOU_KEYS and k != "chi"]
        if unknown:
            raise ValueError(f"ZhouEAMParameterSet: unknown fit key(s) {unknown}")
        self.variables, init = [], []
        for s in self.species:
            for key in self.fit_keys:
                if key != "chi":
                    self.variables.append((f"{s}:{key}", key, (s, key)))
                    init.append(self.elements[s][key])
        if "chi" in self.fit_keys:
            for pair, v in self.chi.items():
                self.variables.append((f"chi:{pair}", "chi", pair))
                init.append(v)
        self._setup_vector(init, "ZhouEAMParameterSet")

    def decode(self, x):
        """{'eam': {'form': 'zhou2004', 'elements', 'chi', 'r_cut'}}."""
        el = {s: dict(p) for s, p in self.elements.items()}
        chi = dict(self.chi)
        for xi, (_, key, target) in zip(np.asarray(x, float), self.variables):
            v = self._value(key, xi)
            if key == "chi":
                chi[target] = v
            else:
                el[target[0]][key] = v
        el = {s: continuous(p) for s, p in el.items()}
        return {"eam": {"form": "zhou2004", "elements": el, "chi": chi, "r_cut": self.r_cut}}

    def build_engine(self, params):
        p = params["eam"]
        return PotentialEngine().add(zhou_eam(p["elements"], self.species, r_cut=p["r_cut"], chi=p["chi"]))

    def potential(self, x=None):
        """The EAMPotential of decode(x) (x0 by default)."""
        p = self.decode(self.x0 if x is None else x)["eam"]
        return zhou_eam(p["elements"], self.species, r_cut=p["r_cut"], chi=p["chi"], width=self.width)

    def table_torch(self, x):
        """P (nf, 43) of decode(x), differentiable in x: the variables set
        into the element rows, continuity re-derived, rows assembled."""
        ns = len(self.species)
        if not hasattr(self, "_plan"):
            el0 = torch.tensor([[self.elements[s][k] for k in ZHOU_KEYS] for s in self.species],
                               dtype=torch.float64)
            chi0 = torch.ones((ns, ns), dtype=torch.float64)
            idx = {s: a for a, s in enumerate(self.species)}
            for pair, v in self.chi.items():
                a, b = (idx[t] for t in pair.split("-"))
                chi0[a, b] = chi0[b, a] = v
            ev, er, ec, cv, c0, c1 = [], [], [], [], [], []
            for v, (_, key, target) in enumerate(self.variables):
                if key == "chi":
                    a, b = (idx[t] for t in target.split("-"))
                    cv += [v, v]
                    c0 += [a, b]
                    c1 += [b, a]
                else:
                    ev.append(v)
                    er.append(idx[target[0]])
                    ec.append(_ZCOL[key])
            logm = torch.tensor([key in self._LOG_KEYS for _, key, _ in self.variables])
            L = lambda q: torch.tensor(q, dtype=torch.long)
            self._plan = (el0, chi0, L(ev), L(er), L(ec), L(cv), L(c0), L(c1), logm)
        el0, chi0, ev, er, ec, cv, c0, c1, logm = self._plan
        vals = torch.where(logm, torch.exp(x), x)
        el = el0.clone().index_put((er, ec), vals[ev]) if len(ev) else el0
        chi = chi0.clone().index_put((c0, c1), vals[cv]) if len(cv) else chi0
        return zhou_table_torch(continuous_torch(el), chi, self.r_cut, self.width)

    def _tables_np(self, X):
        """(P (B, nf, 43),) over the rows of X (B, n_var), in X's dtype: the
        element rows and cross factors set, continuity re-derived, P
        gathered from them by a fixed index map (zhou_table_torch's layout)."""
        ns = len(self.species)
        if not hasattr(self, "_plan"):
            self.table_torch(torch.as_tensor(self.x0))
        el0, chi0, ev, er, ec, cv, c0, c1, _ = [t.numpy() for t in self._plan]
        if not hasattr(self, "_pmap"):
            # src = [el (ns*20), chi (ns*ns), r_cut, width, 0]; P.flat = src[pmap]
            zero = ns * 20 + ns * ns + 2
            rows = []
            for a in range(ns):
                rows.append(list(range(a * 20, a * 20 + 20)) + [zero] * 20 + [zero - 2, zero - 1, zero])
            for a in range(ns):
                rows.append(list(range(a * 20, a * 20 + 20)) + [zero] * 23)
            for a in range(ns):
                for b in range(a, ns):
                    tail = [zero] * 20 if a == b else list(range(b * 20, b * 20 + 20))
                    k = zero if a == b else ns * 20 + a * ns + b
                    rows.append(list(range(a * 20, a * 20 + 20)) + tail + [zero - 2, zero - 1, k])
            self._pmap = np.array(rows, np.int64)
        V = self._vals_np(X)
        B = X.shape[0]
        el = np.repeat(el0[None].astype(X.dtype), B, axis=0)
        chi = np.repeat(chi0[None].astype(X.dtype), B, axis=0)
        if len(ev):
            el[:, er, ec] = V[:, ev]
        if len(cv):
            chi[:, c0, c1] = V[:, cv]
        src = np.concatenate([continuous_np(el).reshape(B, -1), chi.reshape(B, -1),
                              np.broadcast_to(np.array([self.r_cut, self.width, 0.0], X.dtype), (B, 3))], axis=1)
        return (src[:, self._pmap],)


# ---- evaluation with explicit tables and its adjoint ----------------------------

class _TableEval:
    """A batch, its device list and workspaces, evaluated with given tables."""

    def __init__(self, batch, skin):
        self.batch = batch
        self.skin = float(skin)
        self.dlist = None
        self.list_cut = -1.0   # the largest r_cut the current list serves
        self._ws = None
        self._adj_ws = None
        self.lanes = 8

    def autotune(self, tb, tri, candidates=(4, 8, 16), reps=3):
        """Keep the fastest lanes-per-atom tile shape of the evaluation on
        this batch (CUDA events)."""
        times = {}
        for c in candidates:
            self.lanes = c
            self.evaluate(tb, tri)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                self.evaluate(tb, tri)
            b.record()
            b.synchronize()
            times[c] = a.elapsed_time(b) / reps
        self.lanes = min(candidates, key=lambda c: (times[c], c))
        return {"lanes_per_atom": self.lanes, "ms": times}

    def _ensure_list(self, r_cut):
        if self.dlist is None or r_cut > self.list_cut:
            self.dlist = DeviceNeighbourList(r_cut + self.skin).build(self.batch)
            self.list_cut = r_cut
        return self.dlist

    def _tables(self, tb, tri, r_cut=None):
        ns = int(round(tb.shape[0] ** 0.5))
        if r_cut is None:
            r_cut = table_cutoff(tb)
        dl = self._ensure_list(r_cut)
        return dl, _lib.MbfTersoffTables(ns, _lib.ptr(tb), _lib.ptr(tri), r_cut), ns

    def evaluate(self, tb, tri, r_cut=None):
        dl, tabs, _ = self._tables(tb, tri, r_cut)
        b = self.batch
        dev = b.device
        L = _lib.lib()
        need = int(L.mbf_eval_workspace_bytes(b.n_atoms, dl.n_slots, b.n_chunks))
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
        E = torch.empty(b.n_struct, dtype=torch.float64, device=dev)
        F = torch.empty((b.n_atoms, 3), dtype=torch.float64, device=dev)
        W = torch.empty((b.n_struct, 9), dtype=torch.float64, device=dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(L.mbf_tersoff_eval(b.mbf_system(), dl.mbf_nlist(), tabs, b.reduce_plan(), _lib.MBF_FP64, self.lanes,
                                      _lib.ptr(self._ws), self._ws.numel(), _lib.ptr(F), _lib.ptr(E), _lib.ptr(W),
                                      st), "mbf_tersoff_eval")
        return E, F, W

    def adjoint(self, tb, tri, gE, gF, gW, r_cut=None):
        dl, tabs, ns = self._tables(tb, tri, r_cut)
        b = self.batch
        dev = b.device
        L = _lib.lib()
        need = int(L.mbf_tersoff_adjoint_workspace_bytes(dl.n_slots, ns))
        if self._adj_ws is None or self._adj_ws.numel() < need:
            self._adj_ws = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
        d_tb = torch.empty_like(tb)
        d_tri = torch.empty_like(tri)
        g = [None if t is None else t.to(torch.float64).contiguous() for t in (gE, gF, gW)]
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(L.mbf_tersoff_adjoint(b.mbf_system(), dl.mbf_nlist(), tabs, _lib.ptr(g[0]), _lib.ptr(g[1]),
                                         _lib.ptr(g[2]), _lib.ptr(self._adj_ws), self._adj_ws.numel(),
                                         _lib.ptr(d_tb), _lib.ptr(d_tri), st), "mbf_tersoff_adjoint")
        return d_tb, d_tri


class TersoffEFS(torch.autograd.Function):
    """(energy (S,), forces (N, 3), virial (S, 9)) of a batch as a function
    of the Tersoff tables; backward is one mbf_tersoff_adjoint call.  The
    tables may live on the host (a few dozen numbers, decoded there by
    cheap CPU tensor operations): they are copied to the batch's device for
    the evaluation and their gradients come back to where they live."""

    @staticmethod
    def forward(ctx, tb, tri, ev):
        dev = ev.batch.device
        r_cut = table_cutoff(tb)
        tb_d = tb.detach().to(dev, non_blocking=True).contiguous()
        tri_d = tri.detach().to(dev, non_blocking=True).contiguous()
        E, F, W = ev.evaluate(tb_d, tri_d, r_cut)
        ctx.ev = ev
        ctx.r_cut = r_cut
        ctx.home = tb.device
        ctx.save_for_backward(tb_d, tri_d)
        return E, F, W

    @staticmethod
    def backward(ctx, gE, gF, gW):
        tb, tri = ctx.saved_tensors
        d_tb, d_tri = ctx.ev.adjoint(tb, tri, gE, gF, gW, ctx.r_cut)
        return d_tb.to(ctx.home), d_tri.to(ctx.home), None


class _EamTableEval:
    """A batch, its device list and workspaces, evaluated with given Zhou
    rows P (nf, 43) over a fixed function-table skeleton (codes, function
    ids per species; the cutoff is fixed)."""

    def __init__(self, batch, skin, skeleton, r_cut):
        self.batch = batch
        dev = batch.device
        self.r_cut = float(r_cut)
        self.dlist = DeviceNeighbourList(self.r_cut + float(skin)).build(batch)
        self.keep = {k: torch.as_tensor(np.ascontiguousarray(skeleton[k]), device=dev)
                     for k in ("codes", "xo", "nx", "X", "C", "rho_f", "F_f", "phi_f")}
        self.ns = len(skeleton["rho_f"])
        self.nf = len(skeleton["codes"])
        self.fused = 1 if skeleton["fused"] else 0
        self._ws = None
        self._adj_ws = None
        self.lanes = 2

    def _tab(self, P):
        k = self.keep
        return _lib.MbfEamTables(self.ns, self.nf, int(k["X"].shape[0]), _lib.ptr(k["codes"]), _lib.ptr(P),
                                 _lib.ptr(k["xo"]), _lib.ptr(k["nx"]), _lib.ptr(k["X"]), _lib.ptr(k["C"]),
                                 _lib.ptr(k["rho_f"]), _lib.ptr(k["F_f"]), _lib.ptr(k["phi_f"]), self.r_cut,
                                 self.fused)

    def autotune(self, P, candidates=(1, 2, 4, 8), reps=3):
        """Keep the fastest lanes-per-atom of the evaluation (CUDA events)."""
        times = {}
        for c in candidates:
            self.lanes = c
            self.evaluate(P)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                self.evaluate(P)
            b.record()
            b.synchronize()
            times[c] = a.elapsed_time(b) / reps
        self.lanes = min(candidates, key=lambda c: (times[c], c))
        return {"lanes_per_atom": self.lanes, "ms": times}

    def evaluate(self, P):
        b, dl = self.batch, self.dlist
        dev = b.device
        L = _lib.lib()
        need = int(L.mbf_eval_workspace_bytes(b.n_atoms, dl.n_slots, b.n_chunks))
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
        E = torch.empty(b.n_struct, dtype=torch.float64, device=dev)
        F = torch.empty((b.n_atoms, 3), dtype=torch.float64, device=dev)
        W = torch.empty((b.n_struct, 9), dtype=torch.float64, device=dev)
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(L.mbf_eam_eval(b.mbf_system(), dl.mbf_nlist(), self._tab(P), b.reduce_plan(), _lib.MBF_FP64,
                                  self.lanes, _lib.ptr(self._ws), self._ws.numel(), _lib.ptr(F), _lib.ptr(E),
                                  _lib.ptr(W), st), "mbf_eam_eval")
        return E, F, W

    def adjoint(self, P, gE, gF, gW):
        b, dl = self.batch, self.dlist
        dev = b.device
        L = _lib.lib()
        need = int(L.mbf_eam_adjoint_workspace_bytes(b.n_atoms, dl.n_slots, self.ns))
        if self._adj_ws is None or self._adj_ws.numel() < need:
            self._adj_ws = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
        d_P = torch.empty_like(P)
        g = [None if t is None else t.to(torch.float64).contiguous() for t in (gE, gF, gW)]
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(L.mbf_eam_adjoint(b.mbf_system(), dl.mbf_nlist(), self._tab(P), _lib.ptr(g[0]), _lib.ptr(g[1]),
                                     _lib.ptr(g[2]), _lib.ptr(self._adj_ws), self._adj_ws.numel(), _lib.ptr(d_P),
                                     st), "mbf_eam_adjoint")
        return d_P


class EamEFS(torch.autograd.Function):
    """(energy (S,), forces (N, 3), virial (S, 9)) of a batch as a function
    of the Zhou rows P (nf, 43); backward is one mbf_eam_adjoint call.  P
    may live on the host; its gradient comes back there."""

    @staticmethod
    def forward(ctx, P, ev):
        P_d = P.detach().to(ev.batch.device, non_blocking=True).contiguous()
        E, F, W = ev.evaluate(P_d)
        ctx.ev = ev
        ctx.home = P.device
        ctx.save_for_backward(P_d)
        return E, F, W

    @staticmethod
    def backward(ctx, gE, gF, gW):
        (P,) = ctx.saved_tensors
        return ctx.ev.adjoint(P, gE, gF, gW).to(ctx.home), None


def shard_structures(n_atoms, world):
    """Greedy atom-count balance: largest structures first, each to the
    rank with the fewest atoms so far (lowest rank on ties); returns one
    sorted index list per rank."""
    load = [0] * world
    parts = [[] for _ in range(world)]
    for s in sorted(range(len(n_atoms)), key=lambda q: (-int(n_atoms[q]), q)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(s)
        load[r] += int(n_atoms[s])
    return [sorted(p) for p in parts]


def allreduce_sum(vec, world=1, group=None):
    """Sum a tensor over the ranks of a process group in place (the
    reference's _mpi_allreduce_sum_scalar, fitting/loss.py:246-260); a
    no-op for one rank.  Every rank calls it in the same order."""
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(vec, op=dist.ReduceOp.SUM, group=group)
    return vec


def _huber_of_squared(sq, delta):
    """fitting/loss.py:29-48: sq if sqrt(sq) <= delta else 2 delta sqrt(sq) - delta^2."""
    r = torch.sqrt(torch.clamp(sq, min=1e-300))
    return torch.where(r <= delta, sq, 2.0 * delta * r - delta * delta)


class _TersoffModel:
    """Tersoff parameter sets: dense (tb, tri) tables, TersoffEFS."""

    def __init__(self, ps):
        self.ps = ps

    def _tables0(self, device):
        return tables_from_records(self.ps.decode(self.ps.x0)["tersoff"], self.ps.species, device)

    def list_cut(self):
        return table_cutoff(self._tables0("cpu")[0])

    def evaluator(self, batch, skin):
        ev = _TableEval(batch, skin)
        return ev, ev.autotune(*self._tables0(batch.device))

    def efs(self, x_t, ev):
        if hasattr(self.ps, "tables_torch"):
            tb, tri = self.ps.tables_torch(x_t)
        else:
            tb, tri = tables_from_records(self.ps.decode_torch(x_t)["tersoff"], self.ps.species, x_t.device)
        return TersoffEFS.apply(tb, tri, ev)

    def evaluate(self, ev, dtabs, tabs):
        return ev.evaluate(dtabs[0], dtabs[1], table_cutoff(tabs[0]))

    def adjoint(self, ev, dtabs, tabs, gE, gF, gW):
        return ev.adjoint(dtabs[0], dtabs[1], gE, gF, gW, table_cutoff(tabs[0]))


class _ZhouModel:
    """Zhou EAM parameter sets: the analytic rows P (nf, 43), EamEFS."""

    def __init__(self, ps):
        self.ps = ps

    def list_cut(self):
        return self.ps.r_cut

    def evaluator(self, batch, skin):
        ev = _EamTableEval(batch, skin, self.ps.potential().function_table(), self.ps.r_cut)
        P0 = self.ps.table_torch(torch.as_tensor(self.ps.x0)).to(batch.device)
        return ev, ev.autotune(P0)

    def efs(self, x_t, ev):
        return EamEFS.apply(self.ps.table_torch(x_t), ev)

    def evaluate(self, ev, dtabs, tabs):
        return ev.evaluate(dtabs[0])

    def adjoint(self, ev, dtabs, tabs, gE, gF, gW):
        return (ev.adjoint(dtabs[0], gE, gF, gW),)


def _model_of(ps):
    return _ZhouModel(ps) if hasattr(ps, "table_torch") else _TersoffModel(ps)


class PotentialFit:
    """The reference's fit loss (fitting/loss.py:51-260) over a training set
    on the GPU, and its gradient in x, for the Tersoff parameter sets
    (MultiSpeciesTersoffParameterSet, Tersoff1989ParameterSet) and
    ZhouEAMParameterSet.

    structures : dicts with lattice, positions, atom_types, natoms,
                 ref_energy (eV/atom), optional ref_forces (N, 3),
                 ref_stress (3, 3), volume, scale (c_s, squared) and weight
                 (w_trust, linear) -- the reference's keys.
    weights    : energy, forces, stress, r0, eps0 (defaults 1, 1, 0.1, 1, 1)
                 and, for loss_type='huber', huber_delta_energy/forces/stress.
    rank, world, group : with world > 1 this rank takes its share of the
                 structures (shard_structures) and the loss and gradient are
                 summed over the process group (torch.distributed), the
                 reference's MPI split (fitting/loss.py:190-248).
    """

    def __init__(self, param_set, structures, weights=None, loss_type="squared", device=None, skin=0.3,
                 rank=0, world=1, group=None):
        if loss_type not in ("squared", "huber"):
            raise ValueError(f"unknown loss_type '{loss_type}'. Choose 'squared' or 'huber'.")
        weights = dict(weights or {})
        if loss_type == "huber":
            for key in ("huber_delta_energy", "huber_delta_forces", "huber_delta_stress"):
                if key not in weights:
                    raise ValueError(f"loss_type='huber' requires weights['{key}'] (eV)")
        self.ps = param_set
        self.model = _model_of(param_set)
        self.loss_type = loss_type
        self.w = weights
        self.rank, self.world, self.group = int(rank), int(world), group
        self.device = torch.device(device) if device is not None else default_device()
        self.mine = shard_structures([s["natoms"] for s in structures], self.world)[self.rank]
        self._setup([structures[q] for q in self.mine], skin)

    def _setup(self, structs, skin):
        dev = self.device
        sp = self.ps.species
        lats, poss, ids, reps, n_orig, vols = [], [], [], [], [], []
        r_guess = self.model.list_cut()
        for s in structs:
            t = species_ids(s["atom_types"], sp)
            L2, P2, T2, k = replicate_thin(s["lattice"], s["positions"], t, r_guess + skin)
            lats.append(L2)
            poss.append(P2)
            ids.append(T2)
            reps.append(float(np.prod(k)))
            n_orig.append(len(s["positions"]))
            vols.append(float(s.get("volume", abs(np.linalg.det(np.asarray(s["lattice"], float))))))
        self.n_struct = len(structs)
        self.ev = None
        if not structs:
            return
        self.ev, self.tuned = self.model.evaluator(Batch(lats, poss, ids, device=dev), skin)
        off = self.ev.batch.offsets
        idx = np.concatenate([np.arange(off[q], off[q] + n) for q, n in enumerate(n_orig)])
        self._orig = torch.as_tensor(idx, device=dev)
        f64 = dict(dtype=torch.float64, device=dev)
        self._n = torch.tensor(n_orig, **f64)
        self._inv_k = torch.tensor([1.0 / k for k in reps], **f64)
        self._vol = torch.tensor(vols, **f64)
        self._vsup = torch.as_tensor(self.ev.batch.volumes, **f64)
        self._atom_struct = torch.as_tensor(np.repeat(np.arange(len(structs)), n_orig), device=dev)
        self._eref = torch.tensor([float(s["ref_energy"]) for s in structs], **f64)
        fref, fmask, sref, smask = [], [], [], []
        for s, n in zip(structs, n_orig):
            f = s.get("ref_forces")
            fref.append(np.zeros((n, 3)) if f is None else np.asarray(f, float).reshape(n, 3))
            fmask.append(0.0 if f is None else 1.0)
            st = s.get("ref_stress")
            sref.append(np.zeros(9) if st is None else np.asarray(st, float).reshape(9))
            smask.append(0.0 if st is None else 1.0)
        self._fref = torch.as_tensor(np.concatenate(fref), **f64)
        self._fmask = torch.tensor(fmask, **f64)
        self._sref = torch.as_tensor(np.stack(sref), **f64)
        self._smask = torch.tensor(smask, **f64)
        self._cw = torch.tensor([float(s.get("weight", 1.0)) * float(s.get("scale", 1.0)) ** 2 for s in structs],
                                **f64)
        # the fused device loss (mbf_fit_loss): its set description and outputs
        i32 = dict(dtype=torch.int32, device=dev)
        b = self.ev.batch
        fo = np.zeros(len(n_orig), np.int64)
        fo[1:] = np.cumsum(n_orig)[:-1]
        w = self.w
        self._fs_keep = dict(n_orig=torch.tensor(n_orig, **i32), fref_off=torch.as_tensor(fo.astype(np.int32), **i32))
        hub = self.loss_type == "huber"
        self._fs = _lib.MbfFitSet(
            len(structs), b.n_atoms, _lib.ptr(b.struct_off), _lib.ptr(b.atom_struct),
            _lib.ptr(self._fs_keep["n_orig"]), _lib.ptr(self._fs_keep["fref_off"]), _lib.ptr(self._inv_k),
            _lib.ptr(self._eref), _lib.ptr(self._fref), _lib.ptr(self._sref), _lib.ptr(self._vol), _lib.ptr(self._vsup),
            _lib.ptr(self._fmask), _lib.ptr(self._smask), _lib.ptr(self._cw),
            float(w.get("energy", 1.0)), float(w.get("forces", 1.0)), float(w.get("stress", 0.1)),
            float(w.get("r0", 1.0)), float(w.get("eps0", 1.0)), 1 if hub else 0,
            float(w["huber_delta_energy"]) if hub else 0.0, float(w["huber_delta_forces"]) if hub else 0.0,
            float(w["huber_delta_stress"]) if hub else 0.0)
        nws = int(_lib.lib().mbf_fit_loss_workspace_bytes(len(structs)))
        self._fws = torch.empty(max(nws, 256), dtype=torch.uint8, device=dev)
        self._gout = (torch.empty(1, **f64), torch.empty(len(structs), **f64), torch.empty((b.n_atoms, 3), **f64),
                      torch.empty((len(structs), 9), **f64))

    def _local_loss(self, x_t):
        """This rank's loss as a differentiable torch scalar."""
        if self.ev is None:
            return (x_t.sum() * 0.0).to(self.device)
        E, F, W = self.model.efs(x_t, self.ev)
        w = self.w
        w_E, w_F, w_S = float(w.get("energy", 1.0)), float(w.get("forces", 1.0)), float(w.get("stress", 0.1))
        r0, eps0 = float(w.get("r0", 1.0)), float(w.get("eps0", 1.0))
        e = E * self._inv_k
        e_sq = (e - self._n * self._eref) ** 2
        df = F.index_select(0, self._orig) - self._fref
        fs = torch.zeros(self.n_struct, dtype=torch.float64, device=self.device)
        fs = fs.index_add(0, self._atom_struct, (df * df).sum(1))
        f_sq = (r0 ** 2) * fs / (3.0 * self._n)
        sig = W / self._vsup[:, None]
        ds = sig - self._sref
        s_sq = (self._vol * eps0) ** 2 * (ds * ds).mean(1)
        if self.loss_type == "huber":
            e_sq = _huber_of_squared(e_sq, float(w["huber_delta_energy"]))
            f_sq = _huber_of_squared(f_sq, float(w["huber_delta_forces"]))
            s_sq = _huber_of_squared(s_sq, float(w["huber_delta_stress"]))
        per = w_E * e_sq + w_F * f_sq * self._fmask + w_S * s_sq * self._smask
        return (self._cw * per).sum()

    def _reduce(self, vec):
        return allreduce_sum(vec, self.world, self.group)

    def device_step(self, x, grad=True):
        """One step on the device: the tables of x (host, with their
        x-Jacobians by the complex step when grad), the batch evaluation,
        the fused loss (mbf_fit_loss) and, when grad, the adjoint.  Returns
        (loss (1,), table gradients, Jacobians): device tensors, the
        Jacobians numpy; nothing is synchronised."""
        x = np.asarray(x, float)
        if grad:
            tabs, jac = self.ps.table_jacobian(x)
        else:
            tabs, jac = self.ps.tables_np(x), None
        dev = self.device
        dtabs = [torch.from_numpy(t).to(dev, non_blocking=False) for t in tabs]
        E, F, W = self.model.evaluate(self.ev, dtabs, tabs)
        loss, gE, gF, gW = self._gout
        L = _lib.lib()
        st = torch.cuda.current_stream(dev).cuda_stream
        _lib.check(L.mbf_fit_loss(self._fs, _lib.ptr(E), _lib.ptr(F), _lib.ptr(W), _lib.ptr(self._fws),
                                  self._fws.numel(), _lib.ptr(loss), _lib.ptr(gE), _lib.ptr(gF), _lib.ptr(gW), st),
                   "mbf_fit_loss")
        if not grad:
            return loss, (), None
        return loss, self.model.adjoint(self.ev, dtabs, tabs, gE, gF, gW), jac

    def _local(self, x, grad):
        """(loss, gradient or None) of this rank's structures, host numpy."""
        if self.ev is None:
            return 0.0, (np.zeros(len(x)) if grad else None)
        loss, d, jac = self.device_step(x, grad)
        flat = torch.cat([loss] + [t.reshape(-1) for t in d]).cpu().numpy()
        if not grad:
            return float(flat[0]), None
        g = np.zeros(len(x))
        o = 1
        for J, t in zip(jac, d):
            k = t.numel()
            g += np.tensordot(J, flat[o:o + k].reshape(tuple(t.shape)), axes=t.dim())
            o += k
        return float(flat[0]), g

    def _combine(self, vec):
        if self.world > 1:
            vec = self._reduce(torch.as_tensor(vec, device=self.device)).cpu().numpy()
        return vec

    def loss_and_grad(self, x):
        """(loss, dloss/dx) at x; every rank of a group must call it."""
        failed = 0.0
        try:
            loss, g = self._local(x, True)
        except (ValueError, RuntimeError, _lib.MbfError):
            failed, loss, g = 1.0, 0.0, np.zeros(len(x))
        vec = self._combine(np.concatenate([[loss], g, [failed]]))
        if vec[-1] > 0.0:
            return 1e30, np.zeros(len(x))
        return float(vec[0]), vec[1:-1]

    def loss(self, x):
        """The loss at x (1e30 if the parameters cannot be evaluated)."""
        failed = 0.0
        try:
            val, _ = self._local(x, False)
        except (ValueError, RuntimeError, _lib.MbfError):
            failed, val = 1.0, 0.0
        vec = self._combine(np.array([val, failed]))
        return 1e30 if vec[1] > 0.0 else float(vec[0])


TersoffFit = PotentialFit

_FITS = {}


def generic_loss_function(x, param_set, structures, weights, r_cut=None, ewald_alpha=None,
                          coulomb_method="ewald", loss_type="squared"):
    """fitting/loss.py:51 on the GPU for Tersoff and Zhou EAM parameter
    sets: the same value (eV^2; 1e30 when the parameters cannot be
    evaluated).  r_cut, ewald_alpha and coulomb_method concern charges,
    which these sets do not carry; the list radius follows the decoded
    records (Tersoff) or the set's fixed cutoff (EAM)."""
    if loss_type not in ("squared", "huber"):
        raise ValueError(f"generic_loss_function: unknown loss_type '{loss_type}'. Choose 'squared' or 'huber'.")
    key = (id(param_set), id(structures), loss_type, tuple(sorted((k, float(v)) for k, v in weights.items())))
    fit = _FITS.get(key)
    if fit is None:
        fit = _FITS[key] = PotentialFit(param_set, structures, weights, loss_type=loss_type)
    return fit.loss(x)
