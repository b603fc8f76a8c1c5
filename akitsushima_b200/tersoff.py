"""Tersoff bond-order potential on the GPU (reference engine/tersoff.py).

E = sum_{i<j} fc(r_ij) [A exp(-lambda1 r) - b_avg B exp(-lambda2 r)],
b_avg = (b_ij + b_ji) / 2, b_ij = (1 + (beta zeta_ij)^n)^(-1/(2n)),
zeta_ij = sum_k gamma fc(r_ik) g(theta_ijk) exp(lambda3^m (r_ij - r_ik)^m).

Two parameter forms, as the reference (engine/tersoff.py:1135-1169):

* a flat dict (A, B, lambda1, lambda2, lambda3, beta, n, c, d, h, R, D) for
  one species; the reference's single-species path fixes m = 3 and gamma = 1
  (engine/tersoff.py:494, :1431) and so does this one;
* records {(i, j, k): {...}} (LAMMPS convention): pair and bond-order terms
  from (i, j, j), angular terms from (i, j, k); missing entries do not
  interact, with the reference's gating (engine/tersoff.py:528-540, :1665-1702).
"""
import math

import numpy as np
import torch

from . import _lib
from .potential import DevicePotential, nested_records

TERSOFF1989_ELEMENT_KEYS = ("A", "B", "lambda", "mu", "beta", "n", "c", "d", "h", "R", "S")

_TB_KEYS = (("A", 0.0), ("B", 0.0), ("lambda1", 0.0), ("lambda2", 0.0), ("R", 1.0), ("D", 1.0),
            ("beta", 0.0), ("n", 1.0))


class TersoffPotential(DevicePotential):
    """Tersoff potential; ``params`` flat (one species) or records.

    precision : 'fp64' (default) or 'mixed' (float32 cutoff, angular and
                exponential terms; float64 displacements, bond orders and
                accumulation).
    """

    def __init__(self, params, species=None, precision="fp64"):
        super().__init__()
        self.precision = precision
        self.species = list(species) if species else None
        flat = ("A" in params and "lambda1" in params
                and not any(isinstance(k, tuple) for k in params))
        if flat:
            sp0 = self.species[0] if self.species else "__X__"
            self.species = [sp0]
            self._multi = False
            self._flat = dict(params)
            self.R = float(params.get("R", 2.85))
            self.D = float(params.get("D", 0.15))
            self.r_cut = self.R + self.D
            self.p = {(sp0, sp0, sp0): dict(params)}
        else:
            if not self.species:
                raise ValueError("TersoffPotential: 'species' is required when using the "
                                 "multi-species (nested-triple) parameter format.")
            self._multi = True
            self.p = nested_records(params)
            rc = 0.0
            for (i, j, k), v in self.p.items():
                if j == k and "R" in v and "D" in v:
                    rc = max(rc, float(v["R"]) + float(v["D"]))
            self.r_cut = rc if rc > 0 else 3.0
            self.R = self.D = None

    def host_tables(self):
        """Dense species tables: tb (ns*ns, 10) rows [valid A B l1 l2 R D beta
        n 0] and tri (ns^3, 8) rows [valid c d h l3 m gamma 0]."""
        ns = len(self.species)
        tb = np.zeros((ns * ns, 10))
        tri = np.zeros((ns ** 3, 8))
        if not self._multi:
            p = {k: float(v) for k, v in self._flat.items() if not isinstance(v, str)}
            tb[0] = [1.0, p["A"], p["B"], p["lambda1"], p["lambda2"], self.R, self.D,
                     p["beta"], p["n"], 0.0]
            tri[0] = [1.0, p["c"], p["d"], p["h"], p["lambda3"], 3.0, 1.0, 0.0]
            return tb, tri
        for a, sa in enumerate(self.species):
            for b, sb in enumerate(self.species):
                rec = self.p.get((sa, sb, sb))
                if rec is None:
                    tb[a * ns + b] = [0.0, 0, 0, 0, 0, 1.0, 1.0, 0.0, 1.0, 0.0]
                    continue
                tb[a * ns + b] = [1.0] + [float(rec.get(k, d)) for k, d in _TB_KEYS] + [0.0]
        for a, sa in enumerate(self.species):
            for b, sb in enumerate(self.species):
                for c, sc in enumerate(self.species):
                    rec = self.p.get((sa, sb, sc))
                    row = (a * ns + b) * ns + c
                    if rec is None:
                        tri[row] = [0.0, 0.0, 1.0, 0.0, 0.0, 3.0, 1.0, 0.0]
                        continue
                    tri[row] = [1.0, float(rec["c"]), float(rec["d"]), float(rec["h"]),
                                float(rec["lambda3"]), float(rec.get("m", 3.0)),
                                float(rec.get("gamma", 1.0)), 0.0]
        return tb, tri

    def _device_tables(self, device):
        tb, tri = self.host_tables()
        tb_t = torch.as_tensor(np.ascontiguousarray(tb), device=device)
        tri_t = torch.as_tensor(np.ascontiguousarray(tri), device=device)
        st = _lib.MbfTersoffTables(len(self.species), _lib.ptr(tb_t), _lib.ptr(tri_t), self.r_cut)
        return (st, tb_t, tri_t)

    sites_entry = "mbf_tersoff_eval_sites"
    lane_choices = (4, 8, 16)
    lanes_per_atom = 8

    def _call(self, L, sysd, nld, tabs, plan, prec, ws, nbytes, forces, energy, virial, stream):
        return L.mbf_tersoff_eval(sysd, nld, tabs[0], plan, prec, int(self.lanes_per_atom), ws, nbytes, forces, energy,
                                  virial, stream)


def _pair_key(a, b, table, default):
    for k in (f"{a}-{b}", f"{b}-{a}"):
        if k in table:
            return float(table[k])
    return default


def tersoff1989_to_triplets(elements, chi, species=None, omega=None):
    """Tersoff (1989) multicomponent mixing rules expanded to (i, j, k)
    records (Tersoff, PRB 39, 5566, eqs. 1a-1e; reference
    engine/tersoff.py:1968-2034): lambda_ij, mu_ij arithmetic means; A, B,
    R, S geometric means; chi_ij scales B_ij; beta, n, c, d, h of the centre;
    lambda3 = 0, m = 3, gamma = omega_ik (default 1); R = (R_ij + S_ij)/2,
    D = (S_ij - R_ij)/2."""
    species = list(species) if species is not None else list(elements)
    omega = omega or {}
    for s in species:
        if s not in elements:
            raise ValueError(f"tersoff1989: no parameters for element '{s}'")
        missing = [k for k in TERSOFF1989_ELEMENT_KEYS if k not in elements[s]]
        if missing:
            raise ValueError(f"tersoff1989: element '{s}' lacks {missing}")
    out = {}
    for i in species:
        pi = elements[i]
        for j in species:
            pj = elements[j]
            x = 1.0 if i == j else _pair_key(i, j, chi, None)
            if x is None:
                raise ValueError(f"tersoff1989: chi for the {i}-{j} pair is not given.")
            r_ij = math.sqrt(float(pi["R"]) * float(pj["R"]))
            s_ij = math.sqrt(float(pi["S"]) * float(pj["S"]))
            if not s_ij > r_ij:
                raise ValueError(f"tersoff1989: S must exceed R ({i}-{j})")
            for k in species:
                rec = {"c": float(pi["c"]), "d": float(pi["d"]), "h": float(pi["h"]),
                       "lambda3": 0.0, "m": 3.0, "gamma": _pair_key(i, k, omega, 1.0)}
                if j == k:
                    rec.update(A=math.sqrt(float(pi["A"]) * float(pj["A"])),
                               B=x * math.sqrt(float(pi["B"]) * float(pj["B"])),
                               lambda1=0.5 * (float(pi["lambda"]) + float(pj["lambda"])),
                               lambda2=0.5 * (float(pi["mu"]) + float(pj["mu"])),
                               R=0.5 * (r_ij + s_ij), D=0.5 * (s_ij - r_ij),
                               beta=float(pi["beta"]), n=float(pi["n"]))
                out[(i, j, k)] = rec
    return out
