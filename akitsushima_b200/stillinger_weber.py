"""Stillinger-Weber potential on the GPU (reference engine/stillinger_weber.py).

E = sum_{i<j} V2(r_ij) + sum_i sum_{j<k} h(r_ij, r_ik, theta_jik),
V2 = eps A (B xi^-p - xi^-q) exp(1 / (xi - a)), xi = r / sigma;
h  = eps lambda exp(gamma / (x_ij - a)) exp(gamma / (x_ik - a)) (cos - cos0)^2.

Parameter forms as the reference (engine/stillinger_weber.py:840-871): a
flat dict for one species (every key defaults to Stillinger & Weber's Si,
gamma included), or records {(i, j, k): {...}} (LAMMPS .sw convention): the
two-body term and the legs' sigma, a, gamma from (i, j, j), lambda, epsilon
and cos theta0 from (i, j, k), both neighbour orders with lambda/2 each.
"""
import math

import numpy as np
import torch

from . import _lib
from .potential import DevicePotential, nested_records
from .published_parameters import SW_SI_1985


def _effective_two_body(rec):
    if rec is None or float(rec.get("A", 0.0)) == 0.0:
        return None
    return {"epsilon": float(rec.get("epsilon", 1.0)), "sigma": float(rec["sigma"]),
            "a": float(rec["a"]), "A": float(rec["A"]), "B": float(rec.get("B", 0.0)),
            "p": float(rec.get("p", 4)), "q": float(rec.get("q", 0))}


def check_two_body_symmetry(params):
    """Refuse records whose two-body term depends on atom order
    (engine/stillinger_weber.py:714-762): (i, j, j) and (j, i, i) must agree
    on epsilon, sigma, a, A, B, p, q whenever either supplies a term."""
    species = sorted({e for t in params for e in t})
    for x, si in enumerate(species):
        for sj in species[x + 1:]:
            r1 = _effective_two_body(params.get((si, sj, sj)))
            r2 = _effective_two_body(params.get((sj, si, si)))
            if r1 is None and r2 is None:
                continue
            if r1 is None or r2 is None:
                raise ValueError(
                    f"StillingerWeberPotential: only one of ({si},{sj},{sj}) and "
                    f"({sj},{si},{si}) supplies a two-body {si}-{sj} term; the energy would "
                    "depend on atom order.")
            diff = [k for k in r1 if not math.isclose(r1[k], r2[k], rel_tol=1e-12, abs_tol=0.0)]
            if diff:
                raise ValueError(
                    f"StillingerWeberPotential: ({si},{sj},{sj}) and ({sj},{si},{si}) disagree "
                    f"on the two-body parameter(s) {diff}.")


class StillingerWeberPotential(DevicePotential):
    """Stillinger-Weber potential, flat (one species) or records."""

    def __init__(self, params, r_cut=None, species=None, precision="fp64"):
        super().__init__()
        self.precision = precision
        self.species = list(species) if species else None
        flat = (("epsilon" in params or "sigma" in params)
                and not any(isinstance(k, tuple) for k in params)) or params == {}
        if flat and not isinstance(params, list):
            sp0 = self.species[0] if self.species else "__X__"
            self.species = [sp0]
            self._multi = False
            self.p = dict(params)
            q = dict(SW_SI_1985)
            q.update({k: float(v) for k, v in params.items()})
            self._q = q
            self.r_cut = float(r_cut) if r_cut is not None else q["a"] * q["sigma"]
        else:
            if not self.species:
                raise ValueError("StillingerWeberPotential: 'species' is required when using "
                                 "the multi-species (nested-triple) parameter format.")
            self._multi = True
            self.p = nested_records(params)
            check_two_body_symmetry(self.p)
            rc = 0.0
            for (i, j, k), v in self.p.items():
                if j == k:
                    rc = max(rc, float(v["a"]) * float(v["sigma"]))
            self.r_cut = rc if rc > 0 else 4.0

    def host_tables(self):
        """tb (ns*ns, 8) [valid eps sigma a A B p q], leg (ns*ns, 4)
        [sigma a gamma 0], tri (ns^3, 4) [valid eps*lambda/2 cos0 0]; and the
        mask radius."""
        ns = len(self.species)
        tb = np.zeros((ns * ns, 8))
        leg = np.zeros((ns * ns, 4))
        leg[:, 0] = 1.0
        tri = np.zeros((ns ** 3, 4))
        tri[:, 2] = -1.0 / 3.0
        if not self._multi:
            q = self._q
            tb[0] = [1.0, q["epsilon"], q["sigma"], q["a"], q["A"], q["B"], q["p"], q["q"]]
            leg[0] = [q["sigma"], q["a"], q["gamma"], 0.0]
            tri[0] = [1.0, 0.5 * q["epsilon"] * q["lambda"], q["costheta0"], 0.0]
            return tb, leg, tri, q["a"] * q["sigma"]
        for a, sa in enumerate(self.species):
            for b, sb in enumerate(self.species):
                rec = self.p.get((sa, sb, sb))
                if rec is not None:
                    leg[a * ns + b] = [float(rec["sigma"]), float(rec["a"]), float(rec["gamma"]), 0.0]
                two = _effective_two_body(rec)
                if two is not None:
                    tb[a * ns + b] = [1.0, two["epsilon"], two["sigma"], two["a"], two["A"],
                                      two["B"], two["p"], two["q"]]
        for a, sa in enumerate(self.species):
            for b, sb in enumerate(self.species):
                for c, sc in enumerate(self.species):
                    rec = self.p.get((sa, sb, sc))
                    if (rec is None or self.p.get((sa, sb, sb)) is None
                            or self.p.get((sa, sc, sc)) is None):
                        continue
                    tri[(a * ns + b) * ns + c] = [1.0, float(rec.get("epsilon", 1.0)) * 0.5 * float(rec["lambda"]),
                                                  float(rec.get("costheta0", -1.0 / 3.0)), 0.0]
        return tb, leg, tri, self.r_cut

    def _device_tables(self, device):
        tb, leg, tri, rc = self.host_tables()
        t = [torch.as_tensor(np.ascontiguousarray(x), device=device) for x in (tb, leg, tri)]
        st = _lib.MbfSwTables(len(self.species), _lib.ptr(t[0]), _lib.ptr(t[1]), _lib.ptr(t[2]), rc)
        return (st, *t)

    sites_entry = "mbf_sw_eval_sites"
    lane_choices = (4, 8, 16)
    lanes_per_atom = 8

    def _call(self, L, sysd, nld, tabs, plan, prec, ws, nbytes, forces, energy, virial, stream):
        return L.mbf_sw_eval(sysd, nld, tabs[0], plan, prec, int(self.lanes_per_atom), ws, nbytes, forces, energy, virial,
                             stream)
