"""Write the golden fixtures of tests/golden/ by running the reference itself.

Usage (in a container where the reference is importable):

    NUMBA_CACHE_DIR=/tmp/numba_cache python tests/golden/make_golden.py \
        --reference /root/reference

Each fixture is a small .npz holding the inputs (lattice, positions, atom
types, the reference neighbour list's candidate pairs) and the reference's
outputs (energy, forces, stress).  Structures are built with the seeded
generator of the reference's benchmarks/bench_force.py:152-158 (cubic cells of
a fractional basis, Gaussian displacements), strained where a triclinic cell
is wanted (tests/test_multispecies_fit.py:41-47 style).  The fixtures are the
pin of the CPU oracle; nothing at test time imports the reference.
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

DIAMOND = [[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0],
           [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75],
           [0.75, 0.75, 0.25]]
FCC = [[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]]

TERSOFF_SI = {"A": 1830.8, "B": 471.18, "lambda1": 2.4799, "lambda2": 1.7322,
              "lambda3": 0.0, "beta": 1.1e-6, "n": 0.78734, "c": 100390.0,
              "d": 16.217, "h": -0.59825, "R": 2.85, "D": 0.15}
SW_SI = {"epsilon": 2.1683, "sigma": 2.0951, "a": 1.80, "gamma": 1.20,
         "lambda": 21.0, "A": 7.049556277, "B": 0.6022245584, "p": 4.0,
         "q": 0.0, "costheta0": -1 / 3}
TERSOFF_XY = [
    {"i": "X", "j": "Y", "k": "Y", "A": 1830.8, "B": 471.18, "lambda1": 2.4799,
     "lambda2": 1.7322, "R": 2.85, "D": 0.15, "beta": 1.1e-6, "n": 0.78734,
     "c": 100390.0, "d": 16.217, "h": -0.59825, "lambda3": 1.7322},
    {"i": "Y", "j": "X", "k": "X", "A": 1500.0, "B": 400.0, "lambda1": 2.2,
     "lambda2": 1.5, "R": 2.85, "D": 0.15, "beta": 0.9e-6, "n": 0.7,
     "c": 90000.0, "d": 14.0, "h": -0.55, "lambda3": 1.5},
]
_TOMITA_KEYS = ("i", "j", "k", "sigma", "a", "lambda", "gamma", "A", "B", "p", "q")
# Tomita et al., Jpn. J. Appl. Phys. 57, 04FB04 (2018), Table I (GeSn SW).
_TOMITA_ROWS = [
    ("Ge", "Ge", "Ge", 2.181, 1.8110, 32.101, 1.1718, 10.093, 0.6862, 4.6973, 0.6588),
    ("Sn", "Sn", "Sn", 2.503, 1.7825, 28.747, 1.1610, 9.4315, 0.7012, 4.9827, 0.6252),
    ("Ge", "Ge", "Sn", 2.337, 1.7988, 29.858, 1.8136, 0.0, 0.0, 0.0, 0.0),
    ("Ge", "Sn", "Ge", 2.337, 1.7988, 29.858, 0.7232, 0.0, 0.0, 0.0, 0.0),
    ("Ge", "Sn", "Sn", 2.337, 1.7988, 24.460, 1.1484, 9.8864, 0.7021, 4.8537, 0.6482),
    ("Sn", "Ge", "Ge", 2.337, 1.7988, 24.460, 1.1484, 9.8864, 0.7021, 4.8537, 0.6482),
    ("Sn", "Ge", "Sn", 2.337, 1.7988, 26.074, 1.3564, 0.0, 0.0, 0.0, 0.0),
    ("Sn", "Sn", "Ge", 2.337, 1.7988, 26.074, 1.0924, 0.0, 0.0, 0.0, 0.0),
]
SW_GESN = [dict(zip(_TOMITA_KEYS, r), epsilon=1.0, costheta0=-0.333333)
           for r in _TOMITA_ROWS]


def cubic(basis, a, n, types, rattle=0.05, seed=0):
    rng = np.random.default_rng(seed)
    cells = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)])
    frac = (np.asarray(basis, float)[None] + cells[:, None]).reshape(-1, 3)
    pos = frac * a + rng.normal(0.0, rattle, frac.shape)
    return np.eye(3) * a * n, pos, list(types) * len(cells)


def strained(lat, pos, amp, seed):
    """L' = L (I + eps), eps symmetric with entries U(-amp, amp); atoms move
    affinely."""
    rng = np.random.default_rng(seed)
    e = rng.uniform(-amp, amp, (3, 3))
    e = 0.5 * (e + e.T)
    M = np.eye(3) + e
    return lat @ M, pos @ M


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--only", default=None, help="write only this section ('fit_eam')")
    args = ap.parse_args()
    sys.path.insert(0, args.reference)
    os.environ.setdefault("NUMBA_CACHE_DIR", "/tmp/numba_cache")
    import akitsushima as ak
    from akitsushima import NeighbourList

    def save(name, **kw):
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **kw)
        print("wrote", name)

    if args.only == "fit_eam":
        fit_eam(save)
        return

    def nl_pairs(lat, pos, r_cut, skin):
        nl = NeighbourList(r_cut=r_cut, skin_width=skin, backend="cll")
        nl.build(lat, pos)
        i, j = nl.get_candidate_pairs()
        return np.asarray(i, np.int32), np.asarray(j, np.int32)

    # ---- neighbour lists -------------------------------------------------
    cases = []
    lat, pos, _ = cubic(DIAMOND, 5.431, 4, ["Si"] * 8, rattle=0.1, seed=3)
    cases.append(("nl_si512_cubic", lat, pos, 3.0, 0.3))
    lat, pos, _ = cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.1, seed=4)
    lat, pos = strained(lat, pos, 0.03, 5)
    cases.append(("nl_si216_triclinic", lat, pos, 3.77118, 0.3))
    # hexagonal (120 degree) 6x6x3 cell of 2-atom hcp, r_list 4.8 A
    a, c = 3.21, 5.21
    hlat = np.array([[a, 0, 0], [-a / 2, a * np.sqrt(3) / 2, 0], [0, 0, c]])
    basis = np.array([[0, 0, 0], [1 / 3, 2 / 3, 0.5]])
    cells = np.array([[i, j, k] for i in range(6) for j in range(6) for k in range(3)])
    frac = (basis[None] + cells[:, None]).reshape(-1, 3) / np.array([6, 6, 3])
    L6 = hlat * np.array([[6], [6], [3]])
    hpos = frac @ L6 + np.random.default_rng(6).normal(0, 0.05, frac.shape)
    cases.append(("nl_hcp216_hexagonal", L6, hpos, 4.5, 0.3))
    lat, pos, _ = cubic(FCC, 3.58, 5, ["Cu"] * 4, rattle=0.08, seed=7)
    cases.append(("nl_fcc500", lat, pos, 5.805810750600001, 0.3))
    for name, lat, pos, rc, skin in cases:
        i, j = nl_pairs(lat, pos, rc, skin)
        save(name, lattice=lat, positions=pos, r_cut=rc, skin=skin, pair_i=i, pair_j=j)

    # ---- potentials ------------------------------------------------------
    def run(name, cfg, lat, pos, types, skin=0.3):
        fn = ak.force_fn_from_config(cfg)
        i, j = nl_pairs(lat, pos, float(fn.r_cut), skin)
        nl = NeighbourList(r_cut=float(fn.r_cut), skin_width=skin, backend="cll")
        nl.build(lat, pos)
        e, f, s = fn(lat, pos, types, nl)
        save(name, lattice=lat, positions=pos, atom_types=np.array(types),
             r_cut=float(fn.r_cut), skin=skin, pair_i=i, pair_j=j,
             energy=float(e), forces=np.asarray(f), stress=np.asarray(s))

    lat, pos, types = cubic(DIAMOND, 5.431, 4, ["Si"] * 8, rattle=0.05, seed=0)
    run("tersoff_si512", {"type": "Tersoff", "species": ["Si"], "params": TERSOFF_SI},
        lat, pos, types)
    lat2, pos2 = strained(*cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.1, seed=11)[:2], 0.03, 12)
    run("tersoff_si216_triclinic", {"type": "Tersoff", "species": ["Si"],
                                    "params": TERSOFF_SI}, lat2, pos2, ["Si"] * 216)
    xy_types = ["X"] * 4 + ["Y"] * 4
    run("tersoff_xy512", {"type": "Tersoff", "species": ["X", "Y"], "params": TERSOFF_XY},
        lat, pos, xy_types * 64)
    from akitsushima.engine.published_parameters import TERSOFF_1989, ZHOU_2004
    el = TERSOFF_1989["elements"]
    sic_cfg = {"type": "Tersoff", "species": ["Si", "C"],
               "params": {"mixing": "tersoff1989",
                          "elements": {s: dict(el[s]) for s in ("Si", "C")},
                          "chi": {"C-Si": TERSOFF_1989["chi"]["C-Si"]}}}
    zb = ["Si"] * 4 + ["C"] * 4
    for n, seed in ((2, 21), (3, 22)):
        lat3, pos3, t3 = cubic(DIAMOND, 4.36, n, zb, rattle=0.1, seed=seed)
        lat3, pos3 = strained(lat3, pos3, 0.02, seed + 100)
        run(f"tersoff1989_sic{len(t3)}", sic_cfg, lat3, pos3, t3)
    lat, pos, types = cubic(DIAMOND, 5.431, 4, ["Si"] * 8, rattle=0.1, seed=0)
    run("sw_si512", {"type": "SW", "species": ["Si"], "params": SW_SI}, lat, pos, types)
    run("sw_si216_triclinic", {"type": "SW", "species": ["Si"], "params": SW_SI},
        lat2, pos2, ["Si"] * 216)
    rng = np.random.default_rng(1)
    latg, posg, tg = cubic(DIAMOND, 5.762, 4, ["Ge"] * 8, rattle=0.1, seed=2)
    tg = [str(x) for x in rng.choice(["Ge", "Sn"], len(tg), p=[0.75, 0.25])]
    run("sw_gesn512", {"type": "SW", "species": ["Ge", "Sn"], "params": SW_GESN},
        latg, posg, tg)
    latf, posf, tf = cubic(FCC, 3.58, 5, ["Cu"] * 4, rattle=0.08, seed=7)
    tf = [str(x) for x in np.random.default_rng(8).choice(["Cu", "Ni"], len(tf))]
    run("eam_cuni500", {"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"],
                        "species": ["Cu", "Ni"]}, latf, posf, tf)
    latn, posn, tn = cubic(FCC, 3.52, 5, ["Ni"] * 4, rattle=0.05, seed=9)
    run("eam_ni500", {"type": "EAM", "form": "zhou2004", "elements": ["Ni"],
                      "species": ["Ni"]}, latn, posn, tn)
    # setfl spline EAM: tabulate Zhou Cu-Ni, read it back (scipy CubicSpline)
    from akitsushima.engine.eam_zhou import read_setfl, write_setfl, zhou_eam
    zpot = zhou_eam({s: ZHOU_2004[s] for s in ("Cu", "Ni")}, ["Cu", "Ni"])
    path = "/tmp/_golden_cuni.eam.alloy"
    write_setfl(path, zpot, ["Cu", "Ni"], n_rho=2000, n_r=2000)
    spot = read_setfl(path)
    fn = ak.make_force_fn(ak.PotentialEngine().add(spot)) if hasattr(ak, "PotentialEngine") \
        else None
    if fn is None:
        from akitsushima.engine.potential_engine import PotentialEngine
        from akitsushima.fitting.force_fn import make_force_fn
        fn = make_force_fn(PotentialEngine().add(spot))
    i, j = nl_pairs(latf, posf, float(spot.r_cut), 0.3)
    nl = NeighbourList(r_cut=float(spot.r_cut), skin_width=0.3, backend="cll")
    nl.build(latf, posf)
    e, f, s = fn(latf, posf, tf, nl)
    tabs = {}
    for kind, dct in (("F", spot._F), ("rho", spot._rho)):
        for sp_ in ("Cu", "Ni"):
            spec = dct[sp_][0]._ak_spec
            tabs[f"{kind}_{sp_}_x"] = spec[1]
            tabs[f"{kind}_{sp_}_c"] = spec[2]
    for a_, b_ in (("Cu", "Cu"), ("Ni", "Cu"), ("Ni", "Ni")):
        spec = spot._phi[frozenset((a_, b_))][0]._ak_spec
        tabs[f"rphi_{a_}{b_}_x"] = spec[1]
        tabs[f"rphi_{a_}{b_}_c"] = spec[2]
    save("eam_setfl_cuni500", lattice=latf, positions=posf, atom_types=np.array(tf),
         r_cut=float(spot.r_cut), skin=0.3, pair_i=i, pair_j=j, energy=float(e),
         forces=np.asarray(f), stress=np.asarray(s), **tabs)

    # ---- NVE molecular dynamics: the reference's own NVESimulation ----------
    import tempfile
    from akitsushima.solvers.molecular_dynamics import NVESimulation
    latm, posm, tm = cubic(DIAMOND, 5.431, 2, ["Si"] * 8, rattle=0.05, seed=0)
    fn = ak.force_fn_from_config({"type": "Tersoff", "species": ["Si"], "params": TERSOFF_SI})
    with tempfile.TemporaryDirectory() as out_dir:
        sim = NVESimulation(latm, posm, tm, force_fn=fn, r_cut=float(fn.r_cut), timestep=1.0,
                            n_steps=20, temperature=300.0, thermo_every=1, traj_every=1000,
                            output_dir=out_dir, skin_width=0.3, seed=7, verbose=False)
        v0 = sim.velocities.copy()
        sim.run()
        thermo = np.loadtxt(os.path.join(out_dir, "thermo.log"), skiprows=1)
    save("md_nve_si64_tersoff", lattice=latm, positions=posm, atom_types=np.array(tm), seed=7,
         temperature=300.0, dt=1.0, n_steps=20, velocities0=v0, positions_final=sim.positions,
         velocities_final=sim.velocities, thermo=thermo)

    # ---- fitting: SiC Tersoff-1989, the reference's loss and its gradient --
    from akitsushima.engine.tersoff import tersoff1989_to_triplets as ref_mix
    from akitsushima.fitting.loss import generic_loss_function, generic_residuals
    from akitsushima.fitting.parameter_sets import (MultiSpeciesTersoffParameterSet,
                                                    Tersoff1989ParameterSet)
    species = ["Si", "C"]
    el0 = {s: dict(el[s]) for s in species}
    chi0 = {"Si-C": TERSOFF_1989["chi"]["C-Si"]}
    rng = np.random.default_rng(31)
    el_t = {s: {k: (v * rng.uniform(0.95, 1.05) if k in ("A", "B", "lambda", "mu", "c", "d", "h") else v)
                for k, v in el0[s].items()} for s in species}
    chi_t = {"Si-C": chi0["Si-C"] * rng.uniform(0.95, 1.05)}
    target = ak.force_fn_from_config({"type": "Tersoff", "species": species,
                                      "params": ref_mix(el_t, chi_t, species)})
    structs, geo = [], {}
    for q, (n, seed) in enumerate(((2, 41), (2, 42), (3, 43), (3, 44))):
        L, P, T = cubic(DIAMOND, 4.36, n, zb, rattle=0.1, seed=seed)
        L, P = strained(L, P, 0.02, seed + 100)
        nl = NeighbourList(r_cut=float(target.r_cut), skin_width=0.3, backend="cll")
        nl.build(L, P)
        e, f, s = target(L, P, T, nl)
        structs.append({"lattice": L, "positions": P, "atom_types": list(T), "natoms": len(P),
                        "ref_energy": float(e) / len(P), "ref_forces": np.asarray(f),
                        "ref_stress": np.asarray(s)})
        geo.update({f"lattice{q}": L, f"positions{q}": P, f"atom_types{q}": np.array(T),
                    f"ref_energy{q}": float(e) / len(P), f"ref_forces{q}": np.asarray(f),
                    f"ref_stress{q}": np.asarray(s)})
    weights = {"energy": 1.0, "forces": 1.0, "stress": 0.1}
    sets = {"t1989": Tersoff1989ParameterSet(el0, chi0, species),
            "multi": MultiSpeciesTersoffParameterSet(ref_mix(el0, chi0, species), species)}
    out = dict(geo, n_structures=len(structs))
    for tag, ps in sets.items():
        x0 = ps.x0
        lo_b = np.array([b[0] for b in ps.bounds])
        hi_b = np.array([b[1] for b in ps.bounds])
        r0 = generic_residuals(x0, ps, structs, weights, 3.5, None)
        J = np.empty((len(r0), len(x0)))
        for q in range(len(x0)):   # the fit's jacobian_fn (fitting/driver.py:802-816)
            h = 1e-7 * max(1.0, abs(x0[q]))
            if x0[q] + h > hi_b[q]:
                h = -h
            xp = np.array(x0, float)
            xp[q] += h
            J[:, q] = (generic_residuals(xp, ps, structs, weights, 3.5, None) - r0) / h
        x_test = x0 + np.random.default_rng(32).uniform(-0.02, 0.02, len(x0))
        x_test = np.clip(x_test, lo_b, hi_b)
        tab = ps.decode(x_test)["tersoff"]
        keys = sorted(tab)
        out.update({f"{tag}_x0": x0, f"{tag}_names": np.array(ps.variable_names),
                    f"{tag}_lo": lo_b, f"{tag}_hi": hi_b,
                    f"{tag}_loss0": generic_loss_function(x0, ps, structs, weights, 3.5, None),
                    f"{tag}_grad_fd": 2.0 * J.T @ r0, f"{tag}_x_test": x_test,
                    f"{tag}_loss_test": generic_loss_function(x_test, ps, structs, weights, 3.5, None),
                    f"{tag}_decoded_keys": np.array(["|".join(k) for k in keys]),
                    f"{tag}_decoded": np.array([[float(tab[k].get(n, np.nan)) for n in
                                                 ("A", "B", "lambda1", "lambda2", "R", "D", "beta", "n",
                                                  "c", "d", "h", "lambda3", "m", "gamma")] for k in keys])})
    save("fit_sic_t1989", **out)

    fit_eam(save)

    # ---- site terms (heat flux): the reference's engine/site_terms.py -----------
    from akitsushima.engine.site_terms import eam_site_terms, sw_site_terms, tersoff_site_terms
    cases = [
        ("sites_tersoff_si216", {"type": "Tersoff", "species": ["Si"], "params": TERSOFF_SI},
         cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.08, seed=51), tersoff_site_terms),
        ("sites_tersoff1989_sic216", sic_cfg, cubic(DIAMOND, 4.36, 3, zb, rattle=0.08, seed=52),
         tersoff_site_terms),
        ("sites_sw_si216", {"type": "SW", "species": ["Si"], "params": SW_SI},
         cubic(DIAMOND, 5.431, 3, ["Si"] * 8, rattle=0.08, seed=53), sw_site_terms),
        ("sites_eam_cuni256", {"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"],
                               "species": ["Cu", "Ni"]},
         cubic(FCC, 3.58, 4, ["Cu", "Ni", "Cu", "Ni"], rattle=0.08, seed=54), eam_site_terms),
    ]
    for name, cfg, (L, P, T), fun in cases:
        fn = ak.force_fn_from_config(cfg)
        pot = fn.engine._potentials[0]
        st = fun(pot, L, P, list(T))
        vel = np.random.default_rng(55).normal(0, 0.01, P.shape)
        save(name, lattice=L, positions=P, atom_types=np.array(T), e_site=st.e_site, centre=st.centre,
             nbr=st.nbr, vec=st.vec, dUdv=st.dUdv, velocities=vel, virial_flux=st.virial_flux(vel),
             stress=st.stress(abs(np.linalg.det(L))), forces=st.forces())


def fit_eam(save):
    """Zhou (2004) Al-Ni EAM fit: the reference's ZhouEAMParameterSet, its
    loss (fitting/loss.py:51) and the forward-difference gradient of its
    fit (fitting/driver.py:802-816) on two rattled, strained L1_2 Ni3Al
    cells whose targets come from a perturbed parameter set."""
    from akitsushima.engine.published_parameters import ZHOU_2004
    from akitsushima.fitting.loss import generic_loss_function, generic_residuals
    from akitsushima.fitting.parameter_sets import ZhouEAMParameterSet
    species = ["Al", "Ni"]
    el0 = {s: dict(ZHOU_2004[s]) for s in species}
    rng = np.random.default_rng(61)
    el_t = {s: {k: (v * rng.uniform(0.97, 1.03) if k in ("A", "B", "alpha", "beta", "F2", "F3", "eta") else v)
                for k, v in el0[s].items()} for s in species}
    target = ZhouEAMParameterSet(el_t, species, chi={"Al-Ni": 1.04})
    eng = target.build_engine(target.decode(target.x0))
    structs, geo = [], {}
    for q, (n, seed) in enumerate(((4, 62), (5, 63))):
        L, P, T = cubic(FCC, 3.57, n, ["Al", "Ni", "Ni", "Ni"], rattle=0.06, seed=seed)
        L, P = strained(L, P, 0.015, seed + 100)
        e, f, s = eng.compute(L, P, list(T))
        structs.append({"lattice": L, "positions": P, "atom_types": list(T), "natoms": len(P),
                        "ref_energy": float(e) / len(P), "ref_forces": np.asarray(f),
                        "ref_stress": np.asarray(s)})
        geo.update({f"lattice{q}": L, f"positions{q}": P, f"atom_types{q}": np.array(T),
                    f"ref_energy{q}": float(e) / len(P), f"ref_forces{q}": np.asarray(f),
                    f"ref_stress{q}": np.asarray(s)})
    weights = {"energy": 1.0, "forces": 1.0, "stress": 1.0, "r0": 0.1, "eps0": 0.01}
    out = dict(geo, n_structures=len(structs))
    for tag, ps in (("zhou", ZhouEAMParameterSet(el0, species)),
                    ("zhou_chi", ZhouEAMParameterSet(el0, species, fit_keys=["A", "B", "F2", "eta", "chi"]))):
        x0 = ps.x0
        lo_b = np.array([b[0] for b in ps.bounds])
        hi_b = np.array([b[1] for b in ps.bounds])
        r0 = generic_residuals(x0, ps, structs, weights, ps.r_cut, None)
        J = np.empty((len(r0), len(x0)))
        for q in range(len(x0)):   # the fit's jacobian_fn (fitting/driver.py:802-816)
            h = 1e-7 * max(1.0, abs(x0[q]))
            if x0[q] + h > hi_b[q]:
                h = -h
            xp = np.array(x0, float)
            xp[q] += h
            J[:, q] = (generic_residuals(xp, ps, structs, weights, ps.r_cut, None) - r0) / h
        x_test = np.clip(x0 + np.random.default_rng(64).uniform(-0.02, 0.02, len(x0)), lo_b, hi_b)
        dec = ps.decode(x_test)["eam"]
        out.update({f"{tag}_x0": x0, f"{tag}_names": np.array(ps.variable_names), f"{tag}_lo": lo_b,
                    f"{tag}_hi": hi_b, f"{tag}_r_cut": ps.r_cut,
                    f"{tag}_loss0": generic_loss_function(x0, ps, structs, weights, ps.r_cut, None),
                    f"{tag}_grad_fd": 2.0 * J.T @ r0, f"{tag}_x_test": x_test,
                    f"{tag}_loss_test": generic_loss_function(x_test, ps, structs, weights, ps.r_cut, None),
                    f"{tag}_decoded_keys": np.array(list(dec["elements"]["Al"])),
                    f"{tag}_decoded": np.array([[dec["elements"][s][k] for k in dec["elements"]["Al"]]
                                                for s in species]),
                    f"{tag}_decoded_chi": dec["chi"]["Al-Ni"]})
    save("fit_alni_zhou", **out)


if __name__ == "__main__":
    main()
