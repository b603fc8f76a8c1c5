"""Displacement and strain sets of the phonon and elastic solvers, evaluated
as one batch.

The reference's solvers make one force call per configuration: the phonon
force-constant columns (solvers/phonon.py:411-438, and the symmetry-reduced
displacements of :611-628) and the clamped-ion strain points of the elastic
constants (solvers/elastic.py:222-252).  Here the whole set is one batch:
every configuration a structure of a BatchedEvaluator, one neighbour-list
build and one launch sequence per potential, results mapped back per
configuration.  The arithmetic of each configuration is the single-call
path's, so results equal the per-call ones to rounding of the reductions.
"""
import numpy as np

from .batched import BatchedEvaluator

EV_ANG3_TO_GPA = 160.2176621          # constants.py:51 of the reference
VOIGT_PAIRS = ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))   # solvers/elastic.py:46


def _potentials(backend):
    """The potentials behind a force function of this package, a
    PotentialEngine or a single potential."""
    eng = getattr(backend, "engine", None)
    if eng is not None:
        return list(eng.potentials)
    if hasattr(backend, "potentials"):
        return list(backend.potentials)
    return [backend]


def evaluate_many(backend, structures, need_stress=True, skin=0.3, precision=None, device=None):
    """[(energy, forces (N, 3), stress (3, 3) or None)] for every
    (lattice, positions, atom_types) of ``structures``, one batch per
    potential (their sum, as PotentialEngine.compute, engine/potential_engine.py:76-105)."""
    structures = [(np.asarray(l, float), np.asarray(p, float), list(t)) for l, p, t in structures]
    if not structures:
        return []
    e = f = s = None
    for pot in _potentials(backend):
        ev = BatchedEvaluator(pot, structures, skin=skin, precision=precision, device=device)
        e1, f1, s1 = ev.results()
        if e is None:
            e, f, s = e1, f1, s1
        else:
            e = e + e1
            f = [a + b for a, b in zip(f, f1)]
            s = s + s1
    return [(float(e[k]), f[k], s[k] if need_stress else None) for k in range(len(structures))]


def ifc_columns(backend, lattice_sc, positions_sc, atom_types_sc, tasks, delta=0.01, **kw):
    """Force-constant columns -(F(r + delta e_b) - F(r - delta e_b)) / (2 delta)
    for every task (atom j, axis b) -- the reference's _eval_displacement
    (solvers/phonon.py:411-438) -- all 2 len(tasks) displaced supercells in
    one batch.  Returns (len(tasks), N, 3)."""
    pos0 = np.asarray(positions_sc, float)
    structs = []
    for j, b in tasks:
        p = pos0.copy()
        p[j, b] += delta
        m = pos0.copy()
        m[j, b] -= delta
        structs += [(lattice_sc, p, atom_types_sc), (lattice_sc, m, atom_types_sc)]
    res = evaluate_many(backend, structs, need_stress=False, **kw)
    out = np.empty((len(tasks), len(pos0), 3))
    for t in range(len(tasks)):
        out[t] = -(res[2 * t][1] - res[2 * t + 1][1]) / (2.0 * delta)
    return out


def displaced_forces(backend, lattice_sc, positions_sc, atom_types_sc, displacements, **kw):
    """Forces of the supercell with atom j moved by d (3,), for every (j, d)
    -- the symmetry-reduced displacement set of solvers/phonon.py:611-628.
    Returns (len(displacements), N, 3)."""
    pos0 = np.asarray(positions_sc, float)
    structs = []
    for j, d in displacements:
        p = pos0.copy()
        p[j] += np.asarray(d, float)
        structs.append((lattice_sc, p, atom_types_sc))
    res = evaluate_many(backend, structs, need_stress=False, **kw)
    return np.stack([r[1] for r in res]) if res else np.zeros((0, len(pos0), 3))


def strain_matrix(voigt_idx, magnitude):
    """Symmetric strain of one Voigt mode, engineering shear
    (solvers/elastic.py:60-72)."""
    eps = np.zeros((3, 3))
    a, b = VOIGT_PAIRS[voigt_idx]
    if a == b:
        eps[a, b] = magnitude
    else:
        eps[a, b] = eps[b, a] = magnitude / 2.0
    return eps


def clamped_elastic_constants(backend, lattice, positions, atom_types, strains=(0.005, 0.01), **kw):
    """Clamped-ion elastic tensor [GPa] from the reference's strain points:
    the unstrained cell and every Voigt mode at +-each amplitude, fractional
    coordinates fixed (solvers/elastic.py:222-252), C0_ij = -d sigma_i /
    d eta_j from a straight-line least-squares fit per mode (:300-315), all
    points evaluated as one batch.  Returns (C0 (6, 6), stresses, points)."""
    lat0 = np.asarray(lattice, float)
    frac0 = np.asarray(positions, float) @ np.linalg.inv(lat0)
    pts = [(None, 0.0)] + [(j, sg * s) for j in range(6) for s in strains for sg in (+1.0, -1.0)]
    structs = []
    for j, s in pts:
        lat = lat0.copy() if j is None else lat0 @ (np.eye(3) + strain_matrix(j, s))
        structs.append((lat, frac0 @ lat, atom_types))
    res = evaluate_many(backend, structs, need_stress=True, **kw)
    sig = [r[2] for r in res]
    C0 = np.zeros((6, 6))
    for j in range(6):
        idx = [0] + [k for k, (jj, _) in enumerate(pts) if jj == j]
        eta = np.array([pts[k][1] for k in idx])
        A = np.column_stack([eta, np.ones_like(eta)])
        y = np.array([-np.array([sig[k][a, b] for a, b in VOIGT_PAIRS]) for k in idx]) * EV_ANG3_TO_GPA
        coef, *_ = np.linalg.lstsq(A, y, rcond=None)
        C0[:, j] = coef[0]
    return C0, sig, pts
