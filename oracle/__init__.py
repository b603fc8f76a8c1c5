"""CPU oracle for the many-body force path -- TEST INFRASTRUCTURE ONLY.

A restatement of the reference's (akitsushima 0.4.0a4) CPU algorithm for the
neighbour list and the Tersoff / Stillinger-Weber / EAM energy + force +
virial evaluation:

* ``oracle.c`` (built into ``liboracle.so``) restates the numba kernels;
* this module restates the numpy code around them -- the minimum-image
  recompute and cutoff mask, the two-way CSR, the bond order, the species
  tables and the Zhou (2004) EAM set-up -- citing the reference file:line.

Pinning: every function here is checked against golden vectors produced by
the reference itself (``tests/golden/make_golden.py`` imports the reference
and writes ``tests/golden/*.npz``) and against the reference's own ledger
energies (``benchmarks/adr0047.jsonl``); see ``tests/test_oracle_golden.py``.

Who may use it: ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline / reference leg, as the checker or the timed CPU baseline.  The
product package ``akitsushima_b200`` never imports it.
"""
import ctypes
import math
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None
_lib_lock = threading.Lock()

_dp = ctypes.POINTER(ctypes.c_double)
_lp = ctypes.POINTER(ctypes.c_long)
_ip = ctypes.POINTER(ctypes.c_int)
_bp = ctypes.POINTER(ctypes.c_ubyte)
_L = ctypes.c_long
_D = ctypes.c_double


def build():
    """Compile ``liboracle.so`` (gcc, OpenMP) with the Makefile beside it."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(_LIB_PATH) or (
                    os.path.getmtime(_LIB_PATH)
                    < os.path.getmtime(os.path.join(_HERE, "oracle.c"))):
                build()
            _lib = ctypes.CDLL(_LIB_PATH)
            _lib.orc_cll_pairs.restype = _L
            _lib.orc_te_multi_pass3.restype = _D
            _lib.orc_sw_2body.restype = _D
            _lib.orc_sw_3body.restype = _D
            _lib.orc_sw_multi_2body.restype = _D
            _lib.orc_sw_multi_3body.restype = _D
            _lib.orc_eam_kernel.restype = _D
            _lib.orc_num_threads.restype = ctypes.c_int
        return _lib


def set_threads(n):
    """OpenMP threads of the oracle kernels (the reference's numba threads)."""
    lib().orc_set_threads(int(n))


def num_threads():
    return int(lib().orc_num_threads())


def _d(a):
    return a.ctypes.data_as(_dp)


def _l(a):
    return a.ctypes.data_as(_lp)


def _i(a):
    return a.ctypes.data_as(_ip)


def _b(a):
    return a.ctypes.data_as(_bp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)


# ---------------------------------------------------------------------------
#  Neighbour list (engine/neighborlist.py)
# ---------------------------------------------------------------------------

def cell_metrics(lattice):
    """engine/neighborlist.py:170-267: perpendicular widths and sigma_min."""
    lat = np.asarray(lattice, dtype=float)
    volume = abs(float(np.linalg.det(lat)))
    cross = np.array([np.linalg.norm(np.cross(lat[(i + 1) % 3], lat[(i + 2) % 3]))
                      for i in range(3)])
    if volume <= 0.0 or not np.all(cross > 0.0):
        raise ValueError("degenerate (singular) lattice")
    return volume / cross, float(np.linalg.svd(lat, compute_uv=False)[-1])


def check_min_cell(lattice, r_list):
    """engine/neighborlist.py:489-572: refuse r_list >= min width / 2."""
    widths, _ = cell_metrics(lattice)
    if r_list >= float(np.min(widths)) / 2.0:
        raise ValueError("r_cut + skin_width must be < half the smallest "
                         "perpendicular cell width")


def _axis_offsets(nc):
    """engine/neighborlist.py:270-299."""
    if nc == 1:
        return (0,)
    if nc == 2:
        return (0, 1)
    return (-1, 0, 1)


def nl_build(lattice, positions, r_cut, skin=0.5):
    """Candidate pairs within r_cut + skin in canonical order.

    engine/neighborlist.py:574-585 (build), :935-1024 (_build_cell_linked)
    and :1166-1181 (_canonical_pair_order).  Returns (i, j) int32 with i < j
    sorted by (i, j), plus the pair displacements and distances.
    """
    lattice = _f64(lattice)
    positions = _f64(positions)
    r_list = r_cut + skin
    check_min_cell(lattice, r_list)
    N = len(positions)
    inv_lat = np.linalg.inv(lattice)
    widths, _ = cell_metrics(lattice)
    nc = np.maximum(1, np.floor(widths / r_list).astype(int))
    frac = positions @ inv_lat
    frac = frac - np.floor(frac)
    cell_idx = np.clip(np.floor(frac * nc).astype(np.int64), 0, nc - 1)
    nc0, nc1, nc2 = (int(x) for x in nc)
    flat = cell_idx[:, 0] * nc1 * nc2 + cell_idx[:, 1] * nc2 + cell_idx[:, 2]
    # linked list, atoms pushed from N-1 down to 0 (head holds the lowest)
    head = -np.ones(nc0 * nc1 * nc2, dtype=np.int64)
    nxt = -np.ones(N, dtype=np.int64)
    order = np.argsort(flat, kind="stable")
    # the reference's loop `for atom in range(N-1, -1, -1)` leaves each cell's
    # list in ascending atom order; build the same lists without the loop
    sf = flat[order]
    first = np.r_[True, sf[1:] != sf[:-1]]
    head[sf[first]] = order[first]
    same_next = np.r_[sf[1:] == sf[:-1], False]
    nxt[order[same_next]] = order[1:][same_next[:-1]] if N > 1 else []
    offs = np.array([(a, b, c) for a in _axis_offsets(nc0) for b in _axis_offsets(nc1)
                     for c in _axis_offsets(nc2)], dtype=np.int64)
    cidx = _i64(cell_idx)
    L = lib()
    args = [_L(N), _L(nc0), _L(nc1), _L(nc2), _l(cidx), _l(offs), _L(len(offs)),
            _l(head), _l(nxt), _d(positions), _d(lattice), _d(_f64(inv_lat)),
            _D(r_list ** 2)]
    e_i = np.empty(0, np.int32)
    e_d = np.empty(0, np.float64)
    n = L.orc_cll_pairs(*args, _i(e_i), _i(e_i), _d(e_d), _d(e_d), ctypes.c_int(1))
    out_i = np.empty(n, np.int32)
    out_j = np.empty(n, np.int32)
    out_rij = np.empty((n, 3), np.float64)
    out_r = np.empty(n, np.float64)
    L.orc_cll_pairs(*args, _i(out_i), _i(out_j), _d(out_rij), _d(out_r), ctypes.c_int(0))
    # canonical order (i < j already holds for the cell list)
    key = out_i.astype(np.int64) * (int(out_j.max(initial=0)) + 1) + out_j
    o = np.argsort(key, kind="stable")
    return out_i[o].copy(), out_j[o].copy(), out_rij[o].copy(), out_r[o].copy()


def brute_force_pairs(lattice, positions, r_list):
    """O(N^2) minimum-image pair set (tests/test_neighborlist.py:27-42 style)."""
    lattice = _f64(lattice)
    positions = _f64(positions)
    inv = np.linalg.inv(lattice)
    ii, jj = np.triu_indices(len(positions), k=1)
    s = (positions[jj] - positions[ii]) @ inv
    s -= np.round(s)
    d = s @ lattice
    r = np.sqrt((d * d).sum(1))
    keep = (r < r_list) & (r > 1e-10)
    return ii[keep].astype(np.int32), jj[keep].astype(np.int32)


# ---------------------------------------------------------------------------
#  Shared potential preparation
# ---------------------------------------------------------------------------

def mic_mask(lattice, positions, idx_i, idx_j, rc):
    """engine/tersoff.py:1276-1291: fresh minimum-image displacements of the
    candidate pairs and the r < rc, r > 1e-12 mask."""
    lattice = _f64(lattice)
    positions = _f64(positions)
    if len(idx_i) == 0:
        return (np.empty(0, np.int64), np.empty(0, np.int64), np.empty((0, 3)),
                np.empty(0))
    inv = np.linalg.inv(lattice)
    dr = positions[idx_j] - positions[idx_i]
    s = dr @ inv
    s -= np.round(s)
    rij = s @ lattice
    r = np.linalg.norm(rij, axis=1)
    m = (r < rc) & (r > 1e-12)
    return (_i64(idx_i[m]), _i64(idx_j[m]), np.ascontiguousarray(rij[m]),
            np.ascontiguousarray(r[m]))


def two_way_csr(N, idx_i, idx_j, rij, r):
    """engine/tersoff.py:1297-1307: directed neighbour CSR by stable argsort
    of the source atom (row a = its j > a partners, then its i < a ones)."""
    src = np.concatenate([idx_i, idx_j])
    dst = np.concatenate([idx_j, idx_i])
    rdir = np.concatenate([rij, -rij])
    dist = np.concatenate([r, r])
    order = np.argsort(src, kind="stable")
    cnt = np.bincount(src[order], minlength=N)
    start = np.zeros(N + 1, np.int64)
    start[1:] = np.cumsum(cnt)
    return (start, _i64(dst[order]), np.ascontiguousarray(rdir[order]),
            np.ascontiguousarray(dist[order]))


def _volume(lattice):
    return float(abs(np.linalg.det(np.asarray(lattice, float))))


def _all_pairs(N):
    ii, jj = np.triu_indices(N, k=1)
    return ii.astype(np.int32), jj.astype(np.int32)


# ---------------------------------------------------------------------------
#  Tersoff (engine/tersoff.py)
# ---------------------------------------------------------------------------

def tersoff_single(params, lattice, positions, pairs=None):
    """engine/tersoff.py:1233-1513 (_compute_single_species, numba branch)."""
    positions = _f64(positions)
    N = len(positions)
    p = {k: float(v) for k, v in params.items() if not isinstance(v, str)}
    A, B = p["A"], p["B"]
    l1, l2, l3 = p["lambda1"], p["lambda2"], p["lambda3"]
    beta, n, c, d, h = p["beta"], p["n"], p["c"], p["d"], p["h"]
    R, D = p.get("R", 2.85), p.get("D", 0.15)
    rc = R + D
    ii, jj = pairs if pairs is not None else _all_pairs(N)
    ii, jj, rij, r = mic_mask(lattice, positions, ii, jj, rc)
    if len(ii) == 0:
        return 0.0, np.zeros((N, 3)), np.zeros((3, 3))
    nb_start, nb_idx, nb_rij, nb_r = two_way_csr(N, ii, jj, rij, r)
    P = len(ii)
    zij = np.zeros(P)
    zji = np.zeros(P)
    lib().orc_te_zeta(_L(P), _l(ii), _l(jj), _d(rij), _d(r), _l(nb_start), _l(nb_idx),
                      _d(nb_rij), _d(nb_r), _d(zij), _d(zji), _D(l3), _D(c), _D(d),
                      _D(h), _D(R), _D(D))

    def bij(z):
        return np.where(z > 0, (1.0 + (beta * z) ** n) ** (-0.5 / n), 1.0)

    def dbij(z, b):
        safe = np.where(z > 0, z, 1.0)
        bz = (beta * safe) ** n
        return np.where(z > 0, -0.5 * b * bz / (safe * (1.0 + bz)), 0.0)

    b_ij, b_ji = bij(zij), bij(zji)
    db_ij, db_ji = dbij(zij, b_ij), dbij(zji, b_ji)
    fc = np.where(r < R - D, 1.0, np.where(r > R + D, 0.0,
                  0.5 - 0.5 * np.sin(0.5 * np.pi * (r - R) / D)))
    dfc = np.where(r < R - D, 0.0, np.where(r > R + D, 0.0,
                   -0.25 * np.pi / D * np.cos(0.5 * np.pi * (r - R) / D)))
    fr = A * np.exp(-l1 * r)
    fa = -B * np.exp(-l2 * r)
    bavg = 0.5 * (b_ij + b_ji)
    energy = float((fc * (fr + bavg * fa)).sum())
    dEdr = dfc * (fr + bavg * fa) + fc * (-l1 * fr + bavg * (-l2 * fa))
    fij = (dEdr / r)[:, None] * rij
    forces = np.zeros((N, 3))
    np.add.at(forces, ii, fij)
    np.add.at(forces, jj, -fij)
    stress = -np.einsum("ki,kj->ij", fij, rij)
    stress = np.ascontiguousarray(stress)
    lib().orc_te_3body(_L(0), _L(P), _L(N), _l(ii), _l(jj), _d(rij), _d(r),
                       _d(_f64(fc)), _d(_f64(fa)), _d(db_ij), _d(db_ji), _l(nb_start),
                       _l(nb_idx), _d(nb_rij), _d(nb_r), _d(forces), _d(stress),
                       _D(R), _D(D), _D(c), _D(d), _D(h), _D(l3), _D(3.0))
    return energy, forces, stress / _volume(lattice)


class _TeTables(ctypes.Structure):
    _fields_ = [("ns", _L), ("tb_valid", _bp)] + \
        [(k, _dp) for k in ("tb_A", "tb_B", "tb_l1", "tb_l2", "tb_R", "tb_D")] + \
        [("tri_valid", _bp)] + \
        [(k, _dp) for k in ("tri_c", "tri_d", "tri_h", "tri_l3", "tri_m", "tri_gam")]


def tersoff_tables(records, species):
    """engine/tersoff.py:1606-1653: dense (ns, ns) and (ns, ns, ns) tables."""
    ns = len(species)
    T = {"tb_valid": np.zeros((ns, ns), np.uint8)}
    for k, dflt in (("A", 0.0), ("B", 0.0), ("lambda1", 0.0), ("lambda2", 0.0),
                    ("R", 1.0), ("D", 1.0), ("beta", 0.0), ("n", 1.0)):
        T["tb_" + k] = np.full((ns, ns), dflt)
    for a, sa in enumerate(species):
        for b, sb in enumerate(species):
            rec = records.get((sa, sb, sb))
            if rec is None:
                continue
            T["tb_valid"][a, b] = 1
            for k, dflt in (("A", 0.0), ("B", 0.0), ("lambda1", 0.0), ("lambda2", 0.0),
                            ("R", 1.0), ("D", 1.0), ("beta", 0.0), ("n", 1.0)):
                T["tb_" + k][a, b] = float(rec.get(k, dflt))
    T["tri_valid"] = np.zeros((ns, ns, ns), np.uint8)
    for k, dflt in (("c", 0.0), ("d", 1.0), ("h", 0.0), ("lambda3", 0.0), ("m", 3.0),
                    ("gamma", 1.0)):
        T["tri_" + k] = np.full((ns, ns, ns), dflt)
    for a, sa in enumerate(species):
        for b, sb in enumerate(species):
            for c, sc in enumerate(species):
                rec = records.get((sa, sb, sc))
                if rec is None:
                    continue
                T["tri_valid"][a, b, c] = 1
                for k in ("c", "d", "h", "lambda3"):
                    T["tri_" + k][a, b, c] = float(rec[k])
                T["tri_m"][a, b, c] = float(rec.get("m", 3.0))
                T["tri_gamma"][a, b, c] = float(rec.get("gamma", 1.0))
    return {k: np.ascontiguousarray(v) for k, v in T.items()}


def _te_struct(T, ns):
    return _TeTables(ns, _b(T["tb_valid"]), _d(T["tb_A"]), _d(T["tb_B"]),
                     _d(T["tb_lambda1"]), _d(T["tb_lambda2"]), _d(T["tb_R"]),
                     _d(T["tb_D"]), _b(T["tri_valid"]), _d(T["tri_c"]), _d(T["tri_d"]),
                     _d(T["tri_h"]), _d(T["tri_lambda3"]), _d(T["tri_m"]),
                     _d(T["tri_gamma"]))


def tersoff_r_cut(records):
    """engine/tersoff.py:1162-1167."""
    rc = 0.0
    for (i, j, k), v in records.items():
        if j == k and "R" in v and "D" in v:
            rc = max(rc, float(v["R"]) + float(v["D"]))
    return rc if rc > 0 else 3.0


def tersoff_multi(records, species, lattice, positions, atom_types, pairs=None):
    """engine/tersoff.py:1518-1711 (_compute_multi_species, numba branch)."""
    positions = _f64(positions)
    N = len(positions)
    ns = len(species)
    rc = tersoff_r_cut(records)
    index = {s: k for k, s in enumerate(species)}
    tids = np.array([index[t] for t in atom_types], np.int64)
    ii, jj = pairs if pairs is not None else _all_pairs(N)
    ii, jj, rij, r = mic_mask(lattice, positions, ii, jj, rc)
    if len(ii) == 0:
        return 0.0, np.zeros((N, 3)), np.zeros((3, 3))
    nb_start, nb_idx, nb_rij, nb_r = two_way_csr(N, ii, jj, rij, r)
    T = tersoff_tables(records, species)
    st = _te_struct(T, ns)
    P = len(ii)
    zij = np.zeros(P)
    zji = np.zeros(P)
    lib().orc_te_multi_zeta(_L(P), _l(ii), _l(jj), _d(rij), _d(r), _l(tids), _l(nb_start),
                            _l(nb_idx), _d(nb_rij), _d(nb_r), _d(zij), _d(zji),
                            ctypes.byref(st))
    si, sj = tids[ii], tids[jj]
    valid = T["tb_valid"][si, sj].astype(bool)
    b_ij, b_ji = np.ones(P), np.ones(P)
    db_ij, db_ji = np.zeros(P), np.zeros(P)
    for z, bet, nn, bo, dbo in ((zij, T["tb_beta"][si, sj], T["tb_n"][si, sj], b_ij, db_ij),
                                (zji, T["tb_beta"][sj, si], T["tb_n"][sj, si], b_ji, db_ji)):
        m = valid & (z > 0) & (bet != 0.0)
        zz, be, ne = z[m], bet[m], nn[m]
        bz = (be * zz) ** ne
        b = (1.0 + bz) ** (-0.5 / ne)
        bo[m] = b
        dbo[m] = -0.5 * b * bz / (zz * (1.0 + bz))
    forces = np.zeros((N, 3))
    stress = np.zeros((3, 3))
    energy = lib().orc_te_multi_pass3(
        _L(0), _L(P), _L(N), _l(ii), _l(jj), _d(rij), _d(r), _l(tids), _d(b_ij),
        _d(b_ji), _d(db_ij), _d(db_ji), _l(nb_start), _l(nb_idx), _d(nb_rij), _d(nb_r),
        _d(forces), _d(stress), ctypes.byref(st))
    return float(energy), forces, stress / _volume(lattice)


TERSOFF1989_KEYS = ("A", "B", "lambda", "mu", "beta", "n", "c", "d", "h", "R", "S")


def tersoff1989_to_triplets(elements, chi, species=None, omega=None):
    """engine/tersoff.py:1968-2034: Tersoff (1989) mixing rules -> records."""
    species = list(species) if species is not None else list(elements)
    omega = omega or {}

    def pk(a, b, table, default):
        for key in (f"{a}-{b}", f"{b}-{a}"):
            if key in table:
                return float(table[key])
        return default

    out = {}
    for i in species:
        pi = elements[i]
        for j in species:
            pj = elements[j]
            x = 1.0 if i == j else pk(i, j, chi, None)
            if x is None:
                raise ValueError(f"chi for {i}-{j} not given")
            r_ij = math.sqrt(float(pi["R"]) * float(pj["R"]))
            s_ij = math.sqrt(float(pi["S"]) * float(pj["S"]))
            for k in species:
                rec = {"c": float(pi["c"]), "d": float(pi["d"]), "h": float(pi["h"]),
                       "lambda3": 0.0, "m": 3.0, "gamma": pk(i, k, omega, 1.0)}
                if j == k:
                    rec.update(A=math.sqrt(float(pi["A"]) * float(pj["A"])),
                               B=x * math.sqrt(float(pi["B"]) * float(pj["B"])),
                               lambda1=0.5 * (float(pi["lambda"]) + float(pj["lambda"])),
                               lambda2=0.5 * (float(pi["mu"]) + float(pj["mu"])),
                               R=0.5 * (r_ij + s_ij), D=0.5 * (s_ij - r_ij),
                               beta=float(pi["beta"]), n=float(pi["n"]))
                out[(i, j, k)] = rec
    return out


# ---------------------------------------------------------------------------
#  Stillinger-Weber (engine/stillinger_weber.py)
# ---------------------------------------------------------------------------

SW_SI_DEFAULTS = {"epsilon": 2.1682, "sigma": 2.0951, "A": 7.049556, "B": 0.6022246,
                  "p": 4.0, "q": 0.0, "a": 1.80, "lambda": 21.0, "gamma": 1.20,
                  "costheta0": -1.0 / 3.0}


def sw_single(params, lattice, positions, pairs=None):
    """engine/stillinger_weber.py:927-1159 (single species, numba branch)."""
    positions = _f64(positions)
    N = len(positions)
    p = dict(SW_SI_DEFAULTS)
    p.update({k: float(v) for k, v in params.items()})
    rc = p["a"] * p["sigma"]
    ii, jj = pairs if pairs is not None else _all_pairs(N)
    ii, jj, rij, r = mic_mask(lattice, positions, ii, jj, rc)
    if len(ii) == 0:
        return 0.0, np.zeros((N, 3)), np.zeros((3, 3))
    nb_start, nb_idx, nb_rij, nb_r = two_way_csr(N, ii, jj, rij, r)
    forces = np.zeros((N, 3))
    stress = np.zeros((3, 3))
    L = lib()
    e2 = L.orc_sw_2body(_L(len(ii)), _L(N), _l(ii), _l(jj), _d(rij), _d(r), _d(forces),
                        _d(stress), _D(p["epsilon"]), _D(p["sigma"]), _D(p["A"]),
                        _D(p["B"]), _D(p["p"]), _D(p["q"]), _D(p["a"]))
    e3 = L.orc_sw_3body(_L(0), _L(N), _L(N), _l(nb_start), _l(nb_idx), _d(nb_rij),
                        _d(nb_r), _d(forces), _d(stress), _D(p["epsilon"]),
                        _D(p["sigma"]), _D(p["a"]), _D(p["gamma"]), _D(p["lambda"]),
                        _D(p["costheta0"]))
    return float(e2 + e3), forces, stress / _volume(lattice)


def sw_r_cut(records):
    """engine/stillinger_weber.py:867-871."""
    rc = 0.0
    for (i, j, k), v in records.items():
        if j == k:
            rc = max(rc, float(v["a"]) * float(v["sigma"]))
    return rc if rc > 0 else 4.0


def sw_tables(records, species):
    """engine/stillinger_weber.py:1264-1313: dense species tables."""
    ns = len(species)
    T = {"tb_valid": np.zeros((ns, ns), np.uint8), "tb_eps": np.zeros((ns, ns)),
         "tb_sig": np.ones((ns, ns)), "tb_a": np.zeros((ns, ns)), "tb_A": np.zeros((ns, ns)),
         "tb_B": np.zeros((ns, ns)), "tb_p": np.zeros((ns, ns)), "tb_q": np.zeros((ns, ns)),
         "tri_valid": np.zeros((ns, ns, ns), np.uint8), "tri_eps": np.zeros((ns, ns, ns)),
         "tri_lam": np.zeros((ns, ns, ns)), "tri_cos": np.full((ns, ns, ns), -1.0 / 3.0),
         "leg_sig": np.ones((ns, ns)), "leg_a": np.zeros((ns, ns)),
         "leg_gam": np.zeros((ns, ns))}
    for a, sa in enumerate(species):
        for b, sb in enumerate(species):
            tb = records.get((sa, sb, sb))
            if tb is not None:
                T["leg_sig"][a, b] = float(tb["sigma"])
                T["leg_a"][a, b] = float(tb["a"])
                T["leg_gam"][a, b] = float(tb["gamma"])
            if tb is None or float(tb.get("A", 0.0)) == 0.0:
                continue
            T["tb_valid"][a, b] = 1
            T["tb_eps"][a, b] = float(tb.get("epsilon", 1.0))
            T["tb_sig"][a, b] = float(tb["sigma"])
            T["tb_a"][a, b] = float(tb["a"])
            T["tb_A"][a, b] = float(tb["A"])
            T["tb_B"][a, b] = float(tb.get("B", 0.0))
            T["tb_p"][a, b] = float(tb.get("p", 4))
            T["tb_q"][a, b] = float(tb.get("q", 0))
    for a, sa in enumerate(species):
        for b, sb in enumerate(species):
            for c, sc in enumerate(species):
                tri = records.get((sa, sb, sc))
                if (tri is None or records.get((sa, sb, sb)) is None
                        or records.get((sa, sc, sc)) is None):
                    continue
                T["tri_valid"][a, b, c] = 1
                T["tri_eps"][a, b, c] = float(tri.get("epsilon", 1.0))
                T["tri_lam"][a, b, c] = float(tri["lambda"])
                T["tri_cos"][a, b, c] = float(tri.get("costheta0", -1.0 / 3.0))
    return {k: np.ascontiguousarray(v) for k, v in T.items()}


def sw_multi(records, species, lattice, positions, atom_types, pairs=None):
    """engine/stillinger_weber.py:1165-1325 (multi-species, numba branch)."""
    positions = _f64(positions)
    N = len(positions)
    ns = len(species)
    rc = sw_r_cut(records)
    index = {s: k for k, s in enumerate(species)}
    tids = np.array([index[t] for t in atom_types], np.int64)
    ii, jj = pairs if pairs is not None else _all_pairs(N)
    ii, jj, rij, r = mic_mask(lattice, positions, ii, jj, rc)
    if len(ii) == 0:
        return 0.0, np.zeros((N, 3)), np.zeros((3, 3))
    nb_start, nb_idx, nb_rij, nb_r = two_way_csr(N, ii, jj, rij, r)
    T = sw_tables(records, species)
    forces = np.zeros((N, 3))
    stress = np.zeros((3, 3))
    L = lib()
    e2 = L.orc_sw_multi_2body(_L(len(ii)), _L(N), _l(ii), _l(jj), _d(rij), _d(r),
                              _l(tids), _d(forces), _d(stress), _L(ns), _b(T["tb_valid"]),
                              _d(T["tb_eps"]), _d(T["tb_sig"]), _d(T["tb_a"]),
                              _d(T["tb_A"]), _d(T["tb_B"]), _d(T["tb_p"]), _d(T["tb_q"]))
    e3 = L.orc_sw_multi_3body(_L(0), _L(N), _L(N), _l(nb_start), _l(nb_idx), _d(nb_rij),
                              _d(nb_r), _l(tids), _d(forces), _d(stress), _L(ns),
                              _b(T["tri_valid"]), _d(T["tri_eps"]), _d(T["tri_lam"]),
                              _d(T["tri_cos"]), _d(T["leg_sig"]), _d(T["leg_a"]),
                              _d(T["leg_gam"]))
    return float(e2 + e3), forces, stress / _volume(lattice)


# ---------------------------------------------------------------------------
#  EAM (engine/eam.py, engine/_eam_kernels.py, engine/eam_zhou.py)
# ---------------------------------------------------------------------------

ZHOU_KEYS = ("r_e", "f_e", "rho_e", "rho_s", "alpha", "beta", "A", "B", "kappa",
             "lambda", "Fn0", "Fn1", "Fn2", "Fn3", "F0", "F1", "F2", "F3", "eta", "F_e")
_NZ = len(ZHOU_KEYS)


def zhou_continuous(p):
    """engine/eam_zhou.py:47-64: re-derive Fn0, Fn1, F0, F_e."""
    q = {k: float(v) for k, v in p.items()}
    re, rs, eta = q["rho_e"], q["rho_s"], q["eta"]
    F1, F2, F3 = q["F1"], q["F2"], q["F3"]
    y, x = 0.15, -0.15
    t0 = 1.15 * re / rs
    slope0 = (F1 + 2 * F2 * y + 3 * F3 * y * y) / re
    dg = -eta * eta * math.log(t0) * t0 ** (eta - 1.0) / rs
    q["F_e"] = slope0 / dg
    q["F0"] = q["F_e"] * (1 - eta * math.log(t0)) * t0 ** eta - (F1 * y + F2 * y * y + F3 * y ** 3)
    q["Fn0"] = q["F0"] + F1 * x + F2 * x * x + F3 * x ** 3
    q["Fn1"] = 0.85 * (F1 + 2 * F2 * x + 3 * F3 * x * x)
    return q


def _zdecay(r, p, pre, expo, shift):
    x = r / p["r_e"]
    e = pre * np.exp(-expo * (x - 1.0))
    u = x - shift
    den = 1.0 + u ** 20
    return e / den


def zhou_cutoff(p, tol=1e-6):
    """engine/eam_zhou.py:117-125."""
    r = np.linspace(p["r_e"], 5.0 * p["r_e"], 40001)
    phi = _zdecay(r, p, p["A"], p["alpha"], p["kappa"]) - _zdecay(r, p, p["B"], p["beta"], p["lambda"])
    f = _zdecay(r, p, p["f_e"], p["beta"], p["lambda"])
    ok = (np.abs(phi) < tol * max(p["A"], p["B"])) & (f < tol * p["f_e"])
    bad = np.nonzero(~ok)[0]
    return float(r[bad[-1] + 1]) if len(bad) else float(r[0])


class _EamTables(ctypes.Structure):
    _fields_ = [("codes", _lp), ("P", _dp), ("ncol", _L), ("xo", _lp), ("nx", _lp),
                ("X", _dp), ("C", _dp), ("nX", _L)]


class EAMSpec:
    """Function tables of one EAM potential, as engine/_eam_kernels.py:77-121
    (build_tables) lays them out: codes 1 spline, 2 spline/r, 3 Zhou density,
    4 Zhou pair, 5 Zhou cross pair, 6 Zhou embedding."""

    def __init__(self, species, specs, rho_fid, F_fid, phi_fid, r_cut):
        self.species = list(species)
        self.r_cut = float(r_cut)
        nf = len(specs)
        self.codes = np.zeros(nf, np.int64)
        self.P = np.zeros((nf, 2 * _NZ + 3))
        self.xo = np.zeros(nf, np.int64)
        self.nx = np.zeros(nf, np.int64)
        Xs, Cs, off = [], [], 0
        for f, sp in enumerate(specs):
            kind = sp[0]
            if kind in ("spline", "spline_over_r"):
                self.codes[f] = 1 if kind == "spline" else 2
                x, c = np.asarray(sp[1], float), np.asarray(sp[2], float)
                self.xo[f], self.nx[f] = off, len(x)
                Xs.append(x)
                cc = np.zeros((4, len(x)))
                cc[:, :len(x) - 1] = c
                Cs.append(cc)
                off += len(x)
            elif kind == "zhou_embedding":
                self.codes[f] = 6
                self.P[f, :_NZ] = [sp[1][k] for k in ZHOU_KEYS]
            else:
                if kind == "zhou_density":
                    self.codes[f] = 3
                    self.P[f, :_NZ] = [sp[1][k] for k in ZHOU_KEYS]
                    rc, w = sp[2], sp[3]
                elif kind == "zhou_pair":
                    self.codes[f] = 4
                    self.P[f, :_NZ] = [sp[1][k] for k in ZHOU_KEYS]
                    rc, w = sp[2], sp[3]
                else:
                    self.codes[f] = 5
                    self.P[f, :_NZ] = [sp[1][k] for k in ZHOU_KEYS]
                    self.P[f, _NZ:2 * _NZ] = [sp[2][k] for k in ZHOU_KEYS]
                    self.P[f, 2 * _NZ + 2] = float(sp[3])
                    rc, w = sp[4], sp[5]
                self.P[f, 2 * _NZ] = rc
                self.P[f, 2 * _NZ + 1] = w
        self.X = np.ascontiguousarray(np.concatenate(Xs) if Xs else np.zeros(1))
        self.C = np.ascontiguousarray(np.concatenate(Cs, axis=1) if Cs else np.zeros((4, 1)))
        self.rho_fid = np.asarray(rho_fid, np.int64)
        self.F_fid = np.asarray(F_fid, np.int64)
        self.phi_fid = np.ascontiguousarray(phi_fid, np.int64)

    def struct(self):
        return _EamTables(_l(self.codes), _d(self.P), self.P.shape[1], _l(self.xo),
                          _l(self.nx), _d(self.X), _d(self.C), self.X.shape[0])


def zhou_spec(elements, species, r_cut=None, chi=None, width=0.5):
    """engine/eam_zhou.py:128-207 (zhou_eam) expressed as function specs."""
    species = list(species)
    P = {s: zhou_continuous(elements[s]) for s in species}
    if r_cut is None:
        r_cut = max(zhou_cutoff(P[s]) for s in species)
    chi = chi or {}

    def cfac(a, b):
        return float(chi.get(f"{a}-{b}", chi.get(f"{b}-{a}", 1.0))) if a != b else 1.0

    specs = []
    rho_fid = []
    for s in species:
        rho_fid.append(len(specs))
        specs.append(("zhou_density", P[s], r_cut, width))
    F_fid = []
    for s in species:
        F_fid.append(len(specs))
        specs.append(("zhou_embedding", P[s]))
    ns = len(species)
    phi_fid = np.zeros((ns, ns), np.int64)
    for a in range(ns):
        for b in range(a, ns):
            if a == b:
                sp = ("zhou_pair", P[species[a]], r_cut, width)
            else:
                sp = ("zhou_cross", P[species[a]], P[species[b]],
                      cfac(species[a], species[b]), r_cut, width)
            phi_fid[a, b] = phi_fid[b, a] = len(specs)
            specs.append(sp)
    return EAMSpec(species, specs, rho_fid, F_fid, phi_fid, r_cut)


def eam(spec, lattice, positions, atom_types, pairs=None):
    """engine/eam.py:174-256 (numba branch) + engine/_eam_kernels.py:231-307."""
    positions = _f64(positions)
    N = len(positions)
    index = {s: k for k, s in enumerate(spec.species)}
    spc = np.array([index[t] for t in atom_types], np.int64)
    ii, jj = pairs if pairs is not None else _all_pairs(N)
    ii, jj, rij, r = mic_mask(lattice, positions, ii, jj, spec.r_cut)
    if len(ii) == 0:
        return 0.0, np.zeros((N, 3)), np.zeros((3, 3))
    forces = np.zeros((N, 3))
    vir = np.zeros((3, 3))
    st = spec.struct()
    e = lib().orc_eam_kernel(_L(N), _L(len(ii)), _l(ii), _l(jj), _d(rij), _d(r), _l(spc),
                             _l(spec.rho_fid), _l(spec.F_fid), _l(spec.phi_fid),
                             _L(len(spec.species)), ctypes.byref(st), _d(forces), _d(vir))
    return float(e), forces, vir / _volume(lattice)


def zhou_force(elements, species, r_cut=None, chi=None, width=0.5):
    """The force call of a Zhou EAM (zhou_spec) for fit_loss."""
    spec = zhou_spec(elements, species, r_cut, chi, width)
    return lambda lat, pos, types, pairs=None: eam(spec, lat, pos, types, pairs)


# ---- molecular dynamics ------------------------------------------------------
EV_ANG_TO_AMU_ANG_FS2 = (1.60217663e-19 / 1.0e-10) / (1.66053906660e-27) * 1.0e-20
K_B = 1.380649e-23 * 6.241509074e18


def init_velocities_mb(T, masses, rng):
    """solvers/molecular_dynamics.py:195-221 (_init_velocities_mb)."""
    masses = np.asarray(masses, float)
    N = len(masses)
    sigma = np.sqrt(K_B * T * EV_ANG_TO_AMU_ANG_FS2 / masses)
    v = rng.standard_normal((N, 3)) * sigma[:, None]
    v -= np.sum(masses[:, None] * v, axis=0) / masses.sum()
    e_kin = 0.5 * float(np.sum(masses[:, None] * v ** 2)) / EV_ANG_TO_AMU_ANG_FS2
    n_dof = max(3 * N - 3, 1)
    T_act = 2.0 * e_kin / (n_dof * K_B)
    if T_act > 1e-12:
        v *= np.sqrt(T / T_act)
    return v


def nve(force, lattice, positions, masses, velocities, dt, n_steps):
    """Velocity Verlet with the wrap of NVESimulation.run
    (solvers/molecular_dynamics.py:1969-2000); force(positions) -> (E, F).
    Returns per-step (positions, velocities, e_pot, e_kin) lists."""
    lattice = np.asarray(lattice, float)
    r = np.array(positions, float)
    v = np.array(velocities, float)
    m = np.asarray(masses, float)
    e, F = force(r)
    acc = F * EV_ANG_TO_AMU_ANG_FS2 / m[:, None]
    out = []
    for _ in range(n_steps):
        v += 0.5 * dt * acc
        r += dt * v
        frac = r @ np.linalg.inv(lattice)
        frac -= np.floor(frac)
        frac[frac >= 1.0] = 0.0
        r = frac @ lattice
        e, F = force(r)
        acc = F * EV_ANG_TO_AMU_ANG_FS2 / m[:, None]
        v += 0.5 * dt * acc
        e_kin = 0.5 * float(np.sum(m[:, None] * v ** 2)) / EV_ANG_TO_AMU_ANG_FS2
        out.append((r.copy(), v.copy(), e, e_kin))
    return out


# ---- fitting -------------------------------------------------------------------
def fit_loss(records, species, structures, weights, pairs=None, force=None):
    """fitting/loss.py:184-260 (squared loss) with the multi-species Tersoff
    force call: sum_s w_trust c_s^2 [w_E (E - N e_ref)^2 + w_F r0^2
    mean|dF|^2 + w_S (V eps0)^2 mean|dsigma|^2].  pairs: optional list of
    prebuilt (i, j) per structure.  force: optional callable (lattice,
    positions, atom_types, pairs) -> (E, F, stress) used instead of the
    Tersoff call (records is then ignored)."""
    w_E = weights.get("energy", 1.0)
    w_F = weights.get("forces", 1.0)
    w_S = weights.get("stress", 0.1)
    r0 = float(weights.get("r0", 1.0))
    eps0 = float(weights.get("eps0", 1.0))
    total = 0.0
    for q, s in enumerate(structures):
        N = s["natoms"]
        vol = float(s.get("volume", abs(np.linalg.det(s["lattice"]))))
        pq = None if pairs is None else pairs[q]
        if force is not None:
            e, f, st = force(s["lattice"], s["positions"], s["atom_types"], pq)
        else:
            e, f, st = tersoff_multi(records, species, s["lattice"], s["positions"], s["atom_types"], pq)
        tot = w_E * (N * (e / N - s["ref_energy"])) ** 2
        if s.get("ref_forces") is not None:
            tot += w_F * r0 ** 2 * float(np.mean((f - s["ref_forces"]) ** 2))
        if s.get("ref_stress") is not None:
            tot += w_S * (vol * eps0) ** 2 * float(np.mean((st - s["ref_stress"]) ** 2))
        total += float(s.get("weight", 1.0)) * float(s.get("scale", 1.0)) ** 2 * tot
    return total
