"""Seeded synthetic structures of the benchmark configurations.

The generators follow the reference's benchmarks/bench_force.py:152-158:
n^3 conventional cells of a fractional basis (DIAMOND, FCC of
benchmarks/bench_force.py:52-62), Gaussian displacements drawn from
numpy.random.default_rng(seed).  No dataset is involved; the benchmark and
the parity tests at full size build their inputs here, so both see the same
atoms.

* ``make_si(8, sigma=0.05)``: Si diamond 8^3 = 4096 atoms (Tersoff NVE).
* ``make_si(20, sigma=0.1)``: Si diamond 20^3 = 64,000 atoms (SW NVE).
* ``make_cuni(40)``: fcc Cu-Ni 50/50 random alloy, 40^3 = 256,000 atoms.
* ``make_si_set(512)``: 512 strained Si supercells of {1..4}^3 cells.
* ``make_sic_set(256)``: 256 strained zincblende SiC cells of 2^3 / 3^3.
* ``make_ni3al_set(256)``: 256 strained L1_2 Ni3Al cells of 4^3 / 5^3.
* ``make_gesn(20)``: diamond Ge-Sn, 25 % Sn at random, 64,000 atoms.
"""
import numpy as np

DIAMOND = np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0],
                    [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75],
                    [0.75, 0.75, 0.25]], float)
FCC = np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]], float)


def _supercell(basis, reps):
    g = [np.arange(int(r)) for r in reps]
    cells = np.stack(np.meshgrid(*g, indexing="ij"), -1).reshape(-1, 3)
    return (np.asarray(basis, float)[None] + cells[:, None]).reshape(-1, 3), len(cells)


def _strain(rng, amp):
    e = rng.uniform(-amp, amp, (3, 3))
    return np.eye(3) + 0.5 * (e + e.T)


def make_cuni(n_cells=40, a=3.58, sigma=0.08, seed=0):
    """(lattice, positions, species ids) of the fcc Cu-Ni alloy: ids 0 = Cu,
    1 = Ni, uniform at random from seed + 1."""
    rng = np.random.default_rng(seed)
    frac, _ = _supercell(FCC, (n_cells,) * 3)
    pos = frac * a + rng.normal(0.0, sigma, frac.shape)
    ids = np.random.default_rng(seed + 1).integers(0, 2, len(pos)).astype(np.int32)
    return np.eye(3) * a * n_cells, pos, ids


def make_si(n_cells, a=5.431, sigma=0.05, seed=0):
    """(lattice, positions, ["Si"] * N) of an n^3 diamond supercell."""
    rng = np.random.default_rng(seed)
    frac, _ = _supercell(DIAMOND, (n_cells,) * 3)
    pos = frac * a + rng.normal(0.0, sigma, frac.shape)
    return np.eye(3) * a * n_cells, pos, ["Si"] * len(pos)


def make_si_set(n=512, a=5.431, strain=0.03, sigma=0.1, seed=0):
    """Uneven strained Si diamond supercells, {1..4} cells per axis drawn
    uniformly, symmetric strain entries uniform +-strain (triclinic cells):
    a list of (lattice, positions, types)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        reps = rng.integers(1, 5, size=3)
        frac, _ = _supercell(DIAMOND, reps)
        lat = np.diag(reps.astype(float)) * a
        pos = frac * a
        m = _strain(rng, strain)
        lat, pos = lat @ m, pos @ m
        pos = pos + rng.normal(0.0, sigma, pos.shape)
        out.append((lat, pos, ["Si"] * len(pos)))
    return out


def make_sic_set(n=256, a=4.36, strain=0.02, sigma=0.1, seed=0):
    """Zincblende SiC, 2^3 or 3^3 conventional cells (64 or 216 atoms),
    symmetric strain entries uniform +-2 %, Gaussian displacements."""
    rng = np.random.default_rng(seed)
    types8 = ["Si"] * 4 + ["C"] * 4
    out = []
    for _ in range(n):
        m = int(rng.integers(2, 4))
        frac, nc = _supercell(DIAMOND, (m, m, m))
        lat = np.eye(3) * a * m
        pos = frac * a
        M = _strain(rng, strain)
        lat, pos = lat @ M, pos @ M
        pos = pos + rng.normal(0.0, sigma, pos.shape)
        out.append((lat, pos, types8 * nc))
    return out


def make_ni3al_set(n=256, a=3.57, strain=0.02, sigma=0.08, seed=0):
    """L1_2 Ni3Al (Al on the cube corners), 4^3 or 5^3 conventional cells
    (256 or 500 atoms), symmetric strain entries uniform +-2 %, Gaussian
    displacements."""
    rng = np.random.default_rng(seed)
    types4 = ["Al", "Ni", "Ni", "Ni"]
    out = []
    for _ in range(n):
        m = int(rng.integers(4, 6))
        frac, nc = _supercell(FCC, (m, m, m))
        lat = np.eye(3) * a * m
        pos = frac * a
        M = _strain(rng, strain)
        lat, pos = lat @ M, pos @ M
        pos = pos + rng.normal(0.0, sigma, pos.shape)
        out.append((lat, pos, types4 * nc))
    return out


def make_gesn(n_cells=20, a=5.762, sigma=0.1, seed=0, frac_sn=0.25):
    """Diamond Ge-Sn with a fraction frac_sn of Sn at random."""
    lat, pos, _ = make_si(n_cells, a=a, sigma=sigma, seed=seed)
    types = [str(t) for t in np.random.default_rng(seed + 1).choice(["Ge", "Sn"], len(pos),
                                                                    p=[1 - frac_sn, frac_sn])]
    return lat, pos, types
