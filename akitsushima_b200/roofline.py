"""Algorithmic work of the force path, for roofline fractions.

Operation weights: + - * and rint = 1, fused multiply-add = 2, divide and
square root = 4, exp / log / sin / cos / pow = 8.  Counts are per
evaluation of a formula as written in the reference (the minimum work of the
algorithm), not per instruction of any implementation: the owner-computes
kernels evaluate a pair from both of its atoms, and that redundancy is not
credited.

Bytes follow the same rule: each input read once and each output written
once -- positions 24 B, species 4 B, forces 24 B, per-atom energy 8 B per
atom, the two-way CSR 4 B per slot plus 4 B per row offset.
"""

# minimum-image displacement and distance: s = d inv (15), s -= rint(s) (6),
# d = s L (15), r = sqrt(r . r) (9)
MIC = 45
# C2 quintic switch value and derivative (engine/eam_zhou.py:67-71)
SWITCH = 22
# one Zhou element at r: x = r / r_e, two exponentials with their arguments,
# two (x - c)^20 denominators, g = e / den and dg for both, f, df, phi_aa,
# dphi_aa (engine/eam_zhou.py:74-91)
ZHOU_SPECIES = 79
# like pair: one element + switched phi, dphi, rho' ; cross pair: two elements
# + q, dq, phi_ab, dphi_ab (eq. A5) + switched values
ZHOU_LIKE_PAIR = ZHOU_SPECIES + 7
ZHOU_CROSS_PAIR = 2 * ZHOU_SPECIES + 48
# c = phi' + F'_i rho'_j + F'_j rho'_i, f = c / r rij, force, energy, virial
EAM_ASSEMBLE = 34
# density of one neighbour at r (switched), accumulated
EAM_DENSITY = MIC + 15 + 26 + 1
# embedding F(rho), F'(rho) of one atom (eqs. A6-A8, average branch)
EAM_EMBED = 30


def eam_force_flops(n_like_pairs, n_cross_pairs):
    """Force pass: every unordered pair inside the cutoff once."""
    return (n_like_pairs * (MIC + SWITCH + ZHOU_LIKE_PAIR + EAM_ASSEMBLE)
            + n_cross_pairs * (MIC + SWITCH + ZHOU_CROSS_PAIR + EAM_ASSEMBLE))


def eam_density_flops(n_pairs, n_atoms):
    """Density pass: each unordered pair gives two densities."""
    return 2 * n_pairs * EAM_DENSITY + n_atoms * EAM_EMBED


def path_bytes(n_atoms, n_slots):
    """Algorithmic HBM bytes of one evaluation of the path."""
    return n_atoms * (24 + 4 + 24 + 8) + 4 * n_slots + 4 * (n_atoms + 1)


def eam_force_bytes(n_atoms, n_slots):
    """Force pass: positions, species, F'(rho) and the CSR in; forces and
    per-atom energy out."""
    return n_atoms * (24 + 4 + 8 + 24 + 8) + 4 * n_slots + 4 * (n_atoms + 1)
