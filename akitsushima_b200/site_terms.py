"""Site-energy decomposition of the many-body potentials (heat flux).

The reference's SiteTerms (engine/site_terms.py:1-83): for E = sum_i U_i,
U_i a function of the vectors v_m = r_nbr - r_centre of the entries m
centred on i, the arrays

    e_site (N,)   U_i
    centre, nbr (M,), vec (M, 3), dUdv (M, 3) = dU_centre / dv_m

give the forces, the stress and the exact many-body heat flux
J V = sum_i E_i v_i - sum_m v_m (dUdv_m . vel_nbr) (Fan et al., Phys. Rev. B
92, 094301 (2015)).  Here the kernels of the force path produce them in the
same launch as energy and forces (mbf_*_eval_sites); the entries are the
list slots inside the cutoff, centre-major with neighbours ascending.
"""
from dataclasses import dataclass

import numpy as np
import torch

from .neighbourlist import DeviceNeighbourList
from .system import Batch, check_min_image, default_device, species_ids


@dataclass
class SiteTerms:
    e_site: np.ndarray
    centre: np.ndarray
    nbr: np.ndarray
    vec: np.ndarray
    dUdv: np.ndarray

    @property
    def energy(self):
        return float(self.e_site.sum())

    def forces(self):
        F = np.zeros((len(self.e_site), 3))
        np.add.at(F, self.centre, self.dUdv)
        np.add.at(F, self.nbr, -self.dUdv)
        return F

    def stress(self, volume):
        """-(1/V) sum_m dUdv_m (x) v_m, symmetrised (compressive-positive)."""
        S = -np.einsum("ma,mb->ab", self.dUdv, self.vec) / volume
        return 0.5 * (S + S.T)

    def virial_flux(self, velocities):
        """-sum_m v_m (dUdv_m . vel_nbr)  [eV A/fs], not divided by V."""
        c = np.einsum("ma,ma->m", self.dUdv, np.asarray(velocities, float)[self.nbr])
        return -np.einsum("m,ma->a", c, self.vec)

    def heat_flux(self, velocities, masses, conv):
        """J V = sum_i E_i v_i + virial_flux, E_i = 1/2 m_i |v_i|^2 / conv + U_i
        [eV A/fs] (conv = EV_ANG_TO_AMU_ANG_FS2)."""
        v = np.asarray(velocities, float)
        E = 0.5 * np.asarray(masses, float) * np.einsum("ia,ia->i", v, v) / conv + self.e_site
        return np.einsum("i,ia->a", E, v) + self.virial_flux(v)

    @staticmethod
    def combine(parts, n_atoms):
        parts = [p for p in parts if p is not None]
        if not parts:
            z = np.zeros(0, dtype=np.int64)
            return SiteTerms(np.zeros(n_atoms), z, z, np.zeros((0, 3)), np.zeros((0, 3)))
        return SiteTerms(np.sum([p.e_site for p in parts], axis=0), np.concatenate([p.centre for p in parts]),
                         np.concatenate([p.nbr for p in parts]), np.concatenate([p.vec for p in parts]),
                         np.concatenate([p.dUdv for p in parts]))


def potential_site_terms(pot, lattice, positions, atom_types, precision=None, device=None):
    """SiteTerms of one potential of this package on one structure."""
    lattice = np.asarray(lattice, float)
    pos = np.ascontiguousarray(positions, float)
    N = len(pos)
    rc = float(pot.r_cut)
    check_min_image(lattice, rc, f"{type(pot).__name__}.site_terms")
    dev = torch.device(device) if device is not None else default_device()
    batch = Batch.single(lattice, pos, species_ids(atom_types, pot.species), device=dev)
    dl = DeviceNeighbourList(rc).build(batch)
    _, e, dudv, vec = pot.evaluate_sites(batch, dl, precision=precision)
    pot.status(dev)
    n_slots = int(dl.n_slots)
    row_off = dl.row_off[:N + 1].cpu().numpy()
    nbr = dl.nbr[:n_slots].cpu().numpy().astype(np.int64)
    centre = np.repeat(np.arange(N, dtype=np.int64), np.diff(row_off))
    v = vec[:n_slots].cpu().numpy()
    r = np.linalg.norm(v, axis=1)
    live = (r < rc) & (r > 1e-12)
    return SiteTerms(e.cpu().numpy(), centre[live], nbr[live], v[live], dudv[:n_slots].cpu().numpy()[live])


def site_terms(backend, lattice, positions, atom_types, precision=None, device=None):
    """SiteTerms of a force function of this package, a PotentialEngine or a
    single potential (the sum over its potentials, SiteTerms.combine)."""
    eng = getattr(backend, "engine", None)
    pots = list(eng.potentials) if eng is not None else list(getattr(backend, "potentials", [backend]))
    parts = [potential_site_terms(p, lattice, positions, atom_types, precision, device) for p in pots]
    return SiteTerms.combine(parts, len(positions))


# The reference's names (engine/site_terms.py:179, :312, :440).
def sw_site_terms(pot, lattice, positions, atom_types):
    return potential_site_terms(pot, lattice, positions, atom_types)


def tersoff_site_terms(pot, lattice, positions, atom_types):
    return potential_site_terms(pot, lattice, positions, atom_types)


def eam_site_terms(pot, lattice, positions, atom_types):
    return potential_site_terms(pot, lattice, positions, atom_types)
