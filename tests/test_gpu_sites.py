"""Site terms (heat-flux decomposition) against the reference's own
engine/site_terms.py output (tests/golden/sites_*.npz), float64."""
import numpy as np
import pytest

from conftest import SW_SI, TERSOFF_SI, golden

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")
from akitsushima_b200 import site_terms  # noqa: E402
from akitsushima_b200.published_parameters import TERSOFF_1989  # noqa: E402

SIC = {"type": "Tersoff", "species": ["Si", "C"],
       "params": {"mixing": "tersoff1989", "elements": {s: dict(TERSOFF_1989["elements"][s]) for s in ("Si", "C")},
                  "chi": {"C-Si": TERSOFF_1989["chi"]["C-Si"]}}}
CASES = {
    "sites_tersoff_si216": {"type": "Tersoff", "species": ["Si"], "params": TERSOFF_SI},
    "sites_tersoff1989_sic216": SIC,
    "sites_sw_si216": {"type": "SW", "species": ["Si"], "params": SW_SI},
    "sites_eam_cuni256": {"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"], "species": ["Cu", "Ni"]},
}


def _sorted(st):
    o = np.lexsort((st.nbr, st.centre))
    return st.centre[o], st.nbr[o], st.vec[o], st.dUdv[o]


@pytest.mark.parametrize("name", sorted(CASES))
def test_site_terms_match_reference(cuda_device, name):
    g = golden(name)
    L, P, T = g["lattice"], g["positions"], [str(t) for t in g["atom_types"]]
    fn = ak.force_fn_from_config(CASES[name])
    st = site_terms.site_terms(fn, L, P, T)
    np.testing.assert_allclose(st.e_site, g["e_site"], rtol=0, atol=1e-10)
    mine = _sorted(st)
    ref = _sorted(site_terms.SiteTerms(g["e_site"], g["centre"], g["nbr"], g["vec"], g["dUdv"]))
    np.testing.assert_array_equal(mine[0], ref[0])
    np.testing.assert_array_equal(mine[1], ref[1])
    np.testing.assert_allclose(mine[2], ref[2], rtol=0, atol=1e-10)
    np.testing.assert_allclose(mine[3], ref[3], rtol=0, atol=1e-8)
    np.testing.assert_allclose(st.forces(), g["forces"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(st.stress(abs(np.linalg.det(L))), g["stress"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(st.virial_flux(g["velocities"]), g["virial_flux"], rtol=1e-9, atol=1e-10)
    # the decomposition rebuilds the engine's own forces and energy
    e, f, s = fn(L, P, T)
    assert abs(st.energy - e) < 1e-9
    np.testing.assert_allclose(st.forces(), f, rtol=0, atol=1e-8)
