"""mbf_eam_eval_static, the EAM evaluation that allocates nothing.

It exists for callers that cannot allocate device memory (a host program
that owns the device's memory budget and hands its plug-ins only input and
output buffers, or a time-step loop that must not synchronise the device as
cudaMalloc / cudaFree can).  Its scratch is a fixed device array inside the
library.  These tests call it through the C ABI and check that it returns
what mbf_eam_eval (caller-provided workspace) returns, on two calls in a row
with different positions -- the array keeps the previous call's contents, so
the second call shows that nothing leaks from the first -- with its index
check words, read through mbf_eam_eval_static_status (these callers hold
no workspace pointer), clear after each call; and that a structure too
large for the array, or a reduction plan with fewer chunks than
structures, is refused without any work.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

ak = pytest.importorskip("akitsushima_b200")

# the parity tolerance of the float64 tests: 1e-10 relative to the largest
# value; the mixed path is the same kernels, so the same bound holds
REL = 1e-10


def _setup(precision):
    import torch
    from akitsushima_b200 import _lib
    g = golden("eam_cuni500")
    fn = ak.force_fn_from_config({"type": "EAM", "form": "zhou2004", "elements": ["Cu", "Ni"]},
                                 precision=precision)
    pot = fn.engine.potentials[0]
    nl = ak.NeighbourList(fn.r_cut, skin_width=0.3)
    nl.build(g["lattice"], g["positions"])
    batch = nl._batch
    batch.set_types(ak.system.species_ids(list(g["atom_types"]), pot.species))
    return torch, _lib, g, pot, batch, nl.device_list


def _static_call(torch, _lib, pot, batch, dl, precision):
    dev = batch.device
    forces = torch.empty((batch.n_atoms, 3), dtype=torch.float64, device=dev)
    energy = torch.empty(batch.n_struct, dtype=torch.float64, device=dev)
    virial = torch.empty((batch.n_struct, 9), dtype=torch.float64, device=dev)
    tabs = pot.tables(dev)
    prec = _lib.MBF_FP64 if precision == "fp64" else _lib.MBF_MIXED
    rc = _lib.lib().mbf_eam_eval_static(batch.mbf_system(), dl.mbf_nlist(), tabs[0],
                                        batch.reduce_plan(), prec, int(pot.lanes_per_atom),
                                        _lib.ptr(forces), _lib.ptr(energy), _lib.ptr(virial),
                                        torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(rc, "mbf_eam_eval_static")
    # the index-check words of that call, read through the entry point made
    # for these callers (they hold no workspace pointer): all clear
    words = (ctypes.c_int * 4)()
    _lib.check(_lib.lib().mbf_eam_eval_static_status(words, torch.cuda.current_stream(dev).cuda_stream),
               "mbf_eam_eval_static_status")
    assert list(words)[:3] == [0, 0, 0], list(words)
    torch.cuda.synchronize()
    return energy.cpu().numpy(), forces.cpu().numpy(), virial.cpu().numpy()


def _close(a, b):
    scale = max(1.0, float(np.abs(b).max()))
    assert float(np.abs(a - b).max()) <= REL * scale, float(np.abs(a - b).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_static_entry_matches_workspace_entry_on_two_calls(cuda_device, precision):
    torch, _lib, g, pot, batch, dl = _setup(precision)
    rng = np.random.default_rng(42)
    for k in range(2):
        pos = g["positions"] + (0.0 if k == 0 else rng.normal(0.0, 0.02, g["positions"].shape))
        batch.set_positions(pos)
        ref = pot.evaluate(batch, dl, precision=precision)
        torch.cuda.synchronize()
        e0, f0, v0 = ref.energy.cpu().numpy(), ref.forces.cpu().numpy(), ref.virial.cpu().numpy()
        e1, f1, v1 = _static_call(torch, _lib, pot, batch, dl, precision)
        _close(e1, e0)
        _close(f1, f0)
        _close(v1, v0)
        if k == 0 and precision == "fp64":
            assert abs(float(e1[0]) - float(g["energy"])) / 500 < 1e-10


def test_static_entry_refuses_a_short_reduction_plan(cuda_device):
    """A plan with fewer chunks than structures would clear completion
    counters past their region (past the fixed array, here): refused."""
    torch, _lib, g, pot, batch, dl = _setup("fp64")
    dummy = torch.empty(1, dtype=torch.float64, device=batch.device)
    sysd = batch.mbf_system()
    two = _lib.MbfSystem(sysd.n_atoms, 2, sysd.positions, sysd.types, sysd.atom_struct, sysd.struct_off,
                         sysd.cells, sysd.orthorhombic)
    rc = _lib.lib().mbf_eam_eval_static(two, dl.mbf_nlist(), pot.tables(batch.device)[0],
                                        _lib.MbfReducePlan(1, batch.reduce_plan().chunk,
                                                           batch.reduce_plan().chunk_first),
                                        _lib.MBF_FP64, 2, _lib.ptr(dummy), _lib.ptr(dummy), _lib.ptr(dummy),
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == -1


def test_static_entry_refuses_oversized_structure(cuda_device):
    torch, _lib, g, pot, batch, dl = _setup("fp64")
    L = _lib.lib()
    n_atoms = 1_000_000
    n_slots = 80 * n_atoms
    assert L.mbf_eval_workspace_bytes(n_atoms, n_slots, 1) > (32 << 20)
    sysd = _lib.MbfSystem(n_atoms, 1, _lib.ptr(batch.pos), _lib.ptr(batch.types),
                          _lib.ptr(batch.atom_struct), _lib.ptr(batch.struct_off),
                          _lib.ptr(batch.cells), 1)
    nld = _lib.MbfNlist(n_atoms, n_slots, 80, _lib.ptr(dl.row_off), _lib.ptr(dl.nbr),
                        _lib.ptr(dl.rev), _lib.ptr(dl.upper))
    dummy = torch.empty(1, dtype=torch.float64, device=batch.device)
    rc = L.mbf_eam_eval_static(sysd, nld, pot.tables(batch.device)[0], batch.reduce_plan(),
                               _lib.MBF_FP64, 8, _lib.ptr(dummy), _lib.ptr(dummy), _lib.ptr(dummy),
                               torch.cuda.current_stream().cuda_stream)
    assert rc == -6
    assert "no-allocation" in L.mbf_error_string(rc).decode()

