"""ctypes binding of libmbforce.so, the C ABI declared in include/mbforce.h.

The library is built in-tree by ``python -m akitsushima_b200.build`` (or
``__graft_entry__.build()``).  There is no CPU fallback: a missing or stale
library raises here, loudly, instead of computing anything elsewhere.
"""
import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MBF_LIB_PATH") or os.path.join(_HERE, "libmbforce.so")

MBF_OK = 0
MBF_ERR_CAPACITY = -3
MBF_ERR_ROW_TOO_LONG = -4
MBF_FP64 = 0
MBF_MIXED = 1

_vp = ctypes.c_void_p
_i = ctypes.c_int
_ll = ctypes.c_longlong
_d = ctypes.c_double
_sz = ctypes.c_size_t


class MbfSystem(ctypes.Structure):
    _fields_ = [("n_atoms", _i), ("n_struct", _i), ("positions", _vp), ("types", _vp),
                ("atom_struct", _vp), ("struct_off", _vp), ("cells", _vp), ("orthorhombic", _i),
                ("cells_host", _vp)]


class MbfNlist(ctypes.Structure):
    _fields_ = [("n_atoms", _i), ("n_slots", _ll), ("max_row", _i), ("row_off", _vp),
                ("nbr", _vp), ("rev", _vp), ("upper", _vp)]


class MbfReducePlan(ctypes.Structure):
    _fields_ = [("n_chunks", _i), ("chunk", _vp), ("chunk_first", _vp)]


class MbfEamTables(ctypes.Structure):
    _fields_ = [("ns", _i), ("nf", _i), ("nX", _i), ("codes", _vp), ("P", _vp), ("xo", _vp),
                ("nx", _vp), ("X", _vp), ("C", _vp), ("rho_f", _vp), ("F_f", _vp),
                ("phi_f", _vp), ("r_cut", _d), ("zhou_fused", _i),
                ("P_host", _vp), ("rho_f_host", _vp), ("phi_f_host", _vp)]


class MbfFitSet(ctypes.Structure):
    _fields_ = [("n_struct", _i), ("n_atoms", _i)] + \
        [(k, _vp) for k in ("struct_off", "atom_struct", "n_orig", "fref_off", "inv_k", "e_ref", "f_ref",
                            "s_ref", "vol", "vsup", "fmask", "smask", "cw")] + \
        [(k, _d) for k in ("w_e", "w_f", "w_s", "r0", "eps0")] + [("huber", _i)] + \
        [(k, _d) for k in ("delta_e", "delta_f", "delta_s")]


class MbfTersoffTables(ctypes.Structure):
    _fields_ = [("ns", _i), ("tb", _vp), ("tri", _vp), ("r_cut", _d)]


class MbfSwTables(ctypes.Structure):
    _fields_ = [("ns", _i), ("tb", _vp), ("leg", _vp), ("tri", _vp), ("r_cut", _d)]


class MbfError(RuntimeError):
    """A C-ABI call returned an error code."""

    def __init__(self, code, where):
        self.code = code
        super().__init__(f"{where}: {error_string(code)} (code {code})")


_lib = None
_lock = threading.Lock()

_SIGS = {
    "mbf_error_string": (ctypes.c_char_p, [_i]),
    "mbf_version": (_i, []),
    "mbf_nl_workspace_bytes": (_sz, [_i, _i]),
    "mbf_nl_build": (_i, [ctypes.POINTER(MbfSystem), _vp, _i, _d, _vp, _sz, _vp, _vp, _vp, _vp, _ll,
                          ctypes.POINTER(_ll), ctypes.POINTER(_i), _vp]),
    "mbf_nl_rebuild_workspace_bytes": (_sz, [_i, _i, _i]),
    "mbf_nl_rebuild_async": (_i, [ctypes.POINTER(MbfSystem), _vp, _i, _d, _vp, _sz, _vp, _vp, _vp, _vp,
                                  _ll, _i, _vp, _vp]),
    "mbf_nl_max_displacement": (_i, [ctypes.POINTER(MbfSystem), _vp, _vp, _vp, _vp]),
    "mbf_md_kick_drift": (_i, [ctypes.POINTER(MbfSystem), _vp, _vp, _vp, _vp, _d, _vp]),
    "mbf_md_partial_count": (_i, [_i]),
    "mbf_md_kick": (_i, [ctypes.POINTER(MbfSystem), _vp, _vp, _vp, _d, _vp, _vp, _vp, _i, _vp, _vp, _vp]),
    "mbf_md_kick_drift_check": (_i, [ctypes.POINTER(MbfSystem), _vp, _vp, _vp, _vp, _d, _vp, _d, _d, _vp, _vp,
                                     _vp, _i, _vp, _vp, ctypes.c_ulonglong, _vp]),
    "mbf_md_kick_kick_drift_check": (_i, [ctypes.POINTER(MbfSystem), _vp, _vp, _vp, _vp, _d, _vp, _vp, _vp, _i,
                                          _vp, _vp, _d, _d, _vp, _vp, _i, _vp, _vp, ctypes.c_ulonglong, _vp, _vp]),
    "mbf_md_skin_check": (_i, [ctypes.POINTER(MbfSystem), _vp, _d, _d, _vp, _vp, _i, _vp, _vp, _vp,
                               ctypes.c_ulonglong, _vp]),
    "mbf_md_rebuild_done": (_i, [ctypes.POINTER(MbfSystem), _vp, _vp, _vp]),
    "mbf_capture_cond_create": (_i, [_vp, ctypes.POINTER(ctypes.c_ulonglong)]),
    "mbf_capture_if_begin": (_i, [_vp, _vp, ctypes.c_ulonglong]),
    "mbf_capture_if_end": (_i, [_vp]),
    "mbf_nl_half_workspace_bytes": (_sz, [_i]),
    "mbf_nl_half_pairs": (_i, [ctypes.POINTER(MbfNlist), _vp, _vp, _vp, _sz, _vp]),
    "mbf_eval_workspace_bytes": (_sz, [_i, _ll, _i]),
    "mbf_eval_status": (_i, [_vp, ctypes.POINTER(_i), _vp]),
    "mbf_eam_eval": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                          ctypes.POINTER(MbfEamTables), ctypes.POINTER(MbfReducePlan), _i, _i,
                          _vp, _sz, _vp, _vp, _vp, _vp]),
    "mbf_eam_eval_static": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                                 ctypes.POINTER(MbfEamTables), ctypes.POINTER(MbfReducePlan), _i, _i,
                                 _vp, _vp, _vp, _vp]),
    "mbf_eam_eval_static_status": (_i, [ctypes.POINTER(_i), _vp]),
    "mbf_eam_embedding": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                               ctypes.POINTER(MbfEamTables), ctypes.POINTER(MbfReducePlan), _i, _i,
                               _vp, _sz, _vp, _vp]),
    "mbf_eam_forces": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                            ctypes.POINTER(MbfEamTables), ctypes.POINTER(MbfReducePlan), _i, _i,
                            _vp, _sz, _vp, _vp, _vp, _vp, _vp]),
    "mbf_tersoff_eval": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                              ctypes.POINTER(MbfTersoffTables), ctypes.POINTER(MbfReducePlan), _i, _i,
                              _vp, _sz, _vp, _vp, _vp, _vp]),
    "mbf_tersoff_eval_sites": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                                    ctypes.POINTER(MbfTersoffTables), ctypes.POINTER(MbfReducePlan), _i, _i,
                                    _vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "mbf_sw_eval_sites": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                               ctypes.POINTER(MbfSwTables), ctypes.POINTER(MbfReducePlan), _i, _i,
                               _vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "mbf_eam_eval_sites": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                                ctypes.POINTER(MbfEamTables), ctypes.POINTER(MbfReducePlan), _i, _i,
                                _vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "mbf_fit_loss_workspace_bytes": (_sz, [_i]),
    "mbf_fit_loss": (_i, [ctypes.POINTER(MbfFitSet), _vp, _vp, _vp, _vp, _sz, _vp, _vp, _vp, _vp, _vp]),
    "mbf_eam_adjoint_workspace_bytes": (_sz, [_i, _ll, _i]),
    "mbf_eam_adjoint": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                             ctypes.POINTER(MbfEamTables), _vp, _vp, _vp, _vp, _sz, _vp, _vp]),
    "mbf_tersoff_adjoint_workspace_bytes": (_sz, [_ll, _i]),
    "mbf_tersoff_adjoint": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                                 ctypes.POINTER(MbfTersoffTables), _vp, _vp, _vp, _vp, _sz, _vp, _vp, _vp]),
    "mbf_sw_eval": (_i, [ctypes.POINTER(MbfSystem), ctypes.POINTER(MbfNlist),
                         ctypes.POINTER(MbfSwTables), ctypes.POINTER(MbfReducePlan), _i, _i, _vp, _sz,
                         _vp, _vp, _vp, _vp]),
    "mbf_profile_begin": (None, []),
    "mbf_profile_end": (_i, [ctypes.c_char_p, _sz]),
    "mbf_peak_probe": (_i, [_i, _vp, _sz, ctypes.POINTER(_d), _vp]),
}

MBF_STATUS_ROW_TOO_LONG = 1
MBF_STATUS_BAD_INDEX = 2
MBF_STATUS_CAPACITY = 4
MBF_STATUS_SKIN = 8

# Entry points declared in include/mbforce.h (checked by the CPU tests).
EXPORTED = tuple(_SIGS)


def lib():
    """The loaded library; raises if it was not built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build the CUDA extension with "
                    "`python -m akitsushima_b200.build` (nvcc, sm_100a). There is no "
                    "CPU fallback.")
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in _SIGS.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _lib = L
        return _lib


def error_string(code):
    try:
        return lib().mbf_error_string(int(code)).decode()
    except Exception:
        return "error"


def check(code, where):
    if code != MBF_OK:
        raise MbfError(code, where)


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def profile_begin():
    """Start recording CUDA-event timings of every kernel launch."""
    lib().mbf_profile_begin()


def profile_end():
    """Stop recording; {kernel: (launches, total_ms)}."""
    buf = ctypes.create_string_buffer(1 << 16)
    n = lib().mbf_profile_end(buf, len(buf))
    if n < 0:
        raise MbfError(n, "mbf_profile_end")
    out = {}
    for line in buf.value.decode().splitlines():
        name, cnt, ms = line.split()
        out[name] = (int(cnt), float(ms))
    return out
