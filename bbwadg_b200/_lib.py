"""ctypes binding of the native library (include/bbwadg.h).

The library is built in-tree (``python -m bbwadg_b200.build``) as
bbwadg_b200/libbbwadg_b200.so.  There is no fallback: if it is missing or
fails to load, every entry point raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbbwadg_b200.so")

c_int, c_float, c_double, c_void_p = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_void_p
P = ctypes.c_void_p  # device or host pointer


class BBWError(RuntimeError):
    """A bbw_* call returned a non-zero status."""

    def __init__(self, func, status, msg):
        super().__init__("%s failed: %s (%s)" % (func, STATUS.get(status, status), msg))
        self.status = status


STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory",
          4: "call out of sequence", 5: "inconsistent mesh", 6: "operator construction failed",
          7: "unsupported size or option", 8: "bounded device wait gave up"}


class MeshDesc(ctypes.Structure):
    _fields_ = [("N", c_int), ("K", c_int), ("Nq", c_int), ("vgeo", P), ("fgeo", P),
                ("Fmask", P), ("vmapP", P), ("c2q", P), ("Jq", P)]


class OpsDesc(ctypes.Structure):
    _fields_ = [("Dr", P), ("Ds", P), ("Dt", P), ("LIFT", P),
                ("D_ids1", P), ("D_ids2", P), ("D_ids3", P), ("D_ids4", P), ("Dvals4", P),
                ("EEL_nnz", c_int), ("L0_nnz", c_int), ("EEL_ids", P), ("L0_ids", P),
                ("EEL_vals", P), ("L0_vals", P), ("Vq", P), ("Pq", P)]


class CurvedDesc(ctypes.Structure):
    _fields_ = [("N", c_int), ("K", c_int), ("Nq", c_int), ("Nfq", c_int), ("Nq_reduced", c_int),
                ("KCurved", c_int), ("KPlanar", c_int), ("KlistCurved", P), ("KlistPlanar", P),
                ("vgeo", P), ("fgeo", P), ("Jplanar", P), ("Fmask", P), ("vmapP", P),
                ("vgeoq", P), ("Jq", P), ("fgeoq", P), ("Jq_reduced", P), ("c2q", P),
                ("Dr", P), ("Ds", P), ("Dt", P), ("LIFT", P), ("Vq", P), ("Vrq", P), ("Vsq", P),
                ("Vtq", P), ("Pq", P), ("Prq", P), ("Psq", P), ("Ptq", P), ("VfqFace", P),
                ("Pfq", P), ("Vq_reduced", P), ("Pq_reduced", P)]


# name -> (restype, argtypes); every function returns bbw_status unless noted
SIGNATURES = {
    "bbw_status_string": (ctypes.c_char_p, [c_int]),
    "bbw_last_error": (ctypes.c_char_p, []),
    "bbw_version": (ctypes.c_char_p, []),
    "bbw_mesh_connect": (c_int, [c_int, c_int, P, P, P]),
    "bbw_mesh_geometry": (c_int, [c_int, c_int, P, P, P, P, P, P, P, P, P, P, P, P, P]),
    "bbw_mesh_vmapP": (c_int, [c_int, c_int, P, P, P, P, P, P, P]),
    "bbw_ops_build": (c_int, [c_int, P, c_int, P, c_int, ctypes.POINTER(c_void_p)]),
    "bbw_ops_get": (c_int, [c_void_p, ctypes.c_char_p, c_int, P, ctypes.POINTER(ctypes.c_longlong)]),
    "bbw_ops_free": (None, [c_void_p]),
    "bbw_basis_eval": (c_int, [c_int, c_int, c_int, P, P, P, P]),
    "bbw_rk_volume": (c_int, [c_int, c_int, P, P, P, P, P, P, P]),
    "bbw_rk_surface": (c_int, [c_int, c_int, c_int, P, P, P, P, P, P, P]),
    "bbw_rk_update": (c_int, [c_int, c_int, c_float, c_float, c_float, P, P, P, P]),
    "bbw_rk_update_wadg": (c_int, [c_int, c_int, c_int, P, P, P, P, c_float, c_float, c_float,
                                   P, P, P, P]),
    "bbw_rk_volume_bern": (c_int, [c_int, c_int, P, P, P, P, P, P, P, P, P]),
    "bbw_rk_surface_bern": (c_int, [c_int, c_int, c_int, P, P, P, P, c_int, P, P, c_int, P, P,
                                    P, P, P, P]),
    "bbw_rk_surface_bern_slice": (c_int, [c_int, c_int, c_int, P, P, P, P, P, P, c_int, P, P, P,
                                          P, P, P]),
    "bbw_rk_stage_noalloc": (c_int, [c_int, c_int, c_int, c_int, P, P, P, P, P, P, P, P, P, P, P,
                                     P, c_float, c_float, c_float, P, P, P]),
    "bbw_create": (c_int, [ctypes.POINTER(MeshDesc), ctypes.POINTER(OpsDesc), c_int, c_int,
                           ctypes.POINTER(c_void_p)]),
    "bbw_create_ex": (c_int, [ctypes.POINTER(MeshDesc), ctypes.POINTER(OpsDesc), c_int, c_int,
                              c_int, ctypes.POINTER(c_void_p)]),
    "bbw_check": (c_int, [c_void_p]),
    "bbw_destroy": (c_int, [c_void_p]),
    "bbw_set_state": (c_int, [c_void_p, P]),
    "bbw_get_state": (c_int, [c_void_p, P]),
    "bbw_set_residual": (c_int, [c_void_p, P]),
    "bbw_get_residual": (c_int, [c_void_p, P]),
    "bbw_stage": (c_int, [c_void_p, c_float, c_float, c_float]),
    "bbw_steps": (c_int, [c_void_p, c_float, c_int]),
    "bbw_run": (c_int, [c_void_p, c_double, c_float]),
    "bbw_sync": (c_int, [c_void_p]),
    "bbw_stage_ex": (c_int, [c_void_p, c_float, c_float, c_float, c_float]),
    "bbw_set_shots": (c_int, [c_void_p, c_int]),
    "bbw_set_compute_range": (c_int, [c_void_p, c_int]),
    "bbw_gather_elements": (c_int, [c_void_p, c_int, P, P]),
    "bbw_scatter_elements": (c_int, [c_void_p, c_int, P, P]),
    "bbw_stage_part": (c_int, [c_void_p, c_float, c_float, c_float, c_int, c_int]),
    "bbw_stage_commit": (c_int, [c_void_p]),
    "bbw_move_elements": (c_int, [c_void_p, c_int, c_int, c_int, P, P, c_void_p]),
    "bbw_autotune": (c_int, [c_void_p, c_float, c_int, ctypes.POINTER(c_int)]),
    "bbw_set_config": (c_int, [c_void_p, c_int]),
    "bbw_set_grid_limit": (c_int, [c_void_p, c_int]),
    "bbw_set_sources": (c_int, [c_void_p, c_int, P, P, P, c_float, c_float, c_float, c_int]),
    "bbw_set_receivers": (c_int, [c_void_p, c_int, P, P, c_int]),
    "bbw_get_traces": (c_int, [c_void_p, P, ctypes.POINTER(c_int)]),
    "bbw_set_time": (c_int, [c_void_p, c_double]),
    "bbw_get_time": (c_int, [c_void_p, ctypes.POINTER(c_double), ctypes.POINTER(c_int)]),
    "bbw_set_c2q": (c_int, [c_void_p, P]),
    "bbw_forward": (c_int, [c_void_p, c_float, c_int, c_int, ctypes.POINTER(c_void_p)]),
    "bbw_backward": (c_int, [c_void_p, c_void_p, P, P, P]),
    "bbw_tape_free": (c_int, [c_void_p]),
    "bbw_forward_ex": (c_int, [c_void_p, c_float, c_int, c_int, c_int, ctypes.POINTER(c_void_p)]),
    "bbw_tape_kind": (c_int, [c_void_p]),
    "bbw_device_state": (c_int, [c_void_p, ctypes.POINTER(c_void_p), ctypes.POINTER(c_void_p),
                                 ctypes.POINTER(c_void_p)]),
    "bbw_gordon_hall_sphere": (c_int, [c_int, c_int, P, P, P, P, P]),
    "bbw_curved_geometry": (c_int, [c_int, c_int, P, P, P, c_int, P, c_int, P, P, P, P]),
    "bbw_rk_volume_wadg_skew_combine": (c_int, [c_int, c_int, c_int] + [P] * 15 + [P]),
    "bbw_rk_surface_wadg_skew_combine": (c_int, [c_int, c_int, c_int] + [P] * 9 + [P]),
    "bbw_rk_volume_planar": (c_int, [c_int, c_int] + [P] * 8 + [P]),
    "bbw_rk_surface_planar": (c_int, [c_int, c_int] + [P] * 8 + [P]),
    "bbw_curved_create": (c_int, [ctypes.POINTER(CurvedDesc), c_int, ctypes.POINTER(c_void_p)]),
    "bbw_curved_destroy": (c_int, [c_void_p]),
    "bbw_curved_set_state": (c_int, [c_void_p, P]),
    "bbw_curved_get_state": (c_int, [c_void_p, P]),
    "bbw_curved_get_residual": (c_int, [c_void_p, P]),
    "bbw_curved_stage": (c_int, [c_void_p, c_float, c_float, c_float]),
    "bbw_curved_steps": (c_int, [c_void_p, c_float, c_int]),
    "bbw_curved_sync": (c_int, [c_void_p]),
    "bbw_curved_stream": (c_void_p, [c_void_p]),
    "bbw_curved_autotune": (c_int, [c_void_p, c_float, c_int, ctypes.POINTER(c_int)]),
}

_lib = None


def lib():
    """Load the native library (once); raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("bbwadg_b200 native library not built: %s missing "
                               "(run `python -m bbwadg_b200.build`)" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def call(name, *args):
    """Call bbw_<name> and raise BBWError on a non-zero status."""
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        raise BBWError(name, rc, lib().bbw_last_error().decode(errors="replace"))
    return rc


def ptr(a):
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
