"""ctypes binding of libcansfz.so (the C ABI of include/cansfz.h).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import os

from .params import Params

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libcansfz.so")

D = ct.c_double
I = ct.c_int
V = ct.c_void_p          # device or host pointer
PD = ct.POINTER(ct.c_double)

OK = 0
STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA runtime error", 3: "bounded device wait ran out",
    4: "NaN in the divergence check", 5: "maximum divergence too large", 6: "time step too small",
    7: "unsupported on the GPU path", 8: "device allocation failed", 9: "no CUDA device",
}


class Diag(ct.Structure):
    _fields_ = [("time", D), ("istep", ct.c_int64), ("dt", D), ("dto", D), ("dt_cfl", D),
                ("gam", D), ("seps", D), ("divtot", D), ("divmax", D), ("mass12", D * 2),
                ("status", ct.c_int32), ("reserved", ct.c_int32 * 7)]


class Plan(ct.Structure):
    """cansfz_plan: the launch shapes the autotuner chooses."""
    _fields_ = [("phase_slots", ct.c_int32), ("momentum_slots", ct.c_int32), ("zsolve", ct.c_int32),
                ("fp32_transforms", ct.c_int32), ("ms_per_step", D), ("tile_tma", ct.c_int32),
                ("ghost_images", ct.c_int32), ("line_transforms", ct.c_int32),
                ("reserved", ct.c_int32 * 3)]


SIGNATURES = {
    "cansfz_version": (I, []),
    "cansfz_status_string": (ct.c_char_p, [I]),
    "cansfz_create": (I, [ct.POINTER(Params), V, ct.POINTER(V)]),
    "cansfz_destroy": (I, [V]),
    "cansfz_stream": (V, [V]),
    "cansfz_set_fields": (I, [V, V, V, V, V, V, I]),
    "cansfz_get_fields": (I, [V, V, V, V, V, V, I]),
    "cansfz_get_aux": (I, [V, ct.c_char_p, V, I]),
    "cansfz_set_scalar": (I, [V, V, I]),
    "cansfz_init2fl": (I, [V, ct.c_char_p, V, I]),
    "cansfz_initflow": (I, [V, ct.c_char_p]),
    "cansfz_initscal": (I, [V, ct.c_char_p]),
    "cansfz_prepare": (I, [V]),
    "cansfz_step": (I, [V, I]),
    "cansfz_get_diag": (I, [V, ct.POINTER(Diag)]),
    "cansfz_get_status": (I, [V, ct.POINTER(Diag)]),
    "cansfz_rk_2fl": (I, [V, PD, D, D, D, D] + [V] * 10),
    "cansfz_acdi_transport_pf": (I, [V, D, D] + [V] * 12),
    "cansfz_vof_thinc_transport_psi": (I, [V, D] + [V] * 12),
    "cansfz_acdi_cmpt_phi": (I, [V, D, V, V]),
    "cansfz_vof_thinc_cmpt_phi": (I, [V, D, V, V]),
    "cansfz_acdi_set_gamma": (I, [V, D, V, V, V, PD]),
    "cansfz_cmpt_norm_curv_youngs": (I, [V] + [V] * 5),
    "cansfz_clip_field": (I, [V, D, D, V]),
    "cansfz_rk": (I, [V, PD, D, D, PD] + [V] * 12),
    "cansfz_mom_xyz_ad": (I, [V] + [V] * 10),
    "cansfz_mom_xyz_oth": (I, [V, D, PD] + [V] * 9),
    "cansfz_scal_ad": (I, [V] + [V] * 9),
    "cansfz_rk_scal": (I, [V, PD, D] + [V] * 9),
    "cansfz_fillps": (I, [V, D, V, V, V, V]),
    "cansfz_updt_rhs_b": (I, [V, V]),
    "cansfz_solver": (I, [V, V]),
    "cansfz_correc": (I, [V, D, V, V, V, V]),
    "cansfz_updatep": (I, [V, V, V]),
    "cansfz_boundp": (I, [V, I, V]),
    "cansfz_bounduvw": (I, [V, I, V, V, V]),
    "cansfz_chkdt": (I, [V, V, V, V, D, D, PD]),
    "cansfz_chkdiv": (I, [V, V, V, V, PD, PD]),
    "cansfz_bulk_mean_12_stag": (I, [V, I, V, PD]),
    "cansfz_cmpt_mean_mass": (I, [V, V, PD]),
    "cansfz_initgrid": (I, [I, I, D, D, PD, PD, PD, PD]),
    "cansfz_get_grid": (I, [V, PD, PD, PD, PD, PD, PD]),
    # library controls (no reference counterpart)
    "cansfz_set_time": (I, [V, D, ct.c_longlong]),
    "cansfz_set_inivel": (I, [V, ct.c_char_p]),
    "cansfz_kernels_per_step": (I, [V, ct.POINTER(I)]),
    "cansfz_profile_stages": (I, [V, I, PD, I, ct.POINTER(I), ct.c_char_p, I]),
    "cansfz_solver_refined": (I, [V, V, V, I]),
    "cansfz_poisson_residual": (I, [V, V, V, V]),
    "cansfz_xform_matrix": (I, [I, I, I, PD]),
    "cansfz_get_plan": (I, [V, ct.POINTER(Plan)]),
    "cansfz_set_plan": (I, [V, ct.POINTER(Plan)]),
    "cansfz_autotune": (I, [V, ct.c_char_p, ct.POINTER(Plan), ct.c_char_p, I]),
    "cansfz_ensemble_create": (I, [V, I, V, V]),
    "cansfz_ensemble_step": (I, [V, I, V]),
    "cansfz_ensemble_destroy": (I, [V]),
    "cansfz_ensemble_set_batching": (I, [V, I]),
    "cansfz_ensemble_info": (I, [V, ct.POINTER(I), ct.POINTER(I)]),
    "cansfz_solver_static": (I, [ct.POINTER(I), ct.c_char_p, D, V, V, V, V, V, V]),
}

_lib = None


class CansfzError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        super().__init__(f"{what}: status {status} ({STATUS.get(status, 'unknown')})")
        self.status = status


def load():
    """Load libcansfz.so from the source tree (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"{LIBPATH} is not built: run `python cans-fizzy_b200/build.py` "
                               "(or __graft_entry__.build()); there is no CPU fallback")
        L = ct.CDLL(LIBPATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str = "cansfz"):
    if rc != OK:
        raise CansfzError(rc, what)
    return rc
