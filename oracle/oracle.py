"""ORACLE -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper of the C++ restatement of the reference's single-rank CPU
path (oracle/cansfz_oracle.cpp).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use it; the product path never does.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle_cansfz.so")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "cans-fizzy_b200"))

from cansfz.params import Params  # noqa: E402

_lib = None
D = ct.c_double
P = ct.POINTER(ct.c_double)
V = ct.c_void_p


def build():
    """Compile the oracle with its Makefile (g++ -O2 -fopenmp -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Diag(ct.Structure):
    _fields_ = [("time", D), ("istep", ct.c_int64), ("dt", D), ("dto", D), ("dt_cfl", D),
                ("gam", D), ("seps", D), ("divtot", D), ("divmax", D), ("mass12", D * 2),
                ("status", ct.c_int32), ("reserved", ct.c_int32 * 7)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ct.CDLL(LIB)
        sig = {
            "orc_create": (V, [ct.POINTER(Params)]),
            "orc_destroy": (None, [V]),
            "orc_set_threads": (ct.c_int, [ct.c_int]),
            "orc_set_field": (ct.c_int, [V, ct.c_char_p, P]),
            "orc_get_field": (ct.c_int, [V, ct.c_char_p, P]),
            "orc_set_inivel": (None, [V, ct.c_char_p]),
            "orc_set_time": (None, [V, D, ct.c_longlong]),
            "orc_init2fl": (ct.c_int, [V, ct.c_char_p, P, ct.c_int]),
            "orc_initflow": (ct.c_int, [V, ct.c_char_p, D]),
            "orc_prepare": (None, [V]),
            "orc_step": (ct.c_int, [V, ct.c_int]),
            "orc_get_diag": (None, [V, ct.POINTER(Diag)]),
            "orc_get_grid": (None, [V, P, P, P, P, P, P]),
            "orc_seps": (D, [V]),
            "orc_normfft": (D, [V]),
            "orc_solver_data": (None, [V, P, P, P, P]),
            "orc_acdi_transport_pf": (None, [V, D, D] + [P] * 12),
            "orc_vof_thinc_transport_psi": (None, [V, D] + [P] * 12),
            "orc_acdi_cmpt_phi": (None, [V, D, P, P]),
            "orc_vof_thinc_cmpt_phi": (None, [V, D, P, P]),
            "orc_cmpt_norm_curv_youngs": (None, [V] + [P] * 5),
            "orc_mom_xyz_ad": (None, [V] + [P] * 10),
            "orc_mom_xyz_oth": (None, [V, D] + [P] * 10),
            "orc_scal_ad": (None, [V] + [P] * 9),
            "orc_initscal": (ct.c_int, [V, ct.c_char_p]),
            "orc_rk_scal": (ct.c_int, [V, P, D] + [P] * 9),
            "orc_fillps": (None, [V, D, P, P, P, P]),
            "orc_updt_rhs_b": (None, [V, P]),
            "orc_solver": (None, [V, P]),
            "orc_correc": (None, [V, D, P, P, P, P]),
            "orc_updatep": (None, [V, P, P]),
            "orc_clip_field": (None, [V, D, D, P]),
            "orc_rk_2fl": (None, [V, P, D, D, D, D] + [P] * 10),
            "orc_rk": (None, [V, P, D, D, P] + [P] * 12),
            "orc_cmpt_mean_mass": (None, [V, P, P]),
            "orc_boundp": (None, [V, ct.c_int, P]),
            "orc_bounduvw": (None, [V, ct.c_int, P, P, P]),
            "orc_acdi_set_gamma": (D, [V, D, P, P, P]),
            "orc_chkdt_fields": (D, [V, P, P, P, D, D]),
            "orc_chkdiv_fields": (None, [V, P, P, P, P, P]),
            "orc_bulk_mean_12_stag": (D, [V, ct.c_int, P]),
            "orc_r2r": (None, [ct.c_int, ct.c_int, ct.c_int, P]),
            "orc_initgrid": (ct.c_int, [ct.c_int, ct.c_int, D, D, P, P, P, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def ptr(a: np.ndarray):
    """Pointer to a float64 array in Fortran order (the reference layout)."""
    if a.dtype != np.float64 or not (a.flags["F_CONTIGUOUS"] if a.ndim > 1 else a.flags["C_CONTIGUOUS"]):
        raise ValueError("oracle arrays must be float64 and Fortran-contiguous")
    return a.ctypes.data_as(P)


def set_threads(n: int) -> int:
    return lib().orc_set_threads(int(n))


def r2r(kind: int, x: np.ndarray) -> np.ndarray:
    """FFTW-kind r2r transform along the last axis (returns a copy)."""
    y = np.ascontiguousarray(x, dtype=np.float64).copy()
    n = y.shape[-1]
    lib().orc_r2r(kind, n, y.size // n, y.ctypes.data_as(P))  # C-order lines
    return y


class Case:
    """One oracle case: the set-up of program cans and its time loop."""

    FIELDS = ("u", "v", "w", "p", "psi")

    def __init__(self, params: Params):
        self.params = params.copy()
        self.n = params.n
        self.h = lib().orc_create(ct.byref(self.params))
        self.hshape = tuple(x + 2 for x in self.n)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    # halo-layout arrays are Fortran-ordered numpy arrays of shape n+2
    def empty(self):
        return np.zeros(self.hshape, order="F")

    def get(self, name: str) -> np.ndarray:
        interior = name in ("dudtrko", "dvdtrko", "dwdtrko", "dpsidtrko", "dsdtrko") or name.startswith("surf")
        a = np.zeros(self.n if interior else self.hshape, order="F")
        rc = lib().orc_get_field(self.h, name.encode(), ptr(a))
        if rc:
            raise KeyError(name)
        return a

    def set(self, name: str, a: np.ndarray):
        a = np.asfortranarray(a, dtype=np.float64)
        assert a.shape == self.hshape, (a.shape, self.hshape)
        rc = lib().orc_set_field(self.h, name.encode(), ptr(a))
        if rc:
            raise KeyError(name)

    def init2fl(self, inipsi: str, spheres=None):
        sph = np.zeros((0, 4)) if spheres is None else np.ascontiguousarray(spheres, dtype=np.float64)
        lib().orc_init2fl(self.h, inipsi.encode(), sph.ctypes.data_as(P) if sph.size else None,  # rows (x,y,z,r)
                          int(sph.shape[0]))

    def initflow(self, inivel: str, time: float = 0.0):
        lib().orc_initflow(self.h, inivel.encode(), float(time))

    def initscal(self, inisca: str):
        rc = lib().orc_initscal(self.h, inisca.encode())
        if rc:
            raise ValueError(f"initscal: invalid name '{inisca}' or no scalar in this case")

    def set_inivel(self, inivel: str):
        lib().orc_set_inivel(self.h, inivel.encode())

    def prepare(self):
        lib().orc_prepare(self.h)

    def step(self, nsteps: int = 1) -> int:
        return lib().orc_step(self.h, int(nsteps))

    def diag(self) -> Diag:
        d = Diag()
        lib().orc_get_diag(self.h, ct.byref(d))
        return d

    @property
    def seps(self):
        return lib().orc_seps(self.h)

    @property
    def normfft(self):
        return lib().orc_normfft(self.h)

    def grid(self):
        nz = self.n[2]
        arrs = [np.zeros(nz + 2) for _ in range(6)]
        lib().orc_get_grid(self.h, *[ptr(a) for a in arrs])
        return dict(zip(("dzc", "dzf", "zc", "zf", "dzci", "dzfi"), arrs))

    def solver_data(self):
        nx, ny, nz = self.n
        lam = np.zeros((nx, ny), order="F")
        a, b, c = np.zeros(nz), np.zeros(nz), np.zeros(nz)
        lib().orc_solver_data(self.h, ptr(lam), ptr(a), ptr(b), ptr(c))
        return lam, a, b, c

    # per-procedure restatements on host arrays
    def call(self, name: str, *args):
        conv = []
        for a in args:
            if isinstance(a, np.ndarray):
                conv.append(ptr(a))
            else:
                conv.append(a)
        return getattr(lib(), "orc_" + name)(self.h, *conv)
