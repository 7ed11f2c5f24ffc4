"""``cansfz_params`` (include/cansfz.h) as a ctypes structure, filled from a
reference ``input.nml`` (src/param.f90:86-245)."""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import namelist as _nml

ACDI, VOF_THINC = 0, 1
FORM_FP64, FORM_MIXED = 0, 1


class Params(ct.Structure):
    _fields_ = [
        ("ng", ct.c_int32 * 3),
        ("l", ct.c_double * 3),
        ("gtype", ct.c_int32),
        ("gr", ct.c_double),
        ("cfl", ct.c_double),
        ("dtmax", ct.c_double),
        ("dt_f", ct.c_double),
        ("is_solve_ns", ct.c_int32),
        ("is_track_interface", ct.c_int32),
        ("icheck", ct.c_int32),
        ("cbcvel", ct.c_char * 18),
        ("bcvel", ct.c_double * 18),
        ("cbcpre", ct.c_char * 6),
        ("bcpre", ct.c_double * 6),
        ("bforce", ct.c_double * 3),
        ("gacc", ct.c_double * 3),
        ("cbcpsi", ct.c_char * 6),
        ("bcpsi", ct.c_double * 6),
        ("cbcnor", ct.c_char * 18),
        ("bcnor", ct.c_double * 18),
        ("sigma", ct.c_double),
        ("rho12", ct.c_double * 2),
        ("mu12", ct.c_double * 2),
        ("beta12", ct.c_double * 2),
        ("psi_thickness_factor", ct.c_double),
        ("acdi_gam_factor", ct.c_double),
        ("acdi_gam_min", ct.c_double),
        ("interface_capturing", ct.c_int32),
        ("sdf_normals", ct.c_int32),
        ("brackbill", ct.c_int32),
        ("balanced", ct.c_int32),
        ("scalar", ct.c_int32),
        ("boussinesq", ct.c_int32),
        ("cbcsca", ct.c_char * 6),
        ("bcsca", ct.c_double * 6),
        ("ssource", ct.c_double),
        ("ka12", ct.c_double * 2),
        ("cp12", ct.c_double * 2),
        ("form", ct.c_int32),
        ("refine_sweeps", ct.c_int32),
        ("fp32_transforms", ct.c_int32),
        ("reserved", ct.c_int32 * 7),
    ]

    # -- convenience views -------------------------------------------------
    @property
    def n(self):
        return tuple(int(x) for x in self.ng)

    def cbc(self, name):
        """Character BC array as a numpy array in reference index order."""
        raw = bytes(getattr(self, name))
        shape = (2, 3, 3) if len(raw) == 18 else (2, 3)
        return np.array(list(raw.decode()), dtype=object).reshape(shape, order="F")

    def copy(self):
        p = Params()
        ct.memmove(ct.byref(p), ct.byref(self), ct.sizeof(Params))
        return p


def _chars(a) -> bytes:
    flat = np.asarray(a, dtype=object).reshape(-1, order="F")
    return "".join(str(x)[0] for x in flat).encode()


def _dbls(a):
    return [float(x) for x in np.asarray(a, dtype=np.float64).reshape(-1, order="F")]


def from_namelist(nl: _nml.Namelist) -> Params:
    """cansfz_params from a parsed input.nml (plus the optional &cansfz group)."""
    p = Params()
    p.ng[:] = [int(x) for x in nl["ng"]]
    p.l[:] = _dbls(nl["l"])
    p.gtype = int(nl["gtype"])
    p.gr = float(nl["gr"])
    p.cfl = float(nl["cfl"])
    p.dtmax = float(nl["dtmax"])
    p.dt_f = float(nl["dt_f"])
    p.is_solve_ns = int(bool(nl["is_solve_ns"]))
    p.is_track_interface = int(bool(nl["is_track_interface"]))
    p.icheck = int(nl["icheck"])
    p.cbcvel = _chars(nl["cbcvel"])
    p.bcvel[:] = _dbls(nl["bcvel"])
    p.cbcpre = _chars(nl["cbcpre"])
    p.bcpre[:] = _dbls(nl["bcpre"])
    p.bforce[:] = _dbls(nl["bforce"])
    p.gacc[:] = _dbls(nl["gacc"])
    p.cbcpsi = _chars(nl["cbcpsi"])
    p.bcpsi[:] = _dbls(nl["bcpsi"])
    p.cbcnor = _chars(nl["cbcnor"])
    p.bcnor[:] = _dbls(nl["bcnor"])
    p.sigma = float(nl["sigma"])
    p.rho12[:] = _dbls(nl["rho12"])
    p.mu12[:] = _dbls(nl["mu12"])
    p.beta12[:] = _dbls(nl["beta12"])
    vof = bool(nl["interface_capturing_vof"])
    ptf = float(nl["psi_thickness_factor"])
    if vof and ptf == _nml._sp(0.51):
        ptf = 0.50  # the reference's VOF default (src/param.f90:151-153)
    p.psi_thickness_factor = ptf
    p.acdi_gam_factor = float(nl["acdi_gam_factor"])
    p.acdi_gam_min = float(nl["acdi_gam_min"])
    p.interface_capturing = VOF_THINC if vof else ACDI
    p.sdf_normals = int(bool(nl["sdf_normals"]))
    p.brackbill = int(bool(nl["capillary_brackbill_normalization"]))
    p.balanced = int(bool(nl["balanced_capillary_pressure_split"]))
    p.scalar = int(bool(nl["scalar"]))
    p.boussinesq = int(bool(nl["boussinesq_buoyancy"]))
    p.cbcsca = _chars(nl["cbcsca"])
    p.bcsca[:] = _dbls(nl["bcsca"])
    p.ssource = float(nl["ssource"])
    p.ka12[:] = _dbls(nl["ka12"])
    p.cp12[:] = _dbls(nl["cp12"])
    p.form = FORM_MIXED if str(nl["form"]).lower().startswith("mix") else FORM_FP64
    p.refine_sweeps = int(nl["refine_sweeps"])
    p.fp32_transforms = 1 if str(nl["fp32_transforms"]).lower().startswith("fft") else 0
    return p


def from_file(path: str) -> Params:
    return from_namelist(_nml.read(path))


def from_text(text: str) -> Params:
    return from_namelist(_nml.parse(text))
