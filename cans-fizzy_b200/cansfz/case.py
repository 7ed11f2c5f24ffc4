"""High-level host object over the C ABI: one GPU case (the reference's
program cans on a 1x1 pencil), plus the per-procedure entry points with the
reference's argument meaning.

Fields are exchanged in the reference's halo layout: numpy arrays of shape
(nx+2, ny+2, nz+2) in Fortran order, float64.  Device memory and the stream
come from torch (plumbing only; every computation runs in libcansfz).
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from . import lib as _L
from .params import Params


def _dptr(t: torch.Tensor):
    return ct.c_void_p(t.data_ptr())


class DeviceField:
    """A halo-layout (or interior) FP64 field in device memory."""

    def __init__(self, shape, device="cuda"):
        self.shape = tuple(shape)
        self.t = torch.zeros(int(np.prod(shape)), dtype=torch.float64, device=device)

    @property
    def ptr(self):
        return _dptr(self.t)

    def set(self, a: np.ndarray):
        a = np.asarray(a, dtype=np.float64)
        assert a.shape == self.shape, (a.shape, self.shape)
        self.t.copy_(torch.from_numpy(np.ascontiguousarray(a.reshape(-1, order="F"))))
        return self

    def get(self) -> np.ndarray:
        torch.cuda.synchronize()
        return self.t.cpu().numpy().reshape(self.shape, order="F")


class Case:
    """own_stream: the context creates its own CUDA stream instead of using
    torch's current one (cases of an Ensemble need one each; fields then go
    through host arrays, which every entry synchronises)."""

    def __init__(self, params: Params, device: str = "cuda", own_stream: bool = False):
        if not torch.cuda.is_available():
            raise RuntimeError("cansfz needs a CUDA device (B200, sm_100a); there is no CPU fallback")
        self.lib = _L.load()
        self.params = params.copy()
        self.n = params.n
        self.hshape = tuple(x + 2 for x in self.n)
        self.device = device
        self.stream = None if own_stream else torch.cuda.current_stream()
        h = ct.c_void_p()
        st = ct.c_void_p(None if own_stream else self.stream.cuda_stream)
        _L.check(self.lib.cansfz_create(ct.byref(self.params), st, ct.byref(h)), "cansfz_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            torch.cuda.synchronize()
            self.lib.cansfz_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- fields --------------------------------------------------------
    def field(self, a: np.ndarray | None = None) -> DeviceField:
        f = DeviceField(self.hshape, self.device)
        if a is not None:
            f.set(a)
        return f

    def interior(self, a: np.ndarray | None = None) -> DeviceField:
        f = DeviceField(self.n, self.device)
        if a is not None:
            f.set(a)
        return f

    def set_fields(self, u, v, w, p, psi):
        arrs = [np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, order="F")) for x in (u, v, w, p, psi)]
        ptrs = [a.ctypes.data_as(ct.c_void_p) for a in arrs]
        _L.check(self.lib.cansfz_set_fields(self.h, *ptrs, 0), "cansfz_set_fields")

    def get_fields(self):
        outs = [np.zeros(int(np.prod(self.hshape))) for _ in range(5)]
        _L.check(self.lib.cansfz_get_fields(self.h, *[o.ctypes.data_as(ct.c_void_p) for o in outs], 0),
                 "cansfz_get_fields")
        return [o.reshape(self.hshape, order="F") for o in outs]

    # initial conditions computed on the device (no host field arrays)
    def init2fl(self, inipsi: str, spheres=None):
        sph = np.zeros((0, 4)) if spheres is None else np.ascontiguousarray(spheres, dtype=np.float64).reshape(-1, 4)
        ptr = sph.ctypes.data_as(ct.c_void_p) if sph.size else None
        _L.check(self.lib.cansfz_init2fl(self.h, inipsi.encode(), ptr, int(sph.shape[0])), "cansfz_init2fl")

    def initflow(self, inivel: str):
        _L.check(self.lib.cansfz_initflow(self.h, inivel.encode()), "cansfz_initflow")

    def initscal(self, inisca: str):
        _L.check(self.lib.cansfz_initscal(self.h, inisca.encode()), "cansfz_initscal")

    def set_scalar(self, s):
        """The scalar s of a case built with params.scalar = 1 (halo layout)."""
        a = np.ascontiguousarray(np.asarray(s, dtype=np.float64).reshape(-1, order="F"))
        _L.check(self.lib.cansfz_set_scalar(self.h, a.ctypes.data_as(ct.c_void_p), 0), "cansfz_set_scalar")

    def get(self, name: str) -> np.ndarray:
        if name in ("u", "v", "w", "p", "psi"):
            return self.get_fields()[("u", "v", "w", "p", "psi").index(name)]
        interior = name.endswith("dtrko") or name.startswith("surf")
        shape = self.n if interior else self.hshape
        out = np.zeros(int(np.prod(shape)))
        _L.check(self.lib.cansfz_get_aux(self.h, name.encode(), out.ctypes.data_as(ct.c_void_p), 0), name)
        return out.reshape(shape, order="F")

    def set_time(self, time: float, istep: int):
        _L.check(self.lib.cansfz_set_time(self.h, float(time), int(istep)), "cansfz_set_time")

    def set_inivel(self, inivel: str):
        _L.check(self.lib.cansfz_set_inivel(self.h, inivel.encode()), "cansfz_set_inivel")

    def prepare(self):
        _L.check(self.lib.cansfz_prepare(self.h), "cansfz_prepare")

    def step(self, nsteps: int = 1) -> int:
        return self.lib.cansfz_step(self.h, int(nsteps))

    def diag(self) -> _L.Diag:
        d = _L.Diag()
        _L.check(self.lib.cansfz_get_diag(self.h, ct.byref(d)), "cansfz_get_diag")
        return d

    def status(self) -> _L.Diag:
        """The per-step scalars of diag() without the phase masses (NaN)."""
        d = _L.Diag()
        _L.check(self.lib.cansfz_get_status(self.h, ct.byref(d)), "cansfz_get_status")
        return d

    def plan(self) -> _L.Plan:
        q = _L.Plan()
        _L.check(self.lib.cansfz_get_plan(self.h, ct.byref(q)), "cansfz_get_plan")
        return q

    def set_plan(self, q: _L.Plan):
        _L.check(self.lib.cansfz_set_plan(self.h, ct.byref(q)), "cansfz_set_plan")

    def autotune(self, cache_file: str | None = None):
        """Time candidate launch plans on a copy of this case and apply the
        fastest (cansfz_autotune); returns (plan, one-line report)."""
        q = _L.Plan()
        rep = ct.create_string_buffer(256)
        _L.check(self.lib.cansfz_autotune(self.h, cache_file.encode() if cache_file else None, ct.byref(q), rep, 256),
                 "cansfz_autotune")
        return q, rep.value.decode()

    def grid(self):
        nz = self.n[2]
        arrs = [np.zeros(nz + 2) for _ in range(6)]
        _L.check(self.lib.cansfz_get_grid(self.h, *[a.ctypes.data_as(_L.PD) for a in arrs]), "cansfz_get_grid")
        return dict(zip(("dzc", "dzf", "zc", "zf", "dzci", "dzfi"), arrs))

    # ---- per-procedure entries (device fields) ---------------------------
    def call(self, name: str, *args):
        conv = []
        for a in args:
            if isinstance(a, DeviceField):
                conv.append(a.ptr)
            elif isinstance(a, (list, tuple)) and all(isinstance(x, float) for x in a):
                conv.append((ct.c_double * len(a))(*a))
            elif isinstance(a, np.ndarray):
                conv.append(a.ctypes.data_as(_L.PD))
            else:
                conv.append(a)
        rc = getattr(self.lib, "cansfz_" + name)(self.h, *conv)
        _L.check(rc, "cansfz_" + name)
        torch.cuda.synchronize()
        return rc


class Ensemble:
    """Independent cases advanced together: one CUDA graph launch per step
    holds every case's step as a parallel branch (cansfz_ensemble_*).  With
    batch > 1, cases of the same grid and options share batched launches in
    groups of up to `batch` cases."""

    def __init__(self, cases, batch: int = 1):
        self.lib = _L.load()
        self.cases = list(cases)
        arr = (ct.c_void_p * len(self.cases))(*[c.h.value for c in self.cases])
        h = ct.c_void_p()
        _L.check(self.lib.cansfz_ensemble_create(arr, len(self.cases), None, ct.byref(h)), "cansfz_ensemble_create")
        self.h = h
        if batch != 1:
            _L.check(self.lib.cansfz_ensemble_set_batching(self.h, int(batch)), "cansfz_ensemble_set_batching")

    def step(self, nsteps: int = 1):
        st = (ct.c_int * len(self.cases))()
        rc = self.lib.cansfz_ensemble_step(self.h, int(nsteps), st)
        return rc, list(st)

    def groups(self):
        """(number of case groups, cases in groups of two or more) of the
        graph built at the last step."""
        ng, gc = ct.c_int(), ct.c_int()
        _L.check(self.lib.cansfz_ensemble_info(self.h, ct.byref(ng), ct.byref(gc)), "cansfz_ensemble_info")
        return ng.value, gc.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.cansfz_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
