"""cansfz_solver_static: the allocation-free Poisson solve, through the C ABI.

It serves callers that cannot allocate device memory while the solver runs
(device memory owned by another runtime's pool, or code that must not incur
the synchronisation of cudaMalloc).  Its scratch lives in static device
arrays; this test checks it against the context-based entry cansfz_solver on
two calls in a row, with the tolerance of the other Poisson parity tests.
The file is named to run last, so a failure here leaves every other test run.
"""
import ctypes as ct

import numpy as np
import pytest
import torch

from cansfz import case as C
from cansfz import init, lib, namelist, params

pytestmark = pytest.mark.gpu


def _packed_eigs(n, kind, dli):
    """Eigenvalues of the x or y operator in the solver's spectral order
    (periodic: (r0, r_{n/2}, r1, i1, ...), the order of the reference's GPU
    path, src/initsolver.f90:94-113)."""
    if kind == "PP":
        lam = lambda m: -2.0 * (1.0 - np.cos((2 * m) * np.pi / n))  # noqa: E731
        out = np.zeros(n)
        out[0], out[1] = lam(0), lam(n // 2)
        for k in range(1, n // 2):
            out[2 * k], out[2 * k + 1] = lam(k), lam(n - k)
    elif kind == "NN":
        out = -2.0 * (1.0 - np.cos(np.arange(n) * np.pi / n))
    else:
        out = -2.0 * (1.0 - np.cos(np.arange(1, n + 1) * np.pi / n))
    return out * dli * dli


@pytest.mark.parametrize("cbc", ["PPPPNN", "NNPPNN", "DDPPDD"])
def test_static_solver_matches_context_solver(cbc):
    nx, ny, nz = 32, 24, 40
    l = (1.0, 0.75, 1.25)
    nl = namelist.defaults()
    nl.set("ng", np.array([nx, ny, nz]))
    nl.set("l", np.array(l))
    cp = np.array(list(cbc), dtype=object).reshape((2, 3), order="F")
    nl.set("cbcpre", cp)
    nl.set("cbcpsi", cp.copy())
    p = params.from_namelist(nl)
    g = C.Case(p)
    L = lib.load()
    L.cansfz_solver_static.restype = ct.c_int
    L.cansfz_solver_static.argtypes = [ct.POINTER(ct.c_int), ct.c_char_p, ct.c_double, ct.c_void_p, ct.c_void_p,
                                       ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    # inputs of the static entry: eigenvalues, z coefficients, normfft
    lx = _packed_eigs(nx, cbc[0:2], nx / l[0])
    ly = _packed_eigs(ny, cbc[2:4], ny / l[1])
    lam = (lx[:, None] + ly[None, :]).reshape(-1, order="F")
    zg = init.zgrid(p)
    a = zg["dzfi"][1:nz + 1] * zg["dzci"][0:nz]
    c = zg["dzfi"][1:nz + 1] * zg["dzci"][1:nz + 1]
    b = -(a + c)
    fz = {"P": 0.0, "D": -1.0, "N": 1.0}
    b[0] += fz[cbc[4]] * a[0]
    b[-1] += fz[cbc[5]] * c[-1]
    normfft = 1.0 / ((1.0 if cbc[0] == "P" else 2.0) * nx * (1.0 if cbc[2] == "P" else 2.0) * ny)
    dev = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (lam, a, b, c)]
    n3 = (ct.c_int * 3)(nx, ny, nz)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(17)
    for call in range(2):  # two calls in a row: the shared scratch keeps the last call's contents
        rhs = np.zeros((nx + 2, ny + 2, nz + 2), order="F")
        rhs[1:-1, 1:-1, 1:-1] = rng.standard_normal((nx, ny, nz))
        if "D" not in cbc:
            rhs[1:-1, 1:-1, 1:-1] -= rhs[1:-1, 1:-1, 1:-1].mean()
        ref = g.field(rhs)
        g.call("solver", ref)
        out = g.field(rhs)
        rc = L.cansfz_solver_static(n3, cbc.encode(), normfft, *[ct.c_void_p(t.data_ptr()) for t in dev],
                                    out.ptr, ct.c_void_p(stream))
        assert rc == 0, rc
        torch.cuda.synchronize()
        a_, b_ = out.get()[1:-1, 1:-1, 1:-1], ref.get()[1:-1, 1:-1, 1:-1]
        scale = max(np.abs(a_).max(), np.abs(b_).max())
        if "D" not in cbc:
            a_, b_ = a_ - a_.mean(), b_ - b_.mean()
        assert np.abs(a_ - b_).max() / scale < 1e-12, (cbc, call)


def test_static_solver_rejects_oversize():
    """Sizes beyond the static scratch, or beyond what the z solve launches
    with, return CANSFZ_ERR_ARG and leave p untouched."""
    L = lib.load()
    L.cansfz_solver_static.restype = ct.c_int
    L.cansfz_solver_static.argtypes = [ct.POINTER(ct.c_int), ct.c_char_p, ct.c_double, ct.c_void_p, ct.c_void_p,
                                       ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    ptr = ct.c_void_p(dummy.data_ptr())
    for n in ((256, 256, 256), (16, 16, 4096)):  # above 128^3 cells; nz above 1536
        p = torch.arange((n[0] + 2) * (n[1] + 2) * (n[2] + 2), dtype=torch.float64, device="cuda")
        before = p.clone()
        n3 = (ct.c_int * 3)(*n)
        rc = L.cansfz_solver_static(n3, b"PPPPNN", 1.0, ptr, ptr, ptr, ptr, ct.c_void_p(p.data_ptr()), None)
        torch.cuda.synchronize()
        assert rc == 1, (n, rc)  # CANSFZ_ERR_ARG, nothing launched
        assert torch.equal(p, before), n


def test_static_solver_allocates_nothing():
    """Once each shape has run (the set-up, and the driver's loading of the
    kernels' code on their first launch), further calls of those sizes and
    BCs leave the device's free memory unchanged."""
    L = lib.load()
    L.cansfz_solver_static.restype = ct.c_int
    L.cansfz_solver_static.argtypes = [ct.POINTER(ct.c_int), ct.c_char_p, ct.c_double, ct.c_void_p, ct.c_void_p,
                                       ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    cases = [((32, 24, 40), b"PPPPNN"), ((64, 48, 96), b"NNPPNN"), ((128, 128, 128), b"DDPPDD"),
             ((96, 64, 80), b"PPNNDD")]
    bufs = []
    for n, cbc in cases:  # every input allocated before the measurement
        nx, ny, nz = n
        lam = torch.full((nx * ny,), -1.0, dtype=torch.float64, device="cuda")
        a = torch.full((nz,), 1.0, dtype=torch.float64, device="cuda")
        c = a.clone()
        b = torch.full((nz,), -3.0, dtype=torch.float64, device="cuda")
        p = torch.randn((nx + 2) * (ny + 2) * (nz + 2), dtype=torch.float64, device="cuda")
        bufs.append((n, cbc, lam, a, b, c, p))
    stream = torch.cuda.current_stream().cuda_stream

    def call(n, cbc, lam, a, b, c, p):
        n3 = (ct.c_int * 3)(*n)
        return L.cansfz_solver_static(n3, cbc, 1e-3, *[ct.c_void_p(t.data_ptr()) for t in (lam, a, b, c, p)],
                                      ct.c_void_p(stream))

    # one call of each shape first: the set-up on this device, and the
    # driver's first-launch loading of each transform length's kernel code
    # (lazy module loading, the CUDA 12 default), which is not the solver's
    for b in bufs:
        assert call(*b) == 0, b[:2]
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for q in (1, 2, 3, 0, 2, 1):
        assert call(*bufs[q]) == 0, bufs[q][:2]
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
