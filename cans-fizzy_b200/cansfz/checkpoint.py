"""Checkpoint files in the reference's restart format (load_one,
src/load.f90:13-170, as program cans writes and reads them at
src/main.f90:304-330,600-632).

One file per field, `<name>_<ext>.bin` with ext in u, v, w, p, psi (and s
for a case with the scalar, src/main.f90:313-314): the interior
ng(1) x ng(2) x ng(3) array in Fortran order, native FP64, followed by two
reals [time, istep].  The reference aborts on a file whose size is
not (ng(1)*ng(2)*ng(3) + 2) * 8 bytes; read_field() raises instead.
Restarting from these files behaves as the reference does: the AB2
histories are not stored, so the first step after a restart is an Euler step
in both.

save() can hand the host copies to a background thread, so that stepping
continues while the files are written.
"""
from __future__ import annotations

import os
import threading

import numpy as np

FIELDS = ("u", "v", "w", "p", "psi")
SCALAR = ("s",)


class CheckpointError(RuntimeError):
    pass


def _path(datadir: str, name: str, ext: str) -> str:
    return os.path.join(datadir, f"{name}_{ext}.bin")


def write_field(path: str, interior: np.ndarray, time: float, istep: int) -> None:
    a = np.asarray(interior, dtype=np.float64)
    with open(path, "wb") as f:
        f.write(np.asfortranarray(a).tobytes(order="F"))
        f.write(np.array([time, float(istep)], dtype=np.float64).tobytes())


def read_field(path: str, ng) -> tuple[np.ndarray, float, int]:
    ng = tuple(int(x) for x in ng)
    good = (int(np.prod(ng)) + 2) * 8
    size = os.path.getsize(path)
    if size != good:
        raise CheckpointError(f"checkpoint file with incorrect size: {path} | expected size: {good} "
                              f"| actual size: {size}")
    raw = np.fromfile(path, dtype=np.float64)
    a = raw[:-2].reshape(ng, order="F")
    return a, float(raw[-2]), int(round(raw[-1]))


def save_fields(datadir: str, name: str, halo_fields, time: float, istep: int, exts=FIELDS) -> None:
    """Write u, v, w, p, psi (and s with exts = FIELDS + SCALAR; halo-layout
    arrays) as `<name>_<ext>.bin`."""
    os.makedirs(datadir, exist_ok=True)
    for ext, a in zip(exts, halo_fields):
        write_field(_path(datadir, name, ext), a[1:-1, 1:-1, 1:-1], time, istep)


def load_fields(datadir: str, ng, name: str = "fld", exts=FIELDS):
    """Read `<name>_<ext>.bin` into halo-layout arrays (ghosts zero, filled by
    the boundary conditions when the case is prepared); returns the arrays
    (one per ext), time and istep (from the last file read, as the
    reference)."""
    out = []
    time, istep = 0.0, 0
    for ext in exts:
        a, time, istep = read_field(_path(datadir, name, ext), ng)
        h = np.zeros(tuple(n + 2 for n in ng), order="F")
        h[1:-1, 1:-1, 1:-1] = a
        out.append(h)
    return out, time, istep


def save(case, datadir: str, name: str = "fld", background: bool = False):
    """Checkpoint a cansfz Case.  The device-to-host copy is synchronous (it
    must see the current step); with background=True the file writes run on
    a thread, which is returned (join it before the next save)."""
    fields = case.get_fields()
    exts = FIELDS
    if case.params.scalar:
        fields.append(case.get("s"))
        exts = FIELDS + SCALAR
    d = case.diag()
    if not background:
        save_fields(datadir, name, fields, d.time, d.istep, exts)
        return None
    t = threading.Thread(target=save_fields, args=(datadir, name, fields, d.time, d.istep, exts))
    t.start()
    return t


def restore(case, datadir: str, name: str = "fld"):
    """Load a checkpoint into a cansfz Case (fields, time, istep); the caller
    then runs case.prepare(), as program cans does after reading it."""
    exts = FIELDS + SCALAR if case.params.scalar else FIELDS
    fields, time, istep = load_fields(datadir, case.n, name, exts)
    case.set_fields(*fields[:5])
    if case.params.scalar:
        case.set_scalar(fields[5])
    case.set_time(time, istep)
    return time, istep
