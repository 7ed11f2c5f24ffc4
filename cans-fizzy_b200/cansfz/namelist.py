"""Reader for the reference's ``input.nml`` (namelists ``&dns``, ``&scalar``,
``&two_fluid``, ``&cudecomp``; src/param.f90:86-245).

Only the Fortran namelist subset the reference's input files use is
supported: scalar and array assignments with explicit index ranges
(``cbcvel(0:1,1:3,1) = 'D','D', 'P','P', 'D','D'``), strings, logicals
(``T``/``F``/``.true.``/``.false.``), integers and reals (``1.e-4``,
``1.d0``), ``!`` comments, repeat counts (``3*0.``).  Arrays fill in Fortran
(column-major) order over the given ranges, as a Fortran ``read(nml=...)``
does.

The defaults are those of ``read_input`` (src/param.f90:124-150).  Where
the reference writes a default with a default-kind (single-precision)
literal, e.g. ``cfl = 0.95`` or ``acdi_gam_min = 1.e-12``, the value is the
single-precision number promoted to double, as it is in the reference.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

import numpy as np


def _sp(x: float) -> float:
    """A default-kind Fortran real literal promoted to real(8)."""
    return float(np.float32(x))


@dataclass
class Var:
    kind: str            # 'i', 'r', 'l', 's'
    lbounds: tuple       # lower bounds per dim ((): scalar)
    shape: tuple
    default: object


def _arr(kind, lb, shape, default):
    return Var(kind, tuple(lb), tuple(shape), default)


# &dns, &two_fluid, &scalar (src/param.f90:91-120, defaults :124-150)
SCHEMA = {
    "dns": {
        "ng": _arr("i", [1], [3], [128, 128, 128]),
        "l": _arr("r", [1], [3], [1.0, 1.0, 1.0]),
        "gtype": Var("i", (), (), 1),
        "gr": Var("r", (), (), 0.0),
        "cfl": Var("r", (), (), _sp(0.95)),
        "dtmax": Var("r", (), (), _sp(1.0e9)),
        "dt_f": Var("r", (), (), -1.0),
        "is_solve_ns": Var("l", (), (), True),
        "is_track_interface": Var("l", (), (), True),
        "inivel": Var("s", (), (), "zer"),
        "is_wallturb": Var("l", (), (), False),
        "is_forced_hit": Var("l", (), (), False),
        "nstep": Var("i", (), (), 1000),
        "time_max": Var("r", (), (), 1.0),
        "tw_max": Var("r", (), (), 0.5),
        "stop_type": _arr("l", [1], [3], [True, False, False]),
        "restart": Var("l", (), (), False),
        "is_overwrite_save": Var("l", (), (), True),
        "nsaves_max": Var("i", (), (), 0),
        "icheck": Var("i", (), (), 10),
        "iout0d": Var("i", (), (), 10),
        "iout1d": Var("i", (), (), 100),
        "iout2d": Var("i", (), (), 1000),
        "iout3d": Var("i", (), (), 500),
        "isave": Var("i", (), (), 1000),
        "cbcvel": _arr("s", [0, 1, 1], [2, 3, 3], "P"),
        "cbcpre": _arr("s", [0, 1], [2, 3], "P"),
        "bcvel": _arr("r", [0, 1, 1], [2, 3, 3], 0.0),
        "bcpre": _arr("r", [0, 1], [2, 3], 0.0),
        "bforce": _arr("r", [1], [3], 0.0),
        "gacc": _arr("r", [1], [3], 0.0),
        "dims": _arr("i", [1], [2], 0),
    },
    "scalar": {
        "inisca": Var("s", (), (), "zer"),
        "cbcsca": _arr("s", [0, 1], [2, 3], "P"),
        "bcsca": _arr("r", [0, 1], [2, 3], 0.0),
        "ssource": Var("r", (), (), 0.0),
    },
    "two_fluid": {
        "inipsi": Var("s", (), (), "uni"),
        "cbcpsi": _arr("s", [0, 1], [2, 3], "P"),
        "cbcnor": _arr("s", [0, 1, 1], [2, 3, 3], "P"),
        "bcnor": _arr("r", [0, 1, 1], [2, 3, 3], 0.0),
        "bcpsi": _arr("r", [0, 1], [2, 3], 0.0),
        "sigma": Var("r", (), (), 0.0),
        "rho12": _arr("r", [1], [2], 1.0),
        "mu12": _arr("r", [1], [2], _sp(0.01)),
        "ka12": _arr("r", [1], [2], _sp(0.01)),
        "cp12": _arr("r", [1], [2], 1.0),
        "beta12": _arr("r", [1], [2], 1.0),
        "psi_thickness_factor": Var("r", (), (), _sp(0.51)),
    },
    # switches of this library for the reference's compile-time macros and
    # for the two extra forms; not a reference namelist (ignored by it)
    "cansfz": {
        "interface_capturing_vof": Var("l", (), (), False),
        "sdf_normals": Var("l", (), (), True),
        "capillary_brackbill_normalization": Var("l", (), (), True),
        "balanced_capillary_pressure_split": Var("l", (), (), False),
        "scalar": Var("l", (), (), False),
        "boussinesq_buoyancy": Var("l", (), (), False),
        "acdi_gam_factor": Var("r", (), (), 1.0),
        "acdi_gam_min": Var("r", (), (), _sp(1.0e-12)),
        "form": Var("s", (), (), "fp64"),
        "refine_sweeps": Var("i", (), (), -1),
        # the FP32 solve's x/y transforms: 'gemm' (tensor cores where the
        # line lengths allow) or 'fft'
        "fp32_transforms": Var("s", (), (), "gemm"),
    },
    "cudecomp": {},
}


def _default_value(v: Var):
    if not v.shape:
        return v.default
    dt = {"i": np.int64, "r": np.float64, "l": np.bool_, "s": object}[v.kind]
    a = np.empty(v.shape, dtype=dt, order="F")
    if isinstance(v.default, list):
        a[...] = np.array(v.default, dtype=dt).reshape(v.shape, order="F")
    else:
        a[...] = v.default
    return a


@dataclass
class Namelist:
    groups: dict = field(default_factory=dict)

    def __getitem__(self, key):
        for g in self.groups.values():
            if key in g:
                return g[key]
        raise KeyError(key)

    def get(self, key, default=None):
        try:
            return self[key]
        except KeyError:
            return default

    def set(self, key, value):
        for g in self.groups.values():
            if key in g:
                g[key] = value
                return
        raise KeyError(key)


def defaults() -> Namelist:
    nl = Namelist()
    for gname, sch in SCHEMA.items():
        nl.groups[gname] = {k: _default_value(v) for k, v in sch.items()}
    return nl


_TOKEN = re.compile(r"""\s*(?:'([^']*)'|"([^"]*)"|([^,\s]+))\s*,?""")
_ASSIGN = re.compile(r"([A-Za-z_][A-Za-z0-9_]*)\s*(\(([^)]*)\))?\s*=")


def _parse_scalar(tok: str, kind: str):
    t = tok.strip()
    if kind == "s":
        return t
    if kind == "l":
        tl = t.lower().strip(".")
        if tl.startswith("t"):
            return True
        if tl.startswith("f"):
            return False
        raise ValueError(f"bad logical {tok!r}")
    t = t.replace("d", "e").replace("D", "e")
    if kind == "i":
        return int(float(t)) if ("." in t or "e" in t.lower()) else int(t)
    return float(t)


def _tokens(text: str):
    out = []
    pos = 0
    text = text.strip()
    while pos < len(text):
        m = _TOKEN.match(text, pos)
        if not m or m.end() == pos:
            break
        pos = m.end()
        s = m.group(1) if m.group(1) is not None else m.group(2)
        if s is not None:
            out.append(("s", s))
        else:
            tok = m.group(3)
            rep = re.fullmatch(r"(\d+)\*(.*)", tok)
            if rep and rep.group(2):
                out.extend([("t", rep.group(2))] * int(rep.group(1)))
            else:
                out.append(("t", tok))
    return out


def _index_ranges(spec: str | None, var: Var):
    """Fortran index spec -> list of per-dim python ranges (0-based)."""
    if not var.shape:
        return None
    if spec is None:
        return [range(0, s) for s in var.shape]
    parts = [p.strip() for p in spec.split(",")]
    if len(parts) != len(var.shape):
        raise ValueError(f"rank mismatch in index spec {spec!r}")
    rngs = []
    for p, lb, sz in zip(parts, var.lbounds, var.shape):
        if ":" in p:
            a, b = p.split(":")
            lo = int(a) if a.strip() else lb
            hi = int(b) if b.strip() else lb + sz - 1
        else:
            lo = hi = int(p)
        rngs.append(range(lo - lb, hi - lb + 1))
    return rngs


def parse(text: str, base: Namelist | None = None) -> Namelist:
    nl = base if base is not None else defaults()
    # strip comments (outside quotes)
    lines = []
    for line in text.splitlines():
        out, q = [], None
        for ch in line:
            if q:
                out.append(ch)
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
                out.append(ch)
            elif ch == "!":
                break
            else:
                out.append(ch)
        lines.append("".join(out))
    body = "\n".join(lines)
    for gm in re.finditer(r"&(\w+)(.*?)(?:^\s*/|/\s*$|&end)", body, re.S | re.M):
        gname = gm.group(1).lower()
        if gname not in SCHEMA:
            continue
        sch = SCHEMA[gname]
        grp = nl.groups[gname]
        content = gm.group(2)
        assigns = list(_ASSIGN.finditer(content))
        for a_i, am in enumerate(assigns):
            name = am.group(1).lower()
            end = assigns[a_i + 1].start() if a_i + 1 < len(assigns) else len(content)
            vals = _tokens(content[am.end():end])
            if name not in sch:
                continue
            var = sch[name]
            if not var.shape:
                if vals:
                    grp[name] = _parse_scalar(vals[0][1], var.kind)
                continue
            rngs = _index_ranges(am.group(3), var)
            arr = grp[name]
            idx = np.stack(np.meshgrid(*rngs, indexing="ij"), -1).reshape(-1, len(rngs), order="F")
            for (kind, tok), ix in zip(vals, idx):
                arr[tuple(ix)] = _parse_scalar(tok, var.kind)
    return nl


def read(path: str, base: Namelist | None = None) -> Namelist:
    with open(path) as f:
        return parse(f.read(), base)


# defines of the reference's build.conf (configs/flags.mk turns KEY=1 into
# -D_KEY) that select a code path of this library, the &cansfz switch each
# sets, and the value flags.mk assumes when the key is absent
BUILD_DEFINES = {
    "INTERFACE_CAPTURING_VOF": ("interface_capturing_vof", False),
    "SDF_NORMALS": ("sdf_normals", True),
    "CAPILLARY_BRACKBILL_NORMALIZATION": ("capillary_brackbill_normalization", True),
    "BALANCED_CAPILLARY_PRESSURE_SPLIT": ("balanced_capillary_pressure_split", False),
    "SCALAR": ("scalar", False),
    "BOUSSINESQ_BUOYANCY": ("boussinesq_buoyancy", False),
}


def apply_build_conf(nl: Namelist, path: str) -> Namelist:
    """Set the &cansfz switches from a reference build.conf (KEY=VALUE lines,
    '#' comments; a define is on when its value is 1, configs/flags.mk:127-157).
    _BOUSSINESQ_BUOYANCY acts only together with _SCALAR (src/mom.f90:930,1017).
    A build this library does not provide raises ValueError: the HYPRE
    variable-coefficient solver (CONSTANT_COEFFS_POISSON other than 1) and
    SINGLE_PRECISION=1."""
    vals = {}
    with open(path) as f:
        for line in f:
            line = line.split("#", 1)[0].strip()
            if "=" in line:
                key, val = (x.strip() for x in line.split("=", 1))
                vals[key] = val
    if "CONSTANT_COEFFS_POISSON" in vals and vals["CONSTANT_COEFFS_POISSON"] != "1":
        raise ValueError("CONSTANT_COEFFS_POISSON != 1 (the HYPRE solver) is not provided by this library")
    if vals.get("SINGLE_PRECISION", "0") == "1":
        raise ValueError("SINGLE_PRECISION=1 is not provided by this library (see the mixed form instead)")
    g = nl.groups["cansfz"]
    for key, (name, absent) in BUILD_DEFINES.items():
        g[name] = (vals[key] == "1") if key in vals else absent
    g["boussinesq_buoyancy"] = bool(g["boussinesq_buoyancy"]) and bool(g["scalar"])
    return nl


def write(nl: Namelist) -> str:
    """Render a Namelist as input.nml text (every variable, Fortran order)."""
    def fmt(x, kind):
        if kind == "s":
            return f"'{x}'"
        if kind == "l":
            return "T" if x else "F"
        if kind == "i":
            return str(int(x))
        return repr(float(x))

    out = []
    for gname, sch in SCHEMA.items():
        if not sch:
            continue
        out.append(f"&{gname}")
        for name, var in sch.items():
            v = nl.groups[gname][name]
            if not var.shape:
                out.append(f"{name} = {fmt(v, var.kind)}")
            else:
                rng = ",".join(f"{lb}:{lb + s - 1}" for lb, s in zip(var.lbounds, var.shape))
                flat = np.asarray(v).reshape(-1, order="F")
                out.append(f"{name}({rng}) = " + ", ".join(fmt(x, var.kind) for x in flat))
        out.append("/")
        out.append("")
    return "\n".join(out)
