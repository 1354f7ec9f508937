"""LB3D input files: namelist reader and the hot-path parameter set.

LB3D reads three Fortran namelists, &fixed_input, &variable_input and
&lbe_input, from the file given with -f, then re-reads them from an optional
"differential" file given with -d, whose entries override the first
(code/lb3d_config.F90:340-371, :395-404, :815-823).  This module keeps that
input format unchanged: read_input() takes the same two files and returns
the parameters the per-timestep hot path uses, with the reference's
defaults (code/lb3d_config.F90:44-297) and derived values
(omega = 1/tau at :886-893, g_accn_max* defaults at :931-933,
rock_colour -> rock_colour_r/_b at :661-664).
"""
from __future__ import annotations

import ctypes
import dataclasses
import re
from typing import Dict, Optional


# ---------------------------------------------------------------------------
# namelist text -> {group: {name: value}}
# ---------------------------------------------------------------------------
_TOKEN = re.compile(
    r"""\s*(?:
        (?P<str>'(?:[^']|'')*'|"(?:[^"]|"")*")
      | (?P<sep>[=,])
      | (?P<word>[^\s=,'"/]+)
    )""",
    re.X,
)


def _strip_comments(text: str) -> str:
    out = []
    for line in text.splitlines():
        buf, q = [], None
        for ch in line:
            if q:
                buf.append(ch)
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
                buf.append(ch)
            elif ch == "!":
                break
            else:
                buf.append(ch)
        out.append("".join(buf))
    return "\n".join(out)


def _value(tok: str):
    if tok[0] in "'\"":
        return tok[1:-1].replace(tok[0] * 2, tok[0])
    low = tok.lower()
    if low in (".true.", ".t.", "t", "true"):
        return True
    if low in (".false.", ".f.", "f", "false"):
        return False
    if re.fullmatch(r"[+-]?\d+", tok):
        return int(tok)
    return float(low.replace("d", "e"))


def parse_namelists(text: str) -> Dict[str, Dict[str, object]]:
    """Parses every &group ... / block; later blocks of the same group update
    earlier ones, as successive namelist reads do."""
    text = _strip_comments(text)
    groups: Dict[str, Dict[str, object]] = {}
    blocks = []
    i, q, start, name = 0, None, None, None
    while i < len(text):
        ch = text[i]
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "&" and start is None:
            m = re.match(r"&(\w+)", text[i:])
            if m:
                name, start = m.group(1).lower(), i + m.end()
                i = start
                continue
        elif ch == "/" and start is not None:
            blocks.append((name, text[start:i]))
            start = None
        i += 1
    for name, body in blocks:
        vals = groups.setdefault(name, {})
        toks = []
        pos = 0
        while pos < len(body):
            t = _TOKEN.match(body, pos)
            if not t or t.end() == pos:
                break
            pos = t.end()
            for kind in ("str", "sep", "word"):
                if t.group(kind) is not None:
                    toks.append((kind, t.group(kind)))
        i = 0
        while i < len(toks):
            kind, tok = toks[i]
            if kind == "word" and i + 1 < len(toks) and toks[i + 1] == ("sep", "="):
                key = tok.lower()
                j = i + 2
                items = []
                while j < len(toks):
                    k2, t2 = toks[j]
                    if k2 == "sep":
                        j += 1
                        continue
                    if k2 == "word" and j + 1 < len(toks) and toks[j + 1] == ("sep", "="):
                        break
                    items.append(_value(t2))
                    j += 1
                vals[key] = items[0] if len(items) == 1 else items
                i = j
            else:
                i += 1
    return groups


# ---------------------------------------------------------------------------
# hot-path parameter set
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class Params:
    """Parameters of the per-timestep hot path, with the reference defaults
    of code/lb3d_config.F90:44-297.  Component order: red, blue, surfactant."""

    nx: int = 16
    ny: int = 16
    nz: int = 16
    ncomp: int = 3
    tau_r: float = 1.0
    tau_b: float = 1.0
    tau_s: float = 1.0
    tau_d: float = 2.0
    amass_r: float = 1.0
    amass_b: float = 1.0
    amass_s: float = 1.0
    g_br: float = 0.0
    g_bs: float = 0.0
    g_ss: float = 0.0
    g_wr: float = 0.0
    g_wb: float = 0.0
    tau_wr: float = 1.0
    tau_wb: float = 1.0
    beta: float = 1.0
    d_0: float = 1.0
    g_accn: float = 0.0
    g_accn_x: float = 0.0
    g_accn_y: float = 0.0
    g_accn_min: int = 0
    g_accn_max: int = 0
    g_accn_min_x: int = 0
    g_accn_max_x: int = 0
    g_accn_min_y: int = 0
    g_accn_max_y: int = 0
    shear_u: float = 0.0
    shear_omega: float = 0.0
    boundary_cond: int = 0
    inv_fluid: int = 0
    rock_colour_r: float = 0.0
    rock_colour_b: float = 0.0
    bdist: int = 0
    restore: int = 0
    inv_type: int = 0
    pr: float = 0.5
    pg: float = 0.1
    pb: float = 1.0
    fr: float = 1.0
    fg: float = 0.1
    fb: float = 0.5
    # product-only fields (not in the reference's namelists)
    precision: int = 0  # 0: FP64 plain drop-in, 1: FP32 deviation storage
    rho0: float = 0.7  # reference density of the FP32 deviation storage

    # extra, not passed to the kernels
    obs_file: str = "empty.dat"
    obs_folder: str = "../rocks"
    init_cond: int = 0
    n_iteration: int = 100
    restore_string: str = "0000000000-t00000000"
    gr_out_file: str = "default"
    srccpfolder: str = "."
    psifunc: int = 2
    dump_double: bool = True
    dump_format: str = "bin"

    @property
    def lees_edwards(self) -> bool:
        """code/lb3d_bc.F90:61: LE when boundary_cond /= 0 and inv_fluid is 5 or 6."""
        return self.boundary_cond != 0 and self.inv_fluid in (5, 6)

    @property
    def has_rock_file(self) -> bool:
        return self.obs_file.strip() != "empty.dat"

    def finalize(self) -> "Params":
        """Derived values the reference sets after reading its input."""
        if self.g_accn_max == 0:
            self.g_accn_max = self.nz
        if self.g_accn_max_x == 0:
            self.g_accn_max_x = self.nx
        if self.g_accn_max_y == 0:
            self.g_accn_max_y = self.ny
        return self

    def validate(self) -> None:
        """The fatal combinations of code/lb3d_compatibility.F90:105-111 and
        the parts of the input space this implementation covers."""
        if self.ncomp not in (2, 3):
            raise ValueError("ncomp must be 2 (binary, -DNOSURFACTANT) or 3 (ternary)")
        if self.ncomp == 3 and self.lees_edwards:
            raise ValueError("FATAL: Lees Edwards BC are not supported for ternary mixtures")
        if self.ncomp == 3 and self.has_rock_file:
            raise ValueError("FATAL: Obstacles are not supported for ternary mixtures")
        if self.bdist != 2:
            raise ValueError("only the bdist = 2 equilibrium is implemented")
        if self.psifunc != 2:
            raise ValueError("only psifunc = 2 (psi = 1 - exp(-rho)) is implemented")
        recolour = self.boundary_cond != 0 and self.inv_fluid in (7, 8)
        zouhe = self.boundary_cond != 0 and self.inv_fluid in (11, 12)
        if recolour and self.ncomp != 2:
            raise ValueError("Illegal value: inv_fluid 7/8 (recolouring) exists in binary builds only")
        if (self.boundary_cond != 0 and self.inv_fluid >= 0 and not self.lees_edwards
                and not zouhe and not recolour):
            raise ValueError("invasion boundaries (inv_fluid=%d) are not implemented" % self.inv_fluid)
        if self.boundary_cond > 0:
            raise ValueError("boundary_cond > 0 (generated walls) is not implemented")
        if self.precision == 1 and 19 * self.nx * self.ny * self.nz >= 1 << 32:
            raise ValueError("FP32 lattices are limited to 19*sites < 2^32 (226,050,910 sites)")


_PARAM_FIELDS = [f.name for f in dataclasses.fields(Params)]


def params_from_namelists(groups: Dict[str, Dict[str, object]], ncomp: int) -> Params:
    p = Params(ncomp=ncomp)
    flat: Dict[str, object] = {}
    for g in ("fixed_input", "variable_input", "lbe_input"):
        flat.update(groups.get(g, {}))
    for k, v in flat.items():
        if k in _PARAM_FIELDS and k not in ("ncomp", "precision", "rho0", "restore"):
            ftype = type(getattr(p, k))
            if ftype is bool:
                setattr(p, k, bool(v))
            elif ftype is int:
                setattr(p, k, int(v))
            elif ftype is float:
                setattr(p, k, float(v))
            else:
                setattr(p, k, str(v))
    # rock_colour is deprecated in favour of rock_colour_r/_b
    # (code/lb3d_config.F90:661-664)
    rc = float(flat.get("rock_colour", 0.0))
    if rc > 0:
        p.rock_colour_r = rc
    elif rc < 0:
        p.rock_colour_b = rc
    p.restore = 1 if (p.init_cond == 7 or bool(flat.get("restore", False))) else 0
    return p.finalize()


def read_input(path: str, diff_path: Optional[str] = None, ncomp: int = 3) -> Params:
    """Reads an LB3D input file (-f) and its optional differential file (-d).
    ncomp is the compile-time mixture of the reference build: 3 (default),
    2 (-DNOSURFACTANT)."""
    with open(path) as f:
        text = f.read()
    if diff_path:
        with open(diff_path) as f:
            text += "\n" + f.read()
    return params_from_namelists(parse_namelists(text), ncomp)


# ---------------------------------------------------------------------------
# C-ABI mirror of lb3dc_params (include/lb3dc.h)
# ---------------------------------------------------------------------------
_C_FIELDS = [
    ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("ncomp", ctypes.c_int),
    ("tau_r", ctypes.c_double), ("tau_b", ctypes.c_double), ("tau_s", ctypes.c_double),
    ("tau_d", ctypes.c_double),
    ("amass_r", ctypes.c_double), ("amass_b", ctypes.c_double), ("amass_s", ctypes.c_double),
    ("g_br", ctypes.c_double), ("g_bs", ctypes.c_double), ("g_ss", ctypes.c_double),
    ("g_wr", ctypes.c_double), ("g_wb", ctypes.c_double), ("tau_wr", ctypes.c_double),
    ("tau_wb", ctypes.c_double),
    ("beta", ctypes.c_double), ("d_0", ctypes.c_double),
    ("g_accn", ctypes.c_double), ("g_accn_x", ctypes.c_double), ("g_accn_y", ctypes.c_double),
    ("g_accn_min", ctypes.c_int), ("g_accn_max", ctypes.c_int),
    ("g_accn_min_x", ctypes.c_int), ("g_accn_max_x", ctypes.c_int),
    ("g_accn_min_y", ctypes.c_int), ("g_accn_max_y", ctypes.c_int),
    ("shear_u", ctypes.c_double), ("shear_omega", ctypes.c_double),
    ("boundary_cond", ctypes.c_int), ("inv_fluid", ctypes.c_int),
    ("rock_colour_r", ctypes.c_double), ("rock_colour_b", ctypes.c_double),
    ("bdist", ctypes.c_int), ("restore", ctypes.c_int),
    ("inv_type", ctypes.c_int), ("pr", ctypes.c_double), ("pg", ctypes.c_double),
    ("pb", ctypes.c_double), ("fr", ctypes.c_double), ("fg", ctypes.c_double),
    ("fb", ctypes.c_double),
]


class CParams(ctypes.Structure):
    """ctypes mirror of lb3dc_params (include/lb3dc.h)."""

    _fields_ = _C_FIELDS + [("precision", ctypes.c_int), ("rho0", ctypes.c_double)]


def to_cparams(p: Params, struct=CParams):
    c = struct()
    for name, _ in struct._fields_:
        setattr(c, name, getattr(p, name))
    return c
