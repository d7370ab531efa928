"""Reader for the reference's ``&params`` namelist (test infrastructure).

Follows ``read_input_parameters`` (src/input_output.f90:21-132): the same
variable list (:27-40) and the same defaults (:43-62).  Keys are
case-insensitive; ``!`` starts a comment; values may use Fortran ``d``/``e``
exponents, ``.true./.false./T/F`` logicals and quoted strings.
"""
import math
import re

import numpy as _np

# defaults, src/input_output.f90:43-62 (pi as in src/global.f90:30)
_PI = 4.0 * math.atan(1.0)

DEFAULTS = {
    "alpha_stretch": 2.6,
    "lxp": 2.0 * _PI,
    "lzp": 1.0 * _PI,
    "ly_channel": 2.0,
    "min_buffer_width": 0.0,
    # `cg_tol = 1e-8` is a default-real (single precision) literal widened to FP64
    "cg_tol": float(_np.float32(1e-8)),
    "cg_max_iter": 50,
    "t_init": 0.0,
    "body_type": "none",
    "exterior_pressure_gradient": True,
    "x_mass_cte": 0,
    "y_mass_cte": 0,
    "z_mass_cte": 0,
    "dpdx": 0.0,
    "dpdy": 0.0,
    "dpdz": 0.0,
    "body_ramp_up_time": 0.0,
    "perturb_scale": 0.5,
    "qflow_x_0": -999999.0,
    "qflow_z_0": -999999.0,
    # not defaulted by the reference; zero here so the dict is total
    "nx_global": 0, "ny_global": 0, "nz_global": 0, "nxb": 0, "nzb": 0,
    "cfl": 0.0, "nu": 0.0, "nsteps": 0, "nsave": 0, "nstats": 0,
    "nmonitor": 0, "filein": "", "fileout": "", "nstep_init": 0,
    "init_type": 1, "grid_type": 0, "body_param_1": 0.0,
    "body_param_2": 0.0, "body_param_3": 0.0,
    # extension (no reference counterpart): mean y of the plane of
    # body_type 'wall_standing_wave'
    "body_param_4": 0.0,
}

INT_KEYS = {"nx_global", "ny_global", "nz_global", "nxb", "nzb", "x_mass_cte",
            "y_mass_cte", "z_mass_cte", "nsteps", "nsave", "nstats", "nmonitor",
            "nstep_init", "init_type", "grid_type", "cg_max_iter"}
STR_KEYS = {"filein", "fileout", "body_type"}
BOOL_KEYS = {"exterior_pressure_gradient"}
# variables of the namelist group (src/input_output.f90:27-40)
KNOWN_KEYS = set(DEFAULTS) - {"dpdy"}


class NamelistError(ValueError):
    pass


def _strip_comment(line):
    out, quote = [], None
    for ch in line:
        if quote:
            out.append(ch)
            if ch == quote:
                quote = None
        elif ch in "'\"":
            quote = ch
            out.append(ch)
        elif ch == "!":
            break
        else:
            out.append(ch)
    return "".join(out)


def _convert(key, tok):
    tok = tok.strip()
    if key in STR_KEYS:
        if len(tok) >= 2 and tok[0] == tok[-1] and tok[0] in "'\"":
            return tok[1:-1]
        return tok
    if key in BOOL_KEYS:
        t = tok.lower().strip(".")
        if t.startswith("t"):
            return True
        if t.startswith("f"):
            return False
        raise NamelistError(f"bad logical for {key}: {tok!r}")
    num = tok.lower().replace("d", "e")
    if key in INT_KEYS:
        try:
            return int(num)
        except ValueError as exc:
            raise NamelistError(f"bad integer for {key}: {tok!r}") from exc
    try:
        return float(num)
    except ValueError as exc:
        raise NamelistError(f"bad real for {key}: {tok!r}") from exc


def parse_namelist_text(text):
    """Return the parameter dict (lower-case keys) with reference defaults."""
    body = "\n".join(_strip_comment(l) for l in text.splitlines())
    m = re.search(r"&\s*params\b(.*?)(?:^\s*/|/\s*$|&end)", body,
                  re.IGNORECASE | re.DOTALL | re.MULTILINE)
    if not m:
        raise NamelistError("no &params group found")
    group = m.group(1)
    params = dict(DEFAULTS)
    # split on key = value; values end at the next key or newline/comma
    for km in re.finditer(r"([A-Za-z_][A-Za-z0-9_]*)\s*=\s*('[^']*'|\"[^\"]*\"|[^,\n=]+?)\s*(?=,|\n|$)",
                          group):
        key = km.group(1).lower()
        if key not in KNOWN_KEYS:
            raise NamelistError(f"unknown namelist variable {km.group(1)!r}")
        params[key] = _convert(key, km.group(2))
    params["body_type"] = params["body_type"].strip().lower()
    return params


def read_namelist(path):
    with open(path, "r") as fh:
        return parse_namelist_text(fh.read())
