"""Readers for MOSE's own input files, so that a case directory of the
reference (input.ini, MESH/*.tec, INPUT/bc*.txt, INPUT/ic*.tec) runs through
the GPU path unchanged.

* ``read_bc`` follows Read_BCfile (io/IO_BC.f90:136-414): per boundary face
  cell a record line ``b i j k face type`` and, for the types that carry
  data, one list-directed data line.  The records come back in the layout
  of ``mose_gpu_set_bcs``: int32 (b, i, j, k, f, type, bs, is, js, ks, fs,
  d11, d12, d21, d22) and six doubles (401: T0, p0, alpha, beta, rel_fac;
  402: T0, index of its p0 table (``read_series``), alpha, beta, rel_fac;
  403 / 404: T0 / T, mass flux, alpha, beta, rel_fac; 405: mach, T, p, alpha,
  beta, rel_fac; 406: p_back, rel_fac; 407: T0, p0, p_back, alpha, beta,
  rel_fac; 301: qw; 302: Tw).  The direction token ``normal`` becomes the largest double, as
  parse_dir_tok (IO_BC.f90:443-456) does.
* ``read_tecplot`` reads ordered Tecplot ASCII zones with BLOCK data packing
  (the ORION format of MESH/*.tec and INPUT/ic*.tec): node variables on the
  (I, J, K) nodes and, with VARLOCATION, cell-centred variables on the
  (I-1, J-1, K-1) cells, Fortran order (i fastest).
* ``read_input_ini`` maps the [MOSE-*] keys of input.ini onto ``Case``
  numerics (Register_Numerics.f90, Register_Sim_Param.f90).
* ``load_case`` assembles a ``Case`` from a case directory.

Arrays use the layouts of ``mose_b200.cases``: nodes (nk+1, nj+1, ni+1, 3),
primitives (nk, nj, ni, 5) = (rho, u, v, w, p).
"""
from __future__ import annotations

import configparser
import re
import sys
from pathlib import Path

import numpy as np

from .cases import Case, LIMITERS, RIEMANN

# bc types with a data line after the record line (IO_BC.f90:200-410); 102
# (chimera) and 410 (state file) carry a different layout and are read by
# their own branches below
_DATA_LINE = {101, 103, 201, 301, 302, 303, 304, 401, 402, 403, 404, 405, 406, 407, 420, 501, 502}
_HUGE = sys.float_info.max


def _fields(line: str) -> list:
    """List-directed fields of one record (commas or blanks separate)."""
    return [f for f in re.split(r"[,\s]+", line.strip()) if f]


def _dir_tok(tok: str) -> float:
    if "normal" in tok:
        return _HUGE
    try:
        return float(tok.replace("d", "e").replace("D", "e"))
    except ValueError:
        return 0.0


def _num(tok: str) -> float:
    return float(tok.replace("d", "e").replace("D", "e"))


def read_series(path) -> tuple[np.ndarray, np.ndarray, bool]:
    """A 402 p0 table (time_series_type%initialize, Series_Data_m.f90:20-52):
    lines of ``time value`` in bar, after an optional first line holding
    ``periodic``; returns (time, value in Pa, periodic)."""
    lines = [ln for ln in Path(path).read_text().splitlines() if ln.strip()]
    periodic = any("periodic" in ln for ln in lines)
    if periodic:
        lines = lines[1:]
    rows = [[_num(x) for x in _fields(ln)[:2]] for ln in lines]
    arr = np.asarray(rows, dtype=np.float64).reshape(-1, 2)
    return arr[:, 0].copy(), arr[:, 1] * 1e5, periodic


def read_bc(path, series: list | None = None, base=None) -> tuple[np.ndarray, np.ndarray]:
    """bc.txt -> (rec int32 (n, 15), data float64 (n, 6)).  A 402 record's
    p0 table is read from its file (relative to ``base``, by default the case
    directory above INPUT/) and appended to ``series``; the record holds its
    index there."""
    base = Path(base) if base is not None else Path(path).resolve().parent.parent
    lines = [ln for ln in Path(path).read_text().splitlines() if ln.strip()]
    recs, data = [], []
    q = 0
    while q < len(lines):
        f = _fields(lines[q])
        q += 1
        b, i, j, k, face, t = (int(x) for x in f[:6])
        r = [b, i, j, k, face, t] + [0] * 9
        d = [0.0] * 6
        if t in (101, 103, 201):
            g = _fields(lines[q]); q += 1
            r[6:15] = [int(x) for x in g[:9]]
        elif t == 405:
            g = _fields(lines[q]); q += 1
            d = [_num(g[0]), _num(g[1]), _num(g[2]), _dir_tok(g[3]), _dir_tok(g[4]), _num(g[5])]
        elif t == 406:
            g = _fields(lines[q]); q += 1
            d[0], d[1] = _num(g[0]), _num(g[1])
        elif t == 402:                     # T0, p0 file, alpha, beta, rel_fac, ci...
            g = _fields(lines[q]); q += 1
            if series is None:
                raise ValueError(f"{path}: a 402 record needs a list for its p0 table")
            fname = g[1].strip("'\"")
            series.append(read_series(base / fname))
            d = [_num(g[0]), float(len(series) - 1), _dir_tok(g[2]), _dir_tok(g[3]), _num(g[4]), 0.0]
        elif t in (401, 403, 404):         # T0 (T), p0 (mass flux), alpha, beta, rel_fac, ci...
            g = _fields(lines[q]); q += 1
            d = [_num(g[0]), _num(g[1]), _dir_tok(g[2]), _dir_tok(g[3]), _num(g[4]), 0.0]
        elif t == 407:                     # T0, p0, p_back, alpha, beta, rel_fac, ci...
            g = _fields(lines[q]); q += 1
            d = [_num(g[0]), _num(g[1]), _num(g[2]), _dir_tok(g[3]), _dir_tok(g[4]), _num(g[5])]
        elif t in (301, 302):              # qw (Tw), k_rough, eps_wall (IO_BC.f90:241-252)
            g = _fields(lines[q]); q += 1
            d[0] = _num(g[0])
        elif t == 102:
            g = _fields(lines[q]); q += 1
            q += int(g[0]) + int(g[1])        # donor lines
        elif t in _DATA_LINE or t == 410:
            q += 1                            # types off this path: data line skipped
        recs.append(r)
        data.append(d)
    return np.asarray(recs, dtype=np.int32).reshape(-1, 15), np.asarray(data, dtype=np.float64).reshape(-1, 6)


def _zone_header(text: str) -> dict:
    h = {}
    for key in ("I", "J", "K"):
        m = re.search(r"(?<![A-Za-z])" + key + r"\s*=\s*(\d+)", text)
        h[key] = int(m.group(1)) if m else 1
    m = re.search(r"VARLOCATION\s*=\s*\(([^)]*)\)", text, re.IGNORECASE)
    h["cell"] = set()
    if m:
        for part in m.group(1).split(","):
            if "CELLCENTERED" in part.upper():
                r = re.search(r"\[(\d+)(?:-(\d+))?\]", part)
                if r:
                    lo = int(r.group(1))
                    hi = int(r.group(2) or lo)
                    h["cell"].update(range(lo, hi + 1))
    m = re.search(r"DATAPACKING\s*=\s*(\w+)", text, re.IGNORECASE)
    h["packing"] = m.group(1).upper() if m else "BLOCK"
    return h


def read_tecplot(path) -> list[dict]:
    """Ordered Tecplot ASCII zones -> [{"dims": (I, J, K), "nodal": {name:
    array (K, J, I)}, "cell": {name: array (K-1, J-1, I-1)}}, ...]."""
    text = Path(path).read_text()
    m = re.search(r"VARIABLES\s*=\s*(.*?)(?=\n\s*ZONE)", text, re.IGNORECASE | re.DOTALL)
    names = re.findall(r'"([^"]*)"|(\S+)', m.group(1)) if m else []
    names = [a or b for a, b in names]
    names = [n.strip(",") for n in names if n.strip(",")]
    zones = []
    parts = re.split(r"\n\s*ZONE", "\n" + text[m.end():] if m else text)
    for part in parts[1:]:
        # header: up to the first line that is a number
        lines = part.splitlines()
        hdr, q = [], 0
        while q < len(lines):
            s = lines[q].strip()
            if s and re.match(r"^[-+]?(\d|\.\d)", s):
                break
            hdr.append(s)
            q += 1
        h = _zone_header(" ".join(hdr))
        if h["packing"] != "BLOCK":
            raise ValueError(f"{path}: DATAPACKING={h['packing']} (only BLOCK is read)")
        I, J, K = h["I"], h["J"], h["K"]
        nnode, ncell = I * J * K, max(I - 1, 1) * max(J - 1, 1) * max(K - 1, 1)
        vals = np.array(" ".join(lines[q:]).replace("D", "E").replace("d", "e").split(), dtype=np.float64)
        z = {"dims": (I, J, K), "nodal": {}, "cell": {}}
        pos = 0
        for v, name in enumerate(names, start=1):
            if v in h["cell"]:
                z["cell"][name] = vals[pos:pos + ncell].reshape(max(K - 1, 1), max(J - 1, 1), max(I - 1, 1))
                pos += ncell
            else:
                z["nodal"][name] = vals[pos:pos + nnode].reshape(K, J, I)
                pos += nnode
        if pos > len(vals):
            raise ValueError(f"{path}: zone with I={I}, J={J}, K={K} holds {len(vals)} values, needs {pos}")
        zones.append(z)
    return zones


def read_mesh(path) -> list[np.ndarray]:
    """MESH/*.tec -> node arrays (nk+1, nj+1, ni+1, 3), one per block."""
    out = []
    for z in read_tecplot(path):
        xyz = [z["nodal"][k] for k in list(z["nodal"])[:3]]
        out.append(np.ascontiguousarray(np.stack(xyz, axis=-1)))
    return out


def read_ic(path) -> list[np.ndarray]:
    """INPUT/ic*.tec (rho1 u v w p cell centred) -> primitives (nk, nj, ni, 5)."""
    out = []
    for z in read_tecplot(path):
        cols = list(z["cell"].values())
        if len(cols) != 5:
            raise ValueError(f"{path}: {len(cols)} cell-centred variables (one species: rho1 u v w p)")
        out.append(np.ascontiguousarray(np.stack(cols, axis=-1)))
    return out


_TIME_SCHEMES = {"euler": 1, "rk1": 1, "rk2": 2, "rk3": 3}


def read_input_ini(path) -> dict:
    """The numerics of input.ini as Case keyword arguments."""
    cp = configparser.ConfigParser(inline_comment_prefixes=(";", "#"), strict=False)
    cp.read_string(Path(path).read_text())
    num = cp["MOSE-Numerics"] if cp.has_section("MOSE-Numerics") else {}
    par = cp["MOSE-Parameters"] if cp.has_section("MOSE-Parameters") else {}
    kw = {}
    if "cfl" in num:
        kw["cfl"] = float(num["cfl"])
    if "time-scheme" in num:
        kw["n_rk"] = _TIME_SCHEMES[num["time-scheme"].strip().lower()]
    if "time-accurate" in num:
        kw["time_accurate"] = num["time-accurate"].strip().lower() in ("true", ".true.", "t", "1")
    if "riemann-solver" in num:
        kw["riemann"] = num["riemann-solver"].strip()
    if "riemann-options-Minf" in num:
        kw["minf"] = float(num["riemann-options-Minf"])
    rec = num.get("space-reconstruction", "MUSCL").strip()
    if rec.lower() == "first-order":
        kw["limiter"] = "first-order"
    elif "flux-limiter" in num:
        kw["limiter"] = num["flux-limiter"].strip().lower()
    if "time-threshold" in par:
        kw["t_end"] = float(par["time-threshold"])
    if "iter-threshold" in par:
        kw["steps"] = int(par["iter-threshold"])
    unsupported = []
    if rec.upper().endswith("-SD"):
        kw["sd_limiter"] = True
    if "cfl-rise-threshold" in num:
        kw["ramp_iter"] = int(num["cfl-rise-threshold"])
    if "irs-beta" in num:
        kw["irs_beta"] = float(num["irs-beta"])
    if "integration-variables" in num:
        kw["integration"] = num["integration-variables"].strip().lower()
    kw["unsupported"] = unsupported
    return kw


def load_case(case_dir, resolution: str = "", gamma: float | None = None, rgas: float | None = None) -> Case:
    """A reference case directory -> Case.  ``resolution`` selects the
    suffixed files of the multi-resolution 1-D cases ("x4" -> mesh_x4.tec,
    bc_x4.txt, ic_x4.tec).  The gas defaults to test/common/Air (cp =
    1004.5 J/kg/K, M = 28.970418 kg/kmol), the thermo most cases link."""
    d = Path(case_dir)
    sfx = f"_{resolution}" if resolution else ""
    nodes = read_mesh(d / "MESH" / f"mesh{sfx}.tec")
    series: list = []
    rec, data = read_bc(d / "INPUT" / f"bc{sfx}.txt", series, base=d)
    prim = read_ic(d / "INPUT" / f"ic{sfx}.tec")
    kw = read_input_ini(d / "input.ini")
    unsupported = kw.pop("unsupported")
    if rgas is None:
        rgas = 8314.46 / 28.970418
    if gamma is None:
        cp = 1004.5
        gamma = cp / (cp - rgas)
    if kw.get("limiter") is not None and kw["limiter"] not in LIMITERS:
        unsupported.append(f"flux-limiter = {kw['limiter']}")
    if kw.get("integration", "cons") not in ("cons", "prim"):
        unsupported.append(f"integration-variables = {kw.pop('integration')}")
    if kw.get("riemann") is not None and kw["riemann"] not in RIEMANN:
        unsupported.append(f"riemann-solver = {kw['riemann']}")
    case = Case(d.name + sfx, nodes, rec, data, prim, gamma=gamma, rgas=rgas,
                **{k: v for k, v in kw.items() if k in ("cfl", "n_rk", "time_accurate", "riemann", "minf", "limiter",
                                                        "t_end", "steps", "irs_beta", "sd_limiter", "ramp_iter",
                                                        "integration")})
    case.series = series
    case.extra["unsupported"] = unsupported
    return case
