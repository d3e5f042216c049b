"""Builds tests/golden/ein91_x8.npz from the reference's own Ein91 test case
(the HLLE case of its 1-D suite).

Reads, from the MOSE source tree (argv[1], or the MOSE_SOURCE_DIR environment variable):
  test/1D/Ein91/MESH/mesh_x8.tec    node coordinates (Tecplot ASCII, BLOCK)
  test/1D/Ein91/INPUT/ic_x8.tec     initial primitives (cell centred)
  test/1D/Ein91/INPUT/bc_x8.txt     boundary list (bc.txt format)
The numerics come from test/1D/Ein91/input.ini (t = 0.15, CFL 0.9, RK3, time
accurate, MUSCL + van Leer, HLLE) and the gas from test/common/Air (the
thermo MOSE.sh links); the pass criterion from verify.py: relative error at
cells 80, 160 and 240 of the x8 mesh below 1 % (density, velocity) and
1.5 % (pressure) against the exact Riemann solution.  The exact solution is
computed here from the initial states on both sides of the diaphragm with
the exact solver for the ideal-gas Riemann problem (Toro, Riemann Solvers
and Numerical Methods for Fluid Dynamics, ch. 4: pressure function solved
for p*, then the wave pattern sampled at x/t).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from _source import source_tree  # noqa: E402


def _numbers(lines):
    return np.array(" ".join(lines).split(), dtype=np.float64)


def exact_riemann(WL, WR, g, xi):
    """Primitive (rho, u, p) of the exact ideal-gas Riemann solution at the
    similarity coordinates xi = (x - x0) / t."""
    rl, ul, pl = WL
    rr, ur, pr = WR
    al, ar = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)

    def f(p, rk, pk, ak):
        if p > pk:                                   # shock
            A, B = 2.0 / ((g + 1.0) * rk), (g - 1.0) / (g + 1.0) * pk
            return (p - pk) * np.sqrt(A / (p + B))
        return 2.0 * ak / (g - 1.0) * ((p / pk) ** ((g - 1.0) / (2.0 * g)) - 1.0)   # rarefaction

    F = lambda p: f(p, rl, pl, al) + f(p, rr, pr, ar) + (ur - ul)
    lo, hi = 1e-14, 10.0 * max(pl, pr)
    for _ in range(200):                             # F is increasing in p
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if F(mid) < 0.0 else (lo, mid)
    ps = 0.5 * (lo + hi)
    us = 0.5 * (ul + ur) + 0.5 * (f(ps, rr, pr, ar) - f(ps, rl, pl, al))
    out = np.zeros((len(xi), 3))
    gm = (g - 1.0) / (g + 1.0)
    for n, S in enumerate(xi):
        if S <= us:                                  # left of the contact
            if ps > pl:
                SL = ul - al * np.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
                out[n] = (rl, ul, pl) if S <= SL else (rl * (ps / pl + gm) / (gm * ps / pl + 1.0), us, ps)
            else:
                SHL, STL = ul - al, us - al * (ps / pl) ** ((g - 1.0) / (2.0 * g))
                if S <= SHL:
                    out[n] = (rl, ul, pl)
                elif S >= STL:
                    out[n] = (rl * (ps / pl) ** (1.0 / g), us, ps)
                else:
                    c = 2.0 / (g + 1.0) + gm / al * (ul - S)
                    out[n] = (rl * c ** (2.0 / (g - 1.0)), 2.0 / (g + 1.0) * (al + (g - 1.0) / 2.0 * ul + S),
                              pl * c ** (2.0 * g / (g - 1.0)))
        else:                                        # right of the contact
            if ps > pr:
                SR = ur + ar * np.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
                out[n] = (rr, ur, pr) if S >= SR else (rr * (ps / pr + gm) / (gm * ps / pr + 1.0), us, ps)
            else:
                SHR, STR = ur + ar, us + ar * (ps / pr) ** ((g - 1.0) / (2.0 * g))
                if S >= SHR:
                    out[n] = (rr, ur, pr)
                elif S <= STR:
                    out[n] = (rr * (ps / pr) ** (1.0 / g), us, ps)
                else:
                    c = 2.0 / (g + 1.0) - gm / ar * (ur - S)
                    out[n] = (rr * c ** (2.0 / (g - 1.0)), 2.0 / (g + 1.0) * (-ar + (g - 1.0) / 2.0 * ur + S),
                              pr * c ** (2.0 * g / (g - 1.0)))
    return out


def main(root: str | None = None) -> Path:
    root = source_tree(root)
    case = Path(root) / "test" / "1D" / "Ein91"
    mesh = (case / "MESH" / "mesh_x8.tec").read_text().splitlines()
    ni1, nj1, nk1 = 801, 2, 2
    vals = _numbers(mesh[5:])
    n = ni1 * nj1 * nk1
    xyz = vals[:3 * n].reshape(3, nk1, nj1, ni1)
    nodes = np.ascontiguousarray(np.moveaxis(xyz, 0, -1))            # (nk+1, nj+1, ni+1, 3)
    ic = (case / "INPUT" / "ic_x8.tec").read_text().splitlines()
    v = _numbers(ic[2:])
    cells = v[3 * n:].reshape(5, 1, 1, ni1 - 1)                        # rho1 u v w p
    prim = np.ascontiguousarray(np.moveaxis(cells, 0, -1))             # (1, 1, 800, 5)
    rec = []
    for line in (case / "INPUT" / "bc_x8.txt").read_text().splitlines():
        f = line.split()
        if not f:
            continue
        b, i, j, k, face, t = (int(x) for x in f[:6])
        assert t in (0, 400), "the Ein91 list holds only null and extrapolation faces"
        rec.append([b, i, j, k, face, t] + [0] * 9)
    rec = np.asarray(rec, dtype=np.int32)
    R = 8314.46 / 28.970418            # test/common/Air: M = 28.970418, cp = 1004.5
    cp = 1004.5
    gam = cp / (cp - R)
    x = 0.5 * (nodes[0, 0, :-1, 0] + nodes[0, 0, 1:, 0])
    P = prim[0, 0]
    WL, WR = (P[0, 0], P[0, 1], P[0, 4]), (P[-1, 0], P[-1, 1], P[-1, 4])
    exact = exact_riemann(WL, WR, gam, (x - 0.5) / 0.15)
    out = Path(__file__).resolve().parent / "ein91_x8.npz"
    np.savez_compressed(out, nodes=nodes, prim=prim, bc_rec=rec, bc_data=np.zeros((len(rec), 6)), exact=exact,
                        cfl=0.9, t_end=0.15, probes=np.array([80, 160, 240]),
                        threshold_pct=np.array([1.0, 1.0, 1.5]))
    return out


if __name__ == "__main__":
    print(main(*sys.argv[1:]))
