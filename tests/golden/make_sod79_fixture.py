"""Builds tests/golden/sod79_x4.npz from the reference's own Sod79 test case.

Reads, from the MOSE source tree (argv[1], or the MOSE_SOURCE_DIR environment variable):
  test/1D/Sod79/MESH/mesh_x4.tec    node coordinates (Tecplot ASCII, BLOCK)
  test/1D/Sod79/INPUT/ic_x4.tec     initial primitives (cell centred)
  test/1D/Sod79/INPUT/bc_x4.txt     boundary list (bc.txt format)
  test/1D/Sod79/reference/exact.txt exact solution at t = 0.2 (x, rho, u, p, sie)
and stores them in the layouts of mose_b200.cases.  The case numerics come
from test/1D/Sod79/input.ini (cfl 0.9, RK3, time accurate, cons, MUSCL + MC,
SLAU) and MOSE.sh (the x4 mesh), and the pass criterion from check.py:45-84
(1 % at probes 0.2, 0.5, 0.6, 0.8, 0.9 of the cell count).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent))
from _source import source_tree  # noqa: E402


def _numbers(lines):
    return np.array(" ".join(lines).split(), dtype=np.float64)


def main(root: str | None = None) -> Path:
    root = source_tree(root)
    case = Path(root) / "test" / "1D" / "Sod79"
    mesh = (case / "MESH" / "mesh_x4.tec").read_text().splitlines()
    ni1, nj1, nk1 = 401, 2, 2
    vals = _numbers(mesh[5:])
    n = ni1 * nj1 * nk1
    xyz = vals[:3 * n].reshape(3, nk1, nj1, ni1)
    nodes = np.ascontiguousarray(np.moveaxis(xyz, 0, -1))            # (nk+1, nj+1, ni+1, 3)
    ic = (case / "INPUT" / "ic_x4.tec").read_text().splitlines()
    v = _numbers(ic[2:])
    ncell = (ni1 - 1) * (nj1 - 1) * (nk1 - 1)
    cells = v[3 * n:].reshape(5, 1, 1, ni1 - 1)                        # rho1 u v w p
    prim = np.ascontiguousarray(np.moveaxis(cells, 0, -1))             # (1, 1, 400, 5)
    assert prim.shape[2] * prim.shape[1] * prim.shape[0] == ncell
    rec = []
    for line in (case / "INPUT" / "bc_x4.txt").read_text().splitlines():
        f = line.split()
        if not f:
            continue
        b, i, j, k, face, t = (int(x) for x in f[:6])
        assert t in (0, 400), "the Sod79 list holds only null and extrapolation faces"
        rec.append([b, i, j, k, face, t] + [0] * 9)
    rec = np.asarray(rec, dtype=np.int32)
    exact = np.loadtxt(case / "reference" / "exact.txt")
    out = Path(__file__).resolve().parent / "sod79_x4.npz"
    np.savez_compressed(out, nodes=nodes, prim=prim, bc_rec=rec, bc_data=np.zeros((len(rec), 6)), exact=exact,
                        cfl=0.9, t_end=0.2, probes=np.array([0.20, 0.50, 0.60, 0.80, 0.90]), threshold_pct=1.0)
    return out


if __name__ == "__main__":
    print(main(*sys.argv[1:]))
