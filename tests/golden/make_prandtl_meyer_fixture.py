"""Builds tests/golden/prandtl_meyer.npz from the reference's own 2-D
Prandtl-Meyer expansion case (test/2D/euler/prandtl-meyer: MESH/mesh.tec,
INPUT/ic.tec, INPUT/bc.txt, input.ini), read with mose_b200.refio: one
50 x 50 block, supersonic inflow (405), extrapolation (400) and symmetry
(300) faces, HLLE + MUSCL van Leer, RK3, CFL 1.0, local time stepping,
implicit residual smoothing with beta = 0.5.  The case has no verification
script of its own; the tests use it for GPU-oracle parity on the
reference's inputs.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
from mose_b200 import refio  # noqa: E402

sys.path.insert(0, str(Path(__file__).resolve().parent))
from _source import source_tree  # noqa: E402


def main(root: str | None = None) -> Path:
    root = source_tree(root)
    c = refio.load_case(Path(root) / "test" / "2D" / "euler" / "prandtl-meyer")
    assert c.extra["unsupported"] == [], c.extra["unsupported"]
    out = Path(__file__).resolve().parent / "prandtl_meyer.npz"
    np.savez_compressed(out, nodes=c.nodes[0], prim=c.prim[0], bc_rec=c.bc_rec, bc_data=c.bc_data, cfl=c.cfl,
                        n_rk=c.n_rk, time_accurate=c.time_accurate, riemann=c.riemann, limiter=c.limiter,
                        irs_beta=c.irs_beta, steps=c.steps, gamma=c.gamma, rgas=c.rgas)
    return out


if __name__ == "__main__":
    print(main(*sys.argv[1:]))
