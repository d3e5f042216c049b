"""Builds tests/golden/ramp_channel.npz from the reference's own 2-D ramp
channel case (test/2D/euler/ramp-channel: MESH/mesh.tec, INPUT/ic.tec,
INPUT/bc.txt, input.ini), read with mose_b200.refio: one 95 x 100 block,
supersonic inflow (405), extrapolation (400), symmetry (300) and null faces;
HLLE with MUSCL-SD (minmod slopes scaled by the Tramel shock detector), RK3,
CFL 0.9 ramped over the first 100 iterations, local time stepping and
implicit residual smoothing (beta 0.5).  It has no verification script; the
tests use it for GPU-oracle parity on the reference's inputs.
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
    c = refio.load_case(Path(root) / "test" / "2D" / "euler" / "ramp-channel")
    assert c.extra["unsupported"] == [], c.extra["unsupported"]
    out = Path(__file__).resolve().parent / "ramp_channel.npz"
    np.savez_compressed(out, nodes=c.nodes[0], prim=c.prim[0], bc_rec=c.bc_rec, bc_data=c.bc_data, cfl=c.cfl,
                        n_rk=c.n_rk, time_accurate=c.time_accurate, riemann=c.riemann, limiter=c.limiter,
                        irs_beta=c.irs_beta, sd_limiter=c.sd_limiter, ramp_iter=c.ramp_iter, steps=c.steps,
                        gamma=c.gamma, rgas=c.rgas)
    return out


if __name__ == "__main__":
    print(main(*sys.argv[1:]))
