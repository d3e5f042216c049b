"""Builds tests/golden/tor99_x8.npz from one more of the reference's 1-D
verification cases (and, for the record, noh87_x8.npz; see below).

Reads, from the MOSE source tree (argv[1], or the MOSE_SOURCE_DIR environment variable),
through mose_b200.refio: test/1D/<case>/MESH/mesh_x8.tec,
INPUT/ic_x8.tec, INPUT/bc_x8.txt and input.ini (the gas is test/common/Air,
which both cases' MOSE.sh link).

* Tor99 (input.ini: HLLE++, MUSCL van Leer, CFL 0.9, RK3, t = 0.2): a Riemann
  problem with (rho, u, p) = (1, 0.75, 1) | (0.125, 0, 0.1), diaphragm at
  x = 0.3, gamma 1.4 (the states verify.py gives the exact solver).  Its
  verify.py passes when density, velocity, pressure and specific internal
  energy are within 1 % of the exact solution at cells 80, 240, 400, 560,
  720 of the x8 mesh.  The exact solution comes from the ideal-gas Riemann
  solver of make_ein91_fixture.py (Toro ch. 4).
* Noh87 (input.ini: HLLE, first order, CFL 0.5, RK3, t = 1): two streams
  (rho, u, p) = (1, +-1, 1e-15) colliding at x = 0.5.  The planar Noh
  solution at t, gamma 1.4: a shock at |x - 0.5| = t (gamma - 1) / 2 behind
  which rho = (gamma + 1) / (gamma - 1), u = 0, e = 1/2 and p = (gamma - 1)
  rho e; ahead of it the inflow state with e = p = 0.  Its verify.py passes
  when density, velocity (1 %), pressure (1.5 %) and specific internal energy
  (1 %) are within bounds at cells 480 and 640 of the x8 mesh, skipping a
  quantity whose exact value is 0.  Its cold inflow (p = 1e-15: internal
  energy about 20 ulps of the kinetic energy) cannot be carried by the
  closed-form one-species thermo that stands in for FLINT: rounding drift
  of the conservative energy drives the pressure to 0 within ~400 steps,
  and the interface check stops the run, in the oracle as on the GPU.  The
  fixture is kept for that record; no test runs it to its final time.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

from make_ein91_fixture import exact_riemann   # noqa: E402
from mose_b200 import refio                     # noqa: E402

sys.path.insert(0, str(Path(__file__).resolve().parent))
from _source import source_tree  # noqa: E402


def _save(name, case, exact, probes, thresholds, extra):
    out = HERE / f"{name}.npz"
    np.savez_compressed(out, nodes=case.nodes[0], prim=case.prim[0], bc_rec=case.bc_rec, bc_data=case.bc_data,
                        exact=exact, probes=np.asarray(probes), threshold_pct=np.asarray(thresholds),
                        cfl=case.cfl, t_end=case.t_end, riemann=case.riemann, limiter=case.limiter,
                        gamma=case.gamma, rgas=case.rgas, **extra)
    return out


def main(root: str | None = None):
    root = source_tree(root)
    outs = []
    case = refio.load_case(Path(root) / "test" / "1D" / "Tor99", "x8")
    x = 0.5 * (case.nodes[0][0, 0, :-1, 0] + case.nodes[0][0, 0, 1:, 0])
    ex = exact_riemann((1.0, 0.75, 1.0), (0.125, 0.0, 0.1), 1.4, (x - 0.3) / 0.2)
    sie = ex[:, 2] / ((1.4 - 1.0) * ex[:, 0])
    outs.append(_save("tor99_x8", case, np.column_stack([ex, sie]), [80, 240, 400, 560, 720], [1.0, 1.0, 1.0, 1.0],
                      {}))
    case = refio.load_case(Path(root) / "test" / "1D" / "Noh87", "x8")
    x = 0.5 * (case.nodes[0][0, 0, :-1, 0] + case.nodes[0][0, 0, 1:, 0])
    g, t = 1.4, 1.0
    r = np.abs(x - 0.5)
    inside = r < 0.5 * (g - 1.0) * t
    rho = np.where(inside, (g + 1.0) / (g - 1.0), 1.0)
    u = np.where(inside, 0.0, -np.sign(x - 0.5))
    e = np.where(inside, 0.5, 0.0)
    outs.append(_save("noh87_x8", case, np.column_stack([rho, u, (g - 1.0) * rho * e, e]), [480, 640],
                      [1.0, 1.0, 1.5, 1.0], {}))
    return outs


if __name__ == "__main__":
    print(main(*sys.argv[1:]))
