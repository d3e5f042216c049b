"""GPU parity of the Tramel shock detector (Lib_Shock_Detector.f90) and its
two uses: MUSCL-SD slopes (Lib_Reconstruction.f90:24-25) and the SD Riemann
solvers HLLC+ and HLLE++; and of the CFL ramp (cfl-rise-threshold) in
device-driven steps.  The detector calls tanh, whose CUDA and glibc results
may differ in the last bit, so the shock-detector cases are held to the
normwise relative L-infinity bar of 1e-12 per compared state (the ramp case,
without a detector, stays bit for bit).  2-D multi-block cases and 3-D shock
tubes (multi-block, multi-tile with walls, with IRS)."""
from pathlib import Path

import numpy as np
import pytest

from mose_b200 import cases
from mose_b200.cases import Case

from tests.test_gpu_parity import compare_state, solver

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def quad(riemann, sd_limiter=False, limiter="vanleer", **kw):
    c = cases.four_quadrant(seed=6, nbx=3, nby=2, nmin=20, nmax=56, steps=3, limiter=limiter, riemann=riemann,
                            cfl=0.4)
    c.sd_limiter = sd_limiter
    for k, v in kw.items():
        setattr(c, k, v)
    return c


SD_CASES = {
    "hllc_plus": lambda: quad("HLLC+"),
    "hlle_pp": lambda: quad("HLLE++"),
    "muscl_sd_hlle": lambda: quad("HLLE", True, "minmod"),
    "muscl_sd_hllc": lambda: quad("HLLC", True, "vanalbada"),
    "muscl_sd_hllc_plus_irs": lambda: quad("HLLC+", True, irs_beta=0.5, time_accurate=False),
}


@pytest.mark.parametrize("name", sorted(SD_CASES))
def test_shock_detector_steps(oracle_mod, name):
    case = SD_CASES[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(3):
        o.step()
        s.explicit_step()
    compare_state(s, o, len(case.nodes), exact=False, tol=1e-12)
    for _ in range(3):
        o.step()
    s.advance(3)
    compare_state(s, o, len(case.nodes), exact=False, tol=1e-12)


def test_shock_detector_fp64(oracle_mod):
    from mose_b200 import _lib
    case = quad("HLLE++", True)
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_FP64)
    o.step()
    s.explicit_step()
    compare_state(s, o, len(case.nodes), exact=False, tol=1e-12)


def test_cfl_ramp_device_steps_bitwise(oracle_mod):
    """cfl-rise-threshold in fused and graph-replayed steps: the dt pass reads
    the step's iteration from the device counter."""
    case = quad("HLLE", time_accurate=False, ramp_iter=5)
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(3):
        dto, _ = o.step()
        dtg, _ = s.explicit_step()
        assert dtg == dto
    compare_state(s, o, len(case.nodes))
    for _ in range(4):
        o.step()
    s.advance(4)
    compare_state(s, o, len(case.nodes))


def test_ramp_channel_reference_inputs(oracle_mod):
    """The reference's ramp-channel case: its mesh, ic and bc files and
    input.ini numerics (HLLE, MUSCL-SD with minmod, CFL 0.9 ramped over 100
    iterations, local dt, IRS 0.5, inflow angles 'normal')."""
    d = np.load(GOLDEN / "ramp_channel.npz")
    case = Case("ramp_channel", [d["nodes"]], d["bc_rec"], d["bc_data"], [d["prim"]], n_rk=int(d["n_rk"]),
                cfl=float(d["cfl"]), time_accurate=bool(d["time_accurate"]), limiter=str(d["limiter"]),
                riemann=str(d["riemann"]), gamma=float(d["gamma"]), rgas=float(d["rgas"]),
                irs_beta=float(d["irs_beta"]), sd_limiter=bool(d["sd_limiter"]), ramp_iter=int(d["ramp_iter"]))
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(10):
        o.step()
        s.explicit_step()
    compare_state(s, o, 1, exact=False, tol=1e-12)
    for _ in range(30):
        o.step()
    s.advance(30)
    compare_state(s, o, 1, exact=False, tol=1e-12)


V3 = (0, 1, 2, 3, 4)


def tube3d(riemann, sd_limiter=False, limiter="vanleer", ywalls=False, **kw):
    """A 3-D shock tube in the periodic box: the cells with x < 0.5 at twice
    the density and three times the pressure, so the detector switches on at
    the two discontinuities (and their periodic images); 2 x 2 x 2 uneven
    blocks, or multi-tile blocks with slip walls on the y ends."""
    if ywalls:
        c = cases.periodic_box_3d(sizes=[[40, 24], [20], [6, 5]], nb=(2, 1, 2), seed=5, steps=3, limiter=limiter,
                                  riemann=riemann, cfl=0.3, ywalls=True)
    else:
        c = cases.periodic_box_3d(sizes=[[8, 6], [7, 9], [6, 5]], seed=5, steps=3, limiter=limiter, riemann=riemann,
                                  cfl=0.3)
    for nd, P in zip(c.nodes, c.prim):
        left = cases.cell_centres(nd)[..., 0] < 0.5
        P[..., 0] = np.where(left, 2.0 * P[..., 0], P[..., 0])
        P[..., 4] = np.where(left, 3.0 * P[..., 4], P[..., 4])
    c.sd_limiter = sd_limiter
    for k, v in kw.items():
        setattr(c, k, v)
    return c


SD3_CASES = {
    "tube3d_hllc_plus": lambda: tube3d("HLLC+"),
    "tube3d_hlle_pp": lambda: tube3d("HLLE++", limiter="minmod"),
    "tube3d_muscl_sd_hllc": lambda: tube3d("HLLC", True, "vanalbada"),
    "tube3d_ywalls_muscl_sd_hllc_plus": lambda: tube3d("HLLC+", True, ywalls=True),
    "tube3d_muscl_sd_hlle_irs": lambda: tube3d("HLLE", True, irs_beta=0.5, time_accurate=False),
}


@pytest.mark.parametrize("name", sorted(SD3_CASES))
def test_shock_detector_3d_steps(oracle_mod, name):
    """The detector of every 3-D cell over its six face neighbours (its own
    pass over the ghosted state), each face taking its low cell's value (a
    connection face, the boundary cell's)."""
    case = SD3_CASES[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(3):
        o.step()
        s.explicit_step()
    compare_state(s, o, len(case.nodes), exact=False, tol=1e-12, vars_=V3)
    for _ in range(2):
        o.step()
    s.advance(2)
    compare_state(s, o, len(case.nodes), exact=False, tol=1e-12, vars_=V3)


def test_shock_detector_3d_is_active():
    """MUSCL-SD changes the 3-D solution at the discontinuities."""
    a, b = tube3d("HLLC", True, "vanalbada"), tube3d("HLLC", False, "vanalbada")
    sa, sb = solver(a), solver(b)
    sa.explicit_step()
    sb.explicit_step()
    assert not np.array_equal(sa.download_prim(1), sb.download_prim(1))


def test_shock_detector_3d_fp64(oracle_mod):
    from mose_b200 import _lib
    case = tube3d("HLLE++", True)
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_FP64)
    o.step()
    s.explicit_step()
    compare_state(s, o, len(case.nodes), exact=False, tol=1e-12, vars_=V3)
