"""GPU parity of the 3-D path (the k-face march and the plane stage per RK
stage) against the CPU oracle, through the C ABI.  The reference-exact precision must agree
bit for bit, except where the 406 outflow's pow may differ by an ulp between
glibc and CUDA (normwise relative L-infinity bar 1e-12)."""
import numpy as np
import pytest

from mose_b200 import cases
from mose_b200.cases import GC

pytestmark = pytest.mark.gpu


def solver(case, **kw):
    from mose_b200 import Solver
    return Solver(case, **kw)


def interior(P):
    return P[GC:-GC, GC:-GC, GC:-GC]


def compare_state(s, o, nblk, exact=True, tol=1e-12):
    worst = 0.0
    for b in range(1, nblk + 1):
        g = interior(s.download_prim(b))
        r = interior(o.get_prim(b))
        if exact:
            assert np.array_equal(g, r), f"block {b}: max diff {np.abs(g - r).max()}"
        else:
            worst = max(worst, np.abs(g - r).max() / np.abs(r).max())
    if not exact:
        assert worst <= tol, worst
    return worst


SMALL3 = {
    "box_hllc_vanleer": lambda: cases.periodic_box_3d(sizes=[[6, 9], [7, 8], [5, 10]], seed=1, steps=3),
    "box_ausm_minmod": lambda: cases.periodic_box_3d(sizes=[[8, 6], [6, 7], [7, 5]], seed=2, steps=3,
                                                      limiter="minmod", riemann="AUSM+"),
    "box_hllc_vanalbada_1block": lambda: cases.periodic_box_3d(sizes=[[7], [6], [9]], nb=(1, 1, 1), seed=3,
                                                               steps=3, limiter="vanalbada", amp=5e-2),
    # several tiles per block (32 x 8 cells of the (i, j) plane): the tiles of
    # the middle rows have connection faces only, those of the wall rows take
    # the boundary formulas; 40 cells per unit length give metric arrays
    "box_ywalls_tiles": lambda: cases.periodic_box_3d(sizes=[[40, 24], [20], [6, 5]], nb=(2, 1, 2), seed=4,
                                                      steps=3, ywalls=True),
}


@pytest.mark.parametrize("name", sorted(SMALL3))
def test_metrics3d_bitwise(oracle_mod, name):
    case = SMALL3[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for b in range(1, len(case.nodes) + 1):
        vol_o, dl_o, _ = o.get_metrics(b)
        vol_g, dl_g = s.download_metrics(b)
        assert np.array_equal(vol_g[2:-2, 2:-2, 2:-2], vol_o[2:-2, 2:-2, 2:-2])
        assert np.array_equal(dl_g[2:-2, 2:-2, :, 0], dl_o[2:-2, 2:-2, :, 0])
        assert np.array_equal(dl_g[2:-2, :, 2:-2, 1], dl_o[2:-2, :, 2:-2, 1])
        assert np.array_equal(dl_g[:, 2:-2, 2:-2, 2], dl_o[:, 2:-2, 2:-2, 2])
        for d in (1, 2, 3):
            Ng, Ag = s.download_faces(b, d)
            No, Ao = o.get_faces(b, d)
            assert np.array_equal(Ag, Ao) and np.array_equal(Ng, No)


@pytest.mark.parametrize("name", sorted(SMALL3))
def test_residual3d_phase_path_bitwise(oracle_mod, name):
    case = SMALL3[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    o.fill_ghost_cell()
    o.fluxes()
    o.bc_fluxes()
    s.fill_ghost_cell()
    s.fluxes_and_bc_fluxes()
    for b in range(1, len(case.nodes) + 1):
        rg = interior(s.download_residual(b))
        ro = interior(o.get_residual(b))
        assert np.array_equal(rg, ro), f"block {b}: max diff {np.abs(rg - ro).max()}"


@pytest.mark.parametrize("name", sorted(SMALL3))
def test_fused3d_steps_bitwise(oracle_mod, name):
    """Fused steps (the k-face march and the plane stage per RK stage, dt on
    the device, the last stage folding in the next step's CFL pass) and
    graph-replayed advance()."""
    case = SMALL3[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        dto, to = o.step()
        dtg, tg = s.explicit_step()
        assert dtg == dto and tg == to
    compare_state(s, o, len(case.nodes))
    for _ in range(3):
        o.step()
    dtg, tg = s.advance(3)
    assert tg == o.time
    compare_state(s, o, len(case.nodes))


def test_channel3d_curvilinear_boundaries(oracle_mod):
    """Curvilinear 3-D metrics (general-metric kernels), 405 inflow, 406
    outflow (pow), 300 slip walls, 400 extrapolation."""
    case = cases.channel_3d(10, steps=1)
    rng = np.random.default_rng(0)
    case.prim[0][..., 0] *= 1 + 0.05 * rng.standard_normal(case.prim[0].shape[:-1])
    case.prim[0][..., 2] = 0.05 * rng.standard_normal(case.prim[0].shape[:-1])
    case.prim[0][..., 3] = 0.05 * rng.standard_normal(case.prim[0].shape[:-1])
    o = oracle_mod.Oracle(case)
    s = solver(case)
    assert not s.uniform_metrics
    for _ in range(3):
        o.step()
        s.explicit_step()
    compare_state(s, o, 1, exact=False, tol=1e-12)


def perturbed(case, seed=1):
    """The case with every input value of rho, u, v, w, p changed by half an
    ulp (relative 2^-53, seeded signs)."""
    import copy
    c = copy.copy(case)
    rng = np.random.default_rng(seed)
    c.prim = []
    for P in case.prim:
        Q = P.copy()
        for v in (0, 1, 2, 3, 4):
            Q[..., v] = P[..., v] * (1.0 + 2.0 ** -53 * rng.choice([-1.0, 1.0], size=P.shape[:-1]))
        c.prim.append(Q)
    return c


def step_errors(get_a, get_b, base, nb):
    """Per variable: normwise relative error of the state and of the state
    change (a - base against b - base)."""
    out = []
    for v in (0, 1, 2, 3, 4):
        num = max(np.abs(interior(get_a(b))[..., v] - interior(get_b(b))[..., v]).max() for b in range(1, nb + 1))
        den = max(np.abs(interior(get_b(b))[..., v]).max() for b in range(1, nb + 1))
        dnum = max(np.abs((interior(get_a(b)) - base[b - 1])[..., v] - (interior(get_b(b)) - base[b - 1])[..., v]).max()
                   for b in range(1, nb + 1))
        dden = max(np.abs((interior(get_b(b)) - base[b - 1])[..., v]).max() for b in range(1, nb + 1))
        out.append((num / den, dnum / dden))
    return out


@pytest.mark.parametrize("name", sorted(SMALL3))
def test_fp64_3d_within_1e12(oracle_mod, name):
    """One fp64 step within the normwise bar 1e-12 on the state and on the
    state change.  Where a step changes a variable by a few 1e-4 of its size
    (the 40-cell blocks' small dt), a few ulps of the state are already 1e-12
    of the change: there the bar is the larger of 1e-12 and twice the
    oracle's own change under a half-ulp perturbation of its input."""
    from mose_b200 import _lib
    case = SMALL3[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_FP64)
    nb = len(case.nodes)
    base = [interior(o.get_prim(b)).copy() for b in range(1, nb + 1)]
    o.step()
    s.explicit_step()
    errs = step_errors(s.download_prim, o.get_prim, base, nb)
    floors = None
    if max(max(e) for e in errs) > 1e-12:
        op = oracle_mod.Oracle(perturbed(case))
        op.step()
        floors = step_errors(op.get_prim, o.get_prim, base, nb)
    for v, (err, derr) in enumerate(errs):
        fs, fd = floors[v] if floors else (0.0, 0.0)
        assert err <= max(1e-12, 2.0 * fs), (v, err, fs)
        assert derr <= max(1e-12, 2.0 * fd), (v, derr, fd)


@pytest.mark.parametrize("name", ["box_hllc_vanleer", "box_ausm_minmod"])
def test_mixed_3d_density_error(oracle_mod, name):
    from mose_b200 import _lib
    case = SMALL3[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_MIXED)
    for _ in range(5):
        o.step()
        s.explicit_step()
    num = den = 0.0
    for b in range(1, len(case.nodes) + 1):
        g = interior(s.download_prim(b))[..., 0]
        r = interior(o.get_prim(b))[..., 0]
        num += float(((g - r) ** 2).sum())
        den += float((r ** 2).sum())
    assert np.sqrt(num / den) < 1e-6, np.sqrt(num / den)


# every solver of the run-time unit and every limiter on the 3-D sweeps
SOLVERS3 = ["SLAU", "SLAU2", "HLLE", "HLLEM", "LLF", "PLLF", "Hanel", "AUSM+-up", "AUSM+-up2", "HLLC Rotated",
            "exact"]
LIMITERS3 = ["first-order", "mc", "superbee"]


def _box(riemann="HLLC", limiter="vanleer", seed=5, steps=2):
    case = cases.periodic_box_3d(sizes=[[6, 7], [7, 5], [5, 6]], seed=seed, steps=steps, limiter=limiter,
                                 riemann=riemann, amp=5e-2)
    case.minf = 0.3
    return case


@pytest.mark.parametrize("riemann", SOLVERS3)
def test_runtime_solvers_3d(oracle_mod, riemann):
    """The run-time solver unit on the 3-D sweeps: bit for bit, except the
    exact solver (pow: the 1e-12 normwise bar)."""
    case = _box(riemann)
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        o.step()
        s.explicit_step()
    compare_state(s, o, len(case.nodes), exact=riemann != "exact")
    for _ in range(2):
        o.step()
    s.advance(2)
    compare_state(s, o, len(case.nodes), exact=riemann != "exact")


@pytest.mark.parametrize("limiter", LIMITERS3)
@pytest.mark.parametrize("riemann", ["HLLC", "AUSM+", "HLLE"])
def test_limiters_3d(oracle_mod, riemann, limiter):
    case = _box(riemann, limiter)
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(3):
        o.step()
        s.explicit_step()
    compare_state(s, o, len(case.nodes))


@pytest.mark.parametrize("riemann", ["HLLE", "exact"])
def test_runtime_solvers_3d_fp64_within_1e12(oracle_mod, riemann):
    from mose_b200 import _lib
    case = _box(riemann, "vanalbada")
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_FP64)
    o.step()
    s.explicit_step()
    compare_state(s, o, len(case.nodes), exact=False, tol=1e-12)
