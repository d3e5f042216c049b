"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle on
the same seeded inputs.  The reference-exact FP64 mode must agree bit for bit
(max |difference| == 0) except where a transcendental library call (pow in
the 406 outflow) may differ by an ulp between glibc and CUDA; those cases use
the normwise relative L-infinity bar of 1e-12."""
import numpy as np
import pytest

from mose_b200 import cases
from mose_b200.cases import GC

pytestmark = pytest.mark.gpu


def solver(case, **kw):
    from mose_b200 import Solver
    return Solver(case, **kw)


def interior(P):
    """Interior cells of a reference-layout array (nk+4, nj+4, ni+4, 5)."""
    return P[GC:-GC, GC:-GC, GC:-GC]


def rel_linf(a, b):
    den = np.abs(b).max()
    return np.abs(a - b).max() / (den if den > 0 else 1.0)


def compare_state(s, o, nblk, exact=True, tol=1e-12, vars_=(0, 1, 2, 4)):
    worst = 0.0
    for b in range(1, nblk + 1):
        g = interior(s.download_prim(b))[..., list(vars_)]
        r = interior(o.get_prim(b))[..., list(vars_)]
        if exact:
            assert np.array_equal(g, r), f"block {b}: max diff {np.abs(g - r).max()}"
        else:
            worst = max(worst, rel_linf(g, r))
    if not exact:
        assert worst <= tol, worst
    return worst


SMALL = {
    "sod": lambda: cases.sod(200),
    "vortex": lambda: cases.isentropic_vortex(64, steps=3),
    "vortex_minmod_ausm": lambda: cases.isentropic_vortex(40, steps=3, limiter="minmod", riemann="AUSM+"),
    "quadrant": lambda: cases.four_quadrant(seed=2, nbx=3, nby=2, nmin=20, nmax=70, steps=3),
    "quadrant_vanleer_slau": lambda: cases.four_quadrant(seed=5, nbx=2, nby=2, nmin=17, nmax=40, steps=3,
                                                        limiter="vanleer", riemann="SLAU"),
}


@pytest.mark.parametrize("name", sorted(SMALL))
def test_metrics_bitwise(oracle_mod, name):
    case = SMALL[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for b in range(1, len(case.nodes) + 1):
        vol_o, dl_o, _ = o.get_metrics(b)
        vol_g, dl_g = s.download_metrics(b)
        assert np.array_equal(vol_g[2, 2:-2, 2:-2], vol_o[2, 2:-2, 2:-2])
        ni, nj, _ = s.dims[b - 1]
        # dl along i on the i-ghosted rows, along j on the j-ghosted columns
        assert np.array_equal(dl_g[2, 2:-2, :, 0], dl_o[2, 2:-2, :, 0])
        if nj >= 3:
            assert np.array_equal(dl_g[2, :, 2:-2, 1], dl_o[2, :, 2:-2, 1])
        for d in (1, 2):
            Ng, Ag = s.download_faces(b, d)
            No, Ao = o.get_faces(b, d)
            assert np.array_equal(Ag, Ao) and np.array_equal(Ng, No)


@pytest.mark.parametrize("name", sorted(SMALL))
def test_residual_phase_path_bitwise(oracle_mod, name):
    """One residual evaluation (Fill_Ghost_Cell + Fluxes + BC_Fluxes) through
    the phase entry points: R identical to the oracle's."""
    case = SMALL[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    o.fill_ghost_cell()
    o.fluxes()
    o.bc_fluxes()
    s.fill_ghost_cell()
    s.fluxes_and_bc_fluxes()
    for b in range(1, len(case.nodes) + 1):
        rg = interior(s.download_residual(b))[..., [0, 1, 2, 4]]
        ro = interior(o.get_residual(b))[..., [0, 1, 2, 4]]
        assert np.array_equal(rg, ro), f"block {b}: rel {rel_linf(rg, ro):.3e}"


@pytest.mark.parametrize("name", sorted(SMALL))
def test_phase_step_bitwise(oracle_mod, name):
    """A whole Explicit_Step through the separate phases (compute_dt,
    set_global_dt, copy_state, then per stage ghost fill, residual, newstate)."""
    case = SMALL[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        dto, _ = o.step()
        dtg = s.run_phases()
        assert dtg == dto
        compare_state(s, o, len(case.nodes))


@pytest.mark.parametrize("name", sorted(SMALL))
def test_fused_steps_bitwise(oracle_mod, name):
    """The fused step (one kernel per RK stage, dt on the device) over several
    steps, and the graph-replayed advance()."""
    case = SMALL[name]()
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
    ng, no = s.compute_residual(), o.residual_norms()
    np.testing.assert_allclose(ng, no, rtol=1e-12, atol=0)


@pytest.mark.parametrize("n, in_place", [(64, True), (63, False)])
def test_connection_edges_read_in_place(oracle_mod, n, in_place):
    """On an even-sized periodic block the stage kernels read the four 201
    edges' ghost cells from the source cells Ghost_Connection copies there,
    so the fused steps launch no ghost fill; an odd-sized block keeps it.
    Both step bit for bit with the oracle, fused and graph-replayed."""
    case = cases.isentropic_vortex(n, steps=3)
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        dto, to = o.step()
        dtg, tg = s.explicit_step()
        assert dtg == dto and tg == to
    compare_state(s, o, 1)
    for _ in range(3):
        o.step()
    s.advance(3)
    compare_state(s, o, 1)
    _, launches = s.time_kernels(2)
    assert (launches[1] == 0) == in_place, launches


def test_sod_to_final_time_bitwise(oracle_mod):
    """Configuration 1 at 1000 cells integrated to t >= 0.2."""
    case = cases.sod(1000)
    o = oracle_mod.Oracle(case)
    s = solver(case)
    n = 0
    while o.time < case.t_end:
        o.step()
        s.explicit_step()
        n += 1
    assert s.time == o.time
    compare_state(s, o, 1)


def test_sod79_reference_inputs_bitwise(oracle_mod):
    from tests.test_oracle import sod79_case
    case, _ = sod79_case()
    o = oracle_mod.Oracle(case)
    s = solver(case)
    while o.time < case.t_end:
        o.step()
        s.explicit_step()
    compare_state(s, o, 1)


def test_curvilinear_walls_inflow_outflow(oracle_mod):
    """Configuration 5 geometry (small): curvilinear metrics, 405 inflow, 406
    outflow (pow: ulp-level library differences allowed), 300 slip walls."""
    case = cases.curvilinear_channel(48, steps=1)
    # a perturbation so every boundary branch sees non-trivial states
    rng = np.random.default_rng(0)
    case.prim[0][..., 0] *= 1 + 0.05 * rng.standard_normal(case.prim[0].shape[:-1])
    case.prim[0][..., 2] = 0.05 * rng.standard_normal(case.prim[0].shape[:-1])
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(3):
        o.step()
        s.explicit_step()
    compare_state(s, o, 1, exact=False, tol=1e-12)


def test_local_time_stepping(oracle_mod):
    case = cases.four_quadrant(seed=3, nbx=2, nby=2, nmin=16, nmax=30, steps=1)
    case.time_accurate = False
    o = oracle_mod.Oracle(case)
    s = solver(case)
    for _ in range(2):
        o.step()
        s.explicit_step()
    compare_state(s, o, 4)
    for b in range(1, 5):
        assert np.array_equal(s.download_dt(b), o.get_dtlocal(b))


def _per_var_rel(s, o, nblk, vars_=(0, 1, 2, 4), base=None):
    """Normwise relative L-infinity per variable over the whole domain:
    max_cells |gpu - oracle| / max_cells |oracle|, worst variable.  With base
    (the state before the step) it compares the state changes instead."""
    num = {v: 0.0 for v in vars_}
    den = {v: 0.0 for v in vars_}
    for b in range(1, nblk + 1):
        g = interior(s.download_prim(b))
        r = interior(o.get_prim(b))
        if base is not None:
            g = g - base[b - 1]
            r = r - base[b - 1]
        for v in vars_:
            num[v] = max(num[v], float(np.abs(g[..., v] - r[..., v]).max()))
            den[v] = max(den[v], float(np.abs(r[..., v]).max()))
    return max(num[v] / den[v] if den[v] > 0 else num[v] for v in vars_)


@pytest.mark.parametrize("name", sorted(SMALL))
def test_fp64_precision_within_1e12_per_step(oracle_mod, name):
    """The restated FP64 arithmetic (reciprocals, FMA, simplified single-
    species algebra) stays within the 1e-12 normwise relative bar of the
    reference arithmetic over one RK3 step from identical inputs, and the
    residual of one evaluation does too."""
    from mose_b200 import _lib
    case = SMALL[name]()
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_FP64)
    base = [interior(o.get_prim(b)).copy() for b in range(1, len(case.nodes) + 1)]
    dto, _ = o.step()
    dtg, _ = s.explicit_step()
    assert dtg == dto                 # the dt pass is shared by every precision
    err = _per_var_rel(s, o, len(case.nodes))
    assert err <= 1e-12, err
    # the state change of the step, which the residual drives, to the same bar
    derr = _per_var_rel(s, o, len(case.nodes), base=base)
    assert derr <= 1e-12, derr
    # one residual evaluation (the residual phase runs the fp64 arithmetic)
    o2 = oracle_mod.Oracle(case)
    s2 = solver(case, precision=_lib.PRECISION_FP64)
    o2.fill_ghost_cell()
    o2.fluxes()
    o2.bc_fluxes()
    s2.fill_ghost_cell()
    s2.fluxes_and_bc_fluxes()
    num, den = np.zeros(4), np.zeros(4)
    for b in range(1, len(case.nodes) + 1):
        rg = interior(s2.download_residual(b))[..., [0, 1, 2, 4]]
        ro = interior(o2.get_residual(b))[..., [0, 1, 2, 4]]
        num = np.maximum(num, np.abs(rg - ro).reshape(-1, 4).max(axis=0))
        den = np.maximum(den, np.abs(ro).reshape(-1, 4).max(axis=0))
    rerr = float((num / np.where(den > 0, den, 1.0)).max())
    assert rerr <= 1e-12, rerr


@pytest.mark.parametrize("name", ["vortex", "quadrant", "sod"])
def test_mixed_precision_error(oracle_mod, name):
    """FP32 reconstruction + Riemann wave structure, FP64 state, upwind flux
    and compensated accumulation: the density error against the FP64 oracle
    after 5 steps stays below 1e-6 (HLLC) or 1e-5 (the other solvers)."""
    from mose_b200 import _lib
    case = SMALL[name]()
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
    l2 = np.sqrt(num / den)
    tol = 1e-6 if case.riemann == "HLLC" else 1e-5
    assert l2 < tol, l2


@pytest.mark.parametrize("name", ["quadrant", "sod"])
def test_mixed_uniform_detection_tolerates_last_bit_metrics(oracle_mod, name):
    """Nodes placed by floating-point arithmetic (the four-quadrant blocks on
    [0,1]^2, Sod's 200 cells on [0,1]) give metrics that differ in their last
    bits.  The exact and fp64 precisions keep the per-cell metric arrays
    (bitwise uniformity only: a last-bit face-area difference is ~1e-10 of a
    residual); the mixed precision accepts metrics within 1e-9 relative as
    uniform and runs the uniform-grid FP32 pipeline, boundary faces included,
    with its density error against the oracle unchanged in magnitude."""
    from mose_b200 import _lib
    case = SMALL[name]()
    exact = solver(case)
    fp64 = solver(case, precision=_lib.PRECISION_FP64)
    assert not exact.uniform_metrics and not fp64.uniform_metrics
    o = oracle_mod.Oracle(case)
    s = solver(case, precision=_lib.PRECISION_MIXED)
    assert s.uniform_metrics
    for n in range(5):
        dto, _ = o.step()
        dtg, _ = s.explicit_step()
        # the first dt comes from identical states; the later ones from
        # states that carry the FP32 face-state error
        assert abs(dtg - dto) <= (1e-12 if n == 0 else 1e-5) * dto
    num = den = 0.0
    for b in range(1, len(case.nodes) + 1):
        g = interior(s.download_prim(b))[..., 0]
        r = interior(o.get_prim(b))[..., 0]
        num += float(((g - r) ** 2).sum())
        den += float((r ** 2).sum())
    l2 = np.sqrt(num / den)
    assert l2 < 1e-6, l2


def test_device_error_reports_location(oracle_mod):
    """A negative pressure planted in the initial state is reported like the
    reference's stop (code 4/5 with the offending cell), and the context stays
    usable."""
    from mose_b200 import MoseError
    case = cases.isentropic_vortex(32, steps=1)
    case.prim[0][0, 10, 7, 4] = -1.0
    s = solver(case)
    with pytest.raises(MoseError) as ei:
        s.explicit_step()
    assert ei.value.code in (4, 5)
