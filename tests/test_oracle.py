"""Pins the CPU oracle: golden vectors from the reference's own tests and
known answers of the restated algorithm.  CPU only."""
from pathlib import Path

import numpy as np
import pytest

from mose_b200 import cases
from mose_b200.cases import Case

GOLDEN = Path(__file__).resolve().parent / "golden"


def _probe_errors(P, x, exact, gamma, probes):
    """check.py:45-84 of the reference's Sod79 test: relative error (%) of
    rho, u, p, sie at cells int(n * f)."""
    rho, u, p = P[:, 0], P[:, 1], P[:, 4]
    sie = p / ((gamma - 1.0) * rho)
    out = []
    for f in probes:
        i = int(len(rho) * f)
        e = [np.interp(x[i], exact[:, 0], exact[:, c]) for c in (1, 2, 3, 4)]
        out.append([abs(rho[i] - e[0]) / e[0] * 100, abs(u[i] - e[1]) / (e[1] + 1e-10) * 100,
                    abs(p[i] - e[2]) / e[2] * 100, abs(sie[i] - e[3]) / e[3] * 100])
    return np.array(out)


def sod79_case():
    d = np.load(GOLDEN / "sod79_x4.npz")
    R = 8314.46 / 28.970418            # test/common/Air: M = 28.970418, cp = 1004.5
    cp = 1004.5
    gam = cp / (cp - R)
    return Case("sod79", [d["nodes"]], d["bc_rec"], d["bc_data"], [d["prim"]], n_rk=3, cfl=float(d["cfl"]),
                time_accurate=True, limiter="mc", riemann="SLAU", gamma=gam, rgas=R,
                t_end=float(d["t_end"])), d


def test_sod79_reference_case_passes_reference_check(oracle_mod):
    """The reference's Sod79 inputs (mesh_x4, ic_x4, bc_x4) and numerics
    (input.ini: SLAU, MC, CFL 0.9, RK3) reproduce its exact.txt within the
    1 % probe criterion of its check.py."""
    case, d = sod79_case()
    o = oracle_mod.Oracle(case)
    n = 0
    while o.time < case.t_end:
        o.step()
        n += 1
    assert 150 < n < 300
    P = o.get_prim(1)[2, 2, 2:-2]
    x = 0.5 * (d["nodes"][0, 0, :-1, 0] + d["nodes"][0, 0, 1:, 0])
    err = _probe_errors(P, x, d["exact"], case.gamma, d["probes"])
    assert err.max() < float(d["threshold_pct"]), err
    assert err.max() < 0.1     # observed ~0.03 %: a regression guard well inside the 1 % bar


def test_sod_1000_hllc_minmod_matches_exact(oracle_mod):
    """Configuration 1 (1000 cells, MUSCL minmod + HLLC, CFL 0.5) against the
    reference's exact Sod profile at the same probes."""
    case = cases.sod(1000)
    o = oracle_mod.Oracle(case)
    while o.time < case.t_end:
        o.step()
    d = np.load(GOLDEN / "sod79_x4.npz")
    P = o.get_prim(1)[2, 2, 2:-2]
    x = (np.arange(1000) + 0.5) / 1000
    err = _probe_errors(P, x, d["exact"], 1.4, d["probes"])
    assert err.max() < 1.0, err
    # the step count follows from the CFL limit; the reference overshoots t_end by < 1 dt
    assert 0.2 <= o.time < 0.2 + 3e-4


@pytest.mark.parametrize("lim", ["minmod", "vanleer", "vanalbada", "mc", "superbee"])
def test_limiter_known_values(oracle_mod, lim):
    lib = oracle_mod.load()
    L = oracle_mod.LIMITERS[lim]
    f = lambda x, y: lib.orc_limiter(L, x, y)
    # opposite signs: minmod/vanleer/mc/superbee vanish; van Albada is not clipped (r < 0)
    if lim == "vanalbada":
        r = -0.5
        assert f(2.0, -1.0) == pytest.approx(((r * r + r) / (1 + r * r)) * 2.0, rel=0, abs=1e-15)
    else:
        assert f(2.0, -1.0) == 0.0
    # equal slopes are returned unchanged by every limiter (phi(1) = 1)
    assert f(0.3, 0.3) == pytest.approx(0.3, rel=1e-15)
    if lim == "minmod":
        assert f(1.0, 2.0) == 1.0 and f(2.0, 1.0) == 1.0 and f(-3.0, -1.0) == -1.0
    if lim == "vanleer":
        assert f(1.0, 3.0) == pytest.approx(2 * 3.0 / (1 + 3.0), rel=1e-15)   # phi = 2r/(1+r)
    if lim == "superbee":
        assert f(1.0, 3.0) == pytest.approx(2.0, rel=1e-15)
    if lim == "mc":
        assert f(1.0, 3.0) == pytest.approx(2.0, rel=1e-15)
        assert f(1.0, 0.5) == pytest.approx(0.75, rel=1e-15)


RIEMANN_ALL = ["HLLC", "AUSM+", "SLAU", "SLAU2", "HLLE", "HLLEM", "LLF", "PLLF", "Hanel", "AUSM+-up", "AUSM+-up2",
               "HLLC+", "HLLE++", "HLLC Rotated"]


@pytest.mark.parametrize("riemann", RIEMANN_ALL)
def test_riemann_consistency(oracle_mod, riemann):
    """F(U, U) equals the physical Euler flux for every solver."""
    case = cases.sod(8, riemann=riemann)
    case.minf = 0.3
    o = oracle_mod.Oracle(case)
    import ctypes as C
    rng = np.random.default_rng(3)
    for _ in range(20):
        rho, u, v, w, p = rng.uniform(0.2, 2.0), *rng.normal(0, 0.5, 3), rng.uniform(0.2, 2.0)
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        q = np.array([rho, u, v, w, p])
        flux = np.zeros(5)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        o.lib.orc_riemann(o.h, dp(q), dp(q.copy()), dp(n.copy()), dp(flux))
        un = u * n[0] + v * n[1] + w * n[2]
        H = 1.4 / 0.4 * p / rho + 0.5 * (u * u + v * v + w * w)
        ref = np.array([rho * un, rho * un * u + p * n[0], rho * un * v + p * n[1], rho * un * w + p * n[2],
                        rho * un * H])
        np.testing.assert_allclose(flux, ref, rtol=1e-12, atol=1e-13)


def _free_stream(case):
    for p in case.prim:
        p[..., 0] = 1.0
        p[..., 1] = 0.3
        p[..., 2] = -0.2
        p[..., 3] = 0.0
        p[..., 4] = 1.0 / 1.4
    return case


def test_free_stream_preserved_periodic_cartesian(oracle_mod):
    case = _free_stream(cases.isentropic_vortex(32, steps=1))
    o = oracle_mod.Oracle(case)
    P0 = o.get_prim(1).copy()
    for _ in range(3):
        o.step()
    P = o.get_prim(1)
    np.testing.assert_allclose(P[2, 2:-2, 2:-2], P0[2, 2:-2, 2:-2], rtol=0, atol=1e-13)


def test_free_stream_preserved_curvilinear(oracle_mod):
    """Uniform flow on the curvilinear mesh: the interior residual is a sum of
    face-area vectors around each cell, which closes to round-off."""
    case = cases.curvilinear_channel(24, steps=1)
    o = oracle_mod.Oracle(case)
    o.fill_ghost_cell()
    o.fluxes()
    R = o.get_residual(1)[2, 2 + 2:-2 - 2, 2 + 2:-2 - 2]   # cells away from the boundaries
    assert np.abs(R).max() < 1e-13


def test_conservation_periodic(oracle_mod):
    """On a periodic block the summed residual of the conserved variables
    vanishes (every face flux enters two cells with opposite signs)."""
    case = cases.isentropic_vortex(48, steps=1)
    o = oracle_mod.Oracle(case)
    o.fill_ghost_cell()
    o.fluxes()
    o.bc_fluxes()
    R = o.get_residual(1)[2, 2:-2, 2:-2]
    scale = np.abs(R).max(axis=(0, 1))
    tot = np.abs(R.sum(axis=(0, 1)))
    assert np.all(tot[[0, 1, 2, 4]] <= 1e-12 * np.maximum(scale[[0, 1, 2, 4]], 1e-300) * R.shape[0] * R.shape[1])


def test_metrics_uniform_cartesian(oracle_mod):
    case = cases.isentropic_vortex(16, steps=1, L=10.0)
    o = oracle_mod.Oracle(case)
    vol, dl, M = o.get_metrics(1)
    h = 10.0 / 16
    assert np.all(vol[2, 2:-2, 2:-2] == h * h * 1.0)
    assert np.all(dl[2, 2:-2, :, 0] == h) and np.all(dl[2, :, 2:-2, 1] == h)   # incl. ghost dl
    N, A = o.get_faces(1, 1)
    assert np.all(N[..., 0] == 1.0) and np.all(N[..., 1] == 0.0) and np.all(A == h)


def test_sod_first_step_is_deterministic_across_threads(oracle_mod):
    """The OpenMP build (CPU baseline) reproduces the serial oracle bit for bit."""
    case = cases.four_quadrant(seed=1, nbx=2, nby=2, nmin=20, nmax=40, steps=2)
    a = oracle_mod.Oracle(case)
    b = oracle_mod.Oracle(case, nthreads=4, omp=True)
    for _ in range(2):
        a.step()
        b.step()
    for blk in range(1, 5):
        assert np.array_equal(a.get_prim(blk), b.get_prim(blk))


@pytest.mark.parametrize("riemann", RIEMANN_ALL)
def test_riemann_mirror_symmetry(oracle_mod, riemann):
    """Swapping the two states and reversing the normal reverses the flux of
    every conserved quantity (the solvers are symmetric in the face frame)."""
    import ctypes as C
    case = cases.sod(8, riemann=riemann)
    case.minf = 0.3
    o = oracle_mod.Oracle(case)
    rng = np.random.default_rng(11)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    for _ in range(20):
        L = np.array([rng.uniform(0.2, 2.0), *rng.normal(0, 0.6, 3), rng.uniform(0.2, 2.0)])
        R = np.array([rng.uniform(0.2, 2.0), *rng.normal(0, 0.6, 3), rng.uniform(0.2, 2.0)])
        n = rng.normal(size=3)
        if riemann == "HLLC Rotated":
            # its fallback to HLLC for n_z > 0.1 is one-sided in n_z: mirror in 2-D
            n[2], L[3], R[3] = 0.0, 0.0, 0.0
        n /= np.linalg.norm(n)
        f1, f2 = np.zeros(5), np.zeros(5)
        o.lib.orc_riemann(o.h, dp(L), dp(R), dp(n.copy()), dp(f1))
        o.lib.orc_riemann(o.h, dp(R.copy()), dp(L.copy()), dp(-n), dp(f2))
        np.testing.assert_allclose(f1, -f2, rtol=1e-11, atol=1e-12)


def ein91_case():
    d = np.load(GOLDEN / "ein91_x8.npz")
    R = 8314.46 / 28.970418            # test/common/Air
    cp = 1004.5
    return Case("ein91", [d["nodes"]], d["bc_rec"], d["bc_data"], [d["prim"]], n_rk=3, cfl=float(d["cfl"]),
                time_accurate=True, limiter="vanleer", riemann="HLLE", gamma=cp / (cp - R), rgas=R,
                t_end=float(d["t_end"])), d


def test_ein91_reference_case_hlle_passes_reference_check(oracle_mod):
    """The reference's Ein91 inputs (mesh_x8, ic_x8, bc_x8; its HLLE + van
    Leer case, CFL 0.9, RK3) meet its verify.py criterion against the exact
    solution: < 1 % (density, velocity), < 1.5 % (pressure) at cells 80, 160
    and 240."""
    case, d = ein91_case()
    o = oracle_mod.Oracle(case)
    while o.time < case.t_end:
        o.step()
    P = o.get_prim(1)[2, 2, 2:-2]
    ex = d["exact"]
    for i in d["probes"]:
        err = [abs(P[i, 0] - ex[i, 0]) / ex[i, 0] * 100, abs(P[i, 1] - ex[i, 1]) / abs(ex[i, 1] + 1e-10) * 100,
               abs(P[i, 4] - ex[i, 2]) / ex[i, 2] * 100]
        assert all(e < t for e, t in zip(err, d["threshold_pct"])), (i, err)


def test_irs_stage_matches_numpy_restatement(oracle_mod):
    """The oracle's RK stage with implicit residual smoothing equals a numpy
    restatement of Lib_Newstate.f90:40-72 and Lib_IRS.f90 (scale, per
    direction the first ghost layer and two Jacobi sweeps, then the RK
    stage) applied to the oracle's own residual, on a two-block case with
    connection (101) and extrapolation (400) faces."""
    case = cases.four_quadrant(seed=4, nbx=2, nby=1, nmin=9, nmax=14, steps=1, limiter="minmod", riemann="HLLE",
                               cfl=0.4)
    case.irs_beta = 0.6
    case.time_accurate = False
    o = oracle_mod.Oracle(case)
    o.compute_dt()
    o.copy_state()
    o.fill_ghost_cell()
    o.fluxes()
    o.bc_fluxes()
    P0 = [o.get_prim(b).copy() for b in (1, 2)]
    R = [o.get_residual(b).copy() for b in (1, 2)]          # (nk+4, nj+4, ni+4, 5)
    dt = [o.get_dtlocal(b) for b in (1, 2)]
    vol = [o.get_metrics(b)[0] for b in (1, 2)]
    g2 = slice(2, -2)
    for b in range(2):
        R[b][g2, g2, g2] = -(R[b][g2, g2, g2] / vol[b][g2, g2, g2][..., None] * dt[b][..., None] * 1.0)
    beta = case.irs_beta
    rec = case.bc_rec
    inward = {1: (1, 0), 2: (-1, 0), 3: (0, 1), 4: (0, -1)}
    for d in range(2):
        for r in rec:
            b, i, j, f, t = r[0] - 1, r[1], r[2], r[4], r[5]
            if f > 4:
                continue
            gi, gj = i - inward[f][0], j - inward[f][1]
            src = R[r[6] - 1][2, r[8] + 1, r[7] + 1] if t == 101 else R[b][2, j + 1, i + 1]
            R[b][2, gj + 1, gi + 1] = src
        for b in range(2):
            Rs = R[b].copy()
            for _ in range(2):
                Rsn = Rs.copy()
                for k in (2,):
                    if d == 0:
                        Rsn[k, g2, g2] = (R[b][k, g2, g2] + beta * (Rs[k, g2, 1:-3] + Rs[k, g2, 3:-1])) / (1.0 + 2.0 * beta)
                    else:
                        Rsn[k, g2, g2] = (R[b][k, g2, g2] + beta * (Rs[k, 1:-3, g2] + Rs[k, 3:-1, g2])) / (1.0 + 2.0 * beta)
                Rs[:, g2, g2] = Rsn[:, g2, g2]
            R[b][:, g2, g2] = Rs[:, g2, g2]
    o.rk_newstate(1)
    gam, Rg = case.gamma, case.rgas
    cv = Rg / (gam - 1.0)
    for b in range(2):
        p = P0[b][2, g2, g2]
        rho, u, v, w, pr = (p[..., q] for q in range(5))
        T = pr / (rho * Rg)
        U = np.stack([rho, rho * u, rho * v, rho * w, rho * (cv * T + 0.5 * (u * u + v * v + w * w))], -1)
        U = U + (U - U + R[b][2, g2, g2]) * 1.0
        rho = U[..., 0]
        u, v, w = U[..., 1] / rho, U[..., 2] / rho, U[..., 3] / rho
        e = U[..., 4] / rho - 0.5 * (u * u + v * v + w * w)
        want = np.stack([rho, u, v, w, rho * Rg * (e / cv)], -1)
        np.testing.assert_allclose(o.get_prim(b + 1)[2, g2, g2], want, rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("btype", [401, 403, 404, 407])
def test_inlet_boundaries_hold_the_inflow(oracle_mod, btype):
    """The inlet formulas (401 / 403 / 404 / 407) on the curvilinear Mach-0.8
    channel, fed with the free stream's own total or static conditions, keep
    it: after 60 steps the state is finite and the mean density and
    velocity of the four cell columns next to the inflow face stay within a
    few percent of the free stream."""
    g, m = 1.4, 0.8
    p_inf = 1.0 / g
    t0 = p_inf * (1 + 0.5 * (g - 1) * m * m)
    p0 = p_inf * (1 + 0.5 * (g - 1) * m * m) ** (g / (g - 1))
    data = {401: [t0, p0, 0.0, 0.0, 1.0, 0.0], 403: [t0, m, 0.0, 0.0, 1.0, 0.0],
            404: [p_inf, m, 0.0, 0.0, 1.0, 0.0], 407: [t0, p0, p_inf, 0.0, 0.0, 1.0]}[btype]
    case = cases.curvilinear_channel(24, steps=1)
    f1 = case.bc_rec[:, 5] == 405
    case.bc_rec[f1, 5] = btype
    case.bc_data[f1] = data
    o = oracle_mod.Oracle(case)
    for _ in range(60):
        o.step()
    P = o.get_prim(1)[2, 2:-2, 2:-2]
    assert np.isfinite(P).all()
    near = P[:, :4]
    assert abs(near[..., 0].mean() - 1.0) < 0.05 and abs(near[..., 1].mean() - m) < 0.05 * m, near.mean(axis=(0, 1))


def test_far_field_outflow_branch_is_the_406_formula(oracle_mod):
    """Where the boundary cell leaves the domain, 407 takes the back-pressure
    outflow of 406 (Lib_BC_Fluxes_FarField.f90:53-55): the same outflow face
    as 407 or as 406 with the same back pressure gives the same residual."""
    g = 1.4
    p_inf = 1.0 / g
    res = []
    for rec_type, row in ((406, [p_inf, 1.0, 0.0, 0.0, 0.0, 0.0]), (407, [2.0, 2.0, p_inf, 0.0, 0.0, 1.0])):
        case = cases.perturbed_channel(16, steps=1, amp=0.02, seed=1)
        f2 = case.bc_rec[:, 5] == 406
        case.bc_rec[f2, 5] = rec_type
        case.bc_data[f2] = row
        o = oracle_mod.Oracle(case)
        o.fill_ghost_cell()
        o.fluxes()
        o.bc_fluxes()
        res.append(o.get_residual(1))
    assert np.array_equal(res[0], res[1])


def _riemann_flux(o, L, R, n):
    import ctypes as C
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    f = np.zeros(5)
    o.lib.orc_riemann(o.h, dp(np.ascontiguousarray(L, dtype=np.float64)),
                      dp(np.ascontiguousarray(R, dtype=np.float64)), dp(np.ascontiguousarray(n, dtype=np.float64)),
                      dp(f))
    return f


def test_exact_solver_consistency_and_energy_flux(oracle_mod):
    """riemann_exact (Lib_Riemann_Godunov.f90): F(U, U) is the physical flux
    when the velocity is normal to the face; with a tangential velocity its
    energy flux carries only the normal kinetic energy, rho u_n (h + u_n^2/2),
    as the reference's H0(pf, df, sqrt(vel*vel)) forms it."""
    o = oracle_mod.Oracle(cases.sod(8, riemann="exact"))
    rng = np.random.default_rng(5)
    g = 1.4
    for _ in range(20):
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        rho, p, un = rng.uniform(0.2, 2.0), rng.uniform(0.2, 2.0), rng.normal(0, 0.8)
        t = np.cross(n, rng.normal(size=3))
        t *= rng.normal(0, 0.5) / np.linalg.norm(t)
        for vt in (np.zeros(3), t):
            vel = un * n + vt
            q = np.array([rho, *vel, p])
            f = _riemann_flux(o, q, q.copy(), n)
            h = g / (g - 1) * p / rho
            ref = np.array([rho * un, *(rho * un * vel + p * n), rho * un * (h + 0.5 * un * un)])
            np.testing.assert_allclose(f, ref, rtol=1e-12, atol=1e-13)


def test_exact_solver_mirror_symmetry(oracle_mod):
    """Swapping the states and reversing the normal reverses the exact
    solver's flux to within its Newton tolerance (relative pressure change
    1e-5: the two orientations iterate from different starting points)."""
    o = oracle_mod.Oracle(cases.sod(8, riemann="exact"))
    rng = np.random.default_rng(12)
    for _ in range(30):
        L = np.array([rng.uniform(0.2, 2.0), *rng.normal(0, 0.6, 3), rng.uniform(0.2, 2.0)])
        R = np.array([rng.uniform(0.2, 2.0), *rng.normal(0, 0.6, 3), rng.uniform(0.2, 2.0)])
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        f1 = _riemann_flux(o, L, R, n)
        f2 = _riemann_flux(o, R, L, -n)
        np.testing.assert_allclose(f1, -f2, rtol=1e-4, atol=1e-5)


@pytest.mark.parametrize("riemann", ["exact", "HLLC Rotated"])
def test_sod79_inputs_with_exact_and_rotated_solvers(oracle_mod, riemann):
    """The reference's Sod79 inputs with the exact Godunov solver, or the
    rotated HLLC, in place of SLAU still meet its check.py criterion (1 %)."""
    case, d = sod79_case()
    case.riemann = riemann
    o = oracle_mod.Oracle(case)
    while o.time < case.t_end:
        o.step()
    P = o.get_prim(1)[2, 2, 2:-2]
    x = 0.5 * (d["nodes"][0, 0, :-1, 0] + d["nodes"][0, 0, 1:, 0])
    err = _probe_errors(P, x, d["exact"], case.gamma, d["probes"])
    assert err.max() < float(d["threshold_pct"]), err


def _series_update(t, v, periodic, time):
    """update of Series_Data_m.f90:55-86 in plain Python (IEEE doubles, the
    reference's operation order; v_1 where the reference's value is
    undefined, before t_1)."""
    import math
    t_ = time
    if periodic:
        period = t[-1] - t[0]
        if period > 0.0:
            m = math.fmod(t_ - t[0], period)
            if m != 0.0 and ((m < 0.0) != (period < 0.0)):
                m = m + period
            t_ = t[0] + m
    if t_ == t[0]:
        return v[0]
    for i in range(1, len(t)):
        if t[i - 1] < t_ <= t[i]:
            return (v[i] - v[i - 1]) / (t[i] - t[i - 1]) * (t_ - t[i - 1]) + v[i - 1]
    return v[-1] if t_ > t[-1] else v[0]


def test_time_table_update(oracle_mod):
    """The oracle's time-table update equals the plain-Python restatement bit
    for bit (interior points, knots, both ends, periodic wrap in both
    directions) and np.interp to rounding inside the table."""
    case = cases.sod(8)
    t = np.array([0.0, 0.1, 0.25, 0.7])
    v = np.array([1.0, 1.3, 0.8, 1.1])
    case.series = [(t, v, False), (t, v, True)]
    o = oracle_mod.Oracle(case)
    rng = np.random.default_rng(2)
    times = np.concatenate([rng.uniform(-1.5, 3.0, 200), t, [-0.1, 0.7, 5.0, 0.7 * 3, -0.7]])
    for x in times:
        for sid, per in ((0, False), (1, True)):
            assert o.series_eval(sid, float(x)) == _series_update(t, v, per, float(x)), (sid, x)
    inside = rng.uniform(0.0, 0.7, 100)
    np.testing.assert_allclose([o.series_eval(0, float(x)) for x in inside], np.interp(inside, t, v), rtol=1e-14)


def test_time_table_inlet_with_constant_table_is_401(oracle_mod):
    """A 402 inlet whose table holds one p0 at every time gives the 401
    result with that p0, bit for bit (Mod_BC_Fluxes.f90:119-140)."""
    g, m = 1.4, 0.8
    p_inf = 1.0 / g
    t0 = p_inf * (1 + 0.5 * (g - 1) * m * m)
    p0 = p_inf * (1 + 0.5 * (g - 1) * m * m) ** (g / (g - 1))
    out = []
    for btype in (401, 402):
        case = cases.perturbed_channel(16, steps=1, amp=0.02, seed=4)
        f1 = case.bc_rec[:, 5] == 405
        case.bc_rec[f1, 5] = btype
        case.bc_data[f1] = [t0, p0 if btype == 401 else 0.0, 0.0, 0.0, 1.0, 0.0]
        if btype == 402:
            case.series = [(np.array([0.0, 1.0]), np.array([p0, p0]), False)]
        o = oracle_mod.Oracle(case)
        for _ in range(5):
            o.step()
        out.append(o.get_prim(1))
    assert np.array_equal(out[0], out[1])


def _one_euler_stage(oracle_mod, make, integration, cfl, irs=0.0):
    case = make(cfl)
    case.n_rk = 1
    case.integration = integration
    case.irs_beta = irs
    o = oracle_mod.Oracle(case)
    P0 = [o.get_prim(b).copy() for b in range(1, len(case.nodes) + 1)]
    o.step()
    return P0, [o.get_prim(b) for b in range(1, len(case.nodes) + 1)]


def _maxdiff(A, B):
    return max(np.abs(a - b)[2:-2, 2:-2, 2:-2].max() for a, b in zip(A, B))


def test_primitive_update_matches_conservative_to_second_order(oracle_mod):
    """Newstate_Primitive (Lib_Newstate.f90:168-317) linearises the
    conservative update: after one forward-Euler stage from the same state
    the primitive and conservative results differ by O(dt^2), far less than
    the O(dt) change of the state, and the difference shrinks about 4x when
    dt halves (four-quadrant blocks)."""
    make = lambda cfl: cases.four_quadrant(seed=1, nbx=2, nby=2, nmin=12, nmax=20, steps=1, cfl=cfl)
    gaps = []
    for cfl in (0.2, 0.1):
        P0, Pc = _one_euler_stage(oracle_mod, make, "cons", cfl)
        _, Pp = _one_euler_stage(oracle_mod, make, "prim", cfl)
        gap, change = _maxdiff(Pp, Pc), _maxdiff(Pc, P0)
        assert 0.0 < gap < 0.1 * change, (gap, change)
        gaps.append(gap)
    assert 3.0 < gaps[0] / gaps[1] < 5.0, gaps


def test_primitive_update_with_irs_is_continuous_in_beta(oracle_mod):
    """The IRS branch of Newstate_Primitive (:195-231: primitive increments,
    smoothing, RK stage) tends to the plain primitive update as irs-beta
    goes to 0, linearly in beta."""
    make = lambda cfl: cases.isentropic_vortex(40, steps=1, cfl=cfl)
    _, P = _one_euler_stage(oracle_mod, make, "prim", 0.3)
    d = []
    for beta in (2e-3, 1e-3):
        _, Pb = _one_euler_stage(oracle_mod, make, "prim", 0.3, irs=beta)
        d.append(_maxdiff(Pb, P))
    assert 0.0 < d[1] < d[0] < 1e-3 and 1.8 < d[0] / d[1] < 2.2, d


def vv_case(name):
    d = np.load(GOLDEN / f"{name}.npz")
    case = Case(name, [d["nodes"]], d["bc_rec"], d["bc_data"], [d["prim"]], n_rk=3, cfl=float(d["cfl"]),
                time_accurate=True, limiter=str(d["limiter"]), riemann=str(d["riemann"]), gamma=float(d["gamma"]),
                rgas=float(d["rgas"]), t_end=float(d["t_end"]))
    return case, d


def test_tor99_reference_case_passes_reference_check(oracle_mod):
    """The reference's Tor99 inputs (mesh_x8, ic_x8, bc_x8; HLLE++ with the
    Tramel shock detector, van Leer, CFL 0.9, RK3, t = 0.2) meet its
    verify.py criterion: density, velocity, pressure and specific internal
    energy within 1 % of the exact solution at cells 80, 240, 400, 560, 720
    (observed worst 0.07 %)."""
    case, d = vv_case("tor99_x8")
    o = oracle_mod.Oracle(case)
    while o.time < case.t_end:
        o.step()
    P = o.get_prim(1)[2, 2, 2:-2]
    ex = d["exact"]
    sie = P[:, 4] / ((case.gamma - 1.0) * P[:, 0])
    for i in d["probes"]:
        err = [abs(P[i, 0] - ex[i, 0]) / ex[i, 0] * 100, abs(P[i, 1] - ex[i, 1]) / abs(ex[i, 1] + 1e-10) * 100,
               abs(P[i, 4] - ex[i, 2]) / ex[i, 2] * 100, abs(sie[i] - ex[i, 3]) / ex[i, 3] * 100]
        assert all(e < t for e, t in zip(err, d["threshold_pct"])), (i, err)
        assert max(err) < 0.2, (i, err)      # regression guard well inside the 1 % bar


def test_noh87_cold_inflow_is_beyond_the_closed_form_thermo(oracle_mod):
    """The reference's Noh87 inputs: the cold inflow (p = 1e-15) loses its
    pressure to rounding within a few hundred steps under the closed-form
    thermo, and the run stops with the reference's interface-state code
    (4) rather than continuing on a non-physical state."""
    case, _ = vv_case("noh87_x8")
    o = oracle_mod.Oracle(case)
    with pytest.raises(RuntimeError, match="failed: 4"):
        for _ in range(1000):
            o.step()
