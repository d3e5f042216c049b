"""Discrete adjoint of the explicit step (C ABI mose_gpu_adjoint_*) against
central finite differences (step 1e-6) of the forward: one step, a
checkpointed multi-step objective, the CPU oracle's forward (the reference
gradient), and the torch.autograd.Function.  Curvilinear channel: 405
inflow (Mach derivative too), 406 outflow, 300 slip walls; van Albada +
HLLC, SSP-RK3.  Bar: relative error 1e-5."""
import numpy as np
import pytest

from mose_b200 import cases
from mose_b200.cases import GC, to_ref_layout

pytestmark = pytest.mark.gpu

H = 1e-6


def channel(n=16, seed=0):
    case = cases.curvilinear_channel(n, steps=1)
    rng = np.random.default_rng(seed)
    p = case.prim[0]
    p[..., 0] *= 1 + 0.05 * rng.standard_normal(p.shape[:-1])
    p[..., 1] *= 1 + 0.05 * rng.standard_normal(p.shape[:-1])
    p[..., 2] = 0.05 * rng.standard_normal(p.shape[:-1])
    p[..., 4] *= 1 + 0.05 * rng.standard_normal(p.shape[:-1])
    return case


def interior(P):
    return P[GC:-GC, GC:-GC, GC:-GC]


def direction(shape, rng):
    d = rng.standard_normal(shape)
    d[..., 3] = 0.0      # w is not a state of the 2-D path
    return d


def solver(case, **kw):
    from mose_b200 import Solver
    return Solver(case, **kw)


def step_state(s, P0, mach, nsteps):
    s.upload_prim(1, to_ref_layout(P0))
    s.set_time(0.0, 0)
    s.set_inflow_mach(mach)
    for _ in range(nsteps):
        s.explicit_step()
    return interior(s.download_prim(1))


def test_adjoint_step_matches_fd():
    case = channel()
    mach = case.extra["mach"]
    s = solver(case)
    P0 = case.prim[0].copy()
    rng = np.random.default_rng(1)
    lam1 = direction(P0.shape, rng)
    s.upload_prim(1, to_ref_layout(P0))
    s.upload_adjoint(1, to_ref_layout(lam1))
    dM = s.adjoint_step()
    lam0 = interior(s.download_adjoint(1))
    g = lambda P, M: float((lam1 * step_state(s, P, M, 1)).sum())
    for q in range(3):
        d = direction(P0.shape, rng)
        fd = (g(P0 + H * d, mach) - g(P0 - H * d, mach)) / (2 * H)
        adj = float((lam0 * d).sum())
        assert abs(adj - fd) <= 1e-5 * abs(fd), (q, adj, fd)
    fdm = (g(P0, mach + H) - g(P0, mach - H)) / (2 * H)
    assert abs(dM - fdm) <= 1e-5 * max(abs(fdm), 1e-12), (dM, fdm)


def objective(s, P0, mach, nsteps):
    s.upload_prim(1, to_ref_layout(P0))
    s.set_time(0.0, 0)
    s.set_inflow_mach(mach)
    return s.adjoint_forward(nsteps, 4, 1, 3)


def test_checkpointed_gradient_matches_fd():
    case = channel(seed=2)
    mach = case.extra["mach"]
    s = solver(case)
    P0 = case.prim[0].copy()
    n = 12
    J = objective(s, P0, mach, n)
    dM = s.adjoint_backward()
    grad = interior(s.download_adjoint(1))
    assert np.isfinite(J) and np.isfinite(grad).all()
    rng = np.random.default_rng(3)
    for q in range(4):
        d = direction(P0.shape, rng)
        fd = (objective(s, P0 + H * d, mach, n) - objective(s, P0 - H * d, mach, n)) / (2 * H)
        adj = float((grad * d).sum())
        assert abs(adj - fd) <= 1e-5 * abs(fd), (q, adj, fd)
    fdm = (objective(s, P0, mach + H, n) - objective(s, P0, mach - H, n)) / (2 * H)
    assert abs(dM - fdm) <= 1e-5 * abs(fdm), (dM, fdm)


def test_gradient_matches_oracle_fd(oracle_mod):
    """The reference gradient: central differences of the CPU oracle."""
    case = channel(12, seed=4)
    mach = case.extra["mach"]
    n = 8
    s = solver(case)
    P0 = case.prim[0].copy()
    objective(s, P0, mach, n)
    dM = s.adjoint_backward()
    grad = interior(s.download_adjoint(1))

    def J_oracle(P, M):
        c = cases.curvilinear_channel(12, steps=1)
        c.prim[0][...] = P
        c.bc_data[c.bc_rec[:, 5] == 405, 0] = M
        o = oracle_mod.Oracle(c)
        for _ in range(n):
            o.step()
        _, A = o.get_faces(1, 2)                     # j-faces: A[k, j, i], j = 0 is face 3
        p = interior(o.get_prim(1))[0, 0, :, 4]
        return float((p * A[0, 0, :]).sum())

    rng = np.random.default_rng(5)
    for q in range(2):
        d = direction(P0.shape, rng)
        fd = (J_oracle(P0 + H * d, mach) - J_oracle(P0 - H * d, mach)) / (2 * H)
        adj = float((grad * d).sum())
        assert abs(adj - fd) <= 1e-5 * abs(fd), (q, adj, fd)
    fdm = (J_oracle(P0, mach + H) - J_oracle(P0, mach - H)) / (2 * H)
    assert abs(dM - fdm) <= 1e-5 * abs(fdm), (dM, fdm)


def test_autograd_function_matches_direct_api():
    import torch
    from mose_b200.adjoint import wall_pressure
    case = channel(seed=6)
    mach = case.extra["mach"]
    s = solver(case)
    P0 = case.prim[0].copy()
    J_direct = objective(s, P0, mach, 12)
    dM_direct = s.adjoint_backward()
    g_direct = interior(s.download_adjoint(1))
    p = torch.tensor(P0, requires_grad=True)
    m = torch.tensor(mach, dtype=torch.float64, requires_grad=True)
    J = wall_pressure(p, m, s, 12, 4, 1, 3)
    J.backward()
    assert J.item() == J_direct
    assert np.array_equal(p.grad.numpy(), g_direct)
    assert float(m.grad) == dM_direct


def test_gradient_perturbed_channel_64():
    """The adjoint configuration's initial state (uniform Mach-0.8 flow with
    a seeded 5 % cell-wise perturbation) on a 64^2 grid, 30 steps.  Over 30
    steps the objective is piecewise smooth at the scale of a 1e-6 step
    (limiter cut-offs where adjacent slopes change sign, HLLC branches), so
    the differences use a 1e-7 step here."""
    case = cases.perturbed_channel(64, steps=30, seed=8)
    mach = case.extra["mach"]
    s = solver(case)
    P0 = case.prim[0].copy()
    n = 30
    objective(s, P0, mach, n)
    dM = s.adjoint_backward()
    grad = interior(s.download_adjoint(1))
    rng = np.random.default_rng(9)
    for q in range(3):
        d = direction(P0.shape, rng)
        h = 0.1 * H
        fd = (objective(s, P0 + h * d, mach, n) - objective(s, P0 - h * d, mach, n)) / (2 * h)
        adj = float((grad * d).sum())
        assert abs(adj - fd) <= 1e-5 * abs(fd), (q, adj, fd)
    fdm = (objective(s, P0, mach + H, n) - objective(s, P0, mach - H, n)) / (2 * H)
    assert abs(dM - fdm) <= 1e-5 * abs(fdm), (dM, fdm)


def test_uniform_state_has_no_gradient_in_v():
    """At v = 0 exactly (every v-slope zero) the one-step map is not
    differentiable in v: central differences converge to the limiter's
    one-sided directional derivative, which is not linear in the direction.
    A ramp in v over five cells gets limited slopes; each of its single-cell
    parts alone does not, so the differences do not add up."""
    case = cases.curvilinear_channel(16, steps=1)
    mach = case.extra["mach"]
    s = solver(case)
    P0 = case.prim[0].copy()
    rng = np.random.default_rng(10)
    lam1 = direction(P0.shape, rng)
    g = lambda P: float((lam1 * step_state(s, P, mach, 1)).sum())
    fd = lambda d: (g(P0 + H * d) - g(P0 - H * d)) / (2 * H)
    ramp, parts = np.zeros(P0.shape), 0.0
    for k in range(5):
        e = np.zeros(P0.shape)
        e[0, 8, 6 + k, 2] = k + 1.0
        ramp += e
        parts += fd(e)
    whole = fd(ramp)
    assert abs(whole - parts) > 1e-3 * abs(whole), (whole, parts)


def test_fp64_precision_adjoint_matches_fd():
    """The adjoint with its forward and segment recompute in the fp64
    precision (every step's dt from the standalone reference-arithmetic pass,
    so the reverse sweep's dt argmin finds the cell that set it): the
    checkpointed gradient against central differences of the same forward."""
    from mose_b200 import _lib
    case = channel(seed=5)
    mach = case.extra["mach"]
    s = solver(case, precision=_lib.PRECISION_FP64)
    P0 = case.prim[0].copy()
    n = 12
    J = objective(s, P0, mach, n)
    dM = s.adjoint_backward()
    grad = interior(s.download_adjoint(1))
    assert np.isfinite(J) and np.isfinite(grad).all()
    rng = np.random.default_rng(6)
    for q in range(3):
        d = direction(P0.shape, rng)
        fd = (objective(s, P0 + H * d, mach, n) - objective(s, P0 - H * d, mach, n)) / (2 * H)
        adj = float((grad * d).sum())
        assert abs(adj - fd) <= 1e-5 * abs(fd), (q, adj, fd)
    fdm = (objective(s, P0, mach + H, n) - objective(s, P0, mach - H, n)) / (2 * H)
    assert abs(dM - fdm) <= 1e-5 * abs(fdm), (dM, fdm)
    # a plain fused step after the adjoint runs from the standalone dt again
    s.upload_prim(1, to_ref_layout(P0))
    s.set_time(0.0, 0)
    s.explicit_step()


def test_perturbed_channel_512_gradient_against_fd():
    """The 512^2 perturbed channel over 200 RK3 steps, checkpoint interval
    14, the wall-pressure objective on face 3.
    For six seeded cell-wise directions the adjoint directional derivative
    meets its central difference at step 1e-6 within 1e-5, or the direction
    crosses a kink: the objective is piecewise smooth (the limiters cut off
    where adjacent slopes change sign, HLLC selects branches), and a kink
    inside [-h, h] shows as a second difference along the direction that
    changes sign across the step, while the difference at step 1e-7 (fewer
    kinks inside) meets the bar.  dJ/dMach against its central difference
    within 1e-6."""
    import math
    from mose_b200 import Solver
    nsteps = 200
    K = int(round(math.sqrt(nsteps)))
    case = cases.perturbed_channel(512, steps=nsteps, seed=0)
    P0 = case.prim[0].copy()
    mach = case.extra["mach"]
    s = Solver(case)

    def J(P, M=mach):
        s.upload_prim(1, to_ref_layout(P))
        s.set_time(0.0, 0)
        s.set_inflow_mach(M)
        return s.adjoint_forward(nsteps, K, 1, 3)

    J(P0)
    dM = s.adjoint_backward()
    g = interior(s.download_adjoint(1))
    rng = np.random.default_rng(11)
    for q in range(6):
        d = direction(P0.shape, rng)
        adj = float((g * d).sum())
        Jp, Jm = J(P0 + H * d), J(P0 - H * d)
        err = abs(adj - (Jp - Jm) / (2 * H)) / abs(adj)
        if err <= 1e-5:
            continue
        J0, Jp2, Jm2 = J(P0), J(P0 + 2 * H * d), J(P0 - 2 * H * d)
        d2 = [Jm2 - 2 * Jm + J0, Jm - 2 * J0 + Jp, J0 - 2 * Jp + Jp2]
        assert min(d2) < 0 < max(d2), (q, err, d2)
        err7 = abs(adj - (J(P0 + 0.1 * H * d) - J(P0 - 0.1 * H * d)) / (0.2 * H)) / abs(adj)
        assert err7 <= 1e-5, (q, err, err7)
    fdm = (J(P0, mach + H) - J(P0, mach - H)) / (2 * H)
    assert abs(dM - fdm) <= 1e-6 * abs(fdm), (dM, fdm)
    s.close()


def perturbed(case, seed):
    rng = np.random.default_rng(seed)
    for p in case.prim:
        p[..., 0] *= 1 + 0.05 * rng.standard_normal(p.shape[:-1])
        p[..., 1] += 0.05 * rng.standard_normal(p.shape[:-1])
        p[..., 2] += 0.05 * rng.standard_normal(p.shape[:-1])
        p[..., 4] *= 1 + 0.05 * rng.standard_normal(p.shape[:-1])
    return case


def euler_shear_layer_2x2(limiter):
    case = cases.shear_layer(12, nbx=2, nby=2, mu=0.0, warp=0.05, seed=3, steps=1, limiter=limiter)
    case.model = 0
    return perturbed(case, 5)


# name: (case, difference step).  Van Leer's limiter has a kink where
# adjacent slopes change sign; on the perturbed 2 x 2 shear layer two of
# three directions straddle one at step 1e-6 (errors 3.9e-4 and 1.4e-5,
# 9e-8 and 1.5e-9 at step 1e-7), so that case runs at 1e-7.
MULTI = {
    # one periodic block: every ghost record a 101 / 201 connection onto the block itself
    "periodic_vortex_16": (lambda: perturbed(cases.isentropic_vortex(16, steps=1), 4), H),
    # 2 x 2 warped blocks: connections between blocks, 301 / 302 slip walls, corners shared by four blocks
    "shear_layer_2x2_blocks_vanalbada": (lambda: euler_shear_layer_2x2("vanalbada"), H),
    "shear_layer_2x2_blocks_vanleer": (lambda: euler_shear_layer_2x2("vanleer"), 0.1 * H),
}


@pytest.mark.parametrize("name", sorted(MULTI))
def test_adjoint_step_connections_and_blocks(name):
    """One step's transpose against central differences on domains whose
    ghost records are block connections (the transposed fill adds the
    ghosts' adjoint into the source cells of the same or another block) and
    whose boundary faces belong to several blocks."""
    from mose_b200 import Solver
    make, h = MULTI[name]
    case = make()
    s = Solver(case)
    nb = len(case.prim)
    P0 = [p.copy() for p in case.prim]
    rng = np.random.default_rng(2)
    lam1 = [direction(p.shape, rng) for p in P0]
    for b in range(nb):
        s.upload_prim(b + 1, to_ref_layout(P0[b]))
        s.upload_adjoint(b + 1, to_ref_layout(lam1[b]))
    s.set_time(0.0, 0)
    s.adjoint_step()
    lam0 = [interior(s.download_adjoint(b + 1)) for b in range(nb)]

    def g(P):
        for b in range(nb):
            s.upload_prim(b + 1, to_ref_layout(P[b]))
        s.set_time(0.0, 0)
        s.explicit_step()
        return sum(float((lam1[b] * interior(s.download_prim(b + 1))).sum()) for b in range(nb))

    for q in range(3):
        d = [direction(p.shape, rng) for p in P0]
        fd = (g([p + h * x for p, x in zip(P0, d)]) - g([p - h * x for p, x in zip(P0, d)])) / (2 * h)
        adj = sum(float((l * x).sum()) for l, x in zip(lam0, d))
        assert abs(adj - fd) <= 1e-5 * abs(fd), (q, adj, fd)
    s.close()
