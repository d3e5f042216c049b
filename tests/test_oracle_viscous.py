"""The oracle's Navier-Stokes terms (model = 1, laminar; Lib_Diffusive.f90 and
the viscous boundary fluxes) on CPU: the inviscid limit reproduces the Euler
oracle bit for bit, mass is conserved between walls, and a low-Mach shear
layer between no-slip walls decays at the viscous rate exp(-nu pi^2 t)."""
import numpy as np

from mose_b200 import cases
from mose_b200.cases import GC


def interior(P):
    return P[GC:-GC, GC:-GC, GC:-GC]


def test_zero_viscosity_is_the_euler_path(oracle_mod):
    """mu = kappa = 0: every diffusive flux is an exact zero and the VNN limit
    infinite; 301 / 302 walls keep their Euler part (the symmetry flux, with
    extrapolated ghosts), so the states match the Euler oracle (model 0, the
    same records) bit for bit."""
    visc = cases.shear_layer(12, nbx=2, nby=2, mu=0.0, warp=0.05, seed=3)
    visc.kappa = 0.0
    euler = cases.shear_layer(12, nbx=2, nby=2, mu=0.0, warp=0.05, seed=3)
    euler.model = 0
    ov, oe = oracle_mod.Oracle(visc), oracle_mod.Oracle(euler)
    for _ in range(4):
        assert ov.step() == oe.step()
    for b in range(1, 5):
        assert np.array_equal(interior(ov.get_prim(b)), interior(oe.get_prim(b)))


def test_mass_is_conserved_between_walls(oracle_mod):
    """Walls carry no mass flux and the species diffusion of one species is an
    exact zero.  On a uniform grid the two sides of every connection form the
    same face flux (on a warped one the 201 wrap's extrapolated ghost metrics
    make them differ, as in the reference)."""
    case = cases.shear_layer(16, nbx=2, nby=1, mu=0.02, seed=1)
    o = oracle_mod.Oracle(case)

    def mass():
        tot = 0.0
        for b in range(1, 3):
            vol, _, _ = o.get_metrics(b)
            tot += float((interior(o.get_prim(b))[..., 0] * vol[GC:-GC, GC:-GC, GC:-GC]).sum())
        return tot

    m0 = mass()
    for _ in range(20):
        o.step()
    assert abs(mass() - m0) <= 1e-13 * m0


def test_shear_layer_decays_at_the_viscous_rate(oracle_mod):
    """u = u0 sin(pi y) between no-slip walls, Mach 0.02: the mode's
    amplitude decays as exp(-nu pi^2 t), nu = mu / rho (within 1.5 %)."""
    mu, u0 = 0.005, 0.02
    case = cases.shear_layer(32, mu=mu, u0=u0, amp=0.0, cfl=0.5)
    o = oracle_mod.Oracle(case)
    y = cases.cell_centres(case.nodes[0])[0, :, 0, 1]
    shape = np.sin(np.pi * y)

    def amplitude():
        u = interior(o.get_prim(1))[0, :, :, 1].mean(axis=1)
        return float((u * shape).sum() / (shape * shape).sum())

    a0 = amplitude()
    t = 0.0
    while t < 4.0:
        _, t = o.step()
    expect = a0 * np.exp(-mu * np.pi ** 2 * t)
    assert abs(amplitude() - expect) <= 0.015 * expect, (amplitude(), expect)
