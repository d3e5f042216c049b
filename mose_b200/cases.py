"""Synthetic multi-block cases in the reference's data formats.

A case is the data MOSE reads at setup: block node arrays (MESH/*.tec),
the face-by-face boundary list (INPUT/bc.txt) and an initial state
(INPUT/ic.tec), plus the numerics of input.ini.  Arrays use the
reference's Fortran layouts, expressed as C-contiguous numpy arrays with the
fastest Fortran index last:

  nodes[b] : (nk+1, nj+1, ni+1, 3)  == Fortran node(3, 0:ni, 0:nj, 0:nk)
  prim[b]  : (nk,   nj,   ni,   5)  == interior P(5, 1:ni, 1:nj, 1:nk)
  bc_rec   : (nbound, 15) int32     == b i j k f type bs is js ks fs d11 d12 d21 d22
  bc_data  : (nbound, 6)  float64   == 401: T0 p0 alpha beta rel_fac ; 403 / 404: T0 / T g alpha beta
                                      rel_fac ; 405: mach T p alpha beta rel_fac ; 406: p_back rel_fac ;
                                      407: T0 p0 p_back alpha beta rel_fac

The five benchmark configurations are built from seeded synthetic inputs of
the shapes the reference problem statement names; no external dataset is used.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

GC = 2
NPRIM = 5

# limiter / riemann names as in input.ini (Register_Numerics.f90:57-72)
LIMITERS = {"first-order": 0, "none": 0, "minmod": 1, "vanleer": 2, "vanalbada": 3, "mc": 4, "superbee": 5}
RIEMANN = {"HLLC": 0, "AUSM+": 1, "SLAU": 2, "SLAU2": 3, "HLLE": 4, "HLLEM": 5, "LLF": 6, "Rusanov": 6,
           "PLLF": 7, "Hanel": 8, "AUSM+-up": 9, "AUSM+-up2": 10, "HLLC+": 11, "HLLE++": 12,
           "HLLC Rotated": 13, "exact": 14, "Exact": 14}


@dataclass
class Case:
    name: str
    nodes: list
    bc_rec: np.ndarray
    bc_data: np.ndarray
    prim: list
    n_rk: int = 3
    cfl: float = 0.5
    time_accurate: bool = True
    limiter: str = "minmod"
    riemann: str = "HLLC"
    minf: float = 0.0          # riemann-options-Minf (AUSM+-up, AUSM+-up2)
    irs_beta: float = 0.0      # irs-beta: implicit residual smoothing when > 0
    sd_limiter: bool = False   # space-reconstruction MUSCL-SD (shock-detector scaled slopes)
    ramp_iter: int = 0         # cfl-rise-threshold: CFL ramped over the first iterations
    integration: str = "cons"  # integration-variables: 'cons' or 'prim' (primitive RK update)
    model: int = 0             # 0: Euler, 1: laminar Navier-Stokes
    mu: float = 0.0            # laminar viscosity (constant transport properties)
    kappa: float = 0.0         # laminar conductivity
    vnn: float = 0.5           # von Neumann number of the viscous time-step limit
    gamma: float = 1.4
    rgas: float = 1.0
    steps: int = 1
    t_end: float | None = None
    # time tables of 402 inlets: (time, value, periodic) each; a 402 record
    # holds its table's index as its second datum
    series: list = field(default_factory=list)
    extra: dict = field(default_factory=dict)

    @property
    def dims(self):
        return [(n.shape[2] - 1, n.shape[1] - 1, n.shape[0] - 1) for n in self.nodes]

    @property
    def ncells(self) -> int:
        return int(sum(ni * nj * nk for ni, nj, nk in self.dims))


def to_ref_layout(prim: np.ndarray) -> np.ndarray:
    """Interior (nk,nj,ni,5) -> ghosted reference layout (nk+4,nj+4,ni+4,5), ghosts 0."""
    nk, nj, ni, nv = prim.shape
    out = np.zeros((nk + 2 * GC, nj + 2 * GC, ni + 2 * GC, nv), dtype=np.float64)
    out[GC:GC + nk, GC:GC + nj, GC:GC + ni, :] = prim
    return out


def interior(ref: np.ndarray) -> np.ndarray:
    """Ghosted reference layout -> interior view."""
    return ref[GC:-GC, GC:-GC, GC:-GC, :]


def cartesian_nodes(ni: int, nj: int, nk: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0),
                    offs=(0, 0, 0), ntot=None) -> np.ndarray:
    """Uniform Cartesian nodes.  Coordinates are lo + (hi-lo)*(offs+i)/ntot so that
    neighbouring blocks of a global grid share node coordinates bit for bit."""
    ntot = ntot or (ni, nj, nk)
    axes = []
    for n, a, b, o, t in zip((ni, nj, nk), lo, hi, offs, ntot):
        idx = np.arange(n + 1, dtype=np.float64) + o
        axes.append(a + (b - a) * idx / t)
    z, y, x = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    return np.ascontiguousarray(np.stack([x, y, z], axis=-1))


def _face_cells(ni, nj, nk, f):
    """(i, j, k) 1-based of the cells of face f, in file order (k, j, i loops)."""
    if f in (1, 2):
        i = 1 if f == 1 else ni
        return [(i, j, k) for k in range(1, nk + 1) for j in range(1, nj + 1)]
    if f in (3, 4):
        j = 1 if f == 3 else nj
        return [(i, j, k) for k in range(1, nk + 1) for i in range(1, ni + 1)]
    k = 1 if f == 5 else nk
    return [(i, j, k) for j in range(1, nj + 1) for i in range(1, ni + 1)]


def _face_cells_np(ni, nj, nk, f):
    """(n, 3) int array of the 1-based (i, j, k) of face f's cells, in file
    order (k, j, i loops, the last index fastest as _face_cells lists them)."""
    if f in (1, 2):
        k, j = np.meshgrid(np.arange(1, nk + 1), np.arange(1, nj + 1), indexing="ij")
        i = np.full_like(k, 1 if f == 1 else ni)
    elif f in (3, 4):
        k, i = np.meshgrid(np.arange(1, nk + 1), np.arange(1, ni + 1), indexing="ij")
        j = np.full_like(k, 1 if f == 3 else nj)
    else:
        j, i = np.meshgrid(np.arange(1, nj + 1), np.arange(1, ni + 1), indexing="ij")
        k = np.full_like(j, 1 if f == 5 else nk)
    return np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)


def build_bcs(dims, face_spec):
    """Boundary records in bc.txt order.

    face_spec(b, f) -> ("bc", type, data6) | ("conn", type, bs, fs) with 1-based
    blocks.  Connections map face cells with identity orientation
    (d11=1, d12=0, d21=0, d22=1) onto the matching cell of the source face.
    """
    recs, data = [], []
    for b, (ni, nj, nk) in enumerate(dims, start=1):
        for f in range(1, 7):
            spec = face_spec(b, f)
            ijk = _face_cells_np(ni, nj, nk, f)
            r = np.zeros((len(ijk), 15), dtype=np.int32)
            r[:, 0] = b
            r[:, 1:4] = ijk
            r[:, 4] = f
            r[:, 5] = spec[1]
            dd = np.zeros((len(ijk), 6))
            if spec[0] == "bc":
                dd[:] = np.asarray(spec[2], dtype=np.float64)
            else:
                _, t, bs, fs = spec
                sni, snj, snk = dims[bs - 1]
                src = ijk.copy()
                if fs in (1, 2):
                    src[:, 0] = 1 if fs == 1 else sni
                elif fs in (3, 4):
                    src[:, 1] = 1 if fs == 3 else snj
                else:
                    src[:, 2] = 1 if fs == 5 else snk
                r[:, 6] = bs
                r[:, 7:10] = src
                r[:, 10] = fs
                r[:, 11] = 1
                r[:, 14] = 1
            recs.append(r)
            data.append(dd)
    return np.concatenate(recs, axis=0), np.concatenate(data, axis=0)


def cell_centres(nodes: np.ndarray):
    """Cell centres (nk,nj,ni,3) as the mean of the 8 corner nodes."""
    n = nodes
    c = (n[:-1, :-1, :-1] + n[:-1, :-1, 1:] + n[:-1, 1:, :-1] + n[:-1, 1:, 1:] +
         n[1:, :-1, :-1] + n[1:, :-1, 1:] + n[1:, 1:, :-1] + n[1:, 1:, 1:]) / 8.0
    return c


# ---------------------------------------------------------------------------
# The five benchmark configurations
# ---------------------------------------------------------------------------
def sod(ncell: int = 1000, limiter="minmod", riemann="HLLC", cfl=0.5, t_end=0.2) -> Case:
    """1-D Sod shock tube on [0,1], diaphragm at 0.5, transmissive (400) ends."""
    nodes = cartesian_nodes(ncell, 1, 1, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    xc = cell_centres(nodes)[..., 0]
    prim = np.zeros((1, 1, ncell, NPRIM))
    left = xc < 0.5
    prim[..., 0] = np.where(left, 1.0, 0.125)
    prim[..., 4] = np.where(left, 1.0, 0.1)
    spec = lambda b, f: ("bc", 400 if f <= 4 else 0, [0.0] * 6)
    rec, data = build_bcs([(ncell, 1, 1)], spec)
    return Case("sod1d", [nodes], rec, data, [prim], n_rk=3, cfl=cfl, time_accurate=True,
                limiter=limiter, riemann=riemann, gamma=1.4, rgas=1.0, t_end=t_end)


def isentropic_vortex(n: int = 2048, steps: int = 100, limiter="vanalbada", riemann="HLLC",
                      cfl=0.8, L=10.0, strength=5.0, mach=0.5, gamma=1.4) -> Case:
    """2-D isentropic vortex (strength 5, core radius 1) on a periodic [0,L]^2 block,
    free stream rho = p = 1, Mach 0.5 at 45 degrees.  Periodic seams are 201
    (connection with extrapolated ghost metrics)."""
    nodes = cartesian_nodes(n, n, 1, (0.0, 0.0, 0.0), (L, L, 1.0))
    c = cell_centres(nodes)
    x, y = c[..., 0], c[..., 1]
    xc = yc = L / 2
    r2 = (x - xc) ** 2 + (y - yc) ** 2
    ainf = np.sqrt(gamma)
    uinf = vinf = mach * ainf / np.sqrt(2.0)
    f = np.exp(0.5 * (1.0 - r2))
    du = -strength / (2 * np.pi) * f * (y - yc)
    dv = strength / (2 * np.pi) * f * (x - xc)
    T = 1.0 - (gamma - 1.0) * strength ** 2 / (8.0 * gamma * np.pi ** 2) * np.exp(1.0 - r2)
    rho = T ** (1.0 / (gamma - 1.0))
    prim = np.zeros((1, n, n, NPRIM))
    prim[..., 0] = rho
    prim[..., 1] = uinf + du
    prim[..., 2] = vinf + dv
    prim[..., 4] = rho ** gamma

    def spec(b, f):
        if f >= 5:
            return ("bc", 0, [0.0] * 6)
        return ("conn", 201, 1, {1: 2, 2: 1, 3: 4, 4: 3}[f])

    rec, data = build_bcs([(n, n, 1)], spec)
    return Case("vortex2d", [nodes], rec, data, [prim], n_rk=3, cfl=cfl, time_accurate=True,
                limiter=limiter, riemann=riemann, gamma=gamma, rgas=1.0, steps=steps)


def four_quadrant(seed: int = 0, nbx: int = 8, nby: int = 8, nmin: int = 64, nmax: int = 1024,
                  steps: int = 100, limiter="minmod", riemann="AUSM+", cfl=0.5, gamma=1.4,
                  split=(0.5, 0.5)) -> Case:
    """2-D four-quadrant Riemann problem on [0,1]^2 split into nbx x nby blocks
    whose column widths / row heights are drawn from default_rng(seed) in
    [nmin, nmax]; conforming 101 interfaces, transmissive (400) outer faces."""
    rng = np.random.default_rng(seed)
    nx = rng.integers(nmin, nmax + 1, size=nbx)
    ny = rng.integers(nmin, nmax + 1, size=nby)
    Nx, Ny = int(nx.sum()), int(ny.sum())
    ox = np.concatenate([[0], np.cumsum(nx)[:-1]])
    oy = np.concatenate([[0], np.cumsum(ny)[:-1]])
    nodes, prims, dims = [], [], []
    quad = {  # (rho, u, v, p)
        "NE": (1.5, 0.0, 0.0, 1.5), "NW": (0.5323, 1.206, 0.0, 0.3),
        "SW": (0.138, 1.206, 1.206, 0.029), "SE": (0.5323, 0.0, 1.206, 0.3)}
    for by in range(nby):
        for bx in range(nbx):
            ni, nj = int(nx[bx]), int(ny[by])
            nd = cartesian_nodes(ni, nj, 1, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0),
                                 offs=(int(ox[bx]), int(oy[by]), 0), ntot=(Nx, Ny, 1))
            c = cell_centres(nd)
            east, north = c[..., 0] > split[0], c[..., 1] > split[1]
            p = np.zeros((1, nj, ni, NPRIM))
            for key, mask in (("NE", east & north), ("NW", ~east & north),
                              ("SW", ~east & ~north), ("SE", east & ~north)):
                r, u, v, pr = quad[key]
                p[..., 0][mask] = r
                p[..., 1][mask] = u
                p[..., 2][mask] = v
                p[..., 4][mask] = pr
            nodes.append(nd)
            prims.append(p)
            dims.append((ni, nj, 1))

    def spec(b, f):
        bx, by = (b - 1) % nbx, (b - 1) // nbx
        if f >= 5:
            return ("bc", 0, [0.0] * 6)
        nb = {1: (bx - 1, by, 2), 2: (bx + 1, by, 1), 3: (bx, by - 1, 4), 4: (bx, by + 1, 3)}[f]
        if 0 <= nb[0] < nbx and 0 <= nb[1] < nby:
            return ("conn", 101, nb[1] * nbx + nb[0] + 1, nb[2])
        return ("bc", 400, [0.0] * 6)

    rec, data = build_bcs(dims, spec)
    return Case("quadrant2d", nodes, rec, data, prims, n_rk=3, cfl=cfl, time_accurate=True,
                limiter=limiter, riemann=riemann, gamma=gamma, rgas=1.0, steps=steps,
                extra={"nx": nx.tolist(), "ny": ny.tolist(), "seed": seed, "split": split})


def curvilinear_channel(n: int = 512, steps: int = 200, mach: float = 0.8, amp: float = 0.05,
                        limiter="vanalbada", riemann="HLLC", cfl=0.5, gamma=1.4) -> Case:
    """2-D curvilinear block x = xi + a sin(2 pi eta), y = eta + a sin(2 pi xi) on
    [0,1]^2; uniform Mach 0.8 flow, supersonic-static inflow (405) on the left,
    outflow (406) at the free-stream pressure on the right, slip walls (300)."""
    xi = np.arange(n + 1, dtype=np.float64) / n
    eta = np.arange(n + 1, dtype=np.float64) / n
    E, X = np.meshgrid(eta, xi, indexing="ij")
    x = X + amp * np.sin(2 * np.pi * E)
    y = E + amp * np.sin(2 * np.pi * X)
    nodes = np.zeros((2, n + 1, n + 1, 3))
    for k in range(2):
        nodes[k, ..., 0] = x
        nodes[k, ..., 1] = y
        nodes[k, ..., 2] = float(k)
    p_inf = 1.0 / gamma
    prim = np.zeros((1, n, n, NPRIM))
    prim[..., 0] = 1.0
    prim[..., 1] = mach
    prim[..., 4] = p_inf
    T_inf = p_inf / 1.0

    def spec(b, f):
        if f == 1:
            return ("bc", 405, [mach, T_inf, p_inf, 0.0, 0.0, 1.0])
        if f == 2:
            return ("bc", 406, [p_inf, 1.0, 0.0, 0.0, 0.0, 0.0])
        if f in (3, 4):
            return ("bc", 300, [0.0] * 6)
        return ("bc", 0, [0.0] * 6)

    rec, data = build_bcs([(n, n, 1)], spec)
    return Case("channel2d", [nodes], rec, data, [prim], n_rk=3, cfl=cfl, time_accurate=True,
                limiter=limiter, riemann=riemann, gamma=gamma, rgas=1.0, steps=steps,
                extra={"mach": mach})


def perturbed_channel(n: int = 512, steps: int = 200, amp: float = 0.05, seed: int = 0, **kw) -> Case:
    """The curvilinear channel with its uniform Mach-0.8 state carrying seeded
    cell-wise perturbations: relative amplitude `amp` on rho, u and p, and
    v = amp * Mach * N(0, 1).  The wall-pressure objective has no gradient at
    the exactly uniform state: every limited slope is zero there, and the
    limiters (homogeneous of degree 1) have one-sided directional derivatives
    that are not linear in the direction.  The perturbation also breaks the
    ties of the CFL minimum."""
    case = curvilinear_channel(n, steps=steps, **kw)
    rng = np.random.default_rng(seed)
    p = case.prim[0]
    shape = p.shape[:-1]
    for v in (0, 1, 4):
        p[..., v] *= 1 + amp * rng.standard_normal(shape)
    p[..., 2] = amp * case.extra["mach"] * rng.standard_normal(shape)
    return case


def periodic_box_3d(n: int = 128, nb=(2, 2, 2), sizes=None, steps: int = 50, seed: int = 0,
                    limiter="vanleer", riemann="HLLC", cfl=0.3, gamma=1.4, mach=0.3, amp=1e-2,
                    nmodes: int = 16, kmax: int = 8, ywalls: bool = False) -> Case:
    """3-D periodic box [0,1]^3 of nb[0] x nb[1] x nb[2] blocks (n^3 cells each, or
    per-direction block sizes `sizes`), uniform state rho = 1, p = 1/gamma
    (sound speed 1), Mach 0.3 along x, plus `nmodes` seeded Fourier modes with
    integer wavevectors of norm in [1, kmax] and random phases on rho, u, v, w,
    their sum scaled to amplitude `amp`.  Block interfaces are 101 connections,
    the periodic wrap is 201 (connection with extrapolated ghost metrics).
    ywalls: the domain's y ends (faces 3 and 4) are 300 slip walls instead.
    [0,1] with a power-of-two cell count gives dyadic, exactly uniform metrics."""
    rng = np.random.default_rng(seed)
    sizes = sizes or [[n] * nb[0], [n] * nb[1], [n] * nb[2]]
    N = [int(sum(s)) for s in sizes]
    offs = [np.concatenate([[0], np.cumsum(s)[:-1]]).astype(int) for s in sizes]
    modes = []
    while len(modes) < nmodes:
        kv = rng.integers(-kmax, kmax + 1, size=3)
        kn = float(np.sqrt((kv ** 2).sum()))
        if 1.0 <= kn <= kmax:
            modes.append((kv.astype(np.float64), rng.uniform(0.0, 2.0 * np.pi, size=4)))
    nodes, prims, dims, index = [], [], [], {}
    for bz in range(nb[2]):
        for by in range(nb[1]):
            for bx in range(nb[0]):
                ni, nj, nk = int(sizes[0][bx]), int(sizes[1][by]), int(sizes[2][bz])
                nd = cartesian_nodes(ni, nj, nk, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0),
                                     offs=(int(offs[0][bx]), int(offs[1][by]), int(offs[2][bz])), ntot=tuple(N))
                c = cell_centres(nd)
                pert = np.zeros(c.shape[:-1] + (4,))
                for kv, ph in modes:
                    arg = 2.0 * np.pi * (c[..., 0] * kv[0] + c[..., 1] * kv[1] + c[..., 2] * kv[2])
                    for q in range(4):
                        pert[..., q] += np.cos(arg + ph[q])
                pert *= amp / nmodes
                p = np.zeros((nk, nj, ni, NPRIM))
                p[..., 0] = 1.0 + pert[..., 0]
                p[..., 1] = mach + pert[..., 1]
                p[..., 2] = pert[..., 2]
                p[..., 3] = pert[..., 3]
                p[..., 4] = 1.0 / gamma
                index[(bx, by, bz)] = len(nodes) + 1
                nodes.append(nd)
                prims.append(p)
                dims.append((ni, nj, nk))

    def spec(b, f):
        key = [k for k, v in index.items() if v == b][0]
        d = (f - 1) // 2
        step = -1 if f % 2 == 1 else 1
        nbk = list(key)
        nbk[d] += step
        wrap = not (0 <= nbk[d] < nb[d])
        if wrap and ywalls and d == 1:
            return ("bc", 300, [0.0] * 6)
        nbk[d] %= nb[d]
        fs = f + 1 if f % 2 == 1 else f - 1
        return ("conn", 201 if wrap else 101, index[tuple(nbk)], fs)

    rec, data = build_bcs(dims, spec)
    return Case("box3d", nodes, rec, data, prims, n_rk=3, cfl=cfl, time_accurate=True,
                limiter=limiter, riemann=riemann, gamma=gamma, rgas=1.0, steps=steps,
                extra={"sizes": sizes, "seed": seed, "amp": amp, "nmodes": nmodes})


def channel_3d(n: int = 16, steps: int = 10, mach: float = 0.8, amp: float = 0.04,
               limiter="vanalbada", riemann="HLLC", cfl=0.3, gamma=1.4) -> Case:
    """3-D curvilinear channel block on [0,1]^3 (x = xi + a sin(2 pi eta),
    y = eta + a sin(2 pi zeta), z = zeta + a sin(2 pi xi)): supersonic-static
    inflow (405) on face 1, outflow (406) on face 2, slip walls (300) on
    faces 3-4, extrapolation (400) on faces 5-6; uniform Mach-0.8 state."""
    t = np.arange(n + 1, dtype=np.float64) / n
    Z, E, X = np.meshgrid(t, t, t, indexing="ij")
    nodes = np.stack([X + amp * np.sin(2 * np.pi * E), E + amp * np.sin(2 * np.pi * Z),
                      Z + amp * np.sin(2 * np.pi * X)], axis=-1)
    p_inf = 1.0 / gamma
    prim = np.zeros((n, n, n, NPRIM))
    prim[..., 0] = 1.0
    prim[..., 1] = mach
    prim[..., 4] = p_inf

    def spec(b, f):
        if f == 1:
            return ("bc", 405, [mach, p_inf, p_inf, 0.0, 0.0, 1.0])
        if f == 2:
            return ("bc", 406, [p_inf, 1.0, 0.0, 0.0, 0.0, 0.0])
        if f in (3, 4):
            return ("bc", 300, [0.0] * 6)
        return ("bc", 400, [0.0] * 6)

    rec, data = build_bcs([(n, n, n)], spec)
    return Case("channel3d", [np.ascontiguousarray(nodes)], rec, data, [prim], n_rk=3, cfl=cfl,
                time_accurate=True, limiter=limiter, riemann=riemann, gamma=gamma, rgas=1.0, steps=steps,
                extra={"mach": mach})


def shear_layer(n: int = 64, nbx: int = 1, nby: int = 1, steps: int = 10, mu: float = 0.01, prandtl: float = 0.72,
                u0: float = 0.5, amp: float = 0.02, seed: int = 0, tw: float | None = None, top: str = "adiabatic",
                warp: float = 0.0, limiter="vanleer", riemann="HLLC", cfl=0.5, vnn=0.5, gamma=1.4) -> Case:
    """2-D laminar Navier-Stokes channel on [0, 2] x [0, 1]: a shear layer
    u = u0 sin(pi y) between walls, periodic in x, decaying by viscosity;
    rho = 1, p = 1/gamma (sound speed 1) plus seeded cell-wise perturbations
    of relative amplitude `amp` on rho, u, v and p so every gradient term is
    exercised.  Bottom wall (face 3 of the bottom blocks): 302 at temperature
    `tw` (default: the free-stream temperature); top: 301 adiabatic (qw = 0),
    or 300 symmetry with top='symmetry'.  nbx x nby blocks of 2n x n cells
    (101 interfaces, the periodic wrap in x is 201); constant transport
    properties mu and kappa = mu cp / Pr.  warp > 0 moves the nodes to
    y = eta + warp sin(pi xi) sin(pi eta) (walls stay flat, the wrap stays
    periodic), so the metric tensor has off-diagonal terms."""
    rng = np.random.default_rng(seed)
    Nx, Ny = 2 * n * nbx, n * nby
    rgas = 1.0
    p_inf = 1.0 / gamma
    T_inf = p_inf / (1.0 * rgas)
    tw = T_inf if tw is None else tw
    cp = gamma * rgas / (gamma - 1.0)
    nodes, prims, dims = [], [], []
    for by in range(nby):
        for bx in range(nbx):
            ni, nj = 2 * n, n
            nd = cartesian_nodes(ni, nj, 1, (0.0, 0.0, 0.0), (2.0, 1.0, 1.0), offs=(ni * bx, nj * by, 0),
                                 ntot=(Nx, Ny, 1))
            if warp:
                nd[..., 1] = nd[..., 1] + warp * np.sin(np.pi * nd[..., 0]) * np.sin(np.pi * nd[..., 1])
            c = cell_centres(nd)
            p = np.zeros((1, nj, ni, NPRIM))
            shape = p.shape[:-1]
            p[..., 0] = 1.0 * (1 + amp * rng.standard_normal(shape))
            p[..., 1] = u0 * np.sin(np.pi * c[..., 1]) * (1 + amp * rng.standard_normal(shape))
            p[..., 2] = amp * u0 * rng.standard_normal(shape)
            p[..., 4] = p_inf * (1 + amp * rng.standard_normal(shape))
            nodes.append(nd)
            prims.append(p)
            dims.append((ni, nj, 1))

    def spec(b, f):
        bx, by = (b - 1) % nbx, (b - 1) // nbx
        if f >= 5:
            return ("bc", 0, [0.0] * 6)
        if f in (1, 2):   # x: neighbours, the wrap is periodic (201)
            nbx_ = (bx - 1) % nbx if f == 1 else (bx + 1) % nbx
            wrap = (f == 1 and bx == 0) or (f == 2 and bx == nbx - 1)
            return ("conn", 201 if wrap else 101, by * nbx + nbx_ + 1, 2 if f == 1 else 1)
        if f == 3 and by > 0:
            return ("conn", 101, (by - 1) * nbx + bx + 1, 4)
        if f == 4 and by < nby - 1:
            return ("conn", 101, (by + 1) * nbx + bx + 1, 3)
        if f == 3:
            return ("bc", 302, [tw, 0.0, 0.0, 0.0, 0.0, 0.0])
        return ("bc", 300, [0.0] * 6) if top == "symmetry" else ("bc", 301, [0.0] * 6)

    rec, data = build_bcs(dims, spec)
    return Case("shear2d", nodes, rec, data, prims, n_rk=3, cfl=cfl, time_accurate=True, limiter=limiter,
                riemann=riemann, gamma=gamma, rgas=rgas, steps=steps, model=1, mu=mu, kappa=mu * cp / prandtl,
                vnn=vnn, extra={"u0": u0, "tw": tw})
