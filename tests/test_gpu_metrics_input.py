"""Precomputed metrics through mose_gpu_add_block's optional argument (a
block's own Setup_Metrics output, Mod_Metrics.f90:8-107, in the layout the
header documents).  The oracle's metrics handed in unchanged reproduce the
node-derived run bit for bit; perturbed metrics set in the oracle and handed
to the device make both step bit for bit together in the reference-exact
precision, while a device that formed its own metrics from the nodes would
not."""
import numpy as np
import pytest

from mose_b200 import cases
from mose_b200.cases import GC

pytestmark = pytest.mark.gpu


def interior(P):
    return P[GC:-GC, GC:-GC, GC:-GC]


def euler_shear_layer():
    """The warped 2 x 2-block shear layer without the viscous terms: 301 / 302
    faces are then symmetry walls, the wrap in x a 201 connection."""
    case = cases.shear_layer(12, nbx=2, nby=2, mu=0.0, warp=0.05, seed=3, steps=3)
    case.model = 0
    return case


def oracle_metrics(o, b):
    vol, dl, M = o.get_metrics(b)
    return vol, dl, M, [o.get_faces(b, d) for d in (1, 2, 3)]


def perturb(o, nb, seed, eps=1e-3):
    """Scales every metric value of the oracle's blocks by 1 + eps u, u
    uniform in [-1, 1] (face normals keep their direction and length), sets
    them in the oracle and returns the packed arrays for the device."""
    from mose_b200.solver import pack_metrics
    rng = np.random.default_rng(seed)
    packed = []
    for b in range(1, nb + 1):
        vol, dl, M, faces = oracle_metrics(o, b)
        vol = vol * (1 + eps * rng.uniform(-1, 1, vol.shape))
        dl = dl * (1 + eps * rng.uniform(-1, 1, dl.shape))
        M = M * (1 + eps * rng.uniform(-1, 1, M.shape))
        faces = [(N, A * (1 + eps * rng.uniform(-1, 1, A.shape))) for N, A in faces]
        o.set_metrics(b, vol, dl, M)
        for d, (N, A) in enumerate(faces, start=1):
            o.set_faces(b, d, N, A)
        packed.append(pack_metrics(vol, dl, M, faces))
    return packed


CASES = {
    # curvilinear 2-D, symmetry walls, 101 / 201 connections
    "warped_shear_layer_euler": euler_shear_layer,
    # Navier-Stokes on the warped mesh: the metric tensor of interior and first ghost cells
    "warped_shear_layer_viscous": lambda: cases.shear_layer(12, nbx=2, warp=0.06, seed=1, steps=3),
    # 3-D, multi-tile blocks with slip walls (both plane-stage variants)
    "box3d_ywalls": lambda: cases.periodic_box_3d(sizes=[[40, 24], [20], [6, 5]], nb=(2, 1, 2), seed=4, steps=3,
                                                  ywalls=True),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_given_oracle_metrics_match_node_metrics(oracle_mod, name):
    from mose_b200 import Solver
    from mose_b200.solver import pack_metrics
    case = CASES[name]()
    o = oracle_mod.Oracle(case)
    nb = len(case.nodes)
    given = [pack_metrics(*oracle_metrics(o, b)) for b in range(1, nb + 1)]
    s_node = Solver(case)
    s_given = Solver(case, metrics=given)
    assert s_given.uniform_metrics == s_node.uniform_metrics
    for b in range(1, nb + 1):
        for x, y in zip(s_given.download_metrics(b), s_node.download_metrics(b)):
            assert np.array_equal(x, y)
    for _ in range(2):
        assert s_given.explicit_step() == s_node.explicit_step()
    for b in range(1, nb + 1):
        assert np.array_equal(interior(s_given.download_prim(b)), interior(s_node.download_prim(b)))


@pytest.mark.parametrize("name", sorted(CASES))
def test_perturbed_metrics_step_with_the_oracle(oracle_mod, name):
    from mose_b200 import Solver
    case = CASES[name]()
    nb = len(case.nodes)
    o = oracle_mod.Oracle(case)
    given = perturb(o, nb, seed=7)
    s = Solver(case, metrics=given)
    assert not s.uniform_metrics
    s_node = Solver(case)
    for _ in range(3):
        dto, to = o.step()
        dtg, tg = s.explicit_step()
        assert dtg == dto and tg == to
        s_node.explicit_step()
    vs = (0, 1, 2, 3, 4) if case.nodes[0].shape[0] > 2 else (0, 1, 2, 4)
    differs = False
    for b in range(1, nb + 1):
        g, r = interior(s.download_prim(b))[..., vs], interior(o.get_prim(b))[..., vs]
        assert np.array_equal(g, r), f"block {b}: max |diff| {np.abs(g - r).max()}"
        differs |= not np.array_equal(interior(s_node.download_prim(b))[..., vs], r)
    assert differs, "the node-derived run should differ from the perturbed-metric run"


def test_metrics_of_the_wrong_size_are_refused():
    from mose_b200 import Solver
    case = cases.isentropic_vortex(16, steps=1)
    with pytest.raises(ValueError):
        Solver(case, metrics=[np.zeros(10)])
