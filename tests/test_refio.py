"""Readers of MOSE's input files (mose_b200.refio): round trips through
files written in the reference's formats (Tecplot ASCII BLOCK zones,
bc.txt two-line records, input.ini), and, where the reference tree is
present, its own Sod79 and Ein91 inputs against the committed fixtures."""
import os
from pathlib import Path

import numpy as np
import pytest

from mose_b200 import cases, refio

GOLDEN = Path(__file__).resolve().parent / "golden"
# the reference's own test inputs, when MOSE_SOURCE_DIR names a MOSE source tree
REF = Path(os.environ.get("MOSE_SOURCE_DIR", "/nonexistent")) / "test"


def write_tecplot(path, zones, names, ncell_vars=0):
    """zones: list of (nodal arrays list, cell arrays list) in (K, J, I) order."""
    with open(path, "w") as f:
        f.write(" VARIABLES = " + " ".join(f'"{n}"' for n in names) + "\n")
        for b, (nod, cel) in enumerate(zones, start=1):
            K, J, I = nod[0].shape
            loc = f", VARLOCATION=([1-3]=NODAL,[4-{3 + len(cel)}]=CELLCENTERED)" if cel else ""
            f.write(f' ZONE T="BLOCK {b}"\n I={I}, J={J}, K={K}, ZONETYPE=Ordered\n DATAPACKING=BLOCK{loc}\n')
            for a in list(nod) + list(cel):
                for v in a.ravel():
                    f.write(f"{float(v)!r}\n")


def write_bc(path, rec, data):
    with open(path, "w") as f:
        for r, d in zip(rec, data):
            f.write(" ".join(f"{x:7d}" for x in r[:6]) + "\n")
            t = r[5]
            if t in (101, 201):
                f.write(" ".join(f"{x:7d}" for x in r[6:15]) + "\n")
            elif t == 405:
                f.write(f"{float(d[0])!r}, {float(d[1])!r}, {float(d[2])!r}, normal, {float(d[4])!r}, {float(d[5])!r}, 1.0,\n")
            elif t == 406:
                f.write(f"{float(d[0])!r}, {float(d[1])!r}\n")


def test_round_trip_two_blocks(tmp_path):
    case = cases.curvilinear_channel(12, steps=1)
    # a second block joined on face 2 <-> face 1 (connection records with data lines)
    nodes2 = case.nodes[0].copy()
    nodes2[..., 0] += 1.0
    rec, data = cases.build_bcs([(12, 12, 1), (12, 12, 1)], lambda b, f: (
        ("conn", 101, 2, 1) if (b, f) == (1, 2) else ("conn", 101, 1, 2) if (b, f) == (2, 1) else
        ("bc", 405, [0.8, 0.7, 1 / 1.4, 0.0, 0.0, 1.0]) if f == 1 else
        ("bc", 406, [1 / 1.4, 1.0, 0, 0, 0, 0]) if f == 2 else
        ("bc", 300, [0.0] * 6) if f in (3, 4) else ("bc", 0, [0.0] * 6)))
    d = tmp_path / "case"
    (d / "MESH").mkdir(parents=True)
    (d / "INPUT").mkdir()
    write_tecplot(d / "MESH" / "mesh.tec",
                  [([n[..., 0], n[..., 1], n[..., 2]], []) for n in (case.nodes[0], nodes2)], ["X", "Y", "Z"])
    prims = [case.prim[0], case.prim[0] * 1.01]
    write_tecplot(d / "INPUT" / "ic.tec",
                  [([n[..., 0], n[..., 1], n[..., 2]], [p[..., v] for v in range(5)])
                   for n, p in zip((case.nodes[0], nodes2), prims)], ["x", "y", "z", "rho1", "u", "v", "w", "p"])
    write_bc(d / "INPUT" / "bc.txt", rec, data)
    (d / "input.ini").write_text("[MOSE-Parameters]\ntime-threshold = 0.25\n\n[MOSE-Numerics]\ncfl = 0.7\n"
                                 "time-accurate = true\ntime-scheme = RK2\nriemann-solver = AUSM+-up\n"
                                 "riemann-options-Minf = 0.5\nspace-reconstruction = MUSCL\n"
                                 "flux-limiter = vanalbada   ; comment\n")
    c = refio.load_case(d, gamma=1.4, rgas=1.0)
    assert c.dims == [(12, 12, 1), (12, 12, 1)]
    assert all(np.array_equal(a, b) for a, b in zip(c.nodes, (case.nodes[0], nodes2)))
    assert all(np.array_equal(a, b) for a, b in zip(c.prim, prims))
    assert np.array_equal(c.bc_rec, rec)
    want = data.copy()
    want[rec[:, 5] == 405, 3] = np.finfo(np.float64).max      # 'normal' direction sentinel
    assert np.array_equal(c.bc_data, want)
    assert (c.cfl, c.n_rk, c.time_accurate, c.riemann, c.minf, c.limiter, c.t_end) == \
        (0.7, 2, True, "AUSM+-up", 0.5, "vanalbada", 0.25)
    assert c.extra["unsupported"] == []


def test_sd_and_irs_numerics_read(tmp_path):
    ini = tmp_path / "input.ini"
    ini.write_text("[MOSE-Numerics]\nspace-reconstruction = MUSCL-SD\nirs-beta = 0.5\nflux-limiter = mc\n")
    kw = refio.read_input_ini(ini)
    assert kw["unsupported"] == [] and kw["irs_beta"] == 0.5 and kw["sd_limiter"]


@pytest.mark.skipif(not REF.exists(), reason="MOSE_SOURCE_DIR does not name a MOSE source tree")
@pytest.mark.parametrize("name,res,fixture", [("1D/Sod79", "x4", "sod79_x4.npz"), ("1D/Ein91", "x8", "ein91_x8.npz")])
def test_reference_inputs_match_fixtures(name, res, fixture):
    """The readers give, from the reference's own files, exactly the arrays
    the committed fixtures hold (which the oracle and GPU tests run)."""
    c = refio.load_case(REF / name, res)
    d = np.load(GOLDEN / fixture)
    assert np.array_equal(c.nodes[0], d["nodes"])
    assert np.array_equal(c.prim[0], d["prim"])
    assert np.array_equal(c.bc_rec, d["bc_rec"])
    assert c.cfl == float(d["cfl"]) and c.t_end == float(d["t_end"])


def test_inlet_records_read(tmp_path):
    """401 / 403 / 404 / 407 data lines: the numbers in the bc_data layout,
    the token 'normal' as the largest double, species fractions dropped."""
    text = "\n".join([
        "1 1 1 1 1 401", "1.2, 0.95, normal, 0.0, 0.9, 1.0",
        "1 1 2 1 1 403", "1.15 0.8d0 0.1 normal 1.0 1.0",
        "1 1 3 1 1 404", "0.71 -0.8 0.0 0.0 1.0 1.0",
        "1 2 1 1 2 407", "1.2 0.95 0.71 0.05 0.0 0.7 1.0",
    ]) + "\n"
    path = tmp_path / "bc.txt"
    path.write_text(text)
    rec, data = refio.read_bc(path)
    huge = np.finfo(np.float64).max
    assert rec[:, 5].tolist() == [401, 403, 404, 407]
    np.testing.assert_array_equal(data[0], [1.2, 0.95, huge, 0.0, 0.9, 0.0])
    np.testing.assert_array_equal(data[1], [1.15, 0.8, 0.1, huge, 1.0, 0.0])
    np.testing.assert_array_equal(data[2], [0.71, -0.8, 0.0, 0.0, 1.0, 0.0])
    np.testing.assert_array_equal(data[3], [1.2, 0.95, 0.71, 0.05, 0.0, 0.7])


def test_time_table_inlet_read(tmp_path):
    """A 402 record names its p0 table file (Series_Data_m.f90:20-52): the
    table is read relative to the case directory, bar becomes Pa, a first
    line holding 'periodic' marks it periodic, and the record carries the
    table's index."""
    (tmp_path / "INPUT").mkdir()
    (tmp_path / "p0.dat").write_text("0.0 1.0\n0.5 1.2\n1.0 1.1\n")
    (tmp_path / "p0per.dat").write_text("periodic\n0.0 0.9\n0.25 1.0\n")
    text = "\n".join(["1 1 1 1 1 402", "300.0, p0.dat, 0.0, 0.0, 1.0, 1.0",
                      "1 1 2 1 1 402", "300.0 'p0per.dat' normal 0.0 0.8 1.0"]) + "\n"
    (tmp_path / "INPUT" / "bc.txt").write_text(text)
    series = []
    rec, data = refio.read_bc(tmp_path / "INPUT" / "bc.txt", series)
    assert rec[:, 5].tolist() == [402, 402]
    assert data[0, 1] == 0.0 and data[1, 1] == 1.0
    assert data[1, 2] == np.finfo(np.float64).max and data[1, 4] == 0.8
    t, v, per = series[0]
    np.testing.assert_array_equal(t, [0.0, 0.5, 1.0])
    np.testing.assert_array_equal(v, np.array([1.0, 1.2, 1.1]) * 1e5)   # var*1d+5, as the reference scales
    assert not per
    t, v, per = series[1]
    np.testing.assert_array_equal(t, [0.0, 0.25])
    assert per and v[0] == 0.9e5
    with pytest.raises(ValueError):
        refio.read_bc(tmp_path / "INPUT" / "bc.txt")
