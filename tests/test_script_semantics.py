"""Script front end (CPU): the product's parser (tf_open + tf_script_dump),
the oracle's parser and an independent Python reading of the reference's
grammar (oracle/script_ref.py) must agree on every script; reference quirks
are pinned to values derived by hand from the cited reference lines."""
import os

import numpy as np
import pytest

import oracle
import oracle.script_ref as R
import tetfit_b200 as tb
from tetfit_b200.cases import (FitCase, TetCase, batch_cases, grf_materials, random_spheres, write_fit_cavity,
                               write_tet_case)


@pytest.fixture(scope="module")
def libs():
    from tetfit_b200 import build
    build.build()
    oracle.build()
    return tb.lib(), oracle.lib()


def product_parse(path):
    with tb.Discretization(path) as d:
        return d.script()


def all_three(path):
    p = product_parse(path)
    o = oracle.script_dump(path)
    r = R.parse_script(path)
    assert p == r, "product parser disagrees with the independent reading"
    assert o == r, "oracle parser disagrees with the independent reading"
    return r


def product_error(path):
    with pytest.raises(tb.TetfitError) as e:
        tb.Discretization(path)
    return e.value.message


def write(tmp_path, name, text):
    p = os.path.join(str(tmp_path), name)
    with open(p, "w") as f:
        f.write(text)
    return p


GENERATED = [
    ("fit", lambda d: write_fit_cavity(d, FitCase(n=8, steps=10))),
    ("fit_spheres", lambda d: write_fit_cavity(d, FitCase(n=8, steps=10, spheres=random_spheres(6, seed=3)))),
    ("fit_e_source_l2norm", lambda d: write_fit_cavity(d, FitCase(n=6, steps=5, source_type="e",
                                                                  output_mode="l2norm", carrier="gaussian",
                                                                  width=1e-9, delay=2e-9))),
    ("dga", lambda d: write_tet_case(d, TetCase(n=3, method="dga", steps=5))),
    ("gfdtd_two_mat", lambda d: write_tet_case(d, TetCase(n=3, steps=5, split_x=True, eps=(1.5, 3.25)))),
    ("gmsh", lambda d: write_tet_case(d, TetCase(n=3, steps=5, mesh_format="gmsh"))),
    ("batch_member", lambda d: write_tet_case(d, batch_cases(3, n_lo=3, n_hi=4)[2])),
    ("grf", lambda d: write_tet_case(d, TetCase(n=4, steps=5, mat_field=grf_materials(8, grid=8)[0],
                                                eps=grf_materials(8, grid=8)[1]))),
]


@pytest.mark.parametrize("name,make", GENERATED, ids=[g[0] for g in GENERATED])
def test_generated_scripts_agree(tmp_path, libs, name, make):
    all_three(make(str(tmp_path)))


HEADER = """DEFINE mesh 1
   SET type cartesian
   SET xgrid {0,0.25,1}
   SET ygrid {0,0.25,1}
   SET zgrid {0,0.25,1}
   SET file solids.txt
END mesh 1
"""
SOLIDS = """DEFINE solid 1
   SET material 1
   SET type box
   SET corner {0,0,0}
   SET size {1,1,1}
END solid 1
"""


def quirk_script(tmp_path, body):
    write(tmp_path, "solids.txt", SOLIDS)
    return write(tmp_path, "q.fdtd", HEADER + body)


def test_probe_grid_is_read_as_float(tmp_path, libs):
    """Output.hpp:154-164 reads grid values with std::stof (float), stored as
    double; Output.hpp:288-297 accumulates the grid in double."""
    s = quirk_script(tmp_path, """DEFINE output 1
   SET mode probepoint
   SET xgrid { 0.1, 0.1,0.6}
   SET ygrid { 0.5, 1, 0.5}
   SET zgrid { 0, 0.04, 1.05}
   SET grid on
   SET period 1e-10
END output 1
""")
    r = all_three(s)["outputs"]["1"]
    f32 = lambda x: float(np.float32(x))
    assert r["xstart"] == f32(0.1) and r["zstep"] == f32(0.04) and r["zstop"] == f32(1.05)
    assert r["period"] == f32(1e-10)
    # 6 x values (0.1 .. 0.6 in float steps), 1 y value, z from 0 while <= 1.05f: 27 values
    xs, zs = [], []
    x = f32(0.1)
    while x <= f32(0.6):
        xs.append(x)
        x += f32(0.1)
    z = 0.0
    while z <= f32(1.05):
        zs.append(z)
        z += f32(0.04)
    assert len(xs) == 6 and len(zs) == 27
    expect = [[x, f32(0.5), z] for z in zs for x in xs]
    assert r["probes"] == expect


def test_brace_values_rejoined(tmp_path, libs):
    """Discretization.hpp:144-161: a value starting with '{' is re-read from
    the line's first '{' to its first '}', so lists may contain spaces; the
    source `mode` list drops spaces (Source.hpp:228-231) and a short list
    keeps the default "cos" (Source.hpp:53)."""
    s = quirk_script(tmp_path, """DEFINE source 1
   SET type h
   SET profile wave
   SET mode { sin , cos }
   SET center {0.5, 0.25 ,  1}
   SET wavevector {   0.5,0, 0 }
   SET surface 1
END source 1
""")
    r = all_three(s)["sources"]["1"]
    assert r["bfuncs"] == ["sin", "cos", "cos"]
    assert r["center"] == [0.5, 0.25, 1.0]
    assert r["kvec"] == [0.5, 0.0, 0.0]


def test_simulation_source_list_keeps_default(tmp_path, libs):
    """Simulation.hpp:39,55-56: the list starts as {1}; SET source appends and
    sorts/uniques, so `SET source 3` gives {1, 3}."""
    s = quirk_script(tmp_path, """DEFINE simulation 1
   SET method fdtd
   SET source 3
   SET source 2
   SET source 3
   SET mesh 1
   SET duration 1e-9
END simulation 1
""")
    r = all_three(s)["simulations"]["1"]
    assert r["sources"] == [1, 2, 3] and r["method"] == "fdtd" and r["mesh"] == 1


def test_material_tensor_entries(tmp_path, libs):
    """Material.hpp:51-170: scalar settings are relative (times eps0/mu0) and
    reset the tensor to a multiple of the identity; off-diagonal entries are
    stored as given (no eps0 factor); *_vec sets the diagonal only."""
    s = quirk_script(tmp_path, """DEFINE material 1
   SET epsilon_xy 3
   SET epsilon 2
   SET epsilon_yz 0.5
   SET mu_vec {1,2,3}
   SET sigma 0.25
   SET sigma_xz 7
END material 1
""")
    r = all_three(s)["materials"]["1"]
    e0, m0 = R.EPS0, R.MU0
    assert r["eps"] == [[2 * e0, 0, 0], [0, 2 * e0, 0.5], [0, 0.5, 2 * e0]]
    assert r["mu"] == [[m0, 0, 0], [0, 2 * m0, 0], [0, 0, 3 * m0]]
    assert r["sigma"] == [[0.25, 0, 7], [0, 0.25, 0], [7, 0, 0.25]]
    assert m0 == float(np.float64(np.longdouble(4) * np.longdouble("3.141592653589793238") * np.longdouble(1e-7)))


def test_short_lines_reuse_previous_tokens(tmp_path, libs):
    """Discretization.hpp:73: sscanf fills only the tokens a line has, the
    others keep the previous line's: `SET grid` after `SET grid on` runs the
    grid generator again (probes listed twice), and a line of blanks repeats
    the previous instruction."""
    s = quirk_script(tmp_path, """DEFINE output 1
   SET mode probepoint
   SET xgrid {0.5,1,0.5}
   SET ygrid {0.5,1,0.5}
   SET zgrid {0.25,0.5,0.75}
   SET grid on
   SET grid
   \t
END output 1
""")
    r = all_three(s)["outputs"]["1"]
    assert len(r["probes"]) == 6 and r["probes"][:2] == r["probes"][2:4]
    bad = quirk_script(tmp_path, "DEFINE material 1\n   SET epsilon 2\nEND material 1\n   \n")
    msg = "Input file error at line 11: define something before setting variables"
    assert product_error(bad) == msg
    with pytest.raises(R.ScriptError, match="line 11: define something"):
        R.parse_script(bad)
    with pytest.raises(RuntimeError, match="line 11: define something"):
        oracle.script_dump(bad)


def test_bc_surface_table(tmp_path, libs):
    """Discretization.hpp:61,119-128: each bc's END writes its label into the
    100-slot surface table; a later bc on the same surface wins."""
    s = quirk_script(tmp_path, """DEFINE bc 4
   SET type pec
   SET surfaces {1,3, 5}
END bc 4
DEFINE bc 2
   SET type pmc
   SET surface 3
END bc 2
""")
    r = all_three(s)
    t = r["bnd_to_bc"]
    assert len(t) == 100 and t[1] == 4 and t[3] == 2 and t[5] == 4 and sum(1 for v in t if v) == 3
    assert r["bcs"]["4"]["surfs"] == [1, 3, 5] and r["bcs"]["2"]["type"] == "pmc"


def test_solids_file_fields(tmp_path, libs):
    """Solid.hpp:47-233: material read with atoi, radius stored squared;
    solids listed by label (WhichSolid's first-match order)."""
    write(tmp_path, "solids.txt", """DEFINE solid 2
   SET material 3xyz
   SET type sphere
   SET center {0.5,0.5,0.5}
   SET radius 0.25
END solid 2
""" + SOLIDS)
    s = write(tmp_path, "q.fdtd", HEADER)
    r = all_three(s)["solids"]["1"]
    assert list(r) == ["1", "2"]
    assert r["2"]["material"] == 3 and r["2"]["sqr"] == 0.0625 and r["2"]["type"] == "sphere"


ERRORS = [
    ("SET before DEFINE", "   SET epsilon 2\n", 8, "define something before setting variables"),
    ("unknown primitive", "DEFINE widget 1\n", 8,
     "can only define one of the following: material, mesh, refinement, boundary condition, simulation, "
     "output, source"),
    ("END label", "DEFINE material 1\n   SET epsilon 2\nEND material 2\n", 10, "ending unopened definition"),
    ("unknown instruction", "DEFINE material 1\n   PUT epsilon 2\nEND material 1\n", 9,
     "Unknown instruction inside define block"),
    ("unterminated", "DEFINE material 1\n   SET epsilon 2\n", 10, "File ended unexpectedly before ending definition"),
    ("bad carrier", "DEFINE source 1\n   SET carrier square\nEND source 1\n", 9,
     "Unrecognized source carrier! Available: dc, sin, cos, gaussian, ricker"),
    ("bad output mode", "DEFINE output 1\n   SET mode movie\nEND output 1\n", 9,
     "Undefined output mode type! Available: silo, probepoint, maxerror, l2norm"),
    ("bad method", "DEFINE simulation 1\n   SET method rk4\nEND simulation 1\n", 9,
     "Undefined simulation method! Available: fdtd, dga, fem"),
    ("too many coords", "DEFINE source 1\n   SET center {1,2,3,4}\nEND source 1\n", 9,
     "Maximum of three coordinates!"),
    ("unbalanced", "DEFINE source 1\n   SET center {1,2,3\nEND source 1\n", 9, "unbalanced bracket"),
    ("bc type", "DEFINE bc 1\n   SET type open\nEND bc 1\n", 9,
     "Unrecognized boundary condition type! Available: pec, pmc, pml"),
    ("material parameter", "DEFINE material 1\n   SET kappa 2\nEND material 1\n", 9,
     "Unrecognized material parameter! Available: epsilon, mu, sigma, chi"),
]


@pytest.mark.parametrize("name,body,line,msg", ERRORS, ids=[e[0] for e in ERRORS])
def test_error_texts(tmp_path, libs, name, body, line, msg):
    """MyThrow's "Input file error at line N: <msg>" (Utilities.hpp:371-375)
    with the messages of Utilities.hpp:278-317, from all three parsers."""
    s = quirk_script(tmp_path, body)
    want = f"Input file error at line {line}: {msg}"
    assert product_error(s) == want
    with pytest.raises(R.ScriptError) as e:
        R.parse_script(s)
    assert str(e.value) == want
    with pytest.raises(RuntimeError) as e:
        oracle.script_dump(s)
    assert str(e.value) == want


def test_cartesian_y_labels_follow_the_code(tmp_path, libs):
    """Discretization.hpp:5093-5228 labels the y- face 5 and the y+ face 3
    (the reverse of the README).  With PEC on 2, 4, 5, 6 only, the edges in
    the y = 0 plane are PEC and those in the y = 1 plane are natural."""
    s = write_fit_cavity(str(tmp_path), FitCase(n=4, steps=3, pec_surfaces=(2, 4, 5, 6)))
    o = oracle.FitOracle(s)
    en, xyz, _, cl = o.topology()
    p0, p1 = xyz[en[:, 0]], xyz[en[:, 1]]
    inner_x = (np.minimum(p0[:, 0], p1[:, 0]) > 1e-9) & (np.maximum(p0[:, 0], p1[:, 0]) < 1 - 1e-9)
    inner_z = (np.minimum(p0[:, 2], p1[:, 2]) > 1e-9) & (np.maximum(p0[:, 2], p1[:, 2]) < 1 - 1e-9)
    inner = inner_x & inner_z
    on_y0 = inner & (np.abs(p0[:, 1]) < 1e-12) & (np.abs(p1[:, 1]) < 1e-12)
    on_y1 = inner & (np.abs(p0[:, 1] - 1) < 1e-12) & (np.abs(p1[:, 1] - 1) < 1e-12)
    assert on_y0.sum() > 0 and on_y1.sum() == on_y0.sum()
    assert np.all(cl[on_y0] == 1)   # PEC
    assert np.all(cl[on_y1] == 3)   # explicit faces, no source: natural boundary


def test_which_solid_first_match(tmp_path, libs):
    """Discretization.hpp:10110-10122: a cell takes the first solid (by label)
    containing it, so a small box listed before the background keeps its own
    permittivity: M_h of an interior edge inside it is L / (4 da eps)."""
    write(tmp_path, "solids.txt", """DEFINE solid 1
   SET material 1
   SET type box
   SET corner {0,0,0}
   SET size {0.5,0.5,0.5}
END solid 1
DEFINE solid 2
   SET material 2
   SET type box
   SET corner {0,0,0}
   SET size {1,1,1}
END solid 2
""")
    s = write(tmp_path, "q.fdtd", HEADER + """DEFINE material 1
   SET epsilon 4
END material 1
DEFINE material 2
   SET epsilon 1
END material 2
DEFINE simulation 1
   SET method fdtd
   SET mesh 1
   SET duration 1e-10
   SET step 1e-11
END simulation 1
""")
    o = oracle.FitOracle(s)
    en, xyz, _, _ = o.topology()
    mh, _, _, _ = o.coeffs()
    mid = 0.5 * (xyz[en[:, 0]] + xyz[en[:, 1]])
    h = 0.25
    e_in = int(np.argmin(np.linalg.norm(mid - [0.25 + h / 2, 0.25, 0.25], axis=1)))   # inside the small box
    e_out = int(np.argmin(np.linalg.norm(mid - [0.75 - h / 2, 0.75, 0.75], axis=1)))  # background only
    da = h * h / 4
    assert mh[e_in] == pytest.approx(h / (4 * da * 4 * R.EPS0), rel=1e-14)
    assert mh[e_out] == pytest.approx(h / (4 * da * 1 * R.EPS0), rel=1e-14)
