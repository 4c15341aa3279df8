"""GPU tetrahedral paths (dga explicit, gfdtd with the persistent PCG kernel)
against the FP64 CPU oracle, through the C ABI."""
import numpy as np
import pytest

import oracle
import tetfit_b200 as tb
from tetfit_b200.cases import TetCase, write_tet_case

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
TOL_FP32 = 1e-5


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run_pair(script, steps=None, oracle_kw=None, **opts):
    o = oracle.TetOracle(script, **(oracle_kw or {}))
    o.step(o.n_steps if steps is None else steps)
    to, vo, po, _ = o.probes()
    Uo, Bo, Fo = o.state()
    with tb.Discretization(script) as d:
        info = d.prepare(1, **opts)
        d.step(info["n_steps"] if steps is None else steps)
        t, v = d.probes()
        U, B, F = d.state()
        xyz, _ = d.probe_points()
        it, res = d.solver_stats()
        fl = d.flux()
    g = dict(t=t, v=v, U=U, B=B, F=F, xyz=xyz, it=it, res=res, flux=fl, info=info)
    oo = dict(t=to, v=vo, U=Uo, B=Bo, F=Fo, xyz=po, flux=o.flux(), dt=o.dt, n_steps=o.n_steps)
    if o.method == 2:
        oo["it"], oo["res"] = o.cg()
    return g, oo


@pytest.mark.parametrize("n,steps", [(4, 60), (8, 150)])
def test_dga_fp64_matches_oracle(tmp_path, product_lib, oracle_lib, n, steps):
    s = write_tet_case(str(tmp_path), TetCase(n=n, method="dga", steps=steps))
    g, o = run_pair(s)
    assert g["info"]["method"] == "dga" and g["info"]["n_steps"] == o["n_steps"]
    assert g["info"]["dt"] == o["dt"]
    assert np.array_equal(g["xyz"], o["xyz"]) and np.array_equal(g["t"], o["t"])
    for k in ("v", "U", "B", "F", "flux"):
        assert rel(g[k], o[k]) <= TOL_FP64, k
    assert np.abs(o["v"]).max() > 0


@pytest.mark.parametrize("method", ["dga", "gfdtd"])
def test_gmsh_mesh_matches_oracle(tmp_path, product_lib, oracle_lib, method):
    """gmsh input (the reference's conversion to netgen text) on the GPU path
    against the oracle reading the same file."""
    s = write_tet_case(str(tmp_path), TetCase(n=4, method=method, steps=40, mesh_format="gmsh",
                                              split_x=True, eps=(1.5, 3.0)))
    g, o = run_pair(s)
    assert np.array_equal(g["t"], o["t"]) and np.array_equal(g["xyz"], o["xyz"])
    tol = TOL_FP64 if method == "dga" else 1e-8
    for k in ("v", "U", "F"):
        assert rel(g[k], o[k]) <= tol, k
    assert np.abs(o["v"]).max() > 0


@pytest.mark.parametrize("n,steps", [(4, 60), (8, 120)])
def test_gfdtd_fp64_matches_oracle(tmp_path, product_lib, oracle_lib, n, steps):
    s = write_tet_case(str(tmp_path), TetCase(n=n, method="gfdtd", steps=steps))
    g, o = run_pair(s)
    assert g["info"]["method"] == "gfdtd"
    assert np.array_equal(g["t"], o["t"])
    # the same Jacobi-PCG, FP64 in both: iteration counts agree step by step
    assert np.mean(g["it"] == o["it"]) >= 0.95 and np.abs(g["it"] - o["it"]).max() <= 1
    assert np.nanmax(g["res"]) <= 1e-8
    for k in ("v", "U", "B", "F"):
        assert rel(g[k], o[k]) <= 1e-8, k


def test_gfdtd_consistent_mass(tmp_path, product_lib, oracle_lib):
    s = write_tet_case(str(tmp_path), TetCase(n=6, method="gfdtd", steps=80))
    g, o = run_pair(s, oracle_kw=dict(consistent_mass=True), mass="consistent")
    for k in ("v", "U", "F"):
        assert rel(g[k], o[k]) <= 1e-8, k


def test_gfdtd_fp32_error_bound(tmp_path, product_lib, oracle_lib):
    s = write_tet_case(str(tmp_path), TetCase(n=8, method="gfdtd", steps=100))
    g, o = run_pair(s, precision="fp32")
    assert rel(g["v"], o["v"]) <= TOL_FP32
    assert rel(g["U"], o["U"]) <= TOL_FP32


def test_dga_fp32_error_bound(tmp_path, product_lib, oracle_lib):
    s = write_tet_case(str(tmp_path), TetCase(n=8, method="dga", steps=100))
    g, o = run_pair(s, precision="fp32")
    assert rel(g["v"], o["v"]) <= TOL_FP32


@pytest.mark.parametrize("ws", ["zero", "extrapolate"])
def test_gfdtd_warm_starts_same_solution(tmp_path, product_lib, ws):
    s = write_tet_case(str(tmp_path), TetCase(n=6, method="gfdtd", steps=80, tolerance=1e-10))
    res = {}
    for w in ("previous", ws):
        with tb.Discretization(s) as d:
            d.prepare(1, warm_start=w, cg_criterion="rhs")
            d.step(10 ** 6)
            U, _, _ = d.state()
            it, _ = d.solver_stats()
            res[w] = (U, it)
    assert rel(res[ws][0], res["previous"][0]) <= 1e-7
    if ws == "zero":
        assert res["zero"][1].mean() > res["previous"][1].mean()
    else:
        assert res["extrapolate"][1].mean() < res["previous"][1].mean()
