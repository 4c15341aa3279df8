"""GPU FIT path against the FP64 CPU oracle, through the C ABI."""
import numpy as np
import pytest

import oracle
import tetfit_b200 as tb
from tetfit_b200.cases import FitCase, random_spheres, write_fit_cavity

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10   # relative L2, FP64 state
TOL_FP32 = 1e-5    # relative L2, FP32 state vs the FP64 oracle


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run_both(script, precision="fp64", steps=None):
    o = oracle.FitOracle(script)
    o.step(o.n_steps if steps is None else steps)
    to, vo, po, _ = o.probes()
    Uo, Bo, Fo = o.state()
    with tb.Discretization(script) as d:
        info = d.prepare(1, precision=precision)
        d.step(info["n_steps"] if steps is None else steps)
        t, v = d.probes()
        U, B, F = d.state()
        xyz, _ = d.probe_points()
        fl = d.flux()
    return dict(t=t, v=v, U=U, B=B, F=F, xyz=xyz, flux=fl, info=info), \
        dict(t=to, v=vo, U=Uo, B=Bo, F=Fo, xyz=po, flux=o.flux(), dt=o.dt, n_steps=o.n_steps)


@pytest.mark.parametrize("n,steps", [(8, 30), (16, 120), (24, 200)])
def test_cavity_fp64_matches_oracle(tmp_path, product_lib, oracle_lib, n, steps):
    script = write_fit_cavity(str(tmp_path), FitCase(n=n, steps=steps))
    g, o = run_both(script)
    assert g["info"]["n_steps"] == o["n_steps"] == steps
    assert g["info"]["dt"] == o["dt"]
    assert np.array_equal(g["xyz"], o["xyz"])
    assert np.array_equal(g["t"], o["t"])
    assert rel(g["v"], o["v"]) <= TOL_FP64
    assert rel(g["U"], o["U"]) <= TOL_FP64
    assert rel(g["F"], o["F"]) <= TOL_FP64
    assert rel(g["B"], o["B"]) <= TOL_FP64
    assert rel(g["flux"], o["flux"]) <= TOL_FP64
    assert np.abs(o["v"]).max() > 0


def test_cavity_fp64_bitwise_state(tmp_path, product_lib, oracle_lib):
    """The FP64 kernels use the reference's operation order without FMA
    contraction, so the edge and face state is bit-identical to the oracle."""
    script = write_fit_cavity(str(tmp_path), FitCase(n=12, steps=60))
    g, o = run_both(script)
    assert np.array_equal(g["U"], o["U"])
    assert np.array_equal(g["F"], o["F"])
    assert np.array_equal(g["v"][..., :3], o["v"][..., :3])


def test_lossy_spheres_fp64(tmp_path, product_lib, oracle_lib):
    spheres = random_spheres(12, seed=7)
    script = write_fit_cavity(str(tmp_path), FitCase(n=20, steps=100, spheres=spheres))
    g, o = run_both(script)
    for k in ("v", "U", "F", "B"):
        assert rel(g[k], o[k]) <= TOL_FP64, k


def test_cavity_fp32_error_bound(tmp_path, product_lib, oracle_lib):
    script = write_fit_cavity(str(tmp_path), FitCase(n=16, steps=150))
    g, o = run_both(script, precision="fp32")
    assert rel(g["v"], o["v"]) <= TOL_FP32
    assert rel(g["U"], o["U"]) <= TOL_FP32


@pytest.mark.parametrize("src", ["e"])
def test_electric_surface_source(tmp_path, product_lib, oracle_lib, src):
    script = write_fit_cavity(str(tmp_path), FitCase(n=10, steps=50, source_type=src))
    g, o = run_both(script)
    for k in ("v", "U", "F"):
        assert rel(g[k], o[k]) <= TOL_FP64, k


def test_natural_boundary_surface(tmp_path, product_lib, oracle_lib):
    # surface 6 neither PEC nor a source: natural (zero tangential H) boundary
    script = write_fit_cavity(str(tmp_path), FitCase(n=10, steps=80, pec_surfaces=(2, 3, 4, 5)))
    g, o = run_both(script)
    for k in ("v", "U", "F"):
        assert rel(g[k], o[k]) <= TOL_FP64, k


def test_chunked_stepping_matches_single_call(tmp_path, product_lib):
    script = write_fit_cavity(str(tmp_path), FitCase(n=10, steps=100))
    with tb.Discretization(script) as d:
        d.prepare(1, graph_steps=7)
        for _ in range(13):
            d.step(8)
        d.step(1000)
        U1, _, F1 = d.state()
    with tb.Discretization(script) as d:
        d.prepare(1, graph_steps=1)
        d.step(1000)
        U2, _, F2 = d.state()
    assert np.array_equal(U1, U2) and np.array_equal(F1, F2)


@pytest.mark.parametrize("variant", [1, 2, 3, 4, 5, 6])
def test_every_kernel_variant_is_bitwise_identical(tmp_path, product_lib, oracle_lib, variant):
    """The E/H kernel variants the autotuner chooses between (one thread per
    node, z-march over 4 or 16 planes, per-dof coefficient arrays, z-march
    with TMA-staged planes, coefficient classes) give the same FP64 state bit
    for bit, on a lossy multi-material scene."""
    case = FitCase(n=14, steps=50, spheres=random_spheres(5, seed=9))
    script = write_fit_cavity(str(tmp_path), case)
    o = oracle.FitOracle(script)
    o.step(50)
    Uo, _, Fo = o.state()
    with tb.Discretization(script) as d:
        info = d.prepare(1, precision="fp64", fit_variant=variant)
        d.step(50)
        U, _, F = d.state()
        assert d.info()["cg_variant"] == (variant - 1) * 9
    assert np.array_equal(U, Uo) and np.array_equal(F, Fo)


@pytest.mark.parametrize("mode", ["l2norm", "probepoint"])
def test_joule_losses_match_oracle(tmp_path, product_lib, oracle_lib, mode):
    """poynting.dat's third column, 0.25 (U_old + U)^T Si (U_old + U)
    (Discretization.hpp:1902).  The reference fills Si (sigma-bar / length)
    only for l2norm outputs (:5368, :5594-5597): with lossy spheres the loss
    is non-zero there and exactly zero for probe outputs."""
    case = FitCase(n=20, steps=120, spheres=random_spheres(12, seed=7), output_mode=mode)
    script = write_fit_cavity(str(tmp_path), case)
    o = oracle.FitOracle(script)
    o.run()
    lo = o.losses()
    for prec, tol in (("fp64", TOL_FP64), ("fp32", TOL_FP32)):
        with tb.Discretization(script) as d:
            info = d.prepare(1, precision=prec)
            d.step(info["n_steps"])
            lg = d.losses()
            U, _, _ = d.state()
        assert lg.shape == lo.shape == (120,)
        if mode == "probepoint":
            assert not lg.any() and not lo.any()
        else:
            assert lo.max() > 0
            assert rel(lg, lo) <= tol, prec
