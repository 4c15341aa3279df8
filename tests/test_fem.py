"""method fem (Discretization.hpp:1580-1790, 7687-8130): Whitney edge mass,
central differences of the second-order wave equation and the Jacobi-PCG
solve of E / dt^2 each step, on the group engine, against the FP64 oracle."""
import numpy as np
import pytest

import oracle
import tetfit_b200 as tb
from tetfit_b200.cases import TetCase, write_tet_case

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def pair(script, steps=None, **opts):
    o = oracle.TetOracle(script)
    n = o.n_steps if steps is None else steps
    o.step(n)
    to, vo, po, _ = o.probes()
    Uo, Bo, _ = o.state()
    oo = dict(t=to, v=vo, xyz=po, U=Uo, B=Bo, flux=o.flux(), dt=o.dt)
    oo["it"], oo["res"] = o.cg()
    with tb.Discretization(script) as d:
        info = d.prepare(1, **opts)
        d.step(n)
        t, v = d.probes()
        U, B, _ = d.state()
        xyz, _ = d.probe_points()
        it, res = d.solver_stats()
        g = dict(t=t, v=v, xyz=xyz, U=U, B=B, flux=d.flux(), it=it, res=res, info=info)
    return g, oo


@pytest.mark.parametrize("n,steps", [(4, 80), (8, 160)])
def test_fem_fp64_matches_oracle(tmp_path, product_lib, oracle_lib, n, steps):
    s = write_tet_case(str(tmp_path), TetCase(n=n, method="fem", steps=steps, split_x=True, eps=(1.5, 3.0)))
    g, o = pair(s, precision="fp64")
    assert g["info"]["method"] == "fem" and g["info"]["dt"] == o["dt"]
    assert np.array_equal(g["t"], o["t"]) and np.array_equal(g["xyz"], o["xyz"])
    assert np.mean(g["it"] == o["it"]) >= 0.95 and np.abs(g["it"] - o["it"]).max() <= 1
    for k in ("v", "U", "B", "flux"):
        assert rel(g[k], o[k]) <= 1e-8, k
    assert np.abs(o["v"]).max() > 0


def test_fem_tight_tolerance(tmp_path, product_lib, oracle_lib):
    """CG to 1e-13: the kernels (Whitney mass, second-order right-hand side,
    U_older history) agree to 1e-10."""
    s = write_tet_case(str(tmp_path), TetCase(n=6, method="fem", steps=120, tolerance=1e-13))
    g, o = pair(s, precision="fp64")
    for k in ("v", "U", "B", "flux"):
        assert rel(g[k], o[k]) <= 1e-10, k


def test_fem_fp32_error_bound(tmp_path, product_lib, oracle_lib):
    """FP32 state against the FP64 oracle.  fem advances U by its second
    difference, which is O((omega dt)^2) of U, so FP32 rounding of the state
    weighs about 1/(omega dt)^2 times more than in gfdtd's first-order form;
    the bound is 2e-5 (1.3e-5 measured on U, 8e-6 on the probes)."""
    s = write_tet_case(str(tmp_path), TetCase(n=6, method="fem", steps=120))
    g, o = pair(s, precision="fp32")
    assert rel(g["v"], o["v"]) <= 2e-5 and rel(g["U"], o["U"]) <= 2e-5


@pytest.mark.parametrize("src", [dict(source_type="e"), dict(source_type="j"),
                                 dict(carrier="ricker", delay=4e-9)])
def test_fem_sources(tmp_path, product_lib, oracle_lib, src):
    s = write_tet_case(str(tmp_path), TetCase(n=4, method="fem", steps=80, tolerance=1e-13, **src))
    g, o = pair(s, precision="fp64")
    assert np.abs(o["U"]).max() > 0
    for k in ("v", "U", "flux"):
        assert rel(g[k], o[k]) <= 1e-10, k


@pytest.mark.parametrize("mode", ["group", "serial"])
def test_fem_and_gfdtd_members_in_one_batch(tmp_path, product_lib, oracle_lib, mode):
    """fem and gfdtd members of uneven sizes advance together in one group
    (per-member method), each matching its own oracle run."""
    cases = [TetCase(n=4, method="fem", steps=60, seed=11), TetCase(n=6, method="gfdtd", steps=50, seed=12),
             TetCase(n=5, method="fem", steps=70, seed=13, split_x=True, eps=(2.0, 1.25))]
    scripts = [write_tet_case(str(tmp_path / f"m{i}"), c) for i, c in enumerate(cases)]
    with tb.Batch([(s, 1) for s in scripts], precision="fp64", batch_mode=mode) as b:
        b.step(10 ** 6)
        res = [(b.probes(m), b.state(m)[0]) for m in range(len(scripts))]
    for s, ((t, v), U) in zip(scripts, res):
        o = oracle.TetOracle(s)
        o.run()
        to, vo, _, _ = o.probes()
        assert np.array_equal(t, to)
        assert rel(v, vo) <= 1e-8 and rel(U, o.state()[0]) <= 1e-8
