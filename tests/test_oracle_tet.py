"""CPU checks of the tetrahedral oracle: complex invariants, counts and the
relation between the dga, gfdtd and FIT discretisations."""
import numpy as np
import pytest

import oracle
from tetfit_b200.cases import FitCase, TetCase, kuhn_mesh, write_fit_cavity, write_tet_case


def csr_dense(ptr, col, val, ncols):
    m = np.zeros((len(ptr) - 1, ncols))
    for r in range(len(ptr) - 1):
        for k in range(int(ptr[r]), int(ptr[r + 1])):
            m[r, col[k]] += val[k]
    return m


@pytest.mark.parametrize("n", [2, 3, 5])
def test_kuhn_counts_and_numbering(tmp_path, n):
    s = write_tet_case(str(tmp_path), TetCase(n=n, method="dga", steps=3))
    o = oracle.TetOracle(s)
    assert (o.nN, o.nT, o.nE, o.nF) == ((n + 1) ** 3, 6 * n ** 3, 7 * n ** 3 + 9 * n ** 2 + 3 * n,
                                        12 * n ** 3 + 6 * n ** 2)
    e, f, cls, bnd = o.topology()
    # numbering: sorted unique node pairs / triples
    assert np.all(e[:, 0] < e[:, 1]) and np.all(np.diff(e[:, 0].astype(np.int64) * 2**32 + e[:, 1]) > 0)
    fk = f[:, 0].astype(np.int64) * 2**42 + f[:, 1].astype(np.int64) * 2**21 + f[:, 2]
    assert np.all(np.diff(fk) > 0)
    # boundary edges of the 12 n^2 boundary triangles, PEC ones are class 4
    assert set(np.unique(cls)) <= {1, 4}


def test_curl_of_gradient_is_zero(tmp_path):
    # C G = 0 with G the node-edge incidence (edges oriented low -> high node)
    s = write_tet_case(str(tmp_path), TetCase(n=3, method="dga", steps=3))
    o = oracle.TetOracle(s)
    ptr, col, val = o.matrix("C")
    C = csr_dense(ptr, col, val, o.nE)
    e, _, _, _ = o.topology()
    G = np.zeros((o.nE, o.nN))
    G[np.arange(o.nE), e[:, 0]] = -1
    G[np.arange(o.nE), e[:, 1]] = 1
    assert np.abs(C @ G).max() == 0
    assert set(np.unique(val)) == {-1.0, 1.0}
    assert np.all(np.diff(ptr) == 3)


def test_operators_symmetric_positive(tmp_path):
    s = write_tet_case(str(tmp_path), TetCase(n=3, method="gfdtd", steps=3))
    o = oracle.TetOracle(s)
    N = csr_dense(*o.matrix("N"), o.nF)
    E = csr_dense(*o.matrix("E"), o.nE)
    A = csr_dense(*o.matrix("A"), o.n_free)
    for M in (N, E, A):
        assert np.allclose(M, M.T, rtol=1e-12, atol=1e-12 * np.abs(M).max())
    assert np.linalg.eigvalsh(A).min() > 0
    assert np.linalg.eigvalsh(N).min() > 0


def test_dga_agrees_with_fit_on_regular_grid(tmp_path):
    """Same cavity, same source: the dga tet scheme and the Cartesian FIT
    scheme are different discretisations of one problem and must agree
    closely on an unjittered grid."""
    n, steps = 12, 600
    s = write_tet_case(str(tmp_path / "t"), TetCase(n=n, method="dga", steps=steps, jitter=0.0))
    o = oracle.TetOracle(s)
    o.run()
    _, vd, pd, _ = o.probes()
    sf = write_fit_cavity(str(tmp_path / "f"), FitCase(n=n, steps=steps, step=o.dt))
    fo = oracle.FitOracle(sf)
    fo.run()
    _, vf, pf, _ = fo.probes()
    assert np.allclose(pd, pf)
    ey_d, ey_f = vd[:, :, 1], vf[:, :, 1]
    assert np.linalg.norm(ey_d - ey_f) / np.linalg.norm(ey_f) < 0.15


def test_gfdtd_mass_model(tmp_path):
    """The reference's gfdtd eps-mass is four times the consistent one (half
    edge duals without the 1/4): its stability limit doubles, and only the
    consistent form agrees with dga."""
    n, steps = 10, 500
    sd = write_tet_case(str(tmp_path / "d"), TetCase(n=n, method="dga", steps=steps))
    sg = write_tet_case(str(tmp_path / "g"), TetCase(n=n, method="gfdtd", steps=steps))
    od = oracle.TetOracle(sd)
    og_ref = oracle.TetOracle(sg)
    og_con = oracle.TetOracle(sg, consistent_mass=True)
    assert og_ref.dt_estimate / og_con.dt_estimate == pytest.approx(2.0, rel=0.05)
    for o in (od, og_ref, og_con):
        o.run()
    vd = od.probes()[1][1:, :, 1]
    vr = og_ref.probes()[1][:-1, :, 1]
    vc = og_con.probes()[1][:-1, :, 1]
    e_con = np.linalg.norm(vc - vd) / np.linalg.norm(vd)
    e_ref = np.linalg.norm(vr - vd) / np.linalg.norm(vd)
    assert e_con < 0.3 and e_ref > 0.6


def test_gfdtd_cg_criterion_reference(tmp_path):
    s = write_tet_case(str(tmp_path), TetCase(n=5, method="gfdtd", steps=40, tolerance=1e-8))
    o = oracle.TetOracle(s)
    o.run()
    it, err = o.cg()
    assert it.max() <= 100 and it.min() > 0
    assert np.nanmax(err) <= 1e-8


@pytest.mark.parametrize("method", ["gfdtd", "dga"])
def test_gmsh_input_is_the_rounded_netgen_mesh(tmp_path, method):
    """A gmsh mesh goes through the reference's conversion to netgen text,
    which prints coordinates with 6 significant digits
    (Discretization.hpp:5692-5866): it runs exactly as the netgen file of the
    same mesh written with %g coordinates, and not as the full-precision one."""
    kw = dict(n=4, method=method, steps=12, split_x=True, eps=(1.5, 3.0), seed=11)
    runs = []
    for sub, extra in (("g", dict(mesh_format="gmsh")), ("r", dict(coord_fmt="%g")), ("f", {})):
        s = write_tet_case(str(tmp_path / sub), TetCase(**kw, **extra))
        o = oracle.TetOracle(s)
        o.run()
        _, v, _, _ = o.probes()
        U, B, F = o.state()
        o.close()
        runs.append((v, U, B, F))
    for a, b in zip(runs[0], runs[1]):
        assert np.array_equal(a, b)
    assert not np.array_equal(runs[0][1], runs[2][1])


@pytest.mark.parametrize("jitter", [0.0, 0.15])
def test_fem_whitney_mass_constant_field(tmp_path, jitter):
    """fem's edge mass (Discretization.hpp:7902-8060: Whitney functions
    l_a grad l_b - l_b grad l_a on the local edge order ab, bc, ac, ad, bd,
    cd, quadrature 1/40 at the nodes and 9/40 at the face barycentres)
    reproduces a constant field exactly, so for the edge voltages of a
    uniform E0, u.E.u = eps |E0|^2 times the box volume (1 m^3)."""
    n, eps_r = 4, 2.5
    case = TetCase(n=n, method="fem", steps=3, eps=(eps_r,), jitter=jitter)
    s = write_tet_case(str(tmp_path), case)
    o = oracle.TetOracle(s)
    assert o.method == 3
    pts = kuhn_mesh(n, jitter, case.seed)[0]
    e, _, _, _ = o.topology()
    E = csr_dense(*o.matrix("E"), o.nE)
    assert np.allclose(E, E.T, rtol=0, atol=1e-14 * np.abs(E).max())
    for E0 in ([1.0, 0.0, 0.0], [0.3, -1.2, 0.7]):
        u = (pts[e[:, 1]] - pts[e[:, 0]]) @ np.asarray(E0)
        want = 8.854187817e-12 * eps_r * float(np.dot(E0, E0))
        assert u @ E @ u == pytest.approx(want, rel=1e-12)
    # positive definite
    assert np.linalg.eigvalsh(E).min() > 0
