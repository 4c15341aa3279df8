"""Conducting materials on tetrahedra.  gfdtd and fem: the conductivity mass
SigMat (Discretization.hpp:8604-8616 for gfdtd, the same dual basis as the
eps-mass; :8020-8051 for fem, the same Whitney quadrature), the system
SysMat = E + (dt/2) SigMat (gfdtd, :8644) or E / dt^2 + (0.5/dt) SigMat (fem,
:8092-8093), the right-hand-side terms (:1516-1519, :1729-1731) and the
Joule-loss column of poynting.dat (:1518-1546, :1733-1757).  dga: the edge
classes (:6186-6215, :6776-6903) and the node-star operators H, P, Q, Mq of
:9262-9475 stepped as :887-892; dga never fills its SigMat, so its loss
column stays zero.  Magnetic losses (chi) on dga: the face classes
(:6357-6542) and per-tet operators (:9128-9205) stepped as :912-918, for
faces whose tets share chi; fractured faces, whose old values the reference
reads from the electric state (:586), are refused, and so is chi on gfdtd
and fem."""
import numpy as np
import pytest

import oracle
import tetfit_b200 as tb
from tetfit_b200.cases import TetCase, write_tet_case

EPS0_SCRIPT = 8.854187817e-12  # the reference's vacuum permittivity


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def csr(m, n):
    import scipy.sparse as sp
    ptr, col, val = m
    return sp.csr_matrix((val, col.astype(np.int64), ptr.astype(np.int64)), shape=(n, n))


def lossy_case(method, **kw):
    base = dict(n=4, method=method, steps=60, split_x=True, eps=(1.5, 3.0), sigma=(0.0, 0.02),
                carrier="gaussian", width=2e-9, delay=4e-9)
    base.update(kw)
    return TetCase(**base)


@pytest.mark.parametrize("method", ["gfdtd", "fem"])
def test_uniform_conductivity_mass_is_the_scaled_eps_mass(tmp_path, oracle_lib, method):
    """With one material, SigMat is built exactly like E with sigma for eps, so
    SigMat = sigma / (eps_r eps0) E (CPU, oracle)."""
    s = write_tet_case(str(tmp_path), TetCase(n=3, method=method, steps=4, eps=(2.0,), sigma=(0.01,)))
    o = oracle.TetOracle(s)
    E, S = csr(o.matrix("E"), o.nE), csr(o.matrix("Sig"), o.nE)
    o.close()
    assert S.nnz > 0
    d = S - (0.01 / (2.0 * EPS0_SCRIPT)) * E
    assert abs(d).max() <= 1e-12 * abs(S).max()


@pytest.mark.parametrize("method", ["gfdtd", "fem"])
def test_losses_column_follows_the_reference_list(tmp_path, oracle_lib, method):
    """The reference pushes 0.5 a_{i-1} before and (from step 2) a_i after each
    solve into one list and prints its first n entries, so from the third row
    on every odd row is half the even row before it (CPU, oracle)."""
    s = write_tet_case(str(tmp_path), lossy_case(method, steps=40))
    o = oracle.TetOracle(s)
    o.run()
    L = o.losses()
    o.close()
    assert L[0] == 0.0 and np.all(L >= 0) and L.max() > 0
    assert np.array_equal(L[3::2], 0.5 * L[2:-1:2][:len(L[3::2])])


@pytest.mark.parametrize("method", ["gfdtd", "fem", "dga"])
def test_conductivity_damps_the_field(tmp_path, oracle_lib, method):
    """A gaussian pulse in a PEC box: with a conducting half the field left
    after the pulse is smaller than without (CPU, oracle)."""
    norms = {}
    for sig in ((0.0, 0.0), (0.0, 0.02)):
        s = write_tet_case(str(tmp_path / str(sig[1])), lossy_case(method, steps=80, sigma=sig))
        o = oracle.TetOracle(s)
        o.run()
        norms[sig[1]] = np.linalg.norm(o.state()[0])
        o.close()
    assert norms[0.02] < 0.5 * norms[0.0]


def dga_classes(tmp_path, **kw):
    s = write_tet_case(str(tmp_path), lossy_case("dga", **kw))
    o = oracle.TetOracle(s)
    c = o.topology()[2]
    P, nq = o.dga_p()
    o.close()
    return np.bincount(c, minlength=5), P, nq


def test_dga_edge_classes(tmp_path, oracle_lib):
    """Lossless: every free edge is class 1.  One conducting material: every
    free edge is class 2, no node-star fractions.  Half conducting, two eps:
    lossless, uniformly conducting and fractured edges, the last at the
    interface with a block of U_c for each of their ends (CPU, oracle)."""
    n0, _, q0 = dga_classes(tmp_path / "a", sigma=(0.0, 0.0))
    assert n0[2] == n0[3] == 0 and n0[1] > 0 and q0 == 0
    n1, _, q1 = dga_classes(tmp_path / "b", eps=(2.0,), sigma=(0.02,), split_x=False)
    assert n1[1] == n1[3] == 0 and n1[2] > 0 and q1 == 0
    n2, _, q2 = dga_classes(tmp_path / "c")
    assert n2[1] > 0 and n2[2] > 0 and n2[3] > 0 and q2 > 2 * 6


def test_uniformly_conducting_dga_operators(tmp_path, oracle_lib):
    """One material (eps_r, sigma): the star conductivity matrix is sigma /
    (eps_r eps0) times the eps one, so H = E^-1 / (1 + a) and P = (1 - a) /
    (1 + a) with a = dt sigma / (2 eps_r eps0) (CPU, oracle)."""
    ops = {}
    for sig in (0.0, 0.05):
        s = write_tet_case(str(tmp_path / str(sig)), lossy_case("dga", eps=(2.0,), sigma=(sig,), split_x=False))
        o = oracle.TetOracle(s)
        ops[sig] = (csr(o.matrix("H"), o.nE), o.dga_p()[0], o.topology()[2], o.dt)
        o.close()
    H0, _, c0, dt = ops[0.0]
    H1, P1, c1, dt1 = ops[0.05]
    assert dt == dt1
    a = dt * 0.05 / (2 * 2.0 * EPS0_SCRIPT)
    free = c1 == 2
    assert free.sum() > 0 and np.array_equal(c0 == 1, free)
    assert np.abs(P1[free] - (1 - a) / (1 + a)).max() <= 1e-12
    d = H1 - H0 / (1 + a)
    assert abs(d).max() <= 1e-12 * abs(H1).max()


def test_dga_loss_column_stays_zero(tmp_path, oracle_lib):
    """The reference declares dga's SigMat but never fills it (:8701-9475), so
    poynting.dat's loss column is zero on conducting dga runs (CPU, oracle)."""
    s = write_tet_case(str(tmp_path), lossy_case("dga", steps=30))
    o = oracle.TetOracle(s)
    o.run()
    L = o.losses()
    o.close()
    assert len(L) > 0 and np.all(L == 0)


def pair(script, precision="fp64"):
    o = oracle.TetOracle(script)
    o.run()
    to, vo, _, _ = o.probes()
    ref = dict(t=to, v=vo, U=o.state()[0], flux=o.flux(), loss=o.losses(), it=o.cg()[0])
    o.close()
    with tb.Discretization(script) as d:
        d.prepare(1, precision=precision)
        d.step(10 ** 6)
        t, v = d.probes()
        got = dict(t=t, v=v, U=d.state()[0], flux=d.flux(), loss=d.losses(), it=d.solver_stats()[0])
    return got, ref


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["gfdtd", "fem"])
def test_conducting_members_match_oracle(tmp_path, product_lib, oracle_lib, method):
    s = write_tet_case(str(tmp_path), lossy_case(method, tolerance=1e-13))
    g, o = pair(s)
    assert np.array_equal(g["t"], o["t"])
    assert np.abs(o["loss"]).max() > 0
    for k in ("v", "U", "flux", "loss"):
        assert rel(g[k], o[k]) <= 1e-10, k


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["gfdtd", "fem"])
def test_conducting_members_at_reference_tolerance(tmp_path, product_lib, oracle_lib, method):
    """CG to 1e-8 as the configurations run it: iteration counts within one of
    the oracle's step by step; FP32 state within 2e-5 of the FP64 oracle."""
    s = write_tet_case(str(tmp_path), lossy_case(method, n=5))
    g, o = pair(s)
    assert np.abs(g["it"] - o["it"]).max() <= 1 and rel(g["v"], o["v"]) <= 1e-8
    g32, _ = pair(s, precision="fp32")
    assert rel(g32["v"], o["v"]) <= 2e-5 and rel(g32["loss"], o["loss"]) <= 2e-5


@pytest.mark.gpu
def test_conducting_and_lossless_members_in_one_batch(tmp_path, product_lib, oracle_lib):
    cases = [lossy_case("gfdtd", steps=40), TetCase(n=4, method="gfdtd", steps=50, seed=5),
             lossy_case("fem", steps=50, n=5, sigma=(0.01, 0.0))]
    scripts = [write_tet_case(str(tmp_path / f"m{i}"), c) for i, c in enumerate(cases)]
    with tb.Batch([(s, 1) for s in scripts], precision="fp64") as b:
        b.step(10 ** 6)
        res = [(b.probes(m), b.state(m)[0]) for m in range(len(scripts))]
    for s, ((t, v), U) in zip(scripts, res):
        o = oracle.TetOracle(s)
        o.run()
        assert np.array_equal(t, o.probes()[0])
        assert rel(v, o.probes()[1]) <= 1e-8 and rel(U, o.state()[0]) <= 1e-8
        o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("sigma,eps", [((0.0, 0.02), (1.5, 3.0)), ((0.02, 0.02), (1.5, 3.0)),
                                       ((0.01, 0.03), (2.0, 2.0))])
def test_conducting_dga_matches_oracle(tmp_path, product_lib, oracle_lib, sigma, eps):
    """Lossless, uniformly conducting and fractured edges on the GPU against
    the oracle's U_frac restatement: FP64 within 1e-10 on probes, U, F and
    flux; FP32 within 2e-5 on the probes and U.  The fully conducting scene
    ends with F decayed far below its peak, so FP32 rounding taken at the peak
    is larger relative to the final F: 1e-4 there and on the flux history.
    The loss column is zero in both."""
    s = write_tet_case(str(tmp_path), lossy_case("dga", sigma=sigma, eps=eps, steps=80))
    o = oracle.TetOracle(s)
    o.run()
    to, vo, _, _ = o.probes()
    Uo, _, Fo = o.state()
    fo, lo = o.flux(), o.losses()
    o.close()
    for prec, tol, tol_f in (("fp64", 1e-10, 1e-10), ("fp32", 2e-5, 1e-4)):
        with tb.Discretization(s) as d:
            d.prepare(1, precision=prec)
            d.step(10 ** 6)
            t, v = d.probes()
            U, _, F = d.state()
            fl, loss = d.flux(), d.losses()
        assert np.array_equal(t, to)
        assert np.abs(vo).max() > 0 and np.abs(fo).max() > 0
        for name, g, r, t_ in (("v", v, vo, tol), ("U", U, Uo, tol), ("F", F, Fo, tol_f), ("flux", fl, fo, tol_f)):
            assert rel(g, r) <= t_, (prec, name, rel(g, r))
        assert np.all(loss == 0) and np.all(lo == 0)


@pytest.mark.gpu
def test_conducting_dga_state_cannot_be_set(tmp_path, product_lib):
    """The node-star fractions of fractured edges are state that U alone does
    not fix, so tf_set_state refuses U on such a run."""
    s = write_tet_case(str(tmp_path), lossy_case("dga", steps=10))
    with tb.Discretization(s) as d:
        d.prepare(1)
        U, _, F = d.state()
        with pytest.raises(tb.TetfitError) as e:
            d.set_state(U, F)
    assert e.value.code == tb.TF_E_UNSUPPORTED


MU0_SCRIPT = 4e-7 * np.pi  # the reference's vacuum permeability


def test_uniform_magnetic_loss_dga_operators(tmp_path, oracle_lib):
    """One material with chi: every face is class 2, the per-tet loss matrix
    is chi / (mu_r mu0) times the magnetic mass, so the F-update operator is
    the lossless N / (1 + b) and R = (1 - b) / (1 + b), b = dt chi / (2 mu_r
    mu0) (CPU, oracle)."""
    ops = {}
    for chi in (0.0, 400.0):
        s = write_tet_case(str(tmp_path / str(chi)), lossy_case("dga", eps=(2.0,), mu=(1.5,), chi=(chi,),
                                                                split_x=False))
        o = oracle.TetOracle(s)
        ops[chi] = (csr(o.matrix("Nmag"), o.nF), o.dga_r(), o.dt)
        o.close()
    N0, (R0, nr0), dt = ops[0.0]
    N1, (R1, nr1), dt1 = ops[400.0]
    assert dt == dt1 and nr0 == 0 and np.all(R0 == 1) and nr1 == len(R1)
    b = dt * 400.0 / (2 * 1.5 * MU0_SCRIPT)
    assert 0.01 < b < 1
    assert np.abs(R1 - (1 - b) / (1 + b)).max() <= 1e-12
    d = N1 - N0 / (1 + b)
    assert abs(d).max() <= 1e-12 * abs(N1).max()


def test_magnetic_loss_damps_the_field(tmp_path, oracle_lib):
    """A pulse in a PEC box filled with one magnetically lossy material ends
    with less field than without (CPU, oracle)."""
    norms = {}
    for chi in (0.0, 400.0):
        s = write_tet_case(str(tmp_path / str(chi)), lossy_case("dga", steps=80, eps=(2.0,), chi=(chi,), split_x=False,
                                                                sigma=(0.0,)))
        o = oracle.TetOracle(s)
        o.run()
        norms[chi] = np.linalg.norm(o.state()[2])
        o.close()
    assert norms[400.0] < 0.5 * norms[0.0]


@pytest.mark.parametrize("method,kw", [("dga", dict(chi=(0.0, 400.0))), ("dga", dict(chi=(400.0, 400.0), mu=(1.0, 2.0))),
                                       ("gfdtd", dict(chi=(400.0, 400.0)))])
def test_oracle_refuses_unsupported_magnetic_losses(tmp_path, oracle_lib, method, kw):
    """dga faces whose tets differ in chi (or in mu, with chi) are fractured in
    the reference, which reads their old values from the electric state
    (:586); gfdtd and fem have no magnetic-loss path that the oracle follows."""
    s = write_tet_case(str(tmp_path), lossy_case(method, **kw))
    with pytest.raises(Exception):
        oracle.TetOracle(s)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(eps=(2.0,), mu=(1.5,), chi=(400.0,), sigma=(0.0,), split_x=False),
                                dict(eps=(1.5, 3.0), chi=(250.0, 250.0), sigma=(0.0, 0.02))])
def test_magnetic_loss_dga_matches_oracle(tmp_path, product_lib, oracle_lib, kw):
    """Class-2 faces (and, in the second scene, conducting and fractured
    edges as well) on the GPU against the oracle's F_frac restatement: FP64
    within 1e-10 on probes, U, F and flux; FP32 within 2e-5 on the probes and
    U, 1e-4 on the decayed F and the flux history."""
    s = write_tet_case(str(tmp_path), lossy_case("dga", steps=80, **kw))
    o = oracle.TetOracle(s)
    o.run()
    to, vo, _, _ = o.probes()
    Uo, _, Fo = o.state()
    fo = o.flux()
    o.close()
    for prec, tol, tol_f in (("fp64", 1e-10, 1e-10), ("fp32", 2e-5, 1e-4)):
        with tb.Discretization(s) as d:
            d.prepare(1, precision=prec)
            d.step(10 ** 6)
            t, v = d.probes()
            U, _, F = d.state()
            fl = d.flux()
        assert np.array_equal(t, to) and np.abs(vo).max() > 0
        for name, g, r, t_ in (("v", v, vo, tol), ("U", U, Uo, tol), ("F", F, Fo, tol_f), ("flux", fl, fo, tol_f)):
            assert rel(g, r) <= t_, (prec, name, rel(g, r))


@pytest.mark.gpu
@pytest.mark.parametrize("method,kw", [("dga", dict(chi=(0.0, 400.0))), ("gfdtd", dict(chi=(400.0, 400.0)))])
def test_unsupported_magnetic_losses_are_refused(tmp_path, product_lib, method, kw):
    s = write_tet_case(str(tmp_path), lossy_case(method, **kw))
    with tb.Discretization(s) as d:
        with pytest.raises(tb.TetfitError) as e:
            d.prepare(1)
    assert e.value.code == tb.TF_E_UNSUPPORTED


def test_dga_mirror_rows_of_the_first_class_edges(tmp_path, oracle_lib):
    """The reference fills a star's class-1 (class-2) rows from the upper
    triangle and mirrors each entry into the row h_index (p_index) of the
    column's edge, which is 0 for an edge of another class (:6546-6547).  So
    on a half-conducting scene every class-1 or class-2 row holds only edges
    that share a node with it, except the rows of the first class-1 and the
    first class-2 edge, which also collect mirror entries of fractured columns
    from all over the mesh (CPU, oracle)."""
    s = write_tet_case(str(tmp_path), lossy_case("dga"))
    o = oracle.TetOracle(s)
    edges, _, cls, _ = o.topology()
    ptr, col, _ = o.matrix("H")
    o.close()
    near = {}
    for e, (a, b) in enumerate(edges):
        near.setdefault(int(a), set()).add(e)
        near.setdefault(int(b), set()).add(e)
    firsts = {int(np.flatnonzero(cls == c)[0]) for c in (1, 2)}
    extra = {}
    for e in np.flatnonzero((cls == 1) | (cls == 2)):
        cols = set(col[ptr[e]:ptr[e + 1]].tolist())
        allowed = near[int(edges[e][0])] | near[int(edges[e][1])]
        extra[int(e)] = cols - allowed
    assert all(not v for e, v in extra.items() if e not in firsts)
    for e in firsts:
        assert extra[e] and all(cls[c] in (1, 2) for c in extra[e])
