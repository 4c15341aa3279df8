"""Discrete leapfrog energy of a lossless cavity after the source has
switched off: a Gaussian carrier exp(-(t-d)^2/w^2) underflows to
exactly 0 some 27 widths after its delay; from then on the H-source surface is
a natural (zero tangential H) boundary and every other face is PEC, so

    W^{n+1/2} = 1/2 U^n . Me . U^{n+1} + 1/2 F^{n+1/2} . Mmu . F^{n+1/2}

(FIT: Me = 1/M_h, Mmu = M_mu; tets: Me = H^-1 on the interior edges for dga,
the eps-mass E for gfdtd, and Mmu F.F = B.N.B) is invariant.  The GPU state is
read through the C ABI; the operators come from the FP64 oracle."""
import numpy as np
import pytest

import oracle
import tetfit_b200 as tb
from tetfit_b200.cases import FitCase, TetCase, write_fit_cavity, write_tet_case

pytestmark = pytest.mark.gpu


def csr(ptr, col, val, ncols):
    import scipy.sparse as sp
    return sp.csr_matrix((val, col.astype(np.int64), ptr.astype(np.int64)), shape=(len(ptr) - 1, ncols))


def test_fit_cavity_energy_drift(tmp_path, product_lib, oracle_lib):
    n = 16
    dt = FitCase(n=n).dt()
    w = 8 * dt
    case = FitCase(n=n, steps=1700, carrier="gaussian", width=w, delay=4 * w, step=dt)
    s = write_fit_cavity(str(tmp_path), case)
    o = oracle.FitOracle(s)
    mh, _, _, mmu = o.coeffs()
    me = np.where(mh != 0, 1.0 / np.where(mh != 0, mh, 1), 0.0)
    off = int(4 * w / dt + 30 * w / dt) + 2  # source term exactly zero from here on
    with tb.Discretization(s) as d:
        d.prepare(1, precision="fp64")
        d.step(off)

        def energy():
            U0, _, F0 = d.state()
            d.step(1)
            U1, _, _ = d.state()
            return 0.5 * np.dot(U0 * me, U1) + 0.5 * np.dot(F0 * mmu, F0)

        w0 = energy()
        d.step(999)
        w1 = energy()
    assert w0 > 0
    assert abs(w1 - w0) / w0 <= 1e-12, f"relative drift {abs(w1 - w0) / w0:.3e}"


def test_fit_gpu_energy_kernel(tmp_path, product_lib, oracle_lib):
    """tf_energy (fit_energy_kernel, FP64 block reduction on the GPU) of the
    state after a step, (U^n, F^{n+1/2}): W^n = 1/2 U^n . Me . U^n +
    1/2 F^{n+1/2} . Mmu . F^{n-1/2} with F^{n-1/2} recomputed from U^n.  It
    matches the same sum formed in numpy from the states read back before and
    after the step, and it is invariant once the source is off.  FP64 and
    FP32 state (FP64 accumulation in both)."""
    n = 16
    dt = FitCase(n=n).dt()
    w = 8 * dt
    case = FitCase(n=n, steps=1700, carrier="gaussian", width=w, delay=4 * w, step=dt,
                   spheres=[])
    s = write_fit_cavity(str(tmp_path), case)
    o = oracle.FitOracle(s)
    mh, _, _, mmu = o.coeffs()
    me = np.where(mh != 0, 1.0 / np.where(mh != 0, mh, 1), 0.0)
    off = int(4 * w / dt + 30 * w / dt) + 2
    # FP32 state: the drift is the state's rounding over 1000 steps (2.5e-5 seen)
    for prec, tol_np, tol_drift in (("fp64", 1e-12, 1e-12), ("fp32", 1e-6, 1e-4)):
        with tb.Discretization(s) as d:
            d.prepare(1, precision=prec)
            d.step(off)
            _, _, Fprev = d.state()
            d.step(1)
            U0, _, F0 = d.state()
            w_gpu = d.energy()
            w_np = 0.5 * np.dot(U0 * me, U0) + 0.5 * np.dot(F0 * mmu, Fprev)
            assert w_np > 0
            assert abs(w_gpu - w_np) / w_np <= tol_np, (prec, w_gpu, w_np)
            d.step(999)
            w_end = d.energy()
        assert abs(w_end - w_gpu) / w_gpu <= tol_drift, f"{prec}: relative drift {abs(w_end - w_gpu) / w_gpu:.3e}"


@pytest.mark.parametrize("method", ["dga", "gfdtd"])
def test_tet_cavity_energy_drift(tmp_path, product_lib, oracle_lib, method):
    import scipy.sparse.linalg as spla
    n = 5
    dt = TetCase(n=n).dt()
    w = 8 * dt
    case = TetCase(n=n, method=method, steps=2800, carrier="gaussian", width=w, delay=4 * w, step=dt,
                   tolerance=1e-14)
    s = write_tet_case(str(tmp_path), case)
    o = oracle.TetOracle(s)
    N = csr(*o.matrix("N"), o.nF)
    _, _, cls, _ = o.topology()
    interior = cls == 1
    if method == "dga":
        H = csr(*o.matrix("H"), o.nE)[interior][:, interior].tocsc()
        solve = spla.factorized(H)
        me_dot = lambda a, b: np.dot(a[interior], solve(b[interior]))
    else:
        E = csr(*o.matrix("E"), o.nE)
        me_dot = lambda a, b: np.dot(a, E @ b)
    off = int(4 * w / dt + 30 * w / dt) + 2
    with tb.Discretization(s) as d:
        # the reference's stopping test, ||r|| <= 1e-14 ||r_0||, r_0 from the
        # previous solution: the oracle drifts 7e-16 over these steps with it
        d.prepare(1, precision="fp64", cg_maxiter=1000)
        d.step(off)

        def energy():
            U0, B0, _ = d.state()
            d.step(1)
            U1, B1, _ = d.state()
            # dga: state after a step is (U^n, B^{n+1/2}); gfdtd: (U^n, B^{n-1/2})
            Bh = B0 if method == "dga" else B1
            return 0.5 * me_dot(U0, U1) + 0.5 * np.dot(Bh, N @ Bh)

        w0 = energy()
        d.step(999)
        w1 = energy()
        if method == "gfdtd":
            # the GPU reduction of W^n = 1/2 U^n.E.U^n + 1/2 B^{n-1/2}.N.B^{n+1/2}
            # (tf_energy): against numpy on the same states, and its drift
            g0 = d.energy()
            U0, B0, _ = d.state()
            d.step(1)
            _, B1, _ = d.state()
            w_np = 0.5 * me_dot(U0, U0) + 0.5 * np.dot(B0, N @ B1)
            assert abs(g0 - w_np) / w_np <= 1e-12, (g0, w_np)
            d.step(998)
            g1 = d.energy()
            assert abs(g1 - g0) / g0 <= 1e-12, f"GPU energy drift {abs(g1 - g0) / g0:.3e}"
        else:
            # dga: W^n = 1/2 U^n.H^-1.U^{n+1} + 1/2 B^{n+1/2}.N.B^{n+1/2} from the
            # current state alone (tf_energy: a PCG solve with H's class-1
            # block on the GPU): against numpy on the same states, and its drift
            g0 = d.energy()
            w_np = energy()
            assert abs(g0 - w_np) / w_np <= 1e-12, (g0, w_np)
            d.step(998)
            g1 = d.energy()
            assert abs(g1 - g0) / g0 <= 1e-12, f"GPU energy drift {abs(g1 - g0) / g0:.3e}"
    assert w0 > 0
    assert abs(w1 - w0) / w0 <= 1e-12, f"{method}: relative drift {abs(w1 - w0) / w0:.3e}"
