"""Standalone Jacobi-PCG (tf_pcg_solve): SPD systems, both stopping criteria,
the iteration-limit status, and agreement with a CPU reference solve."""
import numpy as np
import pytest

import tetfit_b200 as tb


def laplacian_csr(m, shift=0.1, seed=0):
    """SPD 2-D five-point Laplacian plus a random positive diagonal."""
    rng = np.random.default_rng(seed)
    n = m * m
    rows, cols, vals = [], [], []
    for i in range(m):
        for j in range(m):
            r = i * m + j
            rows.append(r); cols.append(r); vals.append(4.0 + shift + rng.uniform(0, 0.5))
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                ii, jj = i + di, j + dj
                if 0 <= ii < m and 0 <= jj < m:
                    rows.append(r); cols.append(ii * m + jj); vals.append(-1.0)
    order = np.lexsort((cols, rows))
    rows, cols, vals = np.array(rows)[order], np.array(cols)[order], np.array(vals)[order]
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(ptr, rows + 1, 1)
    return np.cumsum(ptr), cols.astype(np.int32), vals


def test_pcg_symbol_exported(product_lib):
    assert hasattr(product_lib, "tf_pcg_solve")


def test_pcg_bad_arguments_report_status(product_lib):
    a = tb.PcgArgs(n=0)
    import ctypes
    it, rs = ctypes.c_int32(), ctypes.c_double()
    assert product_lib.tf_pcg_solve(ctypes.byref(a), ctypes.byref(it), ctypes.byref(rs)) == tb.TF_E_ARG
    assert "tf_pcg_solve" in tb.last_thread_error()


@pytest.mark.gpu
@pytest.mark.parametrize("criterion", [0, 1])
def test_pcg_solves_spd_system(product_lib, criterion):
    import torch
    ptr, col, val = laplacian_csr(40)
    n = len(ptr) - 1
    rng = np.random.default_rng(1)
    b = rng.standard_normal(n)
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    rc, it, rs = tb.pcg_solve(t(ptr), t(col), t(val), t(b), x, tol=1e-10, criterion=criterion)
    assert rc == tb.TF_OK, tb.last_thread_error()
    assert 0 < it < 100
    A = np.zeros((n, n))
    for r in range(n):
        A[r, col[ptr[r]:ptr[r + 1]]] = val[ptr[r]:ptr[r + 1]]
    xs = np.linalg.solve(A, b)
    assert np.linalg.norm(x.cpu().numpy() - xs) / np.linalg.norm(xs) < 1e-8


@pytest.mark.gpu
def test_pcg_iteration_limit_returns_status(product_lib):
    import torch
    ptr, col, val = laplacian_csr(60, shift=0.0)
    n = len(ptr) - 1
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    b = t(np.ones(n))
    rc, it, rs = tb.pcg_solve(t(ptr), t(col), t(val), b, x, tol=1e-14, maxiter=5)
    assert rc == tb.TF_E_SOLVER and it == 5 and rs > 1e-14
    assert "iteration limit" in tb.last_thread_error()
    # warm start from the partial solution converges
    rc, it2, rs2 = tb.pcg_solve(t(ptr), t(col), t(val), b, x, tol=1e-10)
    assert rc == tb.TF_OK and rs2 <= 1e-10
