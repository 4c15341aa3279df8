"""tf_pcg_solve_noalloc against tf_pcg_solve, through the C ABI.

The no-allocation entry point exists for callers that cannot allocate device
memory while they solve: a host whose own pool allocator already holds the
GPU's memory, where a cudaMalloc would fail or fragment that pool, and loops
that must not stall other streams, since cudaMalloc and cudaFree can
synchronize the device.  Its work space is a fixed file-scope device array, so
these tests check that it returns what the allocating entry point returns, on
consecutive calls that reuse the array, and that it refuses systems larger than
the array.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

import tetfit_b200 as tb

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # same kernel and reduction order: results agree to rounding


def spd_csr(m, seed):
    """Five-point Laplacian on an m x m grid with a random positive diagonal shift."""
    rng = np.random.default_rng(seed)
    n = m * m
    rows, cols, vals = [], [], []
    for i in range(m):
        for j in range(m):
            r = i * m + j
            rows.append(r); cols.append(r); vals.append(4.2 + rng.uniform(0.0, 0.5))
            for di, dj in ((1, 0), (-1, 0), (0, 1), (0, -1)):
                ii, jj = i + di, j + dj
                if 0 <= ii < m and 0 <= jj < m:
                    rows.append(r); cols.append(ii * m + jj); vals.append(-1.0)
    order = np.lexsort((cols, rows))
    rows, cols, vals = np.array(rows)[order], np.array(cols)[order], np.array(vals)[order]
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(ptr, rows + 1, 1)
    return np.cumsum(ptr), cols.astype(np.int32), vals


def call(fn, ptr, col, val, b, x, tol=1e-10):
    args = tb.PcgArgs(n=int(ptr.numel() - 1), device=0, row_ptr=ptr.data_ptr(), col=col.data_ptr(),
                      val=val.data_ptr(), b=b.data_ptr(), x=x.data_ptr(), tol=tol, maxiter=0, criterion=0,
                      stream=None)
    it, rs = ctypes.c_int32(), ctypes.c_double()
    rc = fn(ctypes.byref(args), ctypes.byref(it), ctypes.byref(rs))
    return rc, it.value, rs.value


def test_noalloc_matches_allocating_solve_twice(product_lib):
    import torch
    dev = torch.device("cuda:0")
    ptr_h, col_h, val_h = spd_csr(48, seed=3)
    n = len(ptr_h) - 1
    ptr = torch.from_numpy(ptr_h).to(dev)
    col = torch.from_numpy(col_h).to(dev)
    val = torch.from_numpy(val_h).to(dev)
    rng = np.random.default_rng(11)
    for call_no in range(2):  # two calls in a row share the static work space
        b = torch.from_numpy(rng.standard_normal(n)).to(dev)
        x_ref = torch.zeros(n, dtype=torch.float64, device=dev)
        rc_ref, it_ref, rs_ref = call(product_lib.tf_pcg_solve, ptr, col, val, b, x_ref)
        assert rc_ref == tb.TF_OK, tb.last_thread_error()
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        rc, it, rs = call(product_lib.tf_pcg_solve_noalloc, ptr, col, val, b, x)
        assert rc == tb.TF_OK, f"call {call_no}: {tb.last_thread_error()}"
        assert it == it_ref and rs <= 1e-10
        err = (torch.linalg.norm(x - x_ref) / torch.linalg.norm(x_ref)).item()
        assert err <= REL_TOL, f"call {call_no}: relative difference {err:.3e}"


def test_noalloc_rejects_systems_above_its_work_space(product_lib):
    import torch
    n = (1 << 18) + 1
    dev = torch.device("cuda:0")
    ptr = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    col = torch.zeros(1, dtype=torch.int32, device=dev)
    val = torch.zeros(1, dtype=torch.float64, device=dev)
    b = torch.zeros(n, dtype=torch.float64, device=dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)
    rc, _, _ = call(product_lib.tf_pcg_solve_noalloc, ptr, col, val, b, x)
    assert rc == tb.TF_E_ARG
    assert "exceeds the static work space" in tb.last_thread_error()
