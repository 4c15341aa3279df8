"""The host set-up's result does not depend on its thread count: the tet
numbering, operators, node-star inverses, classes, probe location and the
Lanczos dt estimate run in parallel loops and sorts whose outputs are fixed
(tetfit_b200/csrc/host_parallel.hpp: stable sorts, inner products as fixed
chunk sums added in chunk order).  A 40^3 Kuhn box (384,000 tets) splits
every loop into several chunks; its prepared state after a few steps is
bitwise equal with 1, 2 and 7 set-up threads."""
import numpy as np
import pytest

import tetfit_b200 as tb
from tetfit_b200.cases import TetCase, write_tet_case


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["dga", "gfdtd"])
def test_setup_is_independent_of_host_threads(tmp_path, product_lib, method):
    # the Lanczos dt estimate runs beside the pinned step and must agree too
    case = TetCase(n=40, method=method, steps=6, split_x=True, eps=(1.5, 3.0))
    s = write_tet_case(str(tmp_path), case)
    runs = []
    for threads in (1, 2, 7):
        with tb.Discretization(s) as d:
            info = d.prepare(1, precision="fp64", host_threads=threads)
            d.step(3)
            U, B, F = d.state()
            runs.append((info["dt_estimate"], info["nnz_operators"], info["nnz_system"], U, B, F))
    dt0 = runs[0][0]
    assert dt0 > 0
    for r in runs[1:]:
        assert r[0] == dt0 and r[1] == runs[0][1] and r[2] == runs[0][2]
        for a, b in zip(r[3:], runs[0][3:]):
            assert np.array_equal(a, b)
    assert np.abs(runs[0][3]).max() > 0
