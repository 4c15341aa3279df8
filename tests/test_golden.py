"""Committed golden probe fixtures (tests/golden/*.npz, made by
tests/golden/make_golden.py with the FP64 CPU oracle, which
tests/test_analytic.py pins to the reference's analytic H-wave).

CPU: the oracle still reproduces every fixture.  GPU: the product, through
the C ABI in FP64, reproduces them within the parity tolerances (1e-10
relative L2 for fdtd and dga; 1e-8 for gfdtd, whose CG stops at 1e-8)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402
import tetfit_b200 as tb  # noqa: E402

NAMES = sorted(make_golden.CASES)


def load(name):
    z = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    return z["t"], z["v"], z["pts"], z["sel"]


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_fixture(tmp_path, name):
    t0, v0, p0, s0 = load(name)
    t, v, p, s = make_golden.oracle_probes(name, str(tmp_path))
    assert np.array_equal(s, s0) and np.array_equal(t, t0) and np.allclose(p, p0, rtol=0, atol=1e-15)
    assert rel(v, v0) <= 1e-12
    assert np.abs(v0).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_reproduces_fixture(tmp_path, product_lib, name):
    t0, v0, p0, s0 = load(name)
    script = make_golden.script_for(name, str(tmp_path))
    with tb.Discretization(script) as d:
        d.prepare(1, precision="fp64", device=0)
        d.step(10 ** 9)
        t, v = d.probes()
        xyz, _ = d.probe_points()
    assert np.array_equal(t, t0)
    assert np.allclose(xyz[s0], p0, rtol=0, atol=1e-15)
    tol = 1e-8 if name.startswith("gfdtd") else 1e-10
    assert rel(v[:, s0, :], v0) <= tol
