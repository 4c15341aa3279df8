"""Learned warm-start network: the tensor-core forward and backward kernels
(BF16 operands, FP32 accumulation) against the FP64 CPU oracle
(oracle/mlp.py), through the C ABI."""
import numpy as np
import pytest

import tetfit_b200 as tb
from oracle import mlp as omlp

FWD_TOL = 2e-2   # BF16 operands: about 3 significant digits per product
GRAD_TOL = 3e-2


def batch(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 6)).astype(np.float32)
    t = (0.3 * X[:, 0] - 0.2 * X[:, 4] + 0.1 * rng.standard_normal(n)).astype(np.float32)
    return X, t


def test_param_layout_and_init(product_lib):
    p = tb.mlp_init(7)
    assert p.size == omlp.N_PARAM
    W1 = p[omlp.OFF_W1:omlp.OFF_B1].reshape(64, 16)
    assert np.all(W1[:, 6:] == 0) and np.abs(W1[:, :6]).max() > 0
    assert np.all(p[omlp.OFF_B1:omlp.OFF_W2] == 0) and p[omlp.OFF_B3] == 0
    assert np.array_equal(p, tb.mlp_init(7)) and not np.array_equal(p, tb.mlp_init(8))


@pytest.mark.gpu
def test_forward_matches_oracle(product_lib):
    p = tb.mlp_init(3)
    p[omlp.OFF_W3:omlp.OFF_B3] *= 10  # a larger output to compare
    X, _ = batch(1000, 1)
    y = tb.mlp_forward(p, X)
    yo, _ = omlp.forward(p, X)
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) <= FWD_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1000, 4096])
def test_gradient_matches_oracle(product_lib, n):
    p = tb.mlp_init(11)
    p[omlp.OFF_W3:omlp.OFF_B3] *= 10
    X, t = batch(n, 2)
    w = np.where(np.arange(n) % 7 == 0, 0.0, 1.0).astype(np.float32)  # some rows masked
    g, loss = tb.mlp_gradient(p, X, t, w)
    go, lo = omlp.gradient(p, X, t, w)
    assert abs(loss - lo) <= 1e-2 * lo
    for name, a, b in (("W1", omlp.OFF_W1, omlp.OFF_B1), ("b1", omlp.OFF_B1, omlp.OFF_W2),
                       ("W2", omlp.OFF_W2, omlp.OFF_B2), ("b2", omlp.OFF_B2, omlp.OFF_W3),
                       ("W3", omlp.OFF_W3, omlp.OFF_B3), ("b3", omlp.OFF_B3, omlp.N_PARAM)):
        err = np.linalg.norm(g[a:b] - go[a:b]) / max(np.linalg.norm(go[a:b]), 1e-30)
        assert err <= GRAD_TOL, f"{name}: relative error {err:.3e}"
    assert np.all(g[omlp.OFF_W1:omlp.OFF_B1].reshape(64, 16)[:, 6:] == 0)


def test_oracle_gradient_by_finite_differences():
    """The oracle's analytic backward pass against central differences of its
    own FP64 forward pass (no BF16 rounding)."""
    rng = np.random.default_rng(5)
    p = rng.standard_normal(omlp.N_PARAM) * 0.3
    p[omlp.OFF_W1:omlp.OFF_B1].reshape(64, 16)[:, 6:] = 0
    X, t = batch(20, 3)

    def loss(q):
        y, _ = omlp.forward(q, X, bf16_ops=False)
        return np.mean((y - t) ** 2)

    # analytic gradient without rounding
    import oracle.mlp as m
    saved = m.bf16
    m.bf16 = lambda a: np.asarray(a, dtype=np.float64)
    try:
        g, _ = m.gradient(p, X, t)
    finally:
        m.bf16 = saved
    for i in list(range(0, omlp.N_PARAM, 97)) + [omlp.N_PARAM - 1]:
        if omlp.OFF_W1 <= i < omlp.OFF_B1 and (i - omlp.OFF_W1) % 16 >= 6:
            continue
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (loss(p + e) - loss(p - e)) / 2e-6
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), i
