"""Learned CG warm start (warm_start "learned"): the per-edge network trains
on the solver's own solutions during the first learn_steps steps, then its
guess competes with the polynomial extrapolation at every step (the smaller
initial residual wins).  CG still runs to the same tolerance, so the fields
agree with the other warm starts; the tests record the iterations gained."""
import numpy as np
import pytest

import oracle
import tetfit_b200 as tb
from tetfit_b200.cases import TetCase, write_tet_case

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def run(script, steps, **opts):
    with tb.Discretization(script) as d:
        d.prepare(1, cg_criterion="rhs", **opts)
        d.step(steps)
        it, res = d.solver_stats()
        out = dict(it=it, res=res, v=d.probes()[1], U=d.state()[0])
        if opts.get("warm_start") == "learned":
            out["kept"] = d.guess_stats()
            out["loss"] = d.training_loss()
    return out


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-6), ("fp32", 1e-5)])
def test_learned_guess_trains_and_keeps_the_solution(tmp_path, product_lib, oracle_lib, prec, tol):
    steps, learn = 360, 120
    s = write_tet_case(str(tmp_path), TetCase(n=14, method="gfdtd", steps=steps, split_x=True, eps=(1.5, 3.0)))
    ext = run(s, steps, precision=prec, warm_start="extrapolate")
    lrn = run(s, steps, precision=prec, warm_start="learned", learn_steps=learn)
    # same tolerance (||r|| <= 1e-8 ||b||, reached well inside the iteration limit), same fields
    assert lrn["it"].max() < 100
    assert rel(lrn["v"], ext["v"]) <= tol and rel(lrn["U"], ext["U"]) <= tol
    o = oracle.TetOracle(s)
    o.step(steps)
    assert rel(lrn["v"], o.probes()[1]) <= max(tol, 1e-5)
    # training: the loss falls; afterwards the network's guess is used on some steps
    loss = lrn["loss"]
    assert len(loss) >= learn and np.all(np.isfinite(loss))
    assert np.mean(loss[-20:]) < np.mean(loss[:20])
    assert np.all(lrn["kept"][:learn] == 0)
    after = slice(learn + 5, steps)
    it_l, it_e = lrn["it"][after].mean(), ext["it"][after].mean()
    print(f"\n{prec}: mean CG iterations after training: learned {it_l:.2f}, extrapolation {it_e:.2f}, "
          f"network guess kept on {100 * lrn['kept'][after].mean():.0f}% of the steps")
    # never worse than the extrapolation it falls back to (one iteration of slack for rounding)
    assert it_l <= it_e + 0.5


def test_learned_guess_in_a_batch(tmp_path, product_lib, oracle_lib):
    members = []
    for i, (n, e1, e2, f) in enumerate([(6, 1.0, 3.0, 2e8), (9, 2.0, 1.2, 3e8)]):
        c = TetCase(n=n, method="gfdtd", steps=150, split_x=True, eps=(e1, e2), frequency=f, seed=50 + i)
        members.append((write_tet_case(str(tmp_path / f"m{i}"), c), 1))
    with tb.Batch(members, precision="fp32", cg_criterion="rhs", warm_start="learned", learn_steps=60) as b:
        b.step(150)
        res = [(b.probes(m)[1], b.guess_stats(m)) for m in range(b.size)]
        loss = b.training_loss()
        p = b.mlp_params()
    assert len(loss) >= 60 and np.all(np.isfinite(p))
    for (script, _), (v, kept) in zip(members, res):
        o = oracle.TetOracle(script)
        o.step(o.n_steps)
        assert rel(v, o.probes()[1]) <= 1e-5
        assert len(kept) == 150 and np.all(kept[:60] == 0)
