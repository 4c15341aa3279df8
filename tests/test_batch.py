"""Batches of gfdtd simulations (tf_batch_*): members of different mesh sizes,
materials, sources and time steps advanced by one launch sequence and one
persistent CG kernel per step, each checked against its own FP64 CPU oracle
run and against the same member run alone."""
import os

import numpy as np
import pytest

import oracle
import tetfit_b200 as tb
from tetfit_b200.cases import TetCase, write_tet_case


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def members(tmp, specs, **kw):
    out = []
    for i, (n, e1, e2, f) in enumerate(specs):
        case = TetCase(n=n, method="gfdtd", split_x=True, eps=(e1, e2), frequency=f, seed=100 + i, **kw)
        out.append((write_tet_case(os.path.join(str(tmp), f"m{i}"), case), 1))
    return out


SPECS = [(4, 1.0, 3.5, 2e8), (6, 2.5, 1.2, 3.7e8), (5, 1.7, 4.0, 1.1e8)]


def test_batch_reports_the_failing_member(tmp_path, product_lib):
    ms = members(tmp_path, SPECS[:1], steps=5)
    with pytest.raises(tb.TetfitError) as e:
        tb.Batch(ms + [(os.path.join(str(tmp_path), "missing.fdtd"), 1)])
    assert e.value.code == tb.TF_E_SCRIPT and "batch member 1" in e.value.message
    dga = write_tet_case(os.path.join(str(tmp_path), "dga"), TetCase(n=3, method="dga", steps=5))
    with pytest.raises(tb.TetfitError) as e:
        tb.Batch([(dga, 1)])
    assert e.value.code == tb.TF_E_ARG and "gfdtd" in e.value.message
    with pytest.raises(tb.TetfitError) as e:
        tb.Batch(ms, batch_mode=2)
    assert e.value.code == tb.TF_E_ARG


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["group", "serial"])
def test_batch_fp64_members_match_oracle(tmp_path, product_lib, oracle_lib, mode):
    ms = members(tmp_path, SPECS, steps=60)
    with tb.Batch(ms, precision="fp64", batch_mode=mode) as b:
        assert b.step(1000) == 60
        got = []
        for m in range(b.size):
            t, v = b.probes(m)
            U, B, F = b.state(m)
            it, res = b.solver_stats(m)
            got.append((b.info(m), t, v, U, B, F, it, res))
    for (script, _), (info, t, v, U, B, F, it, res) in zip(ms, got):
        o = oracle.TetOracle(script)
        o.step(o.n_steps)
        to, vo, _, _ = o.probes()
        Uo, Bo, Fo = o.state()
        ito, _ = o.cg()
        assert info["dt"] == o.dt and info["step_index"] == o.n_steps
        assert np.array_equal(t, to)
        assert np.abs(it - ito).max() <= 1 and np.mean(it == ito) >= 0.95
        assert np.nanmax(res) <= 1e-8
        for a, c, k in ((v, vo, "probes"), (U, Uo, "U"), (B, Bo, "B"), (F, Fo, "F")):
            assert rel(a, c) <= 1e-8, k


@pytest.mark.gpu
def test_batch_group_equals_members_alone(tmp_path, product_lib):
    """The group image and one image per member give the same fields: the CG
    sums per member, so only the block partition's rounding differs."""
    ms = members(tmp_path, SPECS, steps=40)
    out = {}
    for mode in ("group", "serial"):
        with tb.Batch(ms, precision="fp64", batch_mode=mode) as b:
            b.step(40)
            out[mode] = [(b.probes(m)[1], b.state(m)[0], b.solver_stats(m)[0]) for m in range(b.size)]
    for (vg, Ug, ig), (vs, Us, is_) in zip(out["group"], out["serial"]):
        assert np.abs(ig - is_).max() <= 1
        assert rel(vg, vs) <= 1e-8 and rel(Ug, Us) <= 1e-8


@pytest.mark.gpu
def test_batch_fp32_error_bound(tmp_path, product_lib, oracle_lib):
    ms = members(tmp_path, SPECS, steps=60)
    with tb.Batch(ms, precision="fp32", cg_criterion="rhs") as b:
        b.step(60)
        res = [(b.probes(m)[1], b.state(m)[0]) for m in range(b.size)]
    for (script, _), (v, U) in zip(ms, res):
        o = oracle.TetOracle(script)
        o.step(o.n_steps)
        assert rel(v, o.probes()[1]) <= 1e-5
        assert rel(U, o.state()[0]) <= 1e-5


@pytest.mark.gpu
def test_batch_members_of_different_lengths(tmp_path, product_lib):
    """A member that reaches its last step stops while the others go on; the
    others' results do not depend on it."""
    long_ = members(tmp_path / "a", SPECS[:2], steps=50)
    short = members(tmp_path / "b", SPECS[2:], steps=20)
    with tb.Batch(long_ + short, precision="fp64") as b:
        assert b.step(30) == 30
        assert b.info(2)["step_index"] == 20 and b.info(0)["step_index"] == 30
        b.step(100)
        assert [b.info(m)["step_index"] for m in range(3)] == [50, 50, 20]
        mixed = [b.state(m)[0] for m in range(2)]
        assert len(b.solver_stats(2)[0]) == 20
    with tb.Batch(long_, precision="fp64") as b:
        b.step(50)
        alone = [b.state(m)[0] for m in range(2)]
    for a, c in zip(mixed, alone):
        assert rel(a, c) <= 1e-8


@pytest.mark.gpu
def test_batch_step_io_host_buffers(tmp_path, product_lib):
    ms = members(tmp_path, SPECS, steps=12)
    with tb.Batch(ms, precision="fp64") as b:
        nsrc = [b.info(m)["n_sources"] for m in range(b.size)]
        npr = [b.info(m)["n_probes"] for m in range(b.size)]
        out = np.full(6 * sum(npr), np.nan)
        for _ in range(5):
            assert b.step_io(None, out) == 1
        t, v = b.probes(1)
        o1 = 6 * npr[0]
        assert np.array_equal(out[o1:o1 + 6 * npr[1]], v[-1].ravel())
        zero = np.zeros(sum(nsrc))
        b.step_io(zero, out)
        assert b.info(0)["step_index"] == 6


@pytest.mark.gpu
def test_batch_step_io_routes_each_members_carriers(tmp_path, product_lib):
    """tf_batch_step_io moves every member's carrier values for the step in
    one host-to-device copy and scatters them to the members: a batch driven
    with per-member values matches each member driven alone through
    tf_step_io with its own values (CG to 1e-13, so the two reduction orders
    agree far below the bound), and the probe samples it returns are the
    ones the members record."""
    ms = members(tmp_path, SPECS, steps=30, tolerance=1e-13)
    rng = np.random.default_rng(7)
    steps = 20
    with tb.Batch(ms, precision="fp64") as b:
        nsrc = [b.info(m)["n_sources"] for m in range(b.size)]
        npr = [b.info(m)["n_probes"] for m in range(b.size)]
        car = rng.uniform(-1.0, 1.0, (steps, sum(nsrc)))
        out = np.zeros(6 * sum(npr))
        for k in range(steps):
            b.step_io(car[k], out)
        got = [(b.state(m)[0], b.probes(m)[1]) for m in range(b.size)]
        last = out.copy()
    offs = np.cumsum([0] + nsrc)
    poffs = np.cumsum([0] + [6 * p for p in npr])
    for m, (script, _) in enumerate(ms):
        with tb.Discretization(script) as d:
            d.prepare(1, precision="fp64")
            po = np.zeros(6 * npr[m])
            for k in range(steps):
                d.step_io(car[k, offs[m]:offs[m + 1]], po)
            U = d.state()[0]
            v = d.probes()[1]
        assert np.abs(U).max() > 0
        assert rel(got[m][0], U) <= 1e-11 and rel(got[m][1], v) <= 1e-11
        assert np.array_equal(last[poffs[m]:poffs[m + 1]], got[m][1][-1].ravel())
