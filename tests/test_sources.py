"""Source paths (Discretization.hpp:3907-4202, Source::Compute Source.hpp:313-567):
electric, magnetic and current-density sources, every carrier (sin, cos with
its amplitude-squared quirk, gaussian, ricker), the wave and gaussian
spatial profiles and the radial decay, on FIT, dga and gfdtd, product
against the FP64 oracle (GPU), plus CPU pins of the oracle's carrier
arithmetic."""
import numpy as np
import pytest

import oracle
import tetfit_b200 as tb
from tetfit_b200.cases import FitCase, TetCase, write_fit_cavity, write_tet_case


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


SOURCES = {
    "h_cos_amp2": dict(source_type="h", carrier="cos", amplitude=2.0),
    "h_ricker": dict(source_type="h", carrier="ricker", delay=4e-9),
    "h_gaussian_carrier": dict(source_type="h", carrier="gaussian", width=1.5e-9, delay=4e-9),
    "h_gaussian_profile": dict(source_type="h", profile="gaussian", center=(0.5, 0.5, 0.0), radius=0.3),
    "h_decay": dict(source_type="h", decay=1.0, center=(0.5, 0.5, -0.25)),
    "e_cos": dict(source_type="e", carrier="cos", amplitude=1.5),
    "e_gaussian_profile": dict(source_type="e", profile="gaussian", center=(0.5, 0.5, 0.0), radius=0.4),
    "j_sin": dict(source_type="j"),
    "j_ricker": dict(source_type="j", carrier="ricker", delay=4e-9),
}


def fit_pair(script, steps):
    o = oracle.FitOracle(script)
    o.step(steps)
    to, vo, _, _ = o.probes()
    Uo, _, Fo = o.state()
    with tb.Discretization(script) as d:
        d.prepare(1, precision="fp64")
        d.step(steps)
        t, v = d.probes()
        U, _, F = d.state()
        fl = d.flux()
    return (t, v, U, F, fl), (to, vo, Uo, Fo, o.flux())


def tet_pair(script, steps):
    o = oracle.TetOracle(script)
    o.step(steps)
    to, vo, _, _ = o.probes()
    Uo, _, Fo = o.state()
    with tb.Discretization(script) as d:
        d.prepare(1, precision="fp64")
        d.step(steps)
        t, v = d.probes()
        U, _, F = d.state()
        fl = d.flux()
    return (t, v, U, F, fl), (to, vo, Uo, Fo, o.flux())


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SOURCES))
def test_fit_sources_match_oracle(tmp_path, product_lib, oracle_lib, name):
    s = write_fit_cavity(str(tmp_path), FitCase(n=10, steps=80, **SOURCES[name]))
    g, o = fit_pair(s, 80)
    assert np.array_equal(g[0], o[0])
    if SOURCES[name]["source_type"] == "j":
        # the FIT loop sets I only on the source-surface edges, which it never
        # updates (Discretization.hpp:1855-1861): the fields stay exactly zero
        assert not o[1].any() and not o[2].any()
        assert not g[1].any() and not g[2].any() and not g[3].any()
        return
    assert np.abs(o[1]).max() > 0 and np.abs(o[2]).max() > 0
    for k, nm in enumerate(("t", "probes", "U", "F", "flux")[1:], start=1):
        assert rel(g[k], o[k]) <= 1e-10, nm


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["dga", "gfdtd"])
@pytest.mark.parametrize("name", sorted(SOURCES))
def test_tet_sources_match_oracle(tmp_path, product_lib, oracle_lib, method, name):
    s = write_tet_case(str(tmp_path), TetCase(n=4, method=method, steps=60, tolerance=1e-13, **SOURCES[name]))
    g, o = tet_pair(s, 60)
    assert np.array_equal(g[0], o[0])
    assert np.abs(o[2]).max() > 0
    for k, nm in enumerate(("t", "probes", "U", "F", "flux")[1:], start=1):
        assert rel(g[k], o[k]) <= 1e-10, nm


def test_cos_carrier_squares_the_amplitude(tmp_path, oracle_lib):
    """Source.hpp:315-322: ret = amp, then `cos` multiplies by amp again, so
    the fields of a zero-started linear run scale with amp^2 for cos and with
    amp for sin (CPU, oracle)."""
    def probes(carrier, amp, sub):
        d = tmp_path / sub
        s = write_fit_cavity(str(d), FitCase(n=8, steps=40, carrier=carrier, amplitude=amp))
        o = oracle.FitOracle(s)
        o.run()
        return o.probes()[1]

    c1, c2 = probes("cos", 1.0, "c1"), probes("cos", 2.0, "c2")
    s1, s2 = probes("sin", 1.0, "s1"), probes("sin", 2.0, "s2")
    assert np.abs(c1).max() > 0 and np.abs(s1).max() > 0
    assert rel(c2, 4.0 * c1) <= 1e-13
    assert rel(s2, 2.0 * s1) <= 1e-13


def test_ricker_and_gaussian_carriers(tmp_path, oracle_lib):
    """Source.hpp:323-326 carrier shapes in the oracle: a gaussian carrier
    delayed by a thousand widths underflows to exactly zero, so the fields
    stay zero; a ricker pulse excites them (CPU, oracle)."""
    dt = FitCase(n=8).dt()
    s = write_fit_cavity(str(tmp_path / "g"), FitCase(n=8, steps=30, carrier="gaussian", width=dt,
                                                      delay=1000 * dt))
    o = oracle.FitOracle(s)
    o.run()
    assert not o.probes()[1].any()
    s = write_fit_cavity(str(tmp_path / "r"), FitCase(n=8, steps=30, carrier="ricker", delay=4e-9))
    o = oracle.FitOracle(s)
    o.run()
    assert np.abs(o.probes()[1]).max() > 0
