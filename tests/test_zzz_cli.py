"""The `tetfit` command-line driver (tetfit_b200/csrc/tetfit_main.cpp), the
B200 counterpart of the reference's src/DGA/main/dga_main.cpp.

CPU: usage, missing file and script errors print the reference's message
text and exit with status 1.  GPU: a run writes the reference's files
(<name><label%05d>_probe_E.dat / _probe_H.dat, poynting.dat; columns x y z t
and three components, width 15, 6 significant digits; H times shifted by half
a step) whose values equal the same simulation read back through the C ABI.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

import tetfit_b200 as tb
from tetfit_b200.cases import FitCase, TetCase, write_fit_cavity, write_tet_case


@pytest.fixture(scope="module")
def cli(product_lib):
    from tetfit_b200 import build
    build.build()
    assert os.access(build.CLI, os.X_OK)
    return build.CLI


def run(cli, args, cwd):
    return subprocess.run([cli] + args, cwd=cwd, capture_output=True, text=True, timeout=600)


def test_cli_without_input_prints_reference_usage(cli, tmp_path):
    r = run(cli, [], tmp_path)
    assert r.returncode == 1
    assert 'Input file error at line 0: Input file missing! Correct use is: "tetfit input_file"' in r.stdout


def test_cli_rejects_extra_arguments_and_unknown_options(cli, tmp_path):
    assert run(cli, ["a.fdtd", "b.fdtd"], tmp_path).returncode == 1
    r = run(cli, ["--fast", "a.fdtd"], tmp_path)
    assert r.returncode == 1 and "unknown option --fast" in r.stdout


def test_cli_reports_missing_script(cli, tmp_path):
    r = run(cli, [str(tmp_path / "missing.fdtd")], tmp_path)
    assert r.returncode == 1
    assert "missing.fdtd" in r.stdout


def test_cli_reports_script_errors_with_reference_text(cli, tmp_path):
    p = tmp_path / "bad.fdtd"
    p.write_text("DEFINE bc 1\n  SET type pmx\nEND bc 1\n")
    r = run(cli, [str(p)], tmp_path)
    assert r.returncode == 1
    assert "Input file error at line 2: " in r.stdout
    assert "Unrecognized boundary condition type" in r.stdout


def read_columns(path):
    rows = [list(map(float, line.split())) for line in open(path) if line.strip()]
    return np.array(rows)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["fit", "gfdtd"])
def test_cli_writes_reference_files(cli, tmp_path, kind):
    src = tmp_path / "case"
    src.mkdir()
    if kind == "fit":
        script = write_fit_cavity(str(src), FitCase(n=8, steps=20))
    else:
        script = write_tet_case(str(src), TetCase(n=4, method="gfdtd", steps=12))
    work = tmp_path / "run"
    work.mkdir()
    r = run(cli, [script], work)
    assert r.returncode == 0, r.stdout + r.stderr
    fe = glob.glob(str(work / "*00001_probe_E.dat"))
    fh = glob.glob(str(work / "*00001_probe_H.dat"))
    assert len(fe) == 1 and len(fh) == 1 and (work / "poynting.dat").exists()
    with tb.Discretization(script) as d:
        info = d.prepare(1, precision="fp64", device=0)
        d.step(10 ** 9)
        t, v = d.probes()
        xyz, _ = d.probe_points()
        flux = d.flux()
        dt = d.info()["dt"]
    ns, npr = v.shape[0], v.shape[1]
    assert ns > 0 and npr > 0
    E, H = read_columns(fe[0]), read_columns(fh[0])
    assert E.shape == (ns * npr, 7) and H.shape == (ns * npr, 7)
    # rows: time-major, probes in order; 6 significant digits
    pts = np.tile(xyz, (ns, 1))
    times = np.repeat(t, npr)
    close = lambda a, b: np.allclose(a, b, rtol=1e-5, atol=1e-300)
    assert close(E[:, :3], pts) and close(H[:, :3], pts)
    assert close(E[:, 3], times)
    shift = 0.5 * dt if kind == "gfdtd" else -0.5 * dt
    assert close(H[:, 3], times + shift)
    assert close(E[:, 4:], v[:, :, :3].reshape(-1, 3))
    assert close(H[:, 4:], v[:, :, 3:].reshape(-1, 3))
    P = read_columns(work / "poynting.dat")
    assert P.shape == (len(flux), 3)
    assert close(P[:, 1], flux)
    assert info is not None


@pytest.mark.gpu
def test_cli_digits_round_trip(cli, tmp_path):
    """--digits 17: the probe files carry the values exactly."""
    src = tmp_path / "case"
    src.mkdir()
    script = write_fit_cavity(str(src), FitCase(n=8, steps=10))
    work = tmp_path / "run"
    work.mkdir()
    r = run(cli, ["--digits", "17", script], work)
    assert r.returncode == 0, r.stdout + r.stderr
    E = read_columns(glob.glob(str(work / "*00001_probe_E.dat"))[0])
    with tb.Discretization(script) as d:
        d.prepare(1, precision="fp64", device=0)
        d.step(10 ** 9)
        t, v = d.probes()
    assert np.array_equal(E[:, 3], np.repeat(t, v.shape[1]))
    assert np.array_equal(E[:, 4:], v[:, :, :3].reshape(-1, 3))
