"""Silo-mode field output (ExportFields "silo", Discretization.hpp:2601-2677):
E (Whitney, at the barycentre, vol_barycenter :10479-10484) and H
(GetMagneticField, :3877-3897) of every tet at each print time, written here
as binary .tfd dumps in place of the Silo files (the Silo library is not part
of this build).  The product's per-tet samples are compared with the FP64
oracle, and the files with the samples they were written from."""
import os

import numpy as np
import pytest

import oracle
import tetfit_b200 as tb
from tetfit_b200.cases import TetCase, write_tet_case


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def read_tfd(path):
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:8] == b"TFDUMP1\0"
    nn, nt, sim, k = np.frombuffer(raw, np.int32, 4, 8)
    t = np.frombuffer(raw, np.float64, 1, 24)[0]
    o = 32
    xyz = np.frombuffer(raw, np.float64, 3 * nn, o).reshape(nn, 3)
    o += 24 * nn
    tets = np.frombuffer(raw, np.int32, 4 * nt, o).reshape(nt, 4)
    o += 16 * nt
    E = np.frombuffer(raw, np.float64, 3 * nt, o).reshape(nt, 3)
    o += 24 * nt
    H = np.frombuffer(raw, np.float64, 3 * nt, o).reshape(nt, 3)
    assert o + 24 * nt == len(raw)
    return dict(sim=int(sim), k=int(k), t=float(t), xyz=xyz, tets=tets, E=E, H=H)


def test_oracle_samples_every_tet_in_silo_mode(tmp_path, oracle_lib):
    """The oracle's silo run samples every tet at every print time of the
    probepoint schedule, and the samples carry the field (CPU)."""
    runs = {}
    for mode in ("probepoint", "silo"):
        s = write_tet_case(str(tmp_path / mode), TetCase(n=3, method="dga", steps=20, output_mode=mode))
        o = oracle.TetOracle(s)
        o.run()
        runs[mode] = (o.nT, o.n_probes, o.probes())
        o.close()
    nT, np_silo, (t, v, xyz, _) = runs["silo"]
    assert np_silo == nT and v.shape == (len(t), nT, 6)
    assert np.array_equal(t, runs["probepoint"][2][0])
    assert np.all(np.isfinite(v)) and np.abs(v[-1, :, :3]).max() > 0 and np.abs(v[-1, :, 3:]).max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["dga", "gfdtd", "fem"])
def test_silo_samples_match_oracle(tmp_path, product_lib, oracle_lib, method):
    case = TetCase(n=4, method=method, steps=40, tolerance=1e-13, output_mode="silo", output_period=4 * TetCase(
        n=4, method=method).dt())
    s = write_tet_case(str(tmp_path), case)
    o = oracle.TetOracle(s)
    o.run()
    to, vo, po, _ = o.probes()
    nT = o.nT
    o.close()
    with tb.Discretization(s) as d:
        d.prepare(1, precision="fp64")
        d.step(10 ** 6)
        t, v = d.probes()
        xyz, _ = d.probe_points()
    assert v.shape[1] == nT and np.array_equal(t, to) and np.array_equal(xyz, po)
    assert np.abs(vo).max() > 0
    assert rel(v, vo) <= 1e-10


@pytest.mark.gpu
def test_silo_dump_files(tmp_path, product_lib, monkeypatch):
    """tf_run in silo mode writes one .tfd per print time, named like the
    reference's Silo files (<name><simulation>_<dump>), holding the mesh and
    the per-tet E and H the run sampled."""
    case = TetCase(n=3, method="gfdtd", steps=12, output_mode="silo", output_period=3 * TetCase(
        n=3, method="gfdtd").dt())
    s = write_tet_case(str(tmp_path), case)
    monkeypatch.chdir(tmp_path)
    with tb.Discretization(s) as d:
        d.run_simulation(1, precision="fp64", write_files=True)
        t, v = d.probes()
        xyz, _ = d.probe_points()
    files = sorted(f for f in os.listdir(tmp_path) if f.endswith(".tfd"))
    assert files == [f"zsections00001_{k:05d}.tfd" for k in range(len(t))] and len(t) >= 3
    for k, f in enumerate(files):
        r = read_tfd(tmp_path / f)
        assert r["sim"] == 1 and r["k"] == k and r["t"] == t[k]
        assert np.array_equal(r["E"], v[k, :, :3]) and np.array_equal(r["H"], v[k, :, 3:])
        # the barycentres of the written tets are the sample points
        bary = r["xyz"][r["tets"]].sum(axis=1) / 4.0
        assert np.allclose(bary, xyz, rtol=0, atol=1e-15)
        # ExportMesh's orientation: every written tet has positive volume
        p = r["xyz"][r["tets"]]
        vol = np.einsum("ij,ij->i", p[:, 1] - p[:, 0], np.cross(p[:, 2] - p[:, 0], p[:, 3] - p[:, 0]))
        assert np.all(vol > 0)
