"""Generate the golden probe fixtures of tests/test_golden.py with the FP64
CPU oracle (oracle/, pinned to the reference's analytic H-wave by
tests/test_analytic.py):

    python tests/golden/make_golden.py

Each fixture holds, for one seeded small case (tetfit_b200/cases.py), the
probe sample times and the six field components of every 13th probe.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from tetfit_b200.cases import FitCase, Sphere, TetCase, write_fit_cavity, write_tet_case  # noqa: E402

PROBE_STRIDE = 13
CASES = {
    "fit8": ("fit", FitCase(n=8, steps=40)),
    "fit8_lossy_sphere": ("fit", FitCase(n=8, steps=40, spheres=[Sphere((0.5, 0.5, 0.5), 0.2, 4.0, 0.01)])),
    "dga4": ("tet", TetCase(n=4, method="dga", steps=40)),
    "dga4_two_materials": ("tet", TetCase(n=4, method="dga", steps=40, split_x=True, eps=(1.5, 3.0))),
    "gfdtd4": ("tet", TetCase(n=4, method="gfdtd", steps=30)),
}


def script_for(name, directory):
    kind, case = CASES[name]
    if kind == "fit":
        return write_fit_cavity(directory, case)
    return write_tet_case(directory, case)


def oracle_probes(name, directory):
    kind, _ = CASES[name]
    s = script_for(name, directory)
    o = oracle.FitOracle(s) if kind == "fit" else oracle.TetOracle(s)
    o.run()
    t, v, pts, _ = o.probes()
    o.close()
    sel = np.arange(0, len(pts), PROBE_STRIDE)
    return t, v[:, sel, :], pts[sel], sel


def main():
    for name in CASES:
        with tempfile.TemporaryDirectory() as d:
            t, v, pts, sel = oracle_probes(name, d)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), t=t, v=v, pts=pts, sel=sel)
        print(name, v.shape)


if __name__ == "__main__":
    main()
