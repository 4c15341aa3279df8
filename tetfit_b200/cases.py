"""Workload generators: `.fdtd` scripts, solids files and netgen meshes.

TetFIT reads a `.fdtd` script (grammar: README.md:15-211 of the TetFIT
project), a solids file for Cartesian meshes (Discretization.hpp:4219-4345) and
netgen neutral meshes for tetrahedral ones (Discretization.hpp:5924-6101).  No
example inputs ship with TetFIT, so the workloads used by the tests and the
benchmark are generated here from seeds:

* `fit_cavity` -- the unit-cube PEC cavity driven by an H-wave on surface 1
  (z = zmin), surfaces 2-6 PEC, probe grid {0.1,0.1,0.6} x {0.5,1,0.5} x
  {0,0.04,1.05} (156 probes inside the box), optionally with seeded random
  spheres of lossy dielectric over vacuum.
* `kuhn_box` (tetrahedral) -- n^3 cubes cut into 6 Kuhn tetrahedra with
  seeded interior-vertex jitter; see `write_netgen_kuhn`.

Surface labels on the Cartesian grid follow the reference code
(Discretization.hpp:5084-5232): 1 z-, 2 x-, 3 y+, 4 x+, 5 y-, 6 z+.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

C0 = 1.0 / math.sqrt((4 * math.pi * 1e-7) * 8.854187817e-12)


@dataclass
class Sphere:
    center: tuple
    radius: float
    eps_r: float
    sigma: float


@dataclass
class FitCase:
    n: int = 64
    steps: int = 2000
    courant: float = 0.98
    step: float | None = None        # pinned time step (SET step); default 0.95 of the Yee bound x courant
    frequency: float = 2e8
    spheres: list = field(default_factory=list)
    probes: bool = True
    output_name: str = "zsections"
    source_type: str = "h"
    source_surface: int = 1
    pec_surfaces: tuple = (2, 3, 4, 5, 6)
    carrier: str = "sin"

    def dt(self) -> float:
        if self.step is not None:
            return self.step
        h = 1.0 / self.n
        return 0.95 * self.courant * h / (C0 * math.sqrt(3.0))


def write_fit_cavity(directory: str, case: FitCase, name: str = "cavity") -> str:
    """Write `<name>.fdtd` and `<name>_solids.txt`; return the script path."""
    os.makedirs(directory, exist_ok=True)
    solids = os.path.join(directory, f"{name}_solids.txt")
    script = os.path.join(directory, f"{name}.fdtd")
    nmat = 1 + len(case.spheres)
    with open(solids, "w") as f:
        # spheres first: WhichSolid returns the first solid in label order
        for i, s in enumerate(case.spheres):
            f.write(f"DEFINE solid {i + 1}\n   SET material {i + 1}\n   SET type sphere\n")
            f.write("   SET center {%r,%r,%r}\n" % tuple(float(c) for c in s.center))
            f.write(f"   SET radius {s.radius!r}\nEND solid {i + 1}\n")
        f.write(f"DEFINE solid {nmat}\n   SET material {nmat}\n   SET type box\n")
        f.write("   SET corner {0,0,0}\n   SET size {1,1,1}\n")
        f.write(f"END solid {nmat}\n")
    dt = case.dt()
    duration = (case.steps - 1) * dt
    h = 1.0 / case.n
    lines = []
    lines += ["DEFINE mesh 1", "   SET type cartesian",
              "   SET xgrid {0,%r,1}" % h, "   SET ygrid {0,%r,1}" % h, "   SET zgrid {0,%r,1}" % h,
              f"   SET file {os.path.basename(solids)}", "   SET name cavity", "END mesh 1"]
    for i, s in enumerate(case.spheres):
        lines += [f"DEFINE material {i + 1}", f"   SET epsilon {s.eps_r!r}", "   SET mu 1",
                  f"   SET sigma {s.sigma!r}", f"END material {i + 1}"]
    lines += [f"DEFINE material {nmat}", "   SET epsilon 1", "   SET mu 1", "   SET sigma 0",
              f"END material {nmat}"]
    lines += ["DEFINE bc 1"] + [f"   SET surface {s}" for s in case.pec_surfaces] + ["   SET type pec", "END bc 1"]
    lines += ["DEFINE source 1", f"   SET surface {case.source_surface}", f"   SET type {case.source_type}",
              "   SET profile wave", "   SET mode { sin , cos , cos }", "   SET center {0, 0, 0}",
              "   SET direction x", "   SET amplitude 1", f"   SET frequency {case.frequency!r}",
              f"   SET carrier {case.carrier}", "   SET wavevector { 0.5, 0, 0 }", "END source 1"]
    if case.probes:
        lines += ["DEFINE output 1", f"   SET name {case.output_name}", "   SET mode probepoint",
                  "   SET xgrid { 0.1, 0.1,0.6}", "   SET ygrid { 0.5, 1, 0.5}", "   SET zgrid { 0, 0.04, 1.05}",
                  "   SET grid on", "   SET period 0", "END output 1"]
    lines += ["DEFINE simulation 1", "   SET method fdtd", "   SET mesh 1", "   SET source 1",
              f"   SET duration {duration!r}", f"   SET step {dt!r}",
              f"   SET courant {case.courant!r}"]
    if case.probes:
        lines += ["   SET output 1"]
    lines += ["END simulation 1"]
    with open(script, "w") as f:
        f.write("\n".join(lines) + "\n")
    return script


def random_spheres(count: int, seed: int) -> list:
    """Seeded lossy dielectric spheres: radius U[0.02,0.1] m, eps_r U[1,10],
    sigma log-uniform in [1e-4, 1] S/m, centres uniform in the unit cube."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        out.append(Sphere(center=tuple(rng.uniform(0.0, 1.0, 3)), radius=float(rng.uniform(0.02, 0.1)),
                          eps_r=float(rng.uniform(1.0, 10.0)), sigma=float(10 ** rng.uniform(-4, 0))))
    return out
