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
* `kuhn_mesh` / `write_tet_case` (tetrahedral) -- n^3 cubes cut into 6 Kuhn
  tetrahedra with seeded interior-vertex jitter, written in netgen format.

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
    output_mode: str = "probepoint"  # "l2norm" turns on the reference's FIT Joule-loss column
    source_type: str = "h"
    source_surface: int = 1
    pec_surfaces: tuple = (2, 3, 4, 5, 6)
    carrier: str = "sin"
    width: float | None = None       # gaussian carrier width (s)
    delay: float | None = None       # carrier delay (s)
    profile: str = "wave"            # spatial profile: wave (mode/wavevector) or gaussian (center, radius)
    amplitude: float = 1.0
    center: tuple = (0.0, 0.0, 0.0)
    radius: float | None = None      # gaussian profile radius (m)
    decay: float | None = None       # radial decay exponent about the centre
    direction: str = "x"

    def dt(self) -> float:
        if self.step is not None:
            return float(self.step)
        h = 1.0 / self.n
        return 0.95 * self.courant * h / (C0 * math.sqrt(3.0))


def source_lines(case) -> list:
    """The `source 1` block of a generated script (Source.hpp:60-300)."""
    c = tuple(float(x) for x in case.center)
    lines = ["DEFINE source 1", f"   SET surface {case.source_surface}", f"   SET type {case.source_type}",
             f"   SET profile {case.profile}", "   SET mode { sin , cos , cos }",
             "   SET center {%r, %r, %r}" % c, f"   SET direction {case.direction}",
             f"   SET amplitude {float(case.amplitude)!r}", f"   SET frequency {case.frequency!r}",
             f"   SET carrier {case.carrier}", "   SET wavevector { 0.5, 0, 0 }"]
    if case.width is not None:
        lines += [f"   SET width {float(case.width)!r}"]
    if case.delay is not None:
        lines += [f"   SET delay {float(case.delay)!r}"]
    if case.radius is not None:
        lines += [f"   SET radius {float(case.radius)!r}"]
    if case.decay is not None:
        lines += [f"   SET decay {float(case.decay)!r}"]
    return lines + ["END source 1"]


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
    dt = float(case.dt())
    duration = float((case.steps - 1) * dt)
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
    lines += source_lines(case)
    if case.probes:
        lines += ["DEFINE output 1", f"   SET name {case.output_name}", f"   SET mode {case.output_mode}",
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


# --------------------------------------------------------------- tetrahedral
# Kuhn (Freudenthal) subdivision of a cube into 6 tetrahedra sharing the main
# diagonal; node bits: 1 = +x, 2 = +y, 4 = +z.  The same split in every cube
# keeps the mesh conforming.
KUHN_TETS = ((0, 1, 3, 7), (0, 1, 5, 7), (0, 2, 3, 7), (0, 2, 6, 7), (0, 4, 5, 7), (0, 4, 6, 7))
# domain-surface labels of the generated meshes: 1 z-, 2 x-, 3 y-, 4 x+, 5 y+, 6 z+
SURFACE_LABELS = {("z", 0): 1, ("x", 0): 2, ("y", 0): 3, ("x", 1): 4, ("y", 1): 5, ("z", 1): 6}


def kuhn_mesh(n: int, jitter: float = 0.15, seed: int = 0x7E7F17, material=None):
    """Points [(n+1)^3, 3], tets [6 n^3, 4] (0-based), tet materials, boundary
    triangles [(12 n^2), 3] and their labels, for the unit cube cut into n^3
    cubes of 6 Kuhn tetrahedra.  Interior vertices are moved by
    U[-jitter*h, jitter*h]^3 (seeded); boundary vertices stay on the box.
    `material(centroids) -> labels` assigns tet materials (default 1)."""
    h = 1.0 / n
    g = np.arange(n + 1) * h
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pts = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    idx = np.arange((n + 1) ** 3).reshape((n + 1, n + 1, n + 1), order="F")  # idx[i,j,k]
    rng = np.random.default_rng(seed)
    interior = np.ones((n + 1,) * 3, dtype=bool)
    interior[[0, -1], :, :] = False
    interior[:, [0, -1], :] = False
    interior[:, :, [0, -1]] = False
    inter = interior.ravel(order="F")
    shift = rng.uniform(-jitter * h, jitter * h, size=(int(inter.sum()), 3))
    pts[inter] += shift
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    i, j, k = i.ravel(order="F"), j.ravel(order="F"), k.ravel(order="F")
    corner = [idx[i + (b & 1), j + ((b >> 1) & 1), k + ((b >> 2) & 1)] for b in range(8)]
    tets = np.stack([np.stack([corner[a], corner[b], corner[c], corner[d]], 1) for (a, b, c, d) in KUHN_TETS],
                    1).reshape(-1, 4)
    cent = pts[tets].mean(axis=1)
    mats = np.ones(len(tets), dtype=np.int64) if material is None else np.asarray(material(cent), dtype=np.int64)
    # boundary triangles: the Kuhn faces lying on the box
    tris, labels = [], []
    faces = np.concatenate([tets[:, [0, 1, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 3]], tets[:, [1, 2, 3]]])
    fp = pts[faces]
    for axis, name in enumerate("xyz"):
        for side in (0, 1):
            on = np.all(np.abs(fp[:, :, axis] - side) < 1e-12, axis=1)
            tris.append(faces[on])
            labels.append(np.full(int(on.sum()), SURFACE_LABELS[(name, side)]))
    return pts, tets, mats, np.concatenate(tris), np.concatenate(labels)


def write_netgen(path: str, pts, tets, mats, tris, labels, coord_fmt: str = "%.17g") -> str:
    """Netgen neutral format as TetFIT reads it (Discretization.hpp:5924-6101,
    6612-6654): point count + coordinates, tetrahedron count + `mat p1..p4`,
    triangle count + `label p1 p2 p3`, all node indices 1-based."""
    with open(path, "w") as f:
        f.write(f"{len(pts)}\n")
        np.savetxt(f, pts, fmt=coord_fmt)
        f.write(f"{len(tets)}\n")
        np.savetxt(f, np.column_stack([mats, tets + 1]), fmt="%d")
        f.write(f"{len(tris)}\n")
        np.savetxt(f, np.column_stack([labels, tris + 1]), fmt="%d")
    return path


def write_gmsh(path: str, pts, tets, mats, tris, labels) -> str:
    """ASCII gmsh 2.2 mesh, the layout TetFIT's gmsh conversion reads
    (Discretization.hpp:5692-5866): nodes at full precision, then triangles
    (type 2) and tetrahedra (type 4), each with two tags (physical =
    elementary = the boundary id or material), node indices 1-based."""
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n")
        f.write(f"{len(pts)}\n")
        np.savetxt(f, np.column_stack([np.arange(1, len(pts) + 1), pts]), fmt=["%d", "%.17g", "%.17g", "%.17g"])
        f.write("$EndNodes\n$Elements\n")
        f.write(f"{len(tris) + len(tets)}\n")
        ids = np.arange(1, len(tris) + len(tets) + 1)
        nt = len(tris)
        np.savetxt(f, np.column_stack([ids[:nt], np.full(nt, 2), np.full(nt, 2), labels, labels, tris + 1]), fmt="%d")
        nv = len(tets)
        np.savetxt(f, np.column_stack([ids[nt:], np.full(nv, 4), np.full(nv, 2), mats, mats, tets + 1]), fmt="%d")
        f.write("$EndElements\n")
    return path


@dataclass
class TetCase:
    n: int = 24
    method: str = "gfdtd"            # "dga" (explicit), "gfdtd" or "fem" (PCG each step)
    steps: int = 200
    courant: float = 0.98
    step: float | None = None        # pinned time step; default from the Kuhn-mesh bound below
    tolerance: float = 1e-8
    frequency: float = 2e8
    jitter: float = 0.15
    seed: int = 0x7E7F17
    eps: object = (1.0,)             # eps_r per material label 1, 2, ... (tuple) or {label: eps_r}
    sigma: object = None             # conductivity (S/m) per material label, like eps (None: lossless)
    chi: object = None               # magnetic conductivity per material label, like eps (None: 0)
    mu: object = None                # mu_r per material label, like eps (None: 1)
    split_x: bool = False            # material 1 for x < 0.5, 2 for x >= 0.5
    pec_surfaces: tuple = (2, 3, 4, 5, 6)
    source_surface: int = 1
    source_type: str = "h"
    carrier: str = "sin"
    probes: bool = True
    mat_field: object = None         # optional callable centroids -> labels
    width: float | None = None       # gaussian carrier width (s)
    delay: float | None = None       # carrier delay (s)
    profile: str = "wave"            # spatial profile: wave or gaussian
    amplitude: float = 1.0
    center: tuple = (0.0, 0.0, 0.0)
    radius: float | None = None
    decay: float | None = None
    direction: str = "x"
    mesh_format: str = "netgen"      # "netgen" or "gmsh"
    coord_fmt: str = "%.17g"         # netgen coordinates ("%g": the 6 digits a gmsh conversion keeps)
    output_mode: str = "probepoint"  # "silo": per-tet field dumps at every print time
    output_period: float = 0.0       # SET period of the output (0: every step)

    def dt(self) -> float:
        if self.step is not None:
            return float(self.step)
        # 0.25 h / c0: below the stability limit of the jittered Kuhn meshes
        # for dga and gfdtd; fem (Whitney mass) is stable to about 0.21 h / c0
        return (0.15 if self.method == "fem" else 0.25) * (1.0 / self.n) / C0


def write_tet_case(directory: str, case: TetCase, name: str = "box") -> str:
    os.makedirs(directory, exist_ok=True)
    if case.mat_field is not None:
        material = case.mat_field
    elif case.split_x:
        material = lambda c: np.where(c[:, 0] < 0.5, 1, 2)
    else:
        material = None
    geo = kuhn_mesh(case.n, case.jitter, case.seed, material)
    if case.mesh_format == "gmsh":
        mesh = write_gmsh(os.path.join(directory, f"{name}.msh"), *geo)
    else:
        mesh = write_netgen(os.path.join(directory, f"{name}.mesh"), *geo, coord_fmt=case.coord_fmt)
    dt = float(case.dt())
    duration = float((case.steps - 1) * dt if case.method == "dga" else case.steps * dt)
    lines = ["DEFINE mesh 1", "   SET type tetrahedral", f"   SET mesher {case.mesh_format}",
             f"   SET file {os.path.basename(mesh)}", "   SET name box", "   SET scalefactor 1", "END mesh 1"]
    eps_items = case.eps.items() if isinstance(case.eps, dict) else enumerate(case.eps, start=1)
    per_label = lambda v: dict(v.items() if isinstance(v, dict) else enumerate(v or (), start=1))
    sig, chi, mu = per_label(case.sigma), per_label(case.chi), per_label(case.mu)
    for m, e in eps_items:
        lines += [f"DEFINE material {m}", f"   SET epsilon {float(e)!r}", f"   SET mu {float(mu.get(m, 1.0))!r}",
                  f"   SET sigma {float(sig.get(m, 0.0))!r}", f"   SET chi {float(chi.get(m, 0.0))!r}",
                  f"END material {m}"]
    lines += ["DEFINE bc 1"] + [f"   SET surface {s}" for s in case.pec_surfaces] + ["   SET type pec", "END bc 1"]
    lines += source_lines(case)
    if case.probes:
        lines += ["DEFINE output 1", "   SET name zsections", f"   SET mode {case.output_mode}",
                  "   SET xgrid { 0.1, 0.1,0.6}", "   SET ygrid { 0.5, 1, 0.5}", "   SET zgrid { 0, 0.04, 1.05}",
                  "   SET grid on", f"   SET period {case.output_period!r}", "END output 1"]
    lines += ["DEFINE simulation 1", f"   SET method {case.method}", "   SET solver cg",
              f"   SET tolerance {case.tolerance!r}", "   SET mesh 1", "   SET source 1",
              f"   SET duration {duration!r}", f"   SET step {dt!r}", f"   SET courant {case.courant!r}"]
    if case.probes:
        lines += ["   SET output 1"]
    lines += ["END simulation 1"]
    script = os.path.join(directory, f"{name}.fdtd")
    with open(script, "w") as f:
        f.write("\n".join(lines) + "\n")
    return script


def grf_materials(k_levels: int = 24, corr: float = 0.1, seed: int = 4242, grid: int = 64,
                  lo: float = 1.0, hi: float = 12.0):
    """Seeded 3-D Gaussian random field on the unit cube (Gaussian covariance
    of correlation length `corr`, by FFT filtering of white noise on a
    periodic `grid`^3 lattice), mapped affinely to [lo, hi] and quantised to
    `k_levels` materials.  Returns (material(centroids) -> labels,
    {label: eps_r}, max quantisation error).  Labels skip 7, which TetFIT
    drops (Discretization.hpp:6091), and stay below 100."""
    assert k_levels <= 97
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((grid,) * 3)
    f = np.fft.fftfreq(grid, d=1.0 / grid)
    kx, ky, kz = np.meshgrid(f, f, f, indexing="ij")
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2) * (corr ** 2) / 2)
    field = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    field = (field - field.min()) / (field.max() - field.min())
    eps = lo + (hi - lo) * field
    edges = np.linspace(lo, hi, k_levels + 1)
    centres = 0.5 * (edges[:-1] + edges[1:])
    labels = [l for l in range(1, k_levels + 2) if l != 7][:k_levels]
    table = {labels[q]: float(centres[q]) for q in range(k_levels)}
    qerr = float((hi - lo) / k_levels / 2)

    def material(cent):
        ijk = np.clip((cent * grid).astype(int), 0, grid - 1)
        e = eps[ijk[:, 0], ijk[:, 1], ijk[:, 2]]
        q = np.clip(((e - lo) / (hi - lo) * k_levels).astype(int), 0, k_levels - 1)
        return np.asarray(labels)[q]

    return material, table, qerr


def batch_cases(count: int = 128, n_lo: int = 8, n_hi: int = 48, steps: int = 1000, seed: int = 31337,
                tolerance: float = 1e-8, probes: bool = True) -> list:
    """Independent gfdtd runs for a batch: mesh n ~ U{n_lo..n_hi} cubes per
    side (6 Kuhn tetrahedra each, interior vertices jittered +-0.15 h by a
    per-member seed), eps_r ~ U[1,4] on each x-half (materials 1 and 2), PEC on
    surfaces 2-6, an H-wave source on surface 1 with f ~ U[1e8,4e8] Hz, the
    member's own pinned step 0.25 h / c0 and `steps` steps each."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(n_lo, n_hi + 1))
        e1, e2 = (float(v) for v in rng.uniform(1.0, 4.0, 2))
        f = float(rng.uniform(1e8, 4e8))
        out.append(TetCase(n=n, method="gfdtd", steps=steps, split_x=True, eps=(e1, e2), frequency=f,
                           seed=int(rng.integers(1, 2 ** 31)), tolerance=tolerance, probes=probes))
    return out


def _write_member(arg):
    directory, i, case = arg
    return write_tet_case(os.path.join(directory, f"m{i:04d}"), case)


def write_batch(directory: str, cases: list, processes: int = 0) -> list:
    """Write every member's mesh and script (in parallel worker processes);
    return [(script path, simulation label 1), ...] in member order."""
    import multiprocessing as mp
    args = [(directory, i, c) for i, c in enumerate(cases)]
    procs = processes or min(len(cases), os.cpu_count() or 1, 32)
    if procs <= 1:
        paths = [_write_member(a) for a in args]
    else:
        with mp.get_context("spawn").Pool(procs) as pool:
            paths = pool.map(_write_member, args, chunksize=1)
    return [(p, 1) for p in paths]
