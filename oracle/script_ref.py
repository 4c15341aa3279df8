"""ORACLE -- test infrastructure only.  A second, independent reading of
TetFIT's `.fdtd` script front end, written in Python from the reference's
sources (not from either C++ parser in this repository), so that a misreading
of the grammar in one C++ copy shows up as a disagreement.

Follows:
* the line loop, Discretization.hpp:45-211 -- `sscanf("%s %s %s")` into
  fixed buffers that keep their previous contents when a line has fewer
  tokens (a blank-looking line repeats the previous instruction), a brace
  value re-joined from the line's first '{' to its first '}' (:144-161), the
  bc surface table BndToBC of 100 slots (:61, :119-128);
* the setters Material.hpp:51-170, BoundaryCondition.hpp:47-122,
  Source.hpp:60-300, Output.hpp:58-298, Simulation.hpp:52-97 (SET source
  adds to the default source 1, then sorts and removes duplicates),
  Mesh.hpp:46-203, Solid.hpp:47-233;
* the solids file reader, Discretization.hpp:4219-4345;
* constants Utilities.hpp:92-95 (mu0 evaluated in long double);
* error texts Utilities.hpp:275-317, "Input file error at line N: " prefix
  Utilities.hpp:371-375.

Numbers are converted with the C library's strtod / strtof / strtol (through
ctypes), which is what std::stod / std::stof / std::stoi / std::atoi call.

`parse_script(path)` returns a plain dict (see `_canonical`), the same shape
that the product's `tf_script_dump` and the oracle's `orc_script_dump` print
as JSON.  Documented divergences of the C++ parsers that this module mirrors:
a mesh file that is missing from the working directory is looked up next to
the script; a bc surface label >= 100 is an error instead of a write past the
100-slot table.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

_libc = ctypes.CDLL(None)
_libc.strtod.restype = ctypes.c_double
_libc.strtod.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
_libc.strtol.restype = ctypes.c_long
_libc.strtol.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int]

PI_L = np.longdouble("3.141592653589793238")
MU0 = float(np.float64(np.longdouble(4) * PI_L * np.longdouble(1e-7)))
EPS0 = 8.854187817e-12

DEFINABLES = ["material", "source", "mesh", "bc", "simulation", "geometry", "output", "refinement"]
MESH_DEFINABLES = ["grid", "solid"]
SOLID_TYPES = ["sphere", "box", "cylinder"]
SOURCE_TYPES = ["e", "b", "j", "h", "d"]
PROFILES = ["wave", "gaussian", "const"]
CARRIERS = ["sin", "cos", "gaussian", "dc", "ricker"]
DIRECTIONS = ["x", "y", "z", "r", "psi", "rho", "phi", "theta"]
BC_DIRECTIONS = ["+x", "+y", "+z", "r", "+t", "rho", "-t", "-x", "-y", "-z"]
MODES = ["sin", "cos"]
MESH_TYPES = ["tetrahedral", "cartesian", "none"]
MESHERS = ["netgen", "gmsh", "none"]
OUTPUT_MODES = ["silo", "probepoint", "maxerror", "l2norm"]
METHODS = ["fdtd", "dga", "fem", "dgao2", "frac", "gfdtd", "fraco2", "fdtdo2"]
SOLVERS = ["cg", "agmg"]


class M:  # error texts, Utilities.hpp:278-317
    bc_unknown_type = "Unrecognized boundary condition type! Available: pec, pmc, pml"
    bc_unknown_parameter = "Unrecognized boundary condition parameter! Available: type"
    bc_unknown_direction = "Unrecognized direction! Available: +-x, +-y, +-z, r, +-t, rho"
    src_unknown_direction = "Unrecognized direction! Available: x, y, z"
    src_unknown_type = ("Unrecognized source type!"
                        "Available: e (electric field), b (magnetic field), j (current density)")
    src_unknown_profile = "Unrecognized source profile! Available: const, wave, gaussian"
    src_unknown_carrier = "Unrecognized source carrier! Available: dc, sin, cos, gaussian, ricker"
    coordinates_syntax = "coordinates must be inside braces {...,..,..}"
    unbalanced_bracket = "unbalanced bracket"
    too_many_coords = "Maximum of three coordinates!"
    too_few_coords = "Undefined end to list of coordinates!"
    src_unknown_bf = "Unrecognized base function! Available: sin, cos"
    src_unknown_parameter = "unrecognized parameter for source!"
    material_unknown_parameter = "Unrecognized material parameter! Available: epsilon, mu, sigma, chi"
    mesh_unknown_type = "Undefined mesh type! Available: tetrahedral, cartesian"
    mesh_inexistent_file = "Mesh input file does not exist or it is not in specified path"
    mesh_unknown_mesher = "Undefined mesher! Available: netgen, gmsh"
    mesh_unknown_parameter = "Undefined mesh parameter! Available: file, name, type, mesher, scalefactor"
    sim_unknown_output = "Undefined output mode type! Available: silo, probepoint, maxerror, l2norm"
    sim_unknown_method = "Undefined simulation method! Available: fdtd, dga, fem"
    sim_unknown_solver = "Unavailable solver! Available: cg, agmg"
    sim_unknown_parameter = "Undefined simulation parameter! Available: source, mesh, duration, output"
    out_unknown_parameter = "Undefined output parameter! Available: mode, period, probe, name"
    sim_invalid_coord_system = "Invalid system of coordinates! Available: cartesian, cylindrical, spherical"
    set_wo_define = "define something before setting variables"
    unknown_define = ("can only define one of the following: material, mesh, refinement, boundary condition, "
                      "simulation, output, source")
    grid_unknown_define = "Unknown primivite: can only define solid inside cartesian meshes"
    end_wo_define = "ending unopened definition"
    unknown_instruction = "Unknown instruction inside define block"
    unexpected_end = "File ended unexpectedly before ending definition"
    solid_unknown_parameter = "Unrecognized solid parameter! Available: type, radius, center, corner, size"
    solid_unknown_type = "Unavailable solid type! Available: sphere, box, cylinder"
    solid_negative_value = "Positive definite quantity forced to negative value!"


class ScriptError(Exception):
    pass


def my_throw(line: int, msg: str):
    raise ScriptError(f"Input file error at line {line}: {msg}")


# ------------------------------------------------------------ number parsing
def _conv(fn, s: str, *extra):
    b = s.encode()
    end = ctypes.c_char_p()
    buf = ctypes.create_string_buffer(b)
    endp = ctypes.cast(ctypes.byref(end), ctypes.POINTER(ctypes.c_char_p))
    v = fn(ctypes.cast(buf, ctypes.c_char_p), endp, *extra)
    used = ctypes.cast(end, ctypes.c_void_p).value - ctypes.addressof(buf)
    return v, used


def stod(s: str) -> float:
    v, used = _conv(_libc.strtod, s)
    if used == 0:
        raise ValueError(f"stod: no conversion of {s!r}")
    return float(v)


def stof(s: str) -> float:
    """std::stof: strtof to a float, widened to double where it is stored."""
    v, used = _conv(_libc.strtof, s)
    if used == 0:
        raise ValueError(f"stof: no conversion of {s!r}")
    return float(np.float32(v))


def stoi(s: str) -> int:
    v, used = _conv(_libc.strtol, s, 10)
    if used == 0:
        raise ValueError(f"stoi: no conversion of {s!r}")
    return int(v)


def atoi(s: str) -> int:
    v, _ = _conv(_libc.strtol, s, 10)
    return int(ctypes.c_int(v).value)


def u32(x) -> int:
    """Store a double or int into a uint32_t member (truncation, modulo 2^32)."""
    return int(x) % (1 << 32)


# --------------------------------------------------------- brace lists
def brace_items(line: int, value: str, keep_spaces: bool = True):
    """The coordinate-list loop of the setters (e.g. Source.hpp:90-130):
    items between '{' and '}' separated by ','; spaces dropped for `mode`."""
    if not value or value[0] != "{":
        my_throw(line, M.coordinates_syntax)
    items = []
    i = 1
    n = len(value)
    while i < n and value[i] != "," and value[i] != "}":
        coord = ""
        while i < n and value[i] != "," and value[i] != "}":
            if keep_spaces or value[i] != " ":
                coord += value[i]
            i += 1
        if i == n:
            my_throw(line, M.unbalanced_bracket)
        items.append(coord)
        if value[i] == ",":
            i += 1
    if i == n:
        my_throw(line, M.too_few_coords)
    return items


def three(line: int, value: str, conv, keep_spaces: bool = True):
    items = brace_items(line, value, keep_spaces)
    out = []
    for k, c in enumerate(items):
        if k >= 3:
            my_throw(line, M.too_many_coords)
        out.append(conv(c))
    return out


# ------------------------------------------------------------ primitives
def eye(d):
    return [[d if r == c else 0.0 for c in range(3)] for r in range(3)]


def new_material():
    return dict(eps=eye(EPS0), mu=eye(MU0), sigma=eye(0.0), chi=eye(0.0))


def set_material(m, line, p, v):
    scal = {"epsilon": ("eps", EPS0), "mu": ("mu", MU0), "sigma": ("sigma", None), "chi": ("chi", None)}
    off = {"xy": (0, 1), "xz": (0, 2), "yz": (1, 2)}
    if p in scal:
        key, f = scal[p]
        x = stod(v)
        m[key] = eye(f * x if f is not None else x)
        return
    base, _, suf = p.partition("_")
    if base in scal and suf in off:
        key = scal[base][0]
        r, c = off[suf]
        m[key][r][c] = m[key][c][r] = stod(v)     # no eps0/mu0 factor (Material.hpp:58-61)
        return
    vec = {"eps_vec": ("eps", EPS0), "mu_vec": ("mu", MU0), "sigma_vec": ("sigma", None),
           "chi_vec": ("chi", None)}
    if p in vec:
        key, f = vec[p]
        items = brace_items(line, v)
        for k, c in enumerate(items):
            if k >= 3:
                my_throw(line, M.too_many_coords)
            x = stod(c)
            m[key][k][k] = f * x if f is not None else x
        return
    my_throw(line, M.material_unknown_parameter)


def new_bc():
    return dict(type="none", dir="none", width=0.0, val=0.0, surfs=[])


def set_bc(b, line, p, v):
    if p == "type":
        if v in ("pml", "pmc", "pec"):
            b["type"] = v
            if v != "pml":
                b["val"] = 0.0
        else:
            my_throw(line, M.bc_unknown_type)
    elif p == "direction":
        if v not in BC_DIRECTIONS:
            my_throw(line, M.bc_unknown_direction)
        b["dir"] = v
    elif p == "width":
        b["width"] = stod(v)
    elif p == "surface":
        b["surfs"].append(stoi(v))
    elif p == "surfaces":
        if not v or v[0] != "{":
            my_throw(line, M.coordinates_syntax)
        i, n = 1, len(v)
        while i < n and v[i] != "}":
            coord = ""
            while i < n and v[i] != "," and v[i] != "}":
                coord += v[i]
                i += 1
            if i == n:
                my_throw(line, M.unbalanced_bracket)
            b["surfs"].append(stoi(coord))
            if v[i] == ",":
                i += 1
        if i == n:
            my_throw(line, M.unbalanced_bracket)
    else:
        my_throw(line, M.bc_unknown_parameter)


def new_source():
    return dict(st=" ", prof="dc", carrier="sin", dir="x", amp=0.0, freq=0.0, radius=1.0, decay=0.0, width=1.0,
                delay=0.0, impedance=50.0, kvec=[0.0, 0.0, 0.0], center=[0.0, 0.0, 0.0],
                location=[0.0, 0.0, 0.0], bfuncs=["cos", "cos", "cos"], surfaces=[])


def set_source(s, line, p, v):
    choice = {"direction": ("dir", DIRECTIONS, M.src_unknown_direction),
              "type": ("st", SOURCE_TYPES, M.src_unknown_type),
              "profile": ("prof", PROFILES, M.src_unknown_profile),
              "carrier": ("carrier", CARRIERS, M.src_unknown_carrier)}
    scalar = {"amplitude": "amp", "delay": "delay", "impedance": "impedance", "frequency": "freq",
              "radius": "radius", "decay": "decay", "width": "width"}
    if p in choice:
        key, allowed, msg = choice[p]
        if v not in allowed:
            my_throw(line, msg)
        s[key] = v
    elif p in ("center", "wavevector", "location"):
        key = {"center": "center", "wavevector": "kvec", "location": "location"}[p]
        for k, x in enumerate(three(line, v, stod)):
            s[key][k] = x
    elif p == "mode":
        for k, x in enumerate(three(line, v, str, keep_spaces=False)):
            s["bfuncs"][k] = x
    elif p in ("Xmode", "Ymode", "Zmode"):
        if v not in MODES:
            my_throw(line, M.src_unknown_bf)
        s["bfuncs"]["XYZ".index(p[0])] = v
    elif p in scalar:
        s[scalar[p]] = stod(v)
    elif p in ("kx", "ky", "kz"):
        s["kvec"]["xyz".index(p[1])] = stod(v)
    elif p == "surface":
        s["surfaces"].append(stoi(v))
    else:
        my_throw(line, M.src_unknown_parameter)


def new_output():
    return dict(mode="none", name="simulation", period=0.0, nextprint=1e-15, delay=0.0, ref_sys=0,
                xstart=0.0, xstep=0.0, xstop=0.0, ystart=0.0, ystep=0.0, ystop=0.0,
                zstart=0.0, zstep=0.0, zstop=0.0, probes=[], radiators=[])


def set_output(o, line, p, v):
    if p == "mode":
        if v not in OUTPUT_MODES:
            my_throw(line, M.sim_unknown_output)
        o["mode"] = v
    elif p == "radiator":
        o["radiators"].append(u32(stof(v)))
    elif p == "delay":
        o["nextprint"] = o["delay"] = stod(v)
    elif p == "coordinates":
        if v not in ("cartesian", "cylindrical", "spherical"):
            my_throw(line, M.sim_invalid_coord_system)
        o["ref_sys"] = ("cartesian", "cylindrical", "spherical").index(v)
    elif p == "probe":
        pt = three(line, v, stof)
        o["probes"].append(pt + [0.0] * (3 - len(pt)))
    elif p == "period":
        o["period"] = stof(v)
    elif p in ("xgrid", "ygrid", "zgrid"):
        a = p[0]
        for k, x in enumerate(three(line, v, stof)):
            o[a + ("start", "step", "stop")[k]] = x
    elif p == "grid":
        if v == "on":
            z = o["zstart"]
            while z <= o["zstop"]:
                y = o["ystart"]
                while y <= o["ystop"]:
                    x = o["xstart"]
                    while x <= o["xstop"]:
                        o["probes"].append([x, y, z])
                        x += o["xstep"]
                    y += o["ystep"]
                z += o["zstep"]
        elif v != "off":
            my_throw(line, M.out_unknown_parameter)
    elif p == "error":
        if v not in ("on", "off"):
            my_throw(line, M.out_unknown_parameter)
    elif p == "name":
        o["name"] = v
    else:
        my_throw(line, M.out_unknown_parameter)


def new_simulation():
    return dict(duration=0.0, courant=1.0, step=0.0, tol=1e-8, method="dga", solver="none", analytic="false",
                debug=False, sources=[1], mesh=1, output=0)


def set_simulation(s, line, p, v):
    if p == "source":
        s["sources"] = sorted(set(s["sources"] + [u32(stod(v))]))
    elif p == "mesh":
        s["mesh"] = u32(stod(v))
    elif p == "duration":
        s["duration"] = stod(v)
    elif p == "courant":
        s["courant"] = stod(v)
    elif p == "step":
        s["step"] = stod(v)
    elif p == "output":
        s["output"] = u32(stod(v))
    elif p == "method":
        if v not in METHODS:
            my_throw(line, M.sim_unknown_method)
        s["method"] = v
    elif p == "solver":
        if v not in SOLVERS:
            my_throw(line, M.sim_unknown_solver)
        s["solver"] = v
    elif p == "tolerance":
        s["tol"] = stod(v)
    elif p == "analytic":
        s["analytic"] = v
    elif p == "debug":
        if v not in ("true", "false"):
            my_throw(line, M.sim_unknown_parameter)
        s["debug"] = v == "true"
    else:
        my_throw(line, M.sim_unknown_parameter)


def new_mesh():
    return dict(file="none", name="none", type="none", mesher="none", scale=1.0,
                xmin=0.0, xstep=0.0, xmax=0.0, ymin=0.0, ystep=0.0, ymax=0.0, zmin=0.0, zstep=0.0, zmax=0.0)


def set_mesh(m, line, p, v, base_dir):
    if p == "file":
        path = v
        if not os.path.isfile(path) and path and not path.startswith("/") and base_dir:
            alt = base_dir + "/" + path
            if os.path.isfile(alt):
                path = alt
        if not os.path.isfile(path):
            my_throw(line, M.mesh_inexistent_file)
        m["file"] = path
    elif p == "name":
        m["name"] = v
    elif p == "type":
        if v not in MESH_TYPES:
            my_throw(line, M.mesh_unknown_type)
        m["type"] = v
    elif p == "mesher":
        if v not in MESHERS:
            my_throw(line, M.mesh_unknown_mesher)
        m["mesher"] = v
    elif p in ("xgrid", "ygrid", "zgrid"):
        a = p[0]
        for k, x in enumerate(three(line, v, stod)):
            m[a + ("min", "step", "max")[k]] = x
    elif p == "scalefactor":
        m["scale"] = stod(v)
    else:
        my_throw(line, M.mesh_unknown_parameter)


def new_solid():
    return dict(type="none", material=0, sqr=0.0, center=[0.0, 0.0, 0.0], corner=[0.0, 0.0, 0.0],
                size=[0.0, 0.0, 0.0])


def set_solid(s, line, p, v):
    pre = "In cartesian mesh definition file: "
    try:
        if p == "type":
            if v not in SOLID_TYPES:
                my_throw(line, M.solid_unknown_type)
            s["type"] = v
        elif p == "material":
            s["material"] = u32(atoi(v))
        elif p == "radius":
            r = stod(v)
            if r <= 0:
                my_throw(line, M.solid_negative_value)
            s["sqr"] = r ** 2
        elif p in ("center", "corner", "size"):
            for k, x in enumerate(three(line, v, stod)):
                if p == "size" and x < 0:
                    my_throw(line, M.solid_negative_value)
                s[p][k] = x
        else:
            my_throw(line, M.solid_unknown_parameter)
    except ScriptError as e:
        raise ScriptError(pre + str(e)) from None


# ----------------------------------------------------------- line loop
class _Tokens:
    """The three sscanf buffers; tokens a line does not supply keep their
    previous contents (Discretization.hpp:73)."""

    def __init__(self):
        self.t = ["", "", ""]

    def scan(self, line: str):
        words = [w for w in re.split(r"[ \t\n\v\f\r]+", line) if w]   # C isspace
        for k, w in enumerate(words[:3]):
            self.t[k] = w
        return self.t


def _lines(path):
    with open(path, "rb") as f:
        data = f.read().decode("latin-1")
    # std::getline splits on '\n' only; a final line without '\n' still counts
    parts = data.split("\n")
    if parts and parts[-1] == "":
        parts.pop()
    return parts


def _rejoin(line_no, line, value_buf, val):
    if value_buf[:1] != "{":
        return val
    i = line.find("{")
    j = line.find("}", i)
    if j < 0:
        my_throw(line_no, M.unbalanced_bracket)
    return line[i:j + 1]


def parse_script(path: str) -> dict:
    base_dir = os.path.dirname(path)
    out = dict(materials={}, bcs={}, meshes={}, sources={}, simulations={}, outputs={}, bnd_to_bc=[0] * 100)
    tok = _Tokens()
    in_def = False
    thing, label = "", 0
    line_no = 1
    makers = dict(material=("materials", new_material), bc=("bcs", new_bc), mesh=("meshes", new_mesh),
                  source=("sources", new_source), simulation=("simulations", new_simulation),
                  output=("outputs", new_output))
    for line in _lines(path):
        if len(line) > 0 and line[0] != "#" and line[0] != "\n":
            action, token, value = tok.scan(line)
            if action[:1] != "#":
                if not in_def:
                    if action != "DEFINE":
                        my_throw(line_no, M.set_wo_define)
                    if token not in DEFINABLES:
                        my_throw(line_no, M.unknown_define)
                    thing = token
                    label = u32(stoi(value))
                    in_def = True
                    if thing in makers:
                        key, mk = makers[thing]
                        out[key][label] = mk()
                elif action == "END":
                    if token != thing or u32(atoi(value)) != label:
                        my_throw(line_no, M.end_wo_define)
                    in_def = False
                    if thing == "bc":
                        for sf in out["bcs"][label]["surfs"]:
                            if not 0 <= sf < 100:
                                raise ScriptError(f"bc surface label {sf} outside the 100-slot label table")
                            out["bnd_to_bc"][sf] = label
                elif action != "SET":
                    my_throw(line_no, M.unknown_instruction)
                else:
                    val = _rejoin(line_no, line, value, value)
                    if thing == "material":
                        set_material(out["materials"][label], line_no, token, val)
                    elif thing == "bc":
                        set_bc(out["bcs"][label], line_no, token, val)
                    elif thing == "mesh":
                        set_mesh(out["meshes"][label], line_no, token, val, base_dir)
                    elif thing == "source":
                        set_source(out["sources"][label], line_no, token, val)
                    elif thing == "simulation":
                        set_simulation(out["simulations"][label], line_no, token, val)
                    elif thing == "output":
                        set_output(out["outputs"][label], line_no, token, val)
                    elif thing in ("refinement", "geometry"):
                        raise ScriptError("refinement/geometry primitives are outside the time-stepping path")
                    else:
                        my_throw(line_no, M.unknown_define)
        line_no += 1
    if in_def:
        my_throw(line_no, M.unexpected_end)
    return _canonical(out)


def read_solids(path: str) -> dict:
    pre = "In cartesian mesh definition file: "

    def thr(n, m):
        raise ScriptError(pre + f"Input file error at line {n}: {m}")

    solids = {}
    tok = _Tokens()
    in_def = False
    thing, label = "", 0
    line_no = 1
    for line in _lines(path):
        if len(line) > 0 and line[0] != "#" and line[0] != "\n":
            action, token, value = tok.scan(line)
            if action[:1] != "#":
                if not in_def:
                    if action != "DEFINE":
                        thr(line_no, M.set_wo_define)
                    if token not in MESH_DEFINABLES:
                        thr(line_no, M.grid_unknown_define)
                    thing = token
                    label = u32(stod(value))
                    in_def = True
                    if thing == "solid":
                        solids[label] = new_solid()
                elif action == "END":
                    if token != thing or u32(atoi(value)) != label:
                        thr(line_no, M.end_wo_define)
                    in_def = False
                elif action != "SET":
                    thr(line_no, M.unknown_instruction)
                else:
                    val = _rejoin(line_no, line, value, value)
                    if thing == "solid":
                        set_solid(solids[label], line_no, token, val)
                    else:
                        thr(line_no, M.grid_unknown_define)
        line_no += 1
    if in_def:
        thr(line_no, M.unexpected_end)
    return {str(k): solids[k] for k in sorted(solids)}


def _canonical(d: dict) -> dict:
    """Maps keyed by label strings in ascending label order, the shape the
    C++ dumps print."""
    res = {}
    for k, v in d.items():
        if isinstance(v, dict):
            res[k] = {str(lab): v[lab] for lab in sorted(v)}
        else:
            res[k] = v
    for o in res["outputs"].values():
        o.pop("radiators", None)
    res["solids"] = {lab: read_solids(m["file"]) for lab, m in res["meshes"].items()
                     if m["type"] == "cartesian" and m["file"] != "none"}
    return res
