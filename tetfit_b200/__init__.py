"""B200-native TetFIT leapfrog time-stepping path.

The product is the shared library `libtetfit_b200.so` (C ABI declared in
include/tetfit.h: C++ host code driving sm_100a CUDA kernels).  This module is
a thin ctypes mirror of the reference's driver interface
(src/DGA/Discretization.hpp:45-211 `Discretization(inputfile)`, :289
`RunSimulation(sim, label)`, src/DGA/main/dga_main.cpp:52-62), plus stepwise
access used by tests and the benchmark.  There is no CPU fallback: importing
raises if the library has not been built.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtetfit_b200.so")

TF_OK, TF_E_SCRIPT, TF_E_ARG, TF_E_CUDA, TF_E_UNSUPPORTED, TF_E_STATE, TF_E_SOLVER = 0, -1, -2, -3, -4, -5, -6
FP64, FP32 = 0, 1
METHODS = {0: "fdtd", 1: "dga", 2: "gfdtd", 3: "fem"}


class TetfitError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


class Opts(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("device", ctypes.c_int32), ("write_files", ctypes.c_int32),
                ("verbose", ctypes.c_int32), ("graph_steps", ctypes.c_int32), ("mass_model", ctypes.c_int32),
                ("warm_start", ctypes.c_int32), ("cg_criterion", ctypes.c_int32), ("cg_maxiter", ctypes.c_int32),
                ("batch_mode", ctypes.c_int32), ("host_threads", ctypes.c_int32), ("learn_steps", ctypes.c_int32),
                ("fit_variant", ctypes.c_int32), ("file_digits", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 2)]


class Info(ctypes.Structure):
    _fields_ = [("n_edges", ctypes.c_uint64), ("n_faces", ctypes.c_uint64), ("n_cells", ctypes.c_uint64),
                ("n_probes", ctypes.c_uint64), ("n_steps", ctypes.c_uint64), ("step_index", ctypes.c_uint64),
                ("nx", ctypes.c_uint32), ("ny", ctypes.c_uint32), ("nz", ctypes.c_uint32),
                ("method", ctypes.c_int32), ("dt", ctypes.c_double), ("dt_estimate", ctypes.c_double),
                ("possibly_unstable", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("device_bytes", ctypes.c_uint64), ("kernels_per_step", ctypes.c_uint32),
                ("n_sources", ctypes.c_uint32), ("n_free", ctypes.c_uint64), ("nnz_system", ctypes.c_uint64),
                ("nnz_operators", ctypes.c_uint64), ("cg_blocks", ctypes.c_uint32), ("cg_variant", ctypes.c_int32),
                ("reserved", ctypes.c_uint64 * 3)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}
        d["method"] = METHODS.get(d["method"], d["method"])
        return d


_lib = None


class PcgArgs(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("device", ctypes.c_int32), ("row_ptr", ctypes.c_void_p),
                ("col", ctypes.c_void_p), ("val", ctypes.c_void_p), ("b", ctypes.c_void_p), ("x", ctypes.c_void_p),
                ("tol", ctypes.c_double), ("maxiter", ctypes.c_int32), ("criterion", ctypes.c_int32),
                ("stream", ctypes.c_void_p)]

# name -> (restype, argtypes); every symbol declared in include/tetfit.h
_P = ctypes.c_void_p
_SIGS = {
    "tf_open": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_P)]),
    "tf_simulations": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32,
                                      ctypes.POINTER(ctypes.c_uint32)]),
    "tf_prepare": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(Opts)]),
    "tf_get_info": (ctypes.c_int, [_P, ctypes.POINTER(Info)]),
    "tf_step": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "tf_get_probes": (ctypes.c_int, [_P, _P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "tf_get_probe_points": (ctypes.c_int, [_P, _P, _P, ctypes.c_size_t]),
    "tf_get_state": (ctypes.c_int, [_P, _P, ctypes.c_size_t, _P, ctypes.c_size_t, _P, ctypes.c_size_t]),
    "tf_set_state": (ctypes.c_int, [_P, _P, ctypes.c_size_t, _P, ctypes.c_size_t]),
    "tf_get_flux": (ctypes.c_int, [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "tf_get_losses": (ctypes.c_int, [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "tf_script_dump": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "tf_energy": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double)]),
    "tf_step_io": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(ctypes.c_uint64)]),
    "tf_phase_times": (ctypes.c_int, [_P, ctypes.c_uint64, _P, ctypes.POINTER(ctypes.c_uint64)]),
    "tf_run": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(Opts)]),
    "tf_solver_stats": (ctypes.c_int, [_P, _P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "tf_guess_stats": (ctypes.c_int, [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "tf_training_loss": (ctypes.c_int, [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "tf_batch_guess_stats": (ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "tf_batch_training_loss": (ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_size_t,
                                              ctypes.POINTER(ctypes.c_size_t)]),
    "tf_batch_mlp_params": (ctypes.c_int, [_P, ctypes.c_uint32, _P]),
    "tf_pcg_solve": (ctypes.c_int, [ctypes.POINTER(PcgArgs), ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_double)]),
    "tf_pcg_solve_noalloc": (ctypes.c_int, [ctypes.POINTER(PcgArgs), ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_double)]),
    "tf_barrier_check": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_uint32, ctypes.POINTER(ctypes.c_int32),
                                        ctypes.POINTER(ctypes.c_double)]),
    "tf_batch_open": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_uint32),
                                     ctypes.c_uint32, ctypes.POINTER(Opts), ctypes.POINTER(_P)]),
    "tf_batch_info": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(Info)]),
    "tf_batch_step": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "tf_batch_phase_times": (ctypes.c_int, [_P, ctypes.c_uint64, _P, ctypes.POINTER(ctypes.c_uint64)]),
    "tf_batch_step_io": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(ctypes.c_uint64)]),
    "tf_batch_get_probes": (ctypes.c_int, [_P, ctypes.c_uint32, _P, _P, ctypes.c_size_t,
                                           ctypes.POINTER(ctypes.c_size_t)]),
    "tf_batch_get_probe_points": (ctypes.c_int, [_P, ctypes.c_uint32, _P, _P, ctypes.c_size_t]),
    "tf_batch_get_state": (ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_size_t, _P, ctypes.c_size_t, _P,
                                          ctypes.c_size_t]),
    "tf_batch_get_flux": (ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "tf_batch_energy": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double)]),
    "tf_batch_solver_stats": (ctypes.c_int, [_P, ctypes.c_uint32, _P, _P, ctypes.c_size_t,
                                             ctypes.POINTER(ctypes.c_size_t)]),
    "tf_batch_last_step_ms": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double)]),
    "tf_batch_last_error": (ctypes.c_char_p, [_P]),
    "tf_batch_close": (None, [_P]),
    "tf_mlp_param_count": (ctypes.c_int, []),
    "tf_mlp_init": (ctypes.c_int, [ctypes.c_uint64, _P]),
    "tf_mlp_forward": (ctypes.c_int, [_P, ctypes.c_int64, _P, _P]),
    "tf_mlp_gradient": (ctypes.c_int, [_P, ctypes.c_int64, _P, _P, _P, _P, _P]),
    "tf_last_step_ms": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_double)]),
    "tf_last_error": (ctypes.c_char_p, [_P]),
    "tf_close": (None, [_P]),
    "tf_default_opts": (None, [ctypes.POINTER(Opts)]),
}


def lib():
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m tetfit_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def pcg_solve(row_ptr, col, val, b, x, tol=1e-8, maxiter=0, criterion=0, device=0, stream=None):
    """Jacobi-PCG on a CSR system in device memory (tf_pcg_solve).  Arguments
    are device pointers (ints) or objects with a `data_ptr()` method (e.g.
    torch tensors: int64 row_ptr, int32 col, float64 val/b/x).  Returns
    (status, iterations, relative residual); x is overwritten."""
    def dp(t):
        return t.data_ptr() if hasattr(t, "data_ptr") else int(t)
    n = (len(row_ptr) - 1) if hasattr(row_ptr, "__len__") else None
    a = PcgArgs(n=int(n if n is not None else len(b)), device=device, row_ptr=dp(row_ptr), col=dp(col),
                val=dp(val), b=dp(b), x=dp(x), tol=tol, maxiter=maxiter, criterion=criterion, stream=stream)
    it = ctypes.c_int32()
    rs = ctypes.c_double()
    rc = lib().tf_pcg_solve(ctypes.byref(a), ctypes.byref(it), ctypes.byref(rs))
    return rc, it.value, rs.value


def barrier_check(blocks: int, expected: int, rounds: int = 1, timeout_us: int = 100000, device: int = 0):
    """Self-check of the CG kernels' bounded grid barrier (tf_barrier_check):
    (status, ms) of one launch of `blocks` blocks passing `rounds` barriers
    that wait for `expected` arrivals.  status 0: every barrier completed;
    2: a wait ran out of time (expected > blocks can never complete)."""
    st = ctypes.c_int32()
    ms = ctypes.c_double()
    rc = lib().tf_barrier_check(device, blocks, expected, rounds, timeout_us, ctypes.byref(st), ctypes.byref(ms))
    if rc != TF_OK:
        raise TetfitError(rc, last_thread_error())
    return st.value, ms.value


def mlp_init(seed: int = 1) -> np.ndarray:
    """Initial parameters of the warm-start network (tf_mlp_init)."""
    p = np.zeros(lib().tf_mlp_param_count(), dtype=np.float32)
    lib().tf_mlp_init(seed, _ptr(p))
    return p


def mlp_forward(params, inputs) -> np.ndarray:
    """Network outputs [n] for inputs [n, 6] (tf_mlp_forward, tensor-core kernel)."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    inputs = np.ascontiguousarray(inputs, dtype=np.float32)
    out = np.zeros(len(inputs), dtype=np.float32)
    rc = lib().tf_mlp_forward(_ptr(params), len(inputs), _ptr(inputs), _ptr(out))
    if rc != TF_OK:
        raise TetfitError(rc, last_thread_error())
    return out


def mlp_gradient(params, inputs, targets, weights=None):
    """(gradient[n_params], loss) of sum w (y - t)^2 / n (tf_mlp_gradient)."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    inputs = np.ascontiguousarray(inputs, dtype=np.float32)
    targets = np.ascontiguousarray(targets, dtype=np.float32)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float32)
    g = np.zeros_like(params)
    loss = np.zeros(1, dtype=np.float32)
    rc = lib().tf_mlp_gradient(_ptr(params), len(inputs), _ptr(inputs), _ptr(targets), _ptr(w), _ptr(g), _ptr(loss))
    if rc != TF_OK:
        raise TetfitError(rc, last_thread_error())
    return g, float(loss[0])


def last_thread_error() -> str:
    return lib().tf_last_error(None).decode()


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Discretization:
    """Mirror of TetFIT's `Discretization` driver for one `.fdtd` script.

    `Discretization(path)` parses the script like Discretization.hpp:45-211;
    `run_simulation(label)` runs one simulation end to end like
    RunSimulation (Discretization.hpp:289-2303), writing the same probe and
    poynting files when `write_files=True`.  Script errors raise TetfitError
    whose message is the reference's "Input file error at line N: ..." text.
    """

    def __init__(self, path: str):
        L = lib()
        self._h = _P()
        rc = L.tf_open(os.fsencode(path), ctypes.byref(self._h))
        if rc != TF_OK:
            msg = L.tf_last_error(self._h).decode()
            L.tf_close(self._h)
            self._h = None
            raise TetfitError(rc, msg)

    def _check(self, rc):
        if rc != TF_OK:
            raise TetfitError(rc, lib().tf_last_error(self._h).decode())

    @property
    def simulations(self) -> list:
        n = ctypes.c_uint32()
        self._check(lib().tf_simulations(self._h, None, 0, ctypes.byref(n)))
        arr = (ctypes.c_uint32 * max(n.value, 1))()
        self._check(lib().tf_simulations(self._h, arr, n.value, ctypes.byref(n)))
        return list(arr)[: n.value]

    def script(self) -> dict:
        """The parsed script (tf_script_dump) as a dict."""
        import json
        n = ctypes.c_size_t()
        self._check(lib().tf_script_dump(self._h, None, 0, ctypes.byref(n)))
        buf = ctypes.create_string_buffer(n.value)
        self._check(lib().tf_script_dump(self._h, buf, n.value, ctypes.byref(n)))
        return json.loads(buf.value.decode())

    WARM_STARTS = {"previous": 0, "zero": 1, "extrapolate": 2, "learned": 3}

    @staticmethod
    def _opts(precision="fp64", device=0, write_files=False, verbose=False, graph_steps=0, mass="reference",
              warm_start="previous", cg_criterion="reference", cg_maxiter=0, batch_mode=0, host_threads=0,
              learn_steps=0, fit_variant=0, file_digits=0) -> Opts:
        o = Opts()
        lib().tf_default_opts(ctypes.byref(o))
        o.precision = {"fp64": FP64, "fp32": FP32}[precision] if isinstance(precision, str) else int(precision)
        o.device, o.write_files, o.verbose, o.graph_steps = device, int(write_files), int(verbose), graph_steps
        o.mass_model = {"reference": 0, "consistent": 1}[mass]
        o.warm_start = Discretization.WARM_STARTS[warm_start] if isinstance(warm_start, str) else int(warm_start)
        o.cg_criterion = {"reference": 0, "rhs": 1}[cg_criterion]
        o.cg_maxiter = cg_maxiter
        o.batch_mode = {"group": 0, "serial": 1}[batch_mode] if isinstance(batch_mode, str) else int(batch_mode)
        o.host_threads = host_threads
        o.learn_steps = learn_steps
        o.fit_variant = fit_variant
        o.file_digits = file_digits
        return o

    def prepare(self, label: int, **opts) -> dict:
        o = self._opts(**opts)
        self._check(lib().tf_prepare(self._h, label, ctypes.byref(o)))
        return self.info()

    def run_simulation(self, label: int, **opts) -> dict:
        o = self._opts(**opts)
        self._check(lib().tf_run(self._h, label, ctypes.byref(o)))
        return self.info()

    def info(self) -> dict:
        i = Info()
        self._check(lib().tf_get_info(self._h, ctypes.byref(i)))
        return i.as_dict()

    def step(self, n: int) -> int:
        done = ctypes.c_uint64()
        self._check(lib().tf_step(self._h, n, ctypes.byref(done)))
        return done.value

    def step_io(self, carrier_in=None, probe_out=None) -> int:
        """One step with this step's carrier values from host memory and the
        exported probe sample read back (see tf_step_io)."""
        done = ctypes.c_uint64()
        self._check(lib().tf_step_io(self._h, _ptr(carrier_in), _ptr(probe_out), ctypes.byref(done)))
        return done.value

    def phase_times(self, n: int):
        """Device ms per phase over n steps: sources/BC, E, scatter+flux, probes, H."""
        ms = np.zeros(5)
        done = ctypes.c_uint64()
        self._check(lib().tf_phase_times(self._h, n, _ptr(ms), ctypes.byref(done)))
        return ms, done.value

    def solver_stats(self):
        """gfdtd: (iterations[n_steps_done], final relative residual[n_steps_done])."""
        n = ctypes.c_size_t()
        self._check(lib().tf_solver_stats(self._h, None, None, 0, ctypes.byref(n)))
        it = np.zeros(n.value, dtype=np.int32)
        rs = np.zeros(n.value)
        self._check(lib().tf_solver_stats(self._h, _ptr(it), _ptr(rs), n.value, ctypes.byref(n)))
        return it, rs

    def last_step_ms(self) -> float:
        ms = ctypes.c_double()
        self._check(lib().tf_last_step_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def guess_stats(self):
        """warm_start "learned": per step 1 when the network's guess was kept."""
        n = ctypes.c_size_t()
        self._check(lib().tf_guess_stats(self._h, None, 0, ctypes.byref(n)))
        k = np.zeros(n.value, dtype=np.int8)
        self._check(lib().tf_guess_stats(self._h, _ptr(k), n.value, ctypes.byref(n)))
        return k

    def training_loss(self):
        n = ctypes.c_size_t()
        self._check(lib().tf_training_loss(self._h, None, 0, ctypes.byref(n)))
        v = np.zeros(n.value, dtype=np.float32)
        self._check(lib().tf_training_loss(self._h, _ptr(v), n.value, ctypes.byref(n)))
        return v

    def probes(self):
        """(times[n], values[n, n_probes, 6]) with columns Ex Ey Ez Hx Hy Hz."""
        n = ctypes.c_size_t()
        self._check(lib().tf_get_probes(self._h, None, None, 0, ctypes.byref(n)))
        np_ = self.info()["n_probes"]
        t = np.zeros(n.value)
        v = np.zeros((n.value, np_, 6))
        self._check(lib().tf_get_probes(self._h, _ptr(t), _ptr(v), n.value, ctypes.byref(n)))
        return t, v

    def probe_points(self):
        np_ = self.info()["n_probes"]
        xyz = np.zeros((np_, 3))
        cells = np.zeros(np_, dtype=np.uint64)
        self._check(lib().tf_get_probe_points(self._h, _ptr(xyz), _ptr(cells), np_))
        return xyz, cells

    def state(self):
        """(U[n_edges], B[n_faces], F[n_faces]) in the reference's numbering."""
        i = self.info()
        U, B, F = np.zeros(i["n_edges"]), np.zeros(i["n_faces"]), np.zeros(i["n_faces"])
        self._check(lib().tf_get_state(self._h, _ptr(U), U.size, _ptr(B), B.size, _ptr(F), F.size))
        return U, B, F

    def set_state(self, U, F):
        U = np.ascontiguousarray(U, dtype=np.float64)
        F = np.ascontiguousarray(F, dtype=np.float64)
        self._check(lib().tf_set_state(self._h, _ptr(U), U.size, _ptr(F), F.size))

    def flux(self):
        n = ctypes.c_size_t()
        self._check(lib().tf_get_flux(self._h, None, 0, ctypes.byref(n)))
        f = np.zeros(n.value)
        self._check(lib().tf_get_flux(self._h, _ptr(f), n.value, ctypes.byref(n)))
        return f

    def losses(self):
        """Joule loss of every step taken (the third column of poynting.dat)."""
        n = ctypes.c_size_t()
        self._check(lib().tf_get_losses(self._h, None, 0, ctypes.byref(n)))
        f = np.zeros(n.value)
        self._check(lib().tf_get_losses(self._h, _ptr(f), n.value, ctypes.byref(n)))
        return f

    def energy(self) -> float:
        e = ctypes.c_double()
        self._check(lib().tf_energy(self._h, ctypes.byref(e)))
        return e.value

    def close(self):
        if self._h:
            lib().tf_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many gfdtd simulations advanced together (tf_batch_*).

    `Batch([(script, label), ...], batch_mode="group")` builds every member on
    the host in parallel and lays them out in one device image: each step is
    one launch sequence and one persistent CG kernel for all members, each
    member with its own time step, tolerance, probes and statistics.
    `batch_mode="serial"` keeps each member in its own image and steps them
    one after another, the way the reference runs a script's simulations
    (dga_main.cpp:52-62).  Options as `Discretization.prepare`.
    """

    def __init__(self, members, **opts):
        L = lib()
        members = list(members)
        o = Discretization._opts(**opts)
        paths = (ctypes.c_char_p * len(members))(*[os.fsencode(p) for p, _ in members])
        labels = (ctypes.c_uint32 * len(members))(*[int(l) for _, l in members])
        self._h = _P()
        rc = L.tf_batch_open(paths, labels, len(members), ctypes.byref(o), ctypes.byref(self._h))
        if rc != TF_OK:
            msg = L.tf_batch_last_error(self._h).decode()
            L.tf_batch_close(self._h)
            self._h = None
            raise TetfitError(rc, msg)
        self.size = len(members)

    def _check(self, rc):
        if rc != TF_OK:
            raise TetfitError(rc, lib().tf_batch_last_error(self._h).decode())

    def info(self, m: int) -> dict:
        i = Info()
        self._check(lib().tf_batch_info(self._h, m, ctypes.byref(i)))
        return i.as_dict()

    def step(self, n: int) -> int:
        done = ctypes.c_uint64()
        self._check(lib().tf_batch_step(self._h, n, ctypes.byref(done)))
        return done.value

    def phase_times(self, n: int):
        ms = np.zeros(5)
        done = ctypes.c_uint64()
        self._check(lib().tf_batch_phase_times(self._h, n, _ptr(ms), ctypes.byref(done)))
        return ms, done.value

    def step_io(self, carriers_in=None, probes_out=None) -> int:
        done = ctypes.c_uint64()
        self._check(lib().tf_batch_step_io(self._h, _ptr(carriers_in), _ptr(probes_out), ctypes.byref(done)))
        return done.value

    def last_step_ms(self) -> float:
        ms = ctypes.c_double()
        self._check(lib().tf_batch_last_step_ms(self._h, ctypes.byref(ms)))
        return ms.value

    def probes(self, m: int):
        n = ctypes.c_size_t()
        self._check(lib().tf_batch_get_probes(self._h, m, None, None, 0, ctypes.byref(n)))
        np_ = self.info(m)["n_probes"]
        t, v = np.zeros(n.value), np.zeros((n.value, np_, 6))
        self._check(lib().tf_batch_get_probes(self._h, m, _ptr(t), _ptr(v), n.value, ctypes.byref(n)))
        return t, v

    def probe_points(self, m: int):
        np_ = self.info(m)["n_probes"]
        xyz, cells = np.zeros((np_, 3)), np.zeros(np_, dtype=np.uint64)
        self._check(lib().tf_batch_get_probe_points(self._h, m, _ptr(xyz), _ptr(cells), np_))
        return xyz, cells

    def state(self, m: int):
        i = self.info(m)
        U, B, F = np.zeros(i["n_edges"]), np.zeros(i["n_faces"]), np.zeros(i["n_faces"])
        self._check(lib().tf_batch_get_state(self._h, m, _ptr(U), U.size, _ptr(B), B.size, _ptr(F), F.size))
        return U, B, F

    def flux(self, m: int):
        n = ctypes.c_size_t()
        self._check(lib().tf_batch_get_flux(self._h, m, None, 0, ctypes.byref(n)))
        f = np.zeros(n.value)
        self._check(lib().tf_batch_get_flux(self._h, m, _ptr(f), n.value, ctypes.byref(n)))
        return f

    def guess_stats(self, m: int):
        n = ctypes.c_size_t()
        self._check(lib().tf_batch_guess_stats(self._h, m, None, 0, ctypes.byref(n)))
        k = np.zeros(n.value, dtype=np.int8)
        self._check(lib().tf_batch_guess_stats(self._h, m, _ptr(k), n.value, ctypes.byref(n)))
        return k

    def training_loss(self, m: int = 0):
        n = ctypes.c_size_t()
        self._check(lib().tf_batch_training_loss(self._h, m, None, 0, ctypes.byref(n)))
        v = np.zeros(n.value, dtype=np.float32)
        self._check(lib().tf_batch_training_loss(self._h, m, _ptr(v), n.value, ctypes.byref(n)))
        return v

    def mlp_params(self, m: int = 0):
        p = np.zeros(lib().tf_mlp_param_count(), dtype=np.float32)
        self._check(lib().tf_batch_mlp_params(self._h, m, _ptr(p)))
        return p

    def energy(self, m: int) -> float:
        e = ctypes.c_double()
        self._check(lib().tf_batch_energy(self._h, m, ctypes.byref(e)))
        return e.value

    def solver_stats(self, m: int):
        n = ctypes.c_size_t()
        self._check(lib().tf_batch_solver_stats(self._h, m, None, None, 0, ctypes.byref(n)))
        it, rs = np.zeros(n.value, dtype=np.int32), np.zeros(n.value)
        self._check(lib().tf_batch_solver_stats(self._h, m, _ptr(it), _ptr(rs), n.value, ctypes.byref(n)))
        return it, rs

    def close(self):
        if self._h:
            lib().tf_batch_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
