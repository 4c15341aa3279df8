"""CPU oracle — TEST INFRASTRUCTURE ONLY.

An FP64 C++ restatement of TetFIT's time-stepping path (see the headers of
oracle/*.cpp for the reference lines each part follows), loaded with ctypes.
Only tests/, bench.py's cpu_baseline / reference leg and
__graft_entry__.smoke() may use it, and only as the checker or the timed CPU
baseline; the product (tetfit_b200/) never imports it.

Parity is pinned against fixtures generated by this restatement and against
size-independent properties (energy conservation, analytic waveguide); the
reference ships no tests or golden vectors and cannot be compiled here, so
parity against the reference binary itself is unpinned.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .build import LIB, LIB_OMP, build

_libs = {}


def lib(omp: bool = False):
    path = LIB_OMP if omp else LIB
    if path not in _libs:
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        L.orc_fit_open.restype = P
        L.orc_fit_open.argtypes = [ctypes.c_char_p, ctypes.c_uint, ctypes.c_char_p, ctypes.c_int]
        L.orc_fit_close.argtypes = [P]
        L.orc_fit_info.argtypes = [P, P, P]
        L.orc_fit_step.restype = ctypes.c_longlong
        L.orc_fit_step.argtypes = [P, ctypes.c_longlong]
        L.orc_fit_nsamples.restype = ctypes.c_longlong
        L.orc_fit_nsamples.argtypes = [P]
        L.orc_fit_probes.argtypes = [P, P, P, P, P]
        L.orc_fit_state.argtypes = [P, P, P, P]
        L.orc_fit_flux.argtypes = [P, P]
        L.orc_fit_losses.argtypes = [P, P]
        L.orc_fit_topology.argtypes = [P, P, P, P, P]
        L.orc_fit_coeffs.argtypes = [P, P, P, P, P]
        _libs[path] = L
    return _libs[path]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def script_dump(path: str) -> dict:
    """The oracle front end's parse of a script, as a dict (raises
    RuntimeError with the parser's message on a script error)."""
    import json
    L = lib()
    L.orc_script_dump.restype = ctypes.c_long
    L.orc_script_dump.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_long]
    n = L.orc_script_dump(os.fsencode(path), None, 0)
    buf = ctypes.create_string_buffer(max(n, 4096))
    n = L.orc_script_dump(os.fsencode(path), buf, len(buf))
    if n < 0:
        raise RuntimeError(buf.value.decode())
    return json.loads(buf.value.decode())


class FitOracle:
    """FP64 CPU restatement of one Cartesian FIT simulation."""

    def __init__(self, script: str, label: int = 1, omp: bool = False):
        self.L = lib(omp)
        err = ctypes.create_string_buffer(1024)
        self.h = self.L.orc_fit_open(os.fsencode(script), label, err, 1024)
        if not self.h:
            raise RuntimeError(err.value.decode())
        iv = np.zeros(16, dtype=np.int64)
        dv = np.zeros(16)
        self.L.orc_fit_info(self.h, _p(iv), _p(dv))
        self.nE, self.nF, self.nV, self.n_probes, self.n_steps = (int(x) for x in iv[:5])
        self.N = tuple(int(x) for x in iv[5:8])
        self.possibly_unstable = bool(iv[8])
        self.dt, self.dt_estimate = float(dv[0]), float(dv[1])
        self.steps_done = 0

    def step(self, n: int) -> int:
        d = int(self.L.orc_fit_step(self.h, n))
        self.steps_done += d
        return d

    def run(self) -> int:
        return self.step(self.n_steps)

    def probes(self):
        ns = int(self.L.orc_fit_nsamples(self.h))
        t = np.zeros(ns)
        v = np.zeros((ns, self.n_probes, 6))
        pts = np.zeros((self.n_probes, 3))
        el = np.zeros(self.n_probes, dtype=np.int64)
        self.L.orc_fit_probes(self.h, _p(t), _p(v), _p(pts), _p(el))
        return t, v, pts, el

    def state(self):
        U, F, B = np.zeros(self.nE), np.zeros(self.nF), np.zeros(self.nF)
        self.L.orc_fit_state(self.h, _p(U), _p(F), _p(B))
        return U, B, F

    def flux(self):
        f = np.zeros(self.steps_done)
        self.L.orc_fit_flux(self.h, _p(f))
        return f

    def losses(self):
        """Joule loss of every step taken (Discretization.hpp:1902)."""
        f = np.zeros(self.steps_done)
        self.L.orc_fit_losses(self.h, _p(f))
        return f

    def coeffs(self):
        """(M_h, M_q, M_nu, M_mu) in the reference numbering."""
        mh, mq, mnu, mmu = np.zeros(self.nE), np.zeros(self.nE), np.zeros(self.nF), np.zeros(self.nF)
        self.L.orc_fit_coeffs(self.h, _p(mh), _p(mq), _p(mnu), _p(mmu))
        return mh, mq, mnu, mmu

    def topology(self):
        en = np.zeros((self.nE, 2), dtype=np.uint32)
        npts = self.nV * 8
        xyz = np.zeros((npts, 3))
        fe = np.zeros((self.nF, 4), dtype=np.uint32)
        cl = np.zeros(self.nE, dtype=np.uint32)
        n = self.L.orc_fit_topology(self.h, _p(en), _p(xyz), _p(fe), _p(cl))
        return en, xyz[:n], fe, cl

    def close(self):
        if self.h:
            self.L.orc_fit_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TetOracle:
    """FP64 CPU restatement of one tetrahedral simulation (dga or gfdtd)."""

    def __init__(self, script: str, label: int = 1, omp: bool = False, consistent_mass: bool = False):
        self.L = lib(omp)
        L = self.L
        P = ctypes.c_void_p
        if not getattr(L, "_tet_sigs", False):
            L.orc_tet_open.restype = P
            L.orc_tet_open.argtypes = [ctypes.c_char_p, ctypes.c_uint, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
            L.orc_tet_close.argtypes = [P]
            L.orc_tet_info.argtypes = [P, P, P]
            L.orc_tet_step.restype = ctypes.c_longlong
            L.orc_tet_step.argtypes = [P, ctypes.c_longlong]
            L.orc_tet_nsamples.restype = ctypes.c_longlong
            L.orc_tet_nsamples.argtypes = [P]
            L.orc_tet_probes.argtypes = [P, P, P, P, P]
            L.orc_tet_state.argtypes = [P, P, P, P]
            L.orc_tet_flux.argtypes = [P, P]
            L.orc_tet_losses.argtypes = [P, P]
            L.orc_tet_cg.argtypes = [P, P, P]
            L.orc_tet_topology.argtypes = [P, P, P, P, P]
            L.orc_tet_matrix.restype = ctypes.c_longlong
            L.orc_tet_matrix.argtypes = [P, ctypes.c_int, P, P, P]
            L.orc_tet_dga_p.argtypes = [P, P]
            L.orc_tet_dga_r.argtypes = [P, P]
            L._tet_sigs = True
        err = ctypes.create_string_buffer(1024)
        self.h = L.orc_tet_open(os.fsencode(script), label, int(consistent_mass), err, 1024)
        if not self.h:
            raise RuntimeError(err.value.decode())
        iv = np.zeros(16, dtype=np.int64)
        dv = np.zeros(16)
        L.orc_tet_info(self.h, _p(iv), _p(dv))
        (self.nE, self.nF, self.nT, self.nN, self.n_probes, self.n_steps, self.method, self.n_free,
         self.n_bnd) = (int(x) for x in iv[:9])
        self.possibly_unstable = bool(iv[9])
        self.dt, self.dt_estimate = float(dv[0]), float(dv[1])
        self.steps_done = 0

    def step(self, n: int) -> int:
        d = int(self.L.orc_tet_step(self.h, n))
        self.steps_done += d
        return d

    def run(self) -> int:
        return self.step(self.n_steps)

    def probes(self):
        ns = int(self.L.orc_tet_nsamples(self.h))
        t = np.zeros(ns)
        v = np.zeros((ns, self.n_probes, 6))
        pts = np.zeros((self.n_probes, 3))
        el = np.zeros(self.n_probes, dtype=np.int64)
        self.L.orc_tet_probes(self.h, _p(t), _p(v), _p(pts), _p(el))
        return t, v, pts, el

    def state(self):
        U, F, B = np.zeros(self.nE), np.zeros(self.nF), np.zeros(self.nF)
        self.L.orc_tet_state(self.h, _p(U), _p(F), _p(B))
        return U, B, F

    def flux(self):
        f = np.zeros(self.steps_done)
        self.L.orc_tet_flux(self.h, _p(f))
        return f

    def losses(self):
        """poynting.dat's third column (one entry per step taken)."""
        f = np.zeros(self.steps_done)
        self.L.orc_tet_losses(self.h, _p(f))
        return f

    def cg(self):
        it = np.zeros(self.steps_done, dtype=np.int32)
        er = np.zeros(self.steps_done)
        self.L.orc_tet_cg(self.h, _p(it), _p(er))
        return it, er

    def topology(self):
        e = np.zeros((self.nE, 2), dtype=np.uint32)
        f = np.zeros((self.nF, 3), dtype=np.uint32)
        c = np.zeros(self.nE, dtype=np.uint8)
        b = np.zeros(self.nE, dtype=np.int32)
        self.L.orc_tet_topology(self.h, _p(e), _p(f), _p(c), _p(b))
        return e, f, c, b

    def dga_p(self):
        """dga: (P per edge: 1 on class-1, P_p on class-2 edges, 0 elsewhere;
        number of node-star fractions U_c)."""
        P = np.zeros(self.nE)
        nq = int(self.L.orc_tet_dga_p(self.h, _p(P)))
        return P, nq

    def dga_r(self):
        """dga: (R per face: 1 on class-1, R_r on class-2 faces; number of
        class-2 faces)."""
        R = np.zeros(self.nF)
        nr = int(self.L.orc_tet_dga_r(self.h, _p(R)))
        return R, nr

    def matrix(self, which: str):
        """CSR (ptr, col, val) of one operator: C, N, H (dga), E, Sig (the
        conductivity mass), A (gfdtd, fem) or Nmag (dga: the N or Tr row of
        each face, the operator of the F update)."""
        w = {"C": 0, "N": 1, "H": 2, "E": 3, "A": 4, "Sig": 5, "Nmag": 6}[which]
        nnz = int(self.L.orc_tet_matrix(self.h, w, None, None, None))
        nrows = {0: self.nF, 1: self.nF, 2: self.nE, 3: self.nE, 4: self.n_free, 5: self.nE, 6: self.nF}[w]
        ptr = np.zeros(nrows + 1, dtype=np.uint64)
        col = np.zeros(nnz, dtype=np.uint32)
        val = np.zeros(nnz)
        self.L.orc_tet_matrix(self.h, w, _p(ptr), _p(col), _p(val))
        return ptr, col, val

    def close(self):
        if self.h:
            self.L.orc_tet_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
