"""ctypes binding of the CPU oracle (liblbm_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py to check and time against; the product never
imports it.  Arrays are float64 (or float32 for the diagnostic variant)
``[10, nz, ny, nx]`` in the reference's stored units (rho - 1, scaled moments).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblbm_oracle.so")


class Params(ctypes.Structure):
    _fields_ = [("q", ctypes.c_int), ("nx", ctypes.c_int64), ("ny", ctypes.c_int64), ("nz", ctypes.c_int64),
                ("omega", ctypes.c_double), ("t_omega", ctypes.c_double), ("omega_d2", ctypes.c_double),
                ("tau", ctypes.c_double), ("u_lid", ctypes.c_double)]


def build() -> str:
    subprocess.run(["make", "-s", "-f", os.path.join(HERE, "Makefile")], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = ctypes.CDLL(LIB)
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """One cavity: lattice Q, mesh, relaxation constants and lid speed."""

    def __init__(self, q, nx, ny, nz, Re, u_inf, precision="f64"):
        from cudalbm_b200.casefiles import relaxation

        tau, omega, t_omega, omega_d2 = relaxation(u_inf, Re, nx)
        self.p = Params(q, nx, ny, nz, float(omega), float(t_omega), float(omega_d2), float(tau),
                        float(np.float32(u_inf)))
        self.shape = (10, nz, ny, nx)
        self.dtype = np.float64 if precision == "f64" else np.float32
        sfx = "" if precision == "f64" else "_f32"
        L = lib()
        for name in ("oracle_step", "oracle_function_objects", "oracle_initial_moments", "oracle_run"):
            setattr(self, "_" + name, getattr(L, name + sfx))
            getattr(self, "_" + name).restype = None

    def initial(self, region_values):
        m = np.zeros(self.shape, dtype=self.dtype)
        rv = np.ascontiguousarray(region_values, dtype=np.float32)
        self._oracle_initial_moments(ctypes.byref(self.p), _ptr(rv), _ptr(m))
        return m

    def step(self, m):
        out = np.empty_like(m)
        self._oracle_step(ctypes.byref(self.p), _ptr(np.ascontiguousarray(m, dtype=self.dtype)), _ptr(out))
        return out

    def run(self, m, n, t0=0, fo=None):
        """Advance ``m`` (in place) by n steps from absolute step t0.  ``fo`` is
        an optional dict with any of S, SMean, k, kMean, momentsMean arrays
        (updated in place after each step, as the reference does)."""
        a = np.ascontiguousarray(m, dtype=self.dtype)
        b = np.empty_like(a)
        fo = fo or {}
        args = [_ptr(fo.get(k)) for k in ("S", "SMean", "k", "kMean", "momentsMean")]
        self._oracle_run(ctypes.byref(self.p), _ptr(a), _ptr(b), ctypes.c_int64(t0), ctypes.c_int64(n), *args)
        if a is not m:
            m[...] = a
        return m

    def new_function_objects(self, names):
        nz, ny, nx = self.shape[1:]
        sizes = {"S": 6, "SMean": 6, "k": 1, "kMean": 1, "momentsMean": 10}
        return {k: np.zeros((sizes[k], nz, ny, nx), dtype=self.dtype) for k in names}
