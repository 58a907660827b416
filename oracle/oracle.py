"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle library.

The oracle (oracle/seren_oracle.cpp) is a FP64 restatement of the reference's
Fortran force path and is the checker for the CUDA library; only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it.  Parity is
unpinned: the reference ships no golden vectors and cannot be compiled here.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from seren_b200.cabi import HotPath, Params, bind

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libseren_oracle.so")
KERNTOT = 10000

_lib = None


class Counts(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "grav_cells", "grav_pairs", "grav_nodes", "gradh_tests", "gradh_pairs", "gradh_passes",
        "gradh_walks", "gradh_final_tests", "gradh_final_pairs", "neib_tests", "neib_pairs",
        "hydro_pairs", "hydro_visc")]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off, OpenMP)."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
            os.path.getmtime(os.path.join(HERE, f)) for f in ("seren_oracle.cpp", "seren_oracle.h")):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def library() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = bind(C.CDLL(LIB), "seren_oracle")
        vp = C.c_void_p
        lib.seren_oracle_set_threads.argtypes = [C.c_int32]
        lib.seren_oracle_set_threads.restype = C.c_int
        lib.seren_oracle_direct_gravity.argtypes = [vp, C.POINTER(C.c_int32), C.c_int32,
                                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.seren_oracle_direct_gravity.restype = C.c_int
        lib.seren_oracle_get_counts.argtypes = [vp, C.POINTER(Counts)]
        lib.seren_oracle_get_counts.restype = C.c_int
        lib.seren_oracle_kernel_tables.argtypes = [C.c_int32, C.POINTER(C.c_double)]
        lib.seren_oracle_kernel_tables.restype = C.c_int
        lib.seren_oracle_stage_seconds.argtypes = [vp, C.POINTER(C.c_double)]
        lib.seren_oracle_stage_seconds.restype = C.c_int
        _lib = lib
    return _lib


def set_threads(n: int) -> int:
    return int(library().seren_oracle_set_threads(int(n)))


def kernel_tables(kernel: int = 0) -> np.ndarray:
    """[9, KERNTOT+1] = w0, w1, w2, w3, w4, w5, w6, wh, wg (setup/kernel.F90)."""
    t = np.zeros((9, KERNTOT + 1))
    library().seren_oracle_kernel_tables(kernel, t.ctypes.data_as(C.POINTER(C.c_double)))
    return t


def timestep_sizes(h, a, div_v, sound, alpha, courant_mult=0.2, accel_mult=0.5):
    """Per-particle timesteps, timestep/timestep_size.F90:52-120 (HYDRO,
    ARTIFICIAL_VISCOSITY with beta = 2 alpha, no internal energy), in FP64 with
    the Fortran expressions' order of operations:
    tacc = accel_mult*sqrt(h/(|a| + 1e-20)) (:95-96),
    tcour = courant_mult*h/(c + h|div v| + 0.6(alpha c + beta h|div v|)) (:103-105,
    TVISC_FAC = 0.6 from headers/macros.h:133), dt = min(tacc, tcour)."""
    a = np.asarray(a, dtype=np.float64).reshape(-1, 3)
    h = np.asarray(h, dtype=np.float64)
    dv = np.abs(np.asarray(div_v, dtype=np.float64))
    c = np.asarray(sound, dtype=np.float64)
    beta = 2.0 * alpha
    amag = np.sqrt((a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1]) + a[:, 2] * a[:, 2])
    tacc = accel_mult * np.sqrt(h / (amag + 1.0e-20))
    tcour = (courant_mult * h) / ((c + h * dv) + 0.6 * (alpha * c + (beta * h) * dv))
    return np.minimum(tacc, tcour)


def sink_timesteps(rmh, v, a, radius, sink_mult=0.5):
    """sinks/sink_timestep.F90:28-52 for every sink: min(sink_mult
    sqrt(radius/(|a| + 1e-20)), sink_mult radius/(|v| + 1e-20)) and, with more
    than one sink, sink_mult max(½(radius + radius'), distance)/(|v - v'| + 1e-20)
    for every other sink."""
    rmh, v, a = (np.asarray(x, np.float64).reshape(len(radius), -1) for x in (rmh, v, a))
    radius = np.asarray(radius, np.float64)
    out = np.zeros(len(radius))
    for s in range(len(radius)):
        acc = np.sqrt((a[s, 0] * a[s, 0] + a[s, 1] * a[s, 1]) + a[s, 2] * a[s, 2])
        vel = np.sqrt((v[s, 0] * v[s, 0] + v[s, 1] * v[s, 1]) + v[s, 2] * v[s, 2])
        dt = min(sink_mult * np.sqrt(radius[s] / (acc + 1.0e-20)),
                 (sink_mult * radius[s]) / (vel + 1.0e-20))
        for ss in range(len(radius)):
            if ss == s:
                continue
            d = rmh[ss, 0:3] - rmh[s, 0:3]
            dist = max(0.5 * (radius[s] + radius[ss]),
                       np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]))
            e = v[s] - v[ss]
            dt = min(dt, (sink_mult * dist) / (np.sqrt((e[0] * e[0] + e[1] * e[1]) + e[2] * e[2]) +
                                               1.0e-20))
        out[s] = dt
    return out


def rk2_half(r, v, a, dt):
    """advance/advance_runge_kutta.F90:40-54 at the half step (dt = step/2):
    r + v dt, v + a dt."""
    return r + v * dt, v + a * dt


def rk2_full(r_old, v_old, v_half, a_half, dt):
    """advance/advance_runge_kutta.F90:56-69 at the end of the step: r_old +
    v_half dt, v_old + a dt."""
    return r_old + v_half * dt, v_old + a_half * dt


class Oracle(HotPath):
    def __init__(self, pmax: int, params: Params):
        super().__init__(library(), "seren_oracle", pmax, params)

    def counts(self) -> dict:
        c = Counts()
        self._call("get_counts", self._ctx, C.byref(c))
        return c.as_dict()

    def stage_seconds(self) -> list:
        s = (C.c_double * 6)()
        self._call("stage_seconds", self._ctx, s)
        return list(s)

    def direct_gravity(self, ids) -> tuple:
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        a = np.zeros((ids.size, 3))
        g = np.zeros(ids.size)
        self._call("direct_gravity", self._ctx, ids.ctypes.data_as(C.POINTER(C.c_int32)),
                   ids.size, a.ctypes.data_as(C.POINTER(C.c_double)),
                   g.ctypes.data_as(C.POINTER(C.c_double)))
        return a, g
