"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle library.

The oracle (oracle/seren_oracle.cpp) is a FP64 restatement of the reference's
Fortran force path and is the checker for the CUDA library; only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it.  Parity is
unpinned: the reference ships no golden vectors and cannot be compiled here.
"""
from __future__ import annotations

import ctypes as C
import math
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


def _accrete_pot(d, invhp, hq, mq, w6):
    """gravity/gravity_gradh.F90:11-95, the potential only (zeta/omega = 0);
    accrete_particles.F90:186-188 passes the sink's 1/h as hq."""
    drsqd = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]
    drmag = math.sqrt(drsqd) + 1.0e-20
    invdrmag = 1.0 / drmag
    if invdrmag > 0.5 * invhp:
        kern = min(int((5000.0 * drmag) * invhp), KERNTOT)
        dpot = invhp * w6[kern]
    else:
        dpot = invdrmag
    if drmag < 2.0 * hq:
        invhq = 1.0 / hq
        kern = min(int((5000.0 * drmag) * invhq), KERNTOT)
        dpot = dpot + invhq * w6[kern]
    else:
        dpot = dpot + invdrmag
    return (0.5 * mq) * dpot


def accrete_particles(r, m, h, v, a, sink_rmh, sink_v, sink_a, sink_radius, accrete=None,
                      energy_accrete=False):
    """sinks/accrete_particles.F90:14-365 and main/remove_from_list.F90:10-96
    for particles r [N,3], m, h, v, a [N,3] (all gas) and sinks rmh [S,5] (x,
    y, z, m, h), v, a [S,3], radius [S].  Every particle inside an accreting
    sink's radius goes to the nearest such sink (:82-106; a later sink only
    when strictly nearer); with energy_accrete it must be bound to it
    (:165-205).  Each sink with accreted particles takes their mass and moves
    to the centre of mass, velocity and mass-weighted acceleration, summed in
    particle order, and gains the angular momentum about that centre
    (:233-281).  Returns dead (sink per particle, -1 kept), keep (kept
    particles in order), count per sink, the new sink rmh, v, a and the
    angular momentum added to each sink."""
    r, v, a = (np.asarray(x, np.float64).reshape(-1, 3) for x in (r, v, a))
    m, h = (np.asarray(x, np.float64).ravel() for x in (m, h))
    rmh = np.array(sink_rmh, np.float64).reshape(-1, 5)
    sv = np.array(sink_v, np.float64).reshape(-1, 3)
    sa = np.array(sink_a, np.float64).reshape(-1, 3)
    rad = np.asarray(sink_radius, np.float64).ravel()
    ns, n = rmh.shape[0], r.shape[0]
    acc = [True] * ns if accrete is None else [bool(x) for x in accrete]
    w6 = kernel_tables()[6].tolist()
    dead = [-1] * n
    for p in range(n):
        rp = r[p].tolist()
        flag, best = -1, 0.0
        for s in range(ns):
            if not acc[s]:
                continue
            d = [rp[k] - float(rmh[s, k]) for k in range(3)]
            drsqd = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]
            rads = float(rad[s])
            if drsqd < rads * rads and (flag == -1 or drsqd < best):
                flag, best = s, drsqd
        if flag < 0:
            continue
        if energy_accrete:
            ms, mp = float(rmh[flag, 3]), float(m[p])
            e = [float(sv[flag, k]) - float(v[p, k]) for k in range(3)]
            reduced_mass = (ms * mp) / (ms + mp)
            dpotp = _accrete_pot([float(rmh[flag, k]) - rp[k] for k in range(3)], 1.0 / float(h[p]),
                                 1.0 / float(rmh[flag, 4]), ms, w6)
            total = ((0.5 * reduced_mass) * ((e[0] * e[0] + e[1] * e[1]) + e[2] * e[2])) - dpotp * mp
            if not total < 0.0:
                continue
        dead[p] = flag
    new_rmh, new_v, new_a = rmh.copy(), sv.copy(), sa.copy()
    angmom = np.zeros((ns, 3))
    count = np.zeros(ns, np.int64)
    for s in range(ns):
        if not acc[s]:
            continue
        mine = [p for p in range(n) if dead[p] == s]
        if not mine:
            continue
        ms = float(rmh[s, 3])
        rs, vs = rmh[s, 0:3].tolist(), sv[s].tolist()
        mt = ms
        rc = [ms * x for x in rs]
        vc = [ms * x for x in vs]
        ac = [ms * x for x in sa[s].tolist()]
        for p in mine:
            mp = float(m[p])
            mt = mt + mp
            for k in range(3):
                rc[k] = rc[k] + mp * float(r[p, k])
                vc[k] = vc[k] + mp * float(v[p, k])
                ac[k] = ac[k] + mp * float(a[p, k])
        rc = [x / mt for x in rc]
        vc = [x / mt for x in vc]
        ac = [x / mt for x in ac]
        L = [0.0, 0.0, 0.0]

        def add(L, mq, d, e):
            return [(L[0] + (mq * d[1]) * e[2]) - (mq * d[2]) * e[1],
                    (L[1] + (mq * d[2]) * e[0]) - (mq * d[0]) * e[2],
                    (L[2] + (mq * d[0]) * e[1]) - (mq * d[1]) * e[0]]
        L = add(L, ms, [rs[k] - rc[k] for k in range(3)], [vs[k] - vc[k] for k in range(3)])
        for p in mine:
            L = add(L, float(m[p]), [rc[k] - float(r[p, k]) for k in range(3)],
                    [vc[k] - float(v[p, k]) for k in range(3)])
        new_rmh[s, 0:3], new_rmh[s, 3] = rc, mt
        new_v[s], new_a[s], angmom[s], count[s] = vc, ac, L, len(mine)
    keep = np.array([p for p in range(n) if dead[p] < 0], np.int64)
    return dict(dead=np.array(dead, np.int64), keep=keep, count=count, rmh=new_rmh, v=new_v,
                a=new_a, angmom=angmom)


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
