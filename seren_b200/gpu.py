"""ctypes binding of the CUDA library (the product).

``GpuHotPath`` is a context of libseren_gpu.so with the reference-facing calls
(tree_update, sph_update, get_neib, hydro_forces, grav_forces, sink_forces)
plus the device-resident step (upload, force_step, drift, download).  Loading
raises if the library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import LIB
from .cabi import HotPath, Params, SerenError, bind  # noqa: F401

_lib = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def library(build_if_missing: bool = True) -> C.CDLL:
    """Load libseren_gpu.so (building it with nvcc first if it is missing)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            if not build_if_missing:
                raise RuntimeError(f"{LIB} is missing: run python -m seren_b200.build")
            from .build import build
            build()
        lib = bind(C.CDLL(LIB), "seren_gpu")
        vp = C.c_void_p
        for name, args in (("upload", [vp, C.c_int32, _dp, _dp, _dp]),
                           ("force_step", [vp, C.c_int32]),
                           ("force_step_io", [vp, C.c_int32, _dp, _dp, _dp, C.c_int32, _dp, _dp,
                                              _dp, _dp, _dp, _dp, _dp, _ip]),
                           ("drift", [vp, C.c_double]),
                           ("timestep", [vp, C.c_double, C.c_double, _dp, _dp]),
                           ("rk2_step", [vp, C.c_double]),
                           ("set_sink_motion", [vp, C.c_int32, _dp, _dp]),
                           ("get_sinks", [vp, C.c_int32, _dp, _dp, _dp, _dp]),
                           ("sink_timestep", [vp, C.c_double, _dp]),
                           ("accrete", [vp, C.c_int32, _ip, C.c_int32, _dp, _ip, _ip]),
                           ("sink_search", [vp, C.c_void_p, _ip, _ip, _dp, _ip, _ip]),
                           ("set_build_step", [vp, C.c_int32]),
                           ("set_sinks", [vp, C.c_int32, _dp]),
                           ("download", [vp, _dp, _dp, _dp, _dp, _dp, _dp, _ip]),
                           ("last_step_stats", [vp, _dp, _ip, C.POINTER(C.c_int64)]),
                           ("get_stream", [vp, C.POINTER(C.c_void_p)]),
                           ("fma_peak", [vp, C.c_int32, _dp]),
                           ("block_start", [vp, C.c_void_p]),
                           ("block_step", [vp, C.c_void_p]),
                           ("block_levels", [vp, _ip, C.POINTER(C.c_int64), _ip, _ip]),
                           ("set_clouds", [vp, C.c_int32, _ip]),
                           ("autotune", [vp, C.c_int32, C.c_void_p]),
                           ("set_tuning", [vp, C.c_void_p])):
            fn = getattr(lib, f"seren_gpu_{name}")
            fn.argtypes = args
            fn.restype = C.c_int
        _lib = lib
    return _lib


class SinkSearchParams(C.Structure):
    """seren_gpu_sink_search_params of include/seren_gpu.h."""
    _fields_ = [("rhosink", C.c_double), ("sinkrad", C.c_double)] + [
        (n, C.c_int32) for n in ("hmult_sinkrad", "rho_search", "potmin_search",
                                 "hill_sphere_search", "div_v_search", "div_a_search",
                                 "timescale_search", "reserved")]


class BlockParams(C.Structure):
    """seren_gpu_block_params of include/seren_gpu.h."""
    _fields_ = [("nlevels", C.c_int32), ("level_mode", C.c_int32), ("check_neib", C.c_int32),
                ("reserved", C.c_int32), ("dt_fixed", C.c_double), ("courant_mult", C.c_double),
                ("accel_mult", C.c_double)]


class BlockState(C.Structure):
    """seren_gpu_block_state of include/seren_gpu.h."""
    _fields_ = [("n", C.c_int64), ("nresync", C.c_int64), ("nsteps", C.c_int64),
                ("level_max", C.c_int32), ("level_step", C.c_int32), ("nactive", C.c_int32),
                ("reserved", C.c_int32), ("timestep", C.c_double), ("dt_max", C.c_double),
                ("time", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}


class Tuning(C.Structure):
    """seren_gpu_tuning of include/seren_gpu.h."""
    _fields_ = [("hydro_sub", C.c_int32), ("grav_cap", C.c_int32), ("grav_bps", C.c_int32),
                ("gradh_bps", C.c_int32), ("neib_bps", C.c_int32), ("reserved", C.c_int32),
                ("ms_per_step", C.c_double)]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_ if n != "reserved"}


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


class GpuHotPath(HotPath):
    def __init__(self, pmax: int, params: Params):
        super().__init__(library(), "seren_gpu", pmax, params)
        self.nsink = 0

    # -- device-resident step -------------------------------------------------
    def upload(self, parray, v, csq):
        parray = np.ascontiguousarray(parray, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        csq = np.ascontiguousarray(csq, dtype=np.float64)
        self._call("upload", self._ctx, parray.shape[0], _d(parray), _d(v), _d(csq))
        self.ptot = parray.shape[0]

    def force_step(self, first_call=False):
        self._call("force_step", self._ctx, int(first_call))

    def force_step_io(self, parray, v, csq, first_call=False):
        """One force evaluation from host arrays to host arrays
        (seren_gpu_force_step_io): returns parray, v, csq, rho, omega, a, gpot
        and perm, in tree order."""
        parray = np.ascontiguousarray(parray, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        csq = np.ascontiguousarray(csq, dtype=np.float64)
        n = parray.shape[0]
        out = dict(parray=np.zeros((n, 6)), v=np.zeros((n, 3)), csq=np.zeros(n), rho=np.zeros(n),
                   omega=np.zeros(n), a=np.zeros((n, 3)), gpot=np.zeros(n),
                   perm=np.zeros(n, dtype=np.int32))
        self._call("force_step_io", self._ctx, n, _d(parray), _d(v), _d(csq), int(first_call),
                   _d(out["parray"]), _d(out["v"]), _d(out["csq"]), _d(out["rho"]),
                   _d(out["omega"]), _d(out["a"]), _d(out["gpot"]),
                   out["perm"].ctypes.data_as(_ip))
        self.ptot = n
        return out

    def set_sinks(self, sinks):
        """Sinks ([nsink][5]: x, y, z, m, h) for the device-resident step."""
        s = None if sinks is None else np.ascontiguousarray(np.atleast_2d(sinks), dtype=np.float64)
        ns = 0 if s is None else s.shape[0]
        self._call("set_sinks", self._ctx, ns, None if s is None else _d(s))
        self.nsink = ns

    def set_sink_motion(self, v, radius):
        """Velocities [nsink][3] and radii of the sinks, which rk2_step then
        moves with the gas."""
        v = np.ascontiguousarray(np.atleast_2d(v), dtype=np.float64)
        radius = np.ascontiguousarray(np.atleast_1d(radius), dtype=np.float64)
        self._call("set_sink_motion", self._ctx, v.shape[0], _d(v), _d(radius))

    def get_sinks(self):
        ns = self.nsink
        out = dict(rmh=np.zeros((ns, 5)), v=np.zeros((ns, 3)), a=np.zeros((ns, 3)),
                   gpot=np.zeros(ns))
        self._call("get_sinks", self._ctx, ns, _d(out["rmh"]), _d(out["v"]), _d(out["a"]),
                   _d(out["gpot"]))
        return out

    def sink_timestep(self, sink_mult=0.5):
        d = C.c_double()
        self._call("sink_timestep", self._ctx, C.c_double(sink_mult), C.byref(d))
        return d.value

    def accrete(self, energy_accrete=False, accrete=None, angmom=None):
        """Sink accretion and removal of the accreted particles
        (seren_gpu_accrete).  accrete: per-sink flags (None: every sink);
        angmom [nsink][3] is added to in place when given.  Returns the number
        accreted by each sink; self.ptot becomes the kept count."""
        ns = self.nsink
        flags = None if accrete is None else \
            np.ascontiguousarray(np.atleast_1d(accrete), dtype=np.int32)
        if flags is not None and flags.size != ns:
            raise ValueError("one accrete flag per sink")
        if angmom is not None and (angmom.dtype != np.float64 or angmom.shape != (ns, 3) or
                                   not angmom.flags.c_contiguous):
            raise ValueError("angmom must be a C-contiguous float64 array [nsink][3]")
        cnt = np.zeros(ns, np.int32)
        ptot = C.c_int32()
        self._call("accrete", self._ctx, ns, None if flags is None else flags.ctypes.data_as(_ip),
                   1 if energy_accrete else 0, _d(angmom), cnt.ctypes.data_as(_ip),
                   C.byref(ptot))
        self.ptot = ptot.value
        return cnt

    def sink_search(self, rhosink, sinkrad, hmult_sinkrad=False, rho_search=True,
                    potmin_search=True, hill_sphere_search=True, div_v_search=True,
                    div_a_search=True, timescale_search=False):
        """Sink search and creation (seren_gpu_sink_search); the defaults are
        the reference's (setup/default_parameters.F90:120-129).  Returns a
        dict: created, psink_id, angmom [3], nremoved; self.nsink and
        self.ptot follow."""
        prm = SinkSearchParams(float(rhosink), float(sinkrad), int(hmult_sinkrad), int(rho_search),
                               int(potmin_search), int(hill_sphere_search), int(div_v_search),
                               int(div_a_search), int(timescale_search), 0)
        created, pid, nrem, ptot = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        angmom = np.zeros(3)
        self._call("sink_search", self._ctx, C.cast(C.byref(prm), C.c_void_p), C.byref(created),
                   C.byref(pid), _d(angmom), C.byref(nrem), C.byref(ptot))
        self.ptot = ptot.value
        if created.value:
            self.nsink += 1
        return dict(created=bool(created.value), psink_id=pid.value, angmom=angmom,
                    nremoved=nrem.value)

    def set_build_step(self, nbuildstep: int):
        """Build the tree every nbuildstep device-resident evaluations and
        restock it in between (seren_gpu_set_build_step)."""
        self._call("set_build_step", self._ctx, int(nbuildstep))

    def autotune(self, trials: int = 2) -> dict:
        """Time the kernel knobs on the current state (seren_gpu_autotune) and
        keep the fastest per stage; trials <= 0 applies the choice recorded
        for this size instead."""
        t = Tuning()
        self._call("autotune", self._ctx, int(trials), C.cast(C.byref(t), C.c_void_p))
        return t.as_dict()

    def set_tuning(self, hydro_sub=4, grav_cap=64, grav_bps=0, gradh_bps=0, neib_bps=0):
        t = Tuning(int(hydro_sub), int(grav_cap), int(grav_bps), int(gradh_bps), int(neib_bps), 0,
                   0.0)
        self._call("set_tuning", self._ctx, C.cast(C.byref(t), C.c_void_p))

    def set_clouds(self, counts):
        """The uploaded particles are len(counts) independent clouds, one after
        another (seren_gpu_set_clouds); every force step then builds and walks
        a forest of their trees in single launches."""
        cnt = np.ascontiguousarray(np.atleast_1d(counts), dtype=np.int32)
        self._call("set_clouds", self._ctx, int(cnt.size), cnt.ctypes.data_as(_ip))

    def block_start(self, nlevels=3, level_mode=1, check_neib=1, dt_fixed=1.0,
                    courant_mult=0.2, accel_mult=0.5):
        """Block timesteps from the state of the last force step
        (seren_gpu_block_start)."""
        prm = BlockParams(int(nlevels), int(level_mode), int(check_neib), 0, float(dt_fixed),
                          float(courant_mult), float(accel_mult))
        self._call("block_start", self._ctx, C.cast(C.byref(prm), C.c_void_p))

    def block_step(self) -> dict:
        """One integer step of the block-timestep loop (seren_gpu_block_step);
        returns the time scalars after it."""
        st = BlockState()
        self._call("block_step", self._ctx, C.cast(C.byref(st), C.c_void_p))
        return st.as_dict()

    def block_levels(self) -> dict:
        """Per-particle level state in tree order: nlevel, nlast, nminneib, accdo."""
        n = self.ptot
        out = dict(nlevel=np.zeros(n, np.int32), nlast=np.zeros(n, np.int64),
                   nminneib=np.zeros(n, np.int32), accdo=np.zeros(n, np.int32))
        self._call("block_levels", self._ctx, out["nlevel"].ctypes.data_as(_ip),
                   out["nlast"].ctypes.data_as(C.POINTER(C.c_int64)),
                   out["nminneib"].ctypes.data_as(_ip), out["accdo"].ctypes.data_as(_ip))
        return out

    def drift(self, dt: float):
        self._call("drift", self._ctx, C.c_double(dt))

    def timestep(self, courant_mult=0.2, accel_mult=0.5, per_particle=False):
        """Least particle timestep (seren_gpu_timestep) of the last force
        evaluation; with per_particle, also every particle's (tree order)."""
        dmin = C.c_double()
        dt = np.zeros(self.ptot) if per_particle else None
        self._call("timestep", self._ctx, C.c_double(courant_mult), C.c_double(accel_mult),
                   C.byref(dmin), _d(dt))
        return (dmin.value, dt) if per_particle else dmin.value

    def rk2_step(self, dt: float):
        """One second-order Runge-Kutta step of dt on the device
        (seren_gpu_rk2_step): two force evaluations."""
        self._call("rk2_step", self._ctx, C.c_double(dt))

    def download(self):
        n = self.ptot
        out = dict(parray=np.zeros((n, 6)), v=np.zeros((n, 3)), rho=np.zeros(n),
                   omega=np.zeros(n), a=np.zeros((n, 3)), gpot=np.zeros(n),
                   perm=np.zeros(n, dtype=np.int32))
        self._call("download", self._ctx, _d(out["parray"]), _d(out["v"]), _d(out["rho"]),
                   _d(out["omega"]), _d(out["a"]), _d(out["gpot"]),
                   out["perm"].ctypes.data_as(_ip))
        return out

    def last_step_stats(self):
        """(stage milliseconds [8], kernel launches, work counters [16]) of the
        last force_step; counts[0] cell terms, counts[1] pair terms (the slots
        are listed at seren_gpu_last_step_stats)."""
        ms = (C.c_double * 8)()
        nl = C.c_int32()
        cnt = (C.c_int64 * 16)()
        self._call("last_step_stats", self._ctx, ms, C.byref(nl), cnt)
        return list(ms), nl.value, list(cnt)

    def stream(self) -> int:
        """The cudaStream_t (as an int) all kernels of this context run on."""
        s = C.c_void_p()
        self._call("get_stream", self._ctx, C.byref(s))
        return int(s.value or 0)

    def fma_peak(self, precision: int) -> float:
        """Measured FMA throughput in TFLOP/s of the FP32 (1) or FP64 (0) pipe."""
        t = C.c_double()
        self._call("fma_peak", self._ctx, int(precision), C.byref(t))
        return t.value
