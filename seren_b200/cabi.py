"""ctypes binding of the force-path C ABI (include/seren_gpu.h).

``HotPath`` wraps one context of a library that exports the seren_gpu_* entry
points.  Arrays are numpy float64/int32, C-contiguous, shaped like the
Fortran module arrays they stand for (parray [N, 6], v and a [N, 3], pplist
[N, pp_limit]).  Every call checks the returned status and raises
``SerenError`` with the library's own message.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

__all__ = ["Params", "SerenError", "HotPath", "ERRORS"]

ERRORS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CAPACITY", 3: "ERR_LMAX", 4: "ERR_NONFINITE",
          5: "ERR_WALK", 6: "ERR_NEGATIVE_H", 7: "ERR_CUDA", 8: "ERR_STATE"}


class SerenError(RuntimeError):
    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)} ({code}): {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [("ndim", C.c_int32), ("kernel", C.c_int32), ("visc", C.c_int32),
                ("precision", C.c_int32), ("pp_gather", C.c_int32), ("pp_limit", C.c_int32),
                ("leafmax", C.c_int32), ("lmax", C.c_int32), ("index_base", C.c_int32),
                ("redo_cap", C.c_int32), ("h_fac", C.c_double), ("thetamaxsqd", C.c_double),
                ("alpha", C.c_double), ("alpha_min", C.c_double)]

    @classmethod
    def make(cls, h_fac=1.2, thetamaxsqd=0.25, alpha=1.0, precision=0, kernel=0,
             pp_gather=None, index_base=0, lmax=30, redo_cap=0):
        from .ics import pp_gather_for
        ppg = pp_gather_for(h_fac) if pp_gather is None else int(pp_gather)
        return cls(3, kernel, 0, precision, ppg, 2 * ppg, 8, lmax, index_base, int(redo_cap),
                   float(h_fac), float(thetamaxsqd), float(alpha), 0.1)


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _i(a):
    return None if a is None else a.ctypes.data_as(_ip)


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape)
    return a


def bind(lib: C.CDLL, prefix: str) -> C.CDLL:
    """Declare argument types of the prefix_* entry points on lib."""
    def f(name, args, res=C.c_int):
        fn = getattr(lib, f"{prefix}_{name}")
        fn.argtypes = args
        fn.restype = res
        return fn
    vp = C.c_void_p
    f("create", [C.POINTER(vp), C.c_int64, C.POINTER(Params)])
    f("destroy", [vp], None)
    f("last_error", [vp, C.c_char_p, C.c_int32])
    f("tree_update", [vp, C.c_int32, _dp, C.c_int32, C.c_int32, _ip])
    f("sph_update", [vp, C.c_int32, _ip, C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _ip,
                     C.c_int32])
    f("get_neib", [vp, C.c_int32, _ip, C.c_int32, _dp, _ip, _ip])
    f("h_gather", [vp, C.c_int32, _ip, C.c_int32, _dp])
    f("hydro_forces", [vp, _ip, C.c_int32, _dp, _dp, _dp])
    f("grav_forces", [vp, _ip, C.c_int32, _dp, _dp, C.c_int32, _dp])
    f("sink_forces", [vp, C.c_int32, _dp, _dp, _dp])
    f("tree_export", [vp, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp,
                      _dp])
    return lib


class HotPath:
    """One context of the force hot path behind the C ABI named by prefix."""

    def __init__(self, lib: C.CDLL, prefix: str, pmax: int, params: Params):
        self.lib = lib
        self.prefix = prefix
        self.params = params
        self.pmax = int(pmax)
        self.ptot = 0
        self._ctx = C.c_void_p()
        self._call("create", C.byref(self._ctx), C.c_int64(self.pmax), C.byref(params))

    # -- plumbing -----------------------------------------------------------
    def _fn(self, name):
        return getattr(self.lib, f"{self.prefix}_{name}")

    def _call(self, name, *args):
        rc = self._fn(name)(*args)
        if rc != 0:
            msg = ""
            if self._ctx:
                buf = C.create_string_buffer(512)
                self._fn("last_error")(self._ctx, buf, 512)
                msg = buf.value.decode(errors="replace")
            raise SerenError(rc, f"{self.prefix}_{name}", msg)

    def close(self):
        if self._ctx:
            self._fn("destroy")(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _acc(self, acclist):
        if acclist is None:
            return None, 0
        a = np.ascontiguousarray(acclist, dtype=np.int32)
        return a, a.size

    # -- the reference-facing calls ------------------------------------------
    def tree_update(self, parray, do_build=True, do_reorder=True):
        """Returns (parray in tree order, perm) with perm[new] = old id."""
        parray = _f64(parray).copy()
        n = parray.shape[0]
        perm = np.empty(n, dtype=np.int32)
        self._call("tree_update", self._ctx, n, _d(parray), int(do_build), int(do_reorder),
                   _i(perm))
        self.ptot = n
        return parray, perm

    def sph_update(self, parray, v, first_call=False, acclist=None, lists=True):
        n = self.ptot
        parray = _f64(parray).copy()
        v = _f64(v)
        out = {k: np.zeros(n) for k in ("rho", "omega", "div_v", "drhodt")}
        L = self.params.pp_limit
        pptot = np.zeros(n, dtype=np.int32) if lists else None
        pplist = np.full((n, L), -1, dtype=np.int32) if lists else None
        acc, nacc = self._acc(acclist)
        self._call("sph_update", self._ctx, n, _i(acc), nacc, _d(parray), _d(v), _d(out["rho"]),
                   _d(out["omega"]), _d(out["div_v"]), _d(out["drhodt"]), _i(pptot), _i(pplist),
                   int(first_call))
        out["parray"] = parray
        out["pptot"] = pptot
        out["pplist"] = pplist
        return out

    def get_neib(self, h=None, acclist=None):
        n = self.ptot
        L = self.params.pp_limit
        pptot = np.zeros(n, dtype=np.int32)
        pplist = np.full((n, L), -1, dtype=np.int32)
        hh = None if h is None else _f64(h)
        acc, nacc = self._acc(acclist)
        self._call("get_neib", self._ctx, n, _i(acc), nacc, _d(hh), _i(pptot), _i(pplist))
        return pptot, pplist

    def h_gather(self, parray, acclist=None):
        """Standard-SPH smoothing lengths from exactly pp_gather neighbours
        (sph/h_gather.F90) for the active particles of the last tree; returns
        parray with column 4 (h) updated for them."""
        parray = _f64(parray).copy()
        acc, nacc = self._acc(acclist)
        self._call("h_gather", self._ctx, self.ptot, _i(acc), nacc, _d(parray))
        return parray

    def hydro_forces(self, press, sound, a=None, acclist=None):
        n = self.ptot
        a = np.zeros((n, 3)) if a is None else _f64(a).copy()
        acc, nacc = self._acc(acclist)
        self._call("hydro_forces", self._ctx, _i(acc), nacc, _d(_f64(press)), _d(_f64(sound)),
                   _d(a))
        return a

    def grav_forces(self, a=None, sinks=None, acclist=None):
        n = self.ptot
        a = np.zeros((n, 3)) if a is None else _f64(a).copy()
        gpot = np.zeros(n)
        ns = 0 if sinks is None else int(np.asarray(sinks).shape[0])
        sk = None if sinks is None else _f64(sinks)
        acc, nacc = self._acc(acclist)
        self._call("grav_forces", self._ctx, _i(acc), nacc, _d(a), _d(gpot), ns, _d(sk))
        return a, gpot

    def sink_forces(self, sinks):
        sk = _f64(sinks)
        ns = sk.shape[0]
        sa = np.zeros((ns, 3))
        sp = np.zeros(ns)
        self._call("sink_forces", self._ctx, ns, _d(sk), _d(sa), _d(sp))
        return sa, sp

    def tree_export(self):
        ctot = C.c_int32()
        ltot = C.c_int32()
        self._call("tree_export", self._ctx, C.byref(ctot), C.byref(ltot), *([None] * 13))
        nc = ctot.value + 1
        out = dict(ctot=ctot.value, ltot=ltot.value,
                   leaf=np.zeros(nc, np.int32), nextcell=np.zeros(nc, np.int32),
                   ifopen=np.zeros(nc, np.int32), plist=np.zeros((nc, 8), np.int32),
                   first_cell=np.zeros(ltot.value + 1, np.int32),
                   last_cell=np.zeros(ltot.value + 1, np.int32),
                   grav_r=np.zeros((nc, 3)), grav_m=np.zeros(nc), grav_q=np.zeros((nc, 5)),
                   dminsqd=np.zeros(nc), hydro_r=np.zeros((nc, 3)), rmax=np.zeros(nc),
                   hrangemax=np.zeros(nc))
        o = out
        self._call("tree_export", self._ctx, C.byref(ctot), C.byref(ltot), _i(o["leaf"]),
                   _i(o["nextcell"]), _i(o["ifopen"]), _i(o["plist"]), _i(o["first_cell"]),
                   _i(o["last_cell"]), _d(o["grav_r"]), _d(o["grav_m"]), _d(o["grav_q"]),
                   _d(o["dminsqd"]), _d(o["hydro_r"]), _d(o["rmax"]), _d(o["hrangemax"]))
        return out
