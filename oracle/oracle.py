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
    """sinks/accrete_particles.F90:16-365 and main/remove_from_list.F90:10-96
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


def _is_potmin(r, h, gpot, p):
    """sph/all_sph_gradh.F90:355-471: the particle's -gpot is below every
    gather neighbour's (within 2h, kernel bin <= KERNTOT) and below 0."""
    hp = float(h[p])
    invhp = 1.0 / hp
    dr = r - r[p]
    drsqd = (dr[:, 0] * dr[:, 0] + dr[:, 1] * dr[:, 1]) + dr[:, 2] * dr[:, 2]
    near = drsqd <= (4.0 * hp) * hp
    near[p] = False
    drmag = np.sqrt(drsqd[near]) + 1.0e-20
    ok = ((5000.0 * drmag) * invhp).astype(np.int64) <= KERNTOT
    gmin = 0.0
    if ok.any():
        gmin = min(0.0, float(np.min(-gpot[near][ok])))
    return gmin > -float(gpot[p])


def sink_search(r, m, h, v, a, rho, gpot, sink_rmh, sink_v, sink_a, sink_radius,
                rhosink, sinkrad, hmult_sinkrad=False, rho_search=True, potmin_search=True,
                hill_sphere_search=True, div_v_search=True, div_a_search=True,
                timescale_search=False):
    """sinks/sink_search.F90:25-433 and sinks/create_sink.F90:11-268 on
    particles in tree order (r [N,3], m, h, v [N,3], a [N,3], rho, gpot) with
    existing sinks (rmh [S,5], v, a [S,3], radius [S]).  Returns psink (-1: no sink made), the
    candidates in density order with their flags, and for a new sink its
    state (m, r, v, a, h, radius, angmom), the removed particles (psink and
    its neighbours within the sink radius, in index order) and the kept ones.
    Kept as the reference has them: the Hill test reads the particles' a_grav
    and the sinks' agrav, which only DEBUG_FORCES builds fill
    (sph_sim/sph_grav_forces.F90:128-130; otherwise zero, so the test never
    rejects); div a divides by the
    dot product of the relative acceleration and separation; the particle
    made a sink is the one the last candidate loop visited last (:405-413
    assign psink = p), which can be a candidate that failed that loop's
    test when a lower-density one passed."""
    r, v, a = (np.asarray(x, np.float64).reshape(-1, 3) for x in (r, v, a))
    m, h, rho, gpot = (np.asarray(x, np.float64).ravel() for x in (m, h, rho, gpot))
    rmh = np.array(sink_rmh, np.float64).reshape(-1, 5)
    sv = np.array(sink_v, np.float64).reshape(-1, 3)
    sa = np.array(sink_a, np.float64).reshape(-1, 3)
    srad = np.asarray(sink_radius, np.float64).ravel()
    n, stot = r.shape[0], rmh.shape[0]
    t = kernel_tables()
    w0, w1, w4 = t[0].tolist(), t[1].tolist(), t[4].tolist()
    out = dict(psink=-1, candidates=[], flags=[])
    cand = [p for p in range(n)
            if not (rho_search and rho[p] < rhosink)
            and not (potmin_search and not _is_potmin(r, h, gpot, p))]
    if not cand:
        return out
    cand.sort(key=lambda p: float(rho[p]))          # stable, as insertion_sort_real
    k = len(cand)
    flag = [True] * k
    srho = [float(rho[p]) for p in cand]
    if stot > 0:                                    # :155-200
        for i, p in enumerate(cand):
            rp = r[p].tolist()
            for s in range(stot):
                dr = [float(rmh[s, c]) - rp[c] for c in range(3)]
                drsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2]
                if drsqd < (2.0 * float(srad[s])) * (2.0 * float(srad[s])):
                    flag[i] = False
                if hill_sphere_search:
                    da = [0.0, 0.0, 0.0]                # sink agrav - particle a_grav
                    dadr = (da[0] * dr[0] + da[1] * dr[1]) + da[2] * dr[2]
                    rho_hill = -(3.0 * dadr) / ((4.0 * 3.1415926536) * drsqd)
                    if srho[i] < 3.0 * rho_hill:
                        flag[i] = False
    last = -1                                       # the last candidate a loop visits
    div_v = [0.0] * k
    for i, p in enumerate(cand):                    # :221-300
        if not flag[i]:
            continue
        last = i
        rp, vp, ap = r[p].tolist(), v[p].tolist(), a[p].tolist()
        hp = float(h[p])
        hrange = max(sinkrad * hp, 2.0 * hp) if hmult_sinkrad else max(sinkrad, 2.0 * hp)
        hrangesqd = hrange * hrange
        invhp = 2.0 / hrange
        hfactor = math.pow(invhp, 3.0)
        d = r - r[p]
        dsq = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        rhotemp = (float(m[p]) * w0[0]) * hfactor
        dv_p, da_p, curl = 0.0, 0.0, [0.0, 0.0, 0.0]
        for pp in np.flatnonzero(dsq <= hrangesqd).tolist():
            if pp == p:
                continue
            dr = d[pp].tolist()
            drmag = math.sqrt(float(dsq[pp])) + 1.0e-20
            invdrmag = 1.0 / drmag
            kern = int((5000.0 * drmag) * invhp)
            if kern > KERNTOT:
                continue
            mpp = float(m[pp])
            dv = [float(v[pp, c]) - vp[c] for c in range(3)]
            dvdr = (dv[0] * dr[0] + dv[1] * dr[1]) + dv[2] * dr[2]
            rhotemp = rhotemp + (mpp * hfactor) * w0[kern]
            dv_p = dv_p - ((((mpp * dvdr) * w4[kern]) * hfactor) * invhp) * invdrmag
            dadr = ((float(a[pp, 0]) - ap[0]) * dr[0] + (float(a[pp, 1]) - ap[1]) * dr[1]) + \
                (float(a[pp, 2]) - ap[2]) * dr[2]
            da_p = da_p - ((((mpp * w4[kern]) * hfactor) * invhp) / dadr) * invdrmag
            x = [dv[1] * dr[2] - dv[2] * dr[1], dv[2] * dr[0] - dv[0] * dr[2],
                 dv[0] * dr[1] - dv[1] * dr[0]]
            curl = [curl[c] - ((((mpp * x[c]) * invdrmag) * w1[kern]) * hfactor) * invhp
                    for c in range(3)]
        div_v[i] = dv_p / rhotemp
        if div_a_search and da_p / rhotemp > 0.0:
            flag[i] = False
        if div_v_search and div_v[i] > 0.0:
            flag[i] = False
    if stot > 0:                                    # :328-400, only tacc1 and tcond1 decide
        last = -1
        for i, p in enumerate(cand):
            if not flag[i]:
                continue
            last = i
            rp, vp = r[p].tolist(), v[p].tolist()
            for s in range(stot):
                dr = [float(rmh[s, c]) - rp[c] for c in range(3)]
                drmag = math.sqrt((dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2]) + 1.0e-20
                du = [dr[c] / drmag for c in range(3)]
                dv = [float(sv[s, c]) - vp[c] for c in range(3)]
                drad = drmag - 2.0 * float(srad[s])
                vrad = (dv[0] * du[0] + dv[1] * du[1]) + dv[2] * du[2]
                tacc1 = -drad / vrad
                tcond1 = -1.0 / div_v[i]
                if timescale_search and tcond1 > tacc1:
                    flag[i] = False
    out["candidates"], out["flags"] = cand, flag
    if not any(flag) or last < 0:
        return out
    psink = cand[last]
    out["psink"] = psink
    # create_sink.F90:64-244
    rp, vp = r[psink].tolist(), v[psink].tolist()
    mp, hp = float(m[psink]), float(h[psink])
    msink = mp
    rs = [mp * x for x in rp]
    vs = [mp * x for x in vp]
    asn = [mp * x for x in a[psink].tolist()]
    rads = sinkrad * hp if hmult_sinkrad else sinkrad
    hh = 0.5 * rads
    d = r - r[psink]
    dsq = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
    neib = [pp for pp in np.flatnonzero(dsq <= (4.0 * hh) * hh).tolist() if pp != psink]
    for pp in neib:
        mpp = float(m[pp])
        msink = msink + mpp
        for c in range(3):
            rs[c] = rs[c] + mpp * float(r[pp, c])
            vs[c] = vs[c] + mpp * float(v[pp, c])
            asn[c] = asn[c] + mpp * float(a[pp, c])
    rs = [x / msink for x in rs]
    vs = [x / msink for x in vs]
    asn = [x / msink for x in asn]
    dr = [rs[c] - rp[c] for c in range(3)]
    dv = [vs[c] - vp[c] for c in range(3)]
    L = [(mp * dr[1]) * dv[2] - (mp * dr[2]) * dv[1], (mp * dr[2]) * dv[0] - (mp * dr[0]) * dv[2],
         (mp * dr[0]) * dv[1] - (mp * dr[1]) * dv[0]]
    for pp in neib:
        mpp = float(m[pp])
        dv = [vs[c] - float(v[pp, c]) for c in range(3)]
        dr = [rs[c] - float(r[pp, c]) for c in range(3)]
        L = [(L[0] + (mpp * dr[1]) * dv[2]) - (mpp * dr[2]) * dv[1],
             (L[1] + (mpp * dr[2]) * dv[0]) - (mpp * dr[0]) * dv[2],
             (L[2] + (mpp * dr[0]) * dv[1]) - (mpp * dr[1]) * dv[0]]
    removed = sorted(neib + [psink])
    gone = set(removed)
    out.update(m=msink, r=np.array(rs), v=np.array(vs), a=np.array(asn), h=0.5 * rads,
               radius=rads, angmom=np.array(L), removed=np.array(removed, np.int64),
               keep=np.array([p for p in range(n) if p not in gone], np.int64))
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
