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
        "hydro_pairs", "hydro_visc", "gradh_bisections")]

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


INVLOGETWO = 1.442695041              # headers/macros.h:15
TIMESTEP_LEVEL_DIFF_MAX = 2           # headers/macros.h:185


def _level(dt_max, dt):
    """int(INVLOGETWO*log(dt_max/dt)) + 1 (sph_timesteps.F90:105, :169) with
    libm's log and Fortran's truncation toward zero."""
    return int(INVLOGETWO * math.log(dt_max / dt)) + 1


class BlockSteps:
    """Block timesteps of the reference's main loop for the second-order
    Runge-Kutta scheme with the isothermal grad-h force path
    (sph_sim/sph_integrate.F90:27-136): per call, tree_update on its build
    schedule, the forces of the accdo particles (sph_update, thermal, hydro,
    gravity), sph_timesteps (sph_sim/sph_timesteps.F90:11-341),
    check_neighbour_timesteps (timestep/check_neighbour_timesteps.F90:11-85),
    advance_runge_kutta for every particle (advance/advance_runge_kutta.F90:
    9-111) and, with IMMEDIATE_TIMESTEP_REDUCTION, reduce_timesteps
    (timestep/reduce_timesteps.F90, reduce_particle_timestep.F90).  The forces
    come from `hp` (the C++ oracle); every per-particle array is kept in its
    tree order and permuted at each build, as reorder_particle_arrays does.
    level_mode: 0 free, 1 RESTRICTED_TIMESTEP_LEVELS, 2 FIXED_TIMESTEP_LEVELS;
    check_neib: the CHECK_NEIB_TIMESTEP option (0, 1 or 2).  No sinks."""

    def __init__(self, hp, ic, nlevels=3, level_mode=1, check_neib=1, dt_fixed=1.0,
                 courant_mult=0.2, accel_mult=0.5, nbuildstep=1):
        self.hp, self.alpha = hp, float(ic["alpha"])
        self.nlevels, self.level_mode, self.check_neib = int(nlevels), int(level_mode), int(check_neib)
        self.dt_fixed, self.courant, self.accel = float(dt_fixed), float(courant_mult), float(accel_mult)
        self.nbuildstep = int(nbuildstep)
        # sph_setup: the first evaluation of every particle
        p, perm = hp.tree_update(ic["parray"])
        v = np.ascontiguousarray(ic["v"][perm], dtype=np.float64)
        self.csq = np.ascontiguousarray(ic["sound"][perm] ** 2, dtype=np.float64)
        s = hp.sph_update(p, v, first_call=True)
        self.perm = perm.astype(np.int64)
        self.parray, self.v = s["parray"], v
        self.rho, self.omega, self.div_v = s["rho"], s["omega"], s["div_v"]
        self._forces(None)
        n = p.shape[0]
        # initialize_sph_variables_2.F90:72-73, :157; initialize_seren_variables_2.F90:60-61
        self.r_old, self.v_old = self.parray[:, 0:3].copy(), self.v.copy()
        self.v_half = np.zeros((n, 3))
        self.accdo = np.zeros(n, bool)
        self.nlast = np.zeros(n, np.int64)
        self.nlevel = np.zeros(n, np.int64)
        self.nminneib = np.zeros(n, np.int64)
        self.laststep = np.zeros(n)
        self.n = self.nresync = self.nsteps = 0
        self.level_max = self.level_step = 0
        self.timestep = self.dt_max = self.time = 0.0
        self.since_build = 1
        self.nactive = n

    def _forces(self, act):
        """thermal (sph/thermal.F90:52-59: press = c_s^2 rho, sound = sqrt(press/rho)),
        hydro and gravity for the particles act (None: all)."""
        hp = self.hp
        press = self.csq * self.rho
        self.press, self.sound = press, np.sqrt(press / self.rho)
        a_h = hp.hydro_forces(press, self.sound, acclist=act)
        a, gpot = hp.grav_forces(a_h, acclist=act)
        if act is None:
            self.a, self.gpot = a, gpot
        else:
            self.a[act], self.gpot[act] = a[act], gpot[act]

    def _permute(self, perm):
        for k in ("parray", "v", "csq", "rho", "omega", "div_v", "a", "gpot", "r_old", "v_old",
                  "v_half", "accdo", "nlast", "nlevel", "nminneib", "laststep"):
            setattr(self, k, getattr(self, k)[perm])
        self.perm = self.perm[perm]

    def step(self):
        hp = self.hp
        build = self.since_build >= self.nbuildstep               # main/tree_update.F90
        p, perm = hp.tree_update(self.parray, do_build=build)
        if build:
            self._permute(perm.astype(np.int64))
            self.since_build = 0
        self.since_build += 1
        self.parray[:, 0:3] = p[:, 0:3]
        act = np.nonzero(self.accdo)[0].astype(np.int32)
        self.nactive = int(act.size)
        lists = None
        if act.size:                                               # sph_integrate.F90:36-66
            s = hp.sph_update(self.parray, self.v, acclist=act)
            self.parray[act, 4:6] = s["parray"][act, 4:6]
            for k in ("rho", "omega", "div_v"):
                getattr(self, k)[act] = s[k][act]
            lists = (s["pptot"], s["pplist"])
            self._forces(act)
        self._timesteps()
        if self.check_neib >= 1 and act.size:
            self._check_neighbours(act, lists)
        self._advance()
        if self.check_neib == 2:
            self._reduce()

    def _timesteps(self):
        """sph_sim/sph_timesteps.F90:11-341 (no sinks)."""
        dt_all = timestep_sizes(self.parray[:, 4], self.a, self.div_v, self.sound, self.alpha,
                                self.courant, self.accel)
        n_p = len(dt_all)
        if self.n == self.nresync:                                 # :47-147
            self.n = 0
            self.nlast[:] = 0
            dt_min = float(dt_all.min())
            level_max = self.nlevels - 1
            if self.level_mode == 1:
                level = _level(self.dt_fixed, dt_min)
                dt_min = self.dt_fixed / 2.0 ** level
            elif self.level_mode == 2:
                dt_min = self.dt_fixed / 2.0 ** level_max
            dt_max = dt_min * 2.0 ** level_max
            for p in range(n_p):
                lev = max(min(_level(dt_max, float(dt_all[p])), level_max), 0)
                self.nlevel[p] = lev
                if self.check_neib >= 1:
                    self.nminneib[p] = lev
            self.level_max, self.dt_max = level_max, dt_max
            self.level_step = level_max + 1
            self.nresync = 2 ** self.level_step
            self.timestep = dt_max / float(self.nresync)
        else:                                                      # :152-296
            level_old = self.level_max
            n, level_step = self.n, self.level_step
            p_update = 0
            for p in range(n_p):
                if n == self.nlast[p]:
                    p_update += 1
                    last = int(self.nlevel[p])
                    level = max(_level(self.dt_max, float(dt_all[p])), 0)
                    if level < last and last > 1 and n % 2 ** (level_step - (last - 1)) == 0:
                        self.nlevel[p] = last - 1
                    elif level > last:
                        self.nlevel[p] = level
                    else:
                        self.nlevel[p] = last
            if p_update > 0:
                level_max = int(self.nlevel.max())
                if level_max <= level_old - 1 and level_old > 1 and \
                        n % 2 ** (level_step - (level_old - 1)) == 0:
                    level_max = level_old - 1
                elif level_max < level_old:
                    level_max = level_old
                if self.check_neib >= 1:                           # :236-249
                    D = TIMESTEP_LEVEL_DIFF_MAX
                    for p in range(n_p):
                        self.nminneib[p] = min(int(self.nminneib[p]), level_max)
                        mn, lv = int(self.nminneib[p]), int(self.nlevel[p])
                        if mn - lv > D and self.nlast[p] == n and \
                                n % 2 ** (level_step - mn + D) == 0:
                            self.nlevel[p] = min(mn - D, level_max)
                            self.nminneib[p] = self.nlevel[p]
                        elif self.nlast[p] == n:
                            self.nminneib[p] = lv
                if level_max > level_old:                          # :259-273
                    f = 2 ** (level_max - level_old)
                    self.nlast *= f
                    self.n *= f
                    self.nresync *= f
                elif level_max < level_old:
                    f = 2 ** (level_old - level_max)
                    self.nlast //= f
                    self.n //= f
                    self.nresync //= f
                self.level_max = level_max
                self.level_step = level_max + 1
                self.timestep = self.dt_max / float(self.nresync)
        self.n += 1                                                # :333-336
        self.nsteps += 1
        self.time += self.timestep

    def _check_neighbours(self, act, lists):
        """timestep/check_neighbour_timesteps.F90:41-68: every active
        particle's level reaches its neighbours' nminneib (list of get_neib,
        or the same test on the fly when it overflowed)."""
        pptot, pplist = lists
        L = self.hp.params.pp_limit
        x, h = self.parray[:, 0:3], self.parray[:, 4]
        for p in act:
            lev = int(self.nlevel[p])
            if pptot[p] <= L:
                neib = pplist[p, :pptot[p]] - self.hp.params.index_base
            else:                                                  # get_neib_on_fly
                d = x - x[p]
                r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
                ok = (r2 <= (4.0 * h[p]) * h[p]) | (r2 <= (4.0 * h) * h)
                ok[p] = False
                neib = np.nonzero(ok)[0]
            for pp in neib:
                if lev > self.nminneib[pp] and self.nminneib[pp] != -1:
                    self.nminneib[pp] = lev

    def _advance(self):
        """advance/advance_runge_kutta.F90:20-97 for every particle."""
        dn = self.n - self.nlast
        nfull = 2 ** (self.level_step - self.nlevel)
        nhalf = nfull // 2
        dt = (self.timestep * dn.astype(np.float64))[:, None]
        first = dn <= nhalf
        rp = np.where(first[:, None], self.r_old + self.v_old * dt, self.r_old + self.v_half * dt)
        vp = self.v_old + self.a * dt
        half = first & (dn == nhalf)
        self.v_half[half] = vp[half]
        full = dn == nfull
        self.accdo = half | full
        self.parray[:, 0:3] = rp
        self.v = vp
        self.nlast[full] = self.n
        self.laststep[full] = self.timestep * nfull[full].astype(np.float64)
        self.r_old[full] = rp[full]
        self.v_old[full] = vp[full]

    def _reduce(self):
        """timestep/reduce_timesteps.F90:20-40 with reduce_particle_timestep.F90."""
        D = TIMESTEP_LEVEL_DIFF_MAX
        if np.any(self.nminneib > self.level_max):
            raise RuntimeError("Problem with nminneib > level_max")
        for p in range(len(self.nlevel)):
            mn = int(self.nminneib[p])
            if mn - int(self.nlevel[p]) > D and mn != -1 and self.nlast[p] != self.n and \
                    self.n % 2 ** (self.level_step - mn + D) == 0:
                self.r_old[p] = self.parray[p, 0:3]
                self.v_old[p] = self.v[p]
                self.laststep[p] = self.timestep * float(self.n - self.nlast[p])
                self.nlevel[p] = mn - D
                self.nlast[p] = self.n
                self.nminneib[p] = mn - D
                self.accdo[p] = True


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
