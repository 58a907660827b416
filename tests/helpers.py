"""Shared cases and comparisons for the parity tests."""
from __future__ import annotations

import numpy as np

from seren_b200 import ics
from seren_b200.cabi import Params


def case(name: str):
    """Small seeded workloads covering the configs' regimes (sizes the oracle
    finishes in well under a second)."""
    if name == "sphere4k":
        ic = ics.uniform_sphere(n=4096, seed=1)
        ic["v"] = ics.turbulent_velocity(ic["parray"][:, :3], seed=7, ngrid=32, v_rms=0.2)
    elif name == "sphere32k":          # the reference's CPU-runnable case, full size
        ic = ics.uniform_sphere(n=32768, seed=1, sound=0.1)
    elif name == "turb20k":            # the turbulent core at reduced N
        ic = ics.turbulent_core(n=20000, seed=4, ngrid=32)
    elif name == "plummer16k":         # deep tree, 50 neighbours
        ic = ics.plummer(n=16384, seed=2)
        ic["sound"] = np.full(16384, 0.1)
    elif name == "disc12k":            # thin disc around a sink
        ic = ics.protostellar_disc(n=12000, seed=5)
    elif name == "ragged777":          # ragged size, not a multiple of any tile
        ic = ics.uniform_sphere(n=777, seed=3)
        ic["v"] = np.random.Generator(np.random.PCG64(9)).normal(0, 0.1, (777, 3))
    elif name == "clumps12k":          # three dense Plummer clumps (sink search)
        parts = []
        for centre, seed in (((-1.0, 0.0, 0.0), 11), ((1.0, 0.0, 0.0), 12), ((0.0, 1.0, 0.2), 13)):
            q = ics.plummer(n=4000, seed=seed, a=0.1, mass=1.0 / 3.0, rtrunc=1.0)
            q["parray"][:, 0:3] += np.array(centre)
            q["v"] *= 0.3
            parts.append(q)
        ic = dict(parts[0])
        ic["parray"] = np.vstack([q["parray"] for q in parts])
        ic["v"] = np.vstack([q["v"] for q in parts])
        ic["sound"] = np.full(ic["parray"].shape[0], 0.1)
    elif name == "tiny100":            # just above pp_gather
        ic = ics.uniform_sphere(n=100, seed=5)
    else:
        raise KeyError(name)
    return ic


def params(ic, precision=0, index_base=0, kernel=0, thetamaxsqd=None, redo_cap=0):
    return Params.make(h_fac=ic["h_fac"],
                       thetamaxsqd=ic["thetamaxsqd"] if thetamaxsqd is None else thetamaxsqd,
                       alpha=ic["alpha"], precision=precision, index_base=index_base,
                       kernel=kernel, redo_cap=redo_cap)


def run_pipeline(hp, ic, first_call=True, sinks=None):
    """tree_update -> sph_update -> thermal -> hydro -> gravity, the order of
    sph_setup.F90:42-66; returns everything in tree order."""
    p, perm = hp.tree_update(ic["parray"])
    v = ic["v"][perm - hp.params.index_base]
    s = hp.sph_update(p, v, first_call=first_call)
    sound = ic["sound"][perm - hp.params.index_base]
    press = sound * sound * s["rho"]
    a_h = hp.hydro_forces(press, sound)
    a, gpot = hp.grav_forces(a_h, sinks=sinks)
    return dict(perm=perm, parray=p, v=v, sph=s, press=press, sound=sound, a_hydro=a_h, a=a,
                gpot=gpot)


def rel_rows(x, ref):
    """Per-row |x - ref| / |ref| for [N, k] arrays (|ref| floored at 1e-300)."""
    x = np.asarray(x, float).reshape(len(x), -1)
    ref = np.asarray(ref, float).reshape(len(ref), -1)
    return np.linalg.norm(x - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)


def rel_scaled(x, ref):
    """max |x - ref| / rms |ref| over rows (for fields that pass through zero)."""
    x = np.asarray(x, float).reshape(len(x), -1)
    ref = np.asarray(ref, float).reshape(len(ref), -1)
    scale = np.sqrt(np.mean(np.sum(ref * ref, axis=1))) + 1e-300
    return float(np.max(np.linalg.norm(x - ref, axis=1)) / scale)


def lists_equal(pptot_a, pplist_a, pptot_b, pplist_b, limit):
    if not np.array_equal(pptot_a, pptot_b):
        return False
    for p in range(len(pptot_a)):
        k = int(pptot_a[p])
        if k <= limit and not np.array_equal(pplist_a[p, :k], pplist_b[p, :k]):
            return False
    return True


def deep_clump(a: float, n_core: int = 4000, n_halo: int = 4000):
    """A tight Plummer clump (scale radius a, half the mass) inside a uniform
    halo of radius 10: the root box is ~1e6 clump radii wide, so the octree
    needs more than 21 levels (24 at a = 1e-5, 29 at a = 3e-7)."""
    core = ics.plummer(n=n_core, seed=21, a=a, mass=0.5, rtrunc=20 * a)
    halo = ics.uniform_sphere(n=n_halo, seed=22, radius=10.0, mass=0.5)
    ic = dict(halo)
    ic["parray"] = np.vstack([core["parray"], halo["parray"]])
    ic["v"] = np.vstack([np.zeros((n_core, 3)), halo["v"]])
    ic["sound"] = np.full(n_core + n_halo, 0.1)
    return ic
