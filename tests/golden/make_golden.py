"""Generate the golden fixtures of the force path from the CPU oracle.

The reference ships no golden vectors for this path and cannot be run here
(Fortran, no compiler), so these fixtures are the oracle's own outputs on
small seeded inputs: they pin the oracle against regressions and give the
GPU tests fixed expected values.  Regenerate with
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle  # noqa: E402
from seren_b200 import ics  # noqa: E402
from seren_b200.cabi import Params  # noqa: E402


def make(name, ic, sinks=None):
    n = ic["parray"].shape[0]
    prm = Params.make(h_fac=ic["h_fac"], thetamaxsqd=ic["thetamaxsqd"], alpha=ic["alpha"])
    o = Oracle(n, prm)
    p, perm = o.tree_update(ic["parray"])
    t = o.tree_export()
    v = ic["v"][perm]
    s = o.sph_update(p, v, first_call=True)
    sound = ic["sound"][perm]
    press = sound * sound * s["rho"]
    ah = o.hydro_forces(press, sound)
    a, gpot = o.grav_forces(ah, sinks=sinks)
    out = dict(in_parray=ic["parray"], in_v=ic["v"], in_sound=ic["sound"],
               h_fac=ic["h_fac"], thetamaxsqd=ic["thetamaxsqd"], alpha=ic["alpha"],
               perm=perm, leaf=t["leaf"], nextcell=t["nextcell"], ifopen=t["ifopen"],
               dminsqd=t["dminsqd"], grav_m=t["grav_m"], h=s["parray"][:, 4],
               zeta=s["parray"][:, 5], rho=s["rho"], omega=s["omega"], div_v=s["div_v"],
               pptot=s["pptot"], a_hydro=ah, a=a, gpot=gpot)
    if sinks is not None:
        out["sinks"] = sinks
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, n, "cells", t["ctot"] + 1)


if __name__ == "__main__":
    ic = ics.uniform_sphere(n=777, seed=3)
    ic["v"] = np.random.Generator(np.random.PCG64(9)).normal(0, 0.1, (777, 3))
    make("sphere777", ic)
    ic = ics.turbulent_core(n=3000, seed=4, ngrid=16)
    make("turb3000", ic)
    ic = ics.protostellar_disc(n=2500, seed=5)
    make("disc2500", ic, sinks=ic["sink"])
