"""Golden fixtures (tests/golden/*.npz, made by make_golden.py from the oracle).

CPU: the oracle reproduces its committed outputs bit for bit.
GPU: the CUDA path reproduces the integer fixtures exactly and the floating
point ones within 1e-12 relative (1e-11 for the summed accelerations).
"""
import glob
import os

import numpy as np
import pytest

from seren_b200.cabi import Params
from tests.helpers import rel_rows, rel_scaled

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))


def _run(hp_cls, f):
    d = np.load(f)
    n = d["in_parray"].shape[0]
    prm = Params.make(h_fac=float(d["h_fac"]), thetamaxsqd=float(d["thetamaxsqd"]),
                      alpha=float(d["alpha"]))
    hp = hp_cls(n, prm)
    p, perm = hp.tree_update(d["in_parray"])
    t = hp.tree_export()
    v = d["in_v"][perm]
    s = hp.sph_update(p, v, first_call=True)
    sound = d["in_sound"][perm]
    ah = hp.hydro_forces(sound * sound * s["rho"], sound)
    a, gpot = hp.grav_forces(ah, sinks=d["sinks"] if "sinks" in d else None)
    return d, dict(perm=perm, leaf=t["leaf"], nextcell=t["nextcell"], ifopen=t["ifopen"],
                   dminsqd=t["dminsqd"], grav_m=t["grav_m"], h=s["parray"][:, 4],
                   zeta=s["parray"][:, 5], rho=s["rho"], omega=s["omega"], div_v=s["div_v"],
                   pptot=s["pptot"], a_hydro=ah, a=a, gpot=gpot)


def test_fixtures_present():
    assert len(FILES) >= 3


@pytest.mark.parametrize("f", FILES, ids=[os.path.basename(x) for x in FILES])
def test_oracle_reproduces_golden(f):
    from oracle.oracle import Oracle
    d, r = _run(Oracle, f)
    for k, val in r.items():
        assert np.array_equal(val, d[k]), k


@pytest.mark.gpu
@pytest.mark.parametrize("f", FILES, ids=[os.path.basename(x) for x in FILES])
def test_gpu_reproduces_golden(f):
    from seren_b200.gpu import GpuHotPath
    d, r = _run(GpuHotPath, f)
    for k in ("perm", "leaf", "nextcell", "ifopen", "pptot", "dminsqd", "grav_m"):
        assert np.array_equal(r[k], d[k]), k
    for k in ("h", "rho", "omega", "gpot"):
        assert rel_rows(r[k], d[k]).max() < 1e-12, k
    for k in ("zeta", "div_v", "a_hydro"):
        assert rel_scaled(r[k], d[k]) < 1e-12, k
    assert rel_rows(r["a"], d["a"]).max() < 1e-11
