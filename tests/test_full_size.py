"""The benchmark configurations at their full sizes, against the accuracy bars
of the mixed-precision path.

* Plummer sphere, N = 1,048,576, gravity only, softening = the grad-h h for
  50 neighbours: the mixed-precision tree gravity against the oracle's FP64
  direct sum (sph/direct_sph_gravity.F90:64-79) on 4,096 particles chosen
  with seed 3, at theta^2 = 0.09, 0.25 and 0.49 (theta = 0.3, 0.5, 0.7).
* Turbulent core, N = 4,194,304, and protostellar disc with a sink,
  N = 8,388,608: two force evaluations (first call, drift, second call) in
  each precision on the device; mixed against FP64 within rms 1e-4 in the
  total acceleration and 1e-5 in density, and the mixed gravity against the
  FP64 direct sum on 256 particles.

Sizes at which the oracle cannot run the whole path are checked through
these size-independent properties: the FP64 direct sum on a subset, and the
FP64 GPU path (itself bit-exact or within 1e-12 of the oracle on the smaller
cases of test_gpu_parity.py).
"""
import os

import numpy as np
import pytest

from seren_b200 import ics
from tests.helpers import params, rel_rows

pytestmark = pytest.mark.gpu

DT = 1.0e-3
RMS_VS_DIRECT = 1e-3      # mixed tree gravity vs the FP64 direct sum
RMS_VS_FP64 = 1e-4        # mixed vs the FP64 GPU path, total acceleration
RHO_VS_FP64 = 1e-5        # mixed vs the FP64 GPU path, |d rho| / rho


def _rms(x):
    return float(np.sqrt(np.mean(np.asarray(x) ** 2)))


def _gravity_vs_direct(ic, parray, ids, precisions=(1, 0), thetas=None):
    """Gravity-only accelerations of the GPU tree walks for one state (parray
    with the solved h and zeta) against the oracle's FP64 direct sum for the
    particles ids (in tree order); returns {(precision, theta^2): (rms, max)}
    and the rms between the mixed and FP64 walks."""
    from oracle.oracle import Oracle, set_threads
    from seren_b200.gpu import GpuHotPath
    set_threads(os.cpu_count() or 1)
    n = parray.shape[0]
    o = Oracle(n, params(ic, 0))
    _, permo = o.tree_update(parray)
    ad, _ = o.direct_gravity(ids)
    o.close()
    out, walks = {}, {}
    for th in thetas or (ic["thetamaxsqd"],):
        for prec in precisions:
            g = GpuHotPath(n, params(ic, prec, thetamaxsqd=th))
            _, permg = g.tree_update(parray)
            assert np.array_equal(permg, permo), "GPU and oracle trees order the particles alike"
            ag, _ = g.grav_forces(np.zeros((n, 3)))
            g.close()
            err = rel_rows(ag[ids], ad)
            out[(prec, th)] = (_rms(err), float(err.max()))
            walks[(prec, th)] = ag
        if set(precisions) == {0, 1}:
            out[("mixed_vs_fp64", th)] = _rms(rel_rows(walks[(1, th)], walks[(0, th)]))
    return out


def _solved_state(ic, precision, sinks=None):
    """First call (h guess + grad-h), a drift and a second force evaluation on
    the device; returns the downloaded state (tree order)."""
    from seren_b200.gpu import GpuHotPath
    n = ic["parray"].shape[0]
    g = GpuHotPath(n, params(ic, precision))
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    if sinks is not None:
        g.set_sinks(sinks)
    g.force_step(first_call=True)
    g.drift(DT)
    g.force_step(first_call=False)
    st = g.download()
    g.close()
    return st


def test_plummer_1m_gravity_vs_direct_sum():
    ic = ics.plummer(n=1048576, seed=2)
    from seren_b200.gpu import GpuHotPath
    n = ic["parray"].shape[0]
    g = GpuHotPath(n, params(ic, 0))
    p, perm = g.tree_update(ic["parray"])
    s = g.sph_update(p, ic["v"][perm], first_call=True, lists=False)
    g.close()
    parray = s["parray"]                     # tree order, with the solved h and zeta
    ids = np.sort(np.random.Generator(np.random.PCG64(3)).choice(n, 4096, replace=False))
    ids = ids.astype(np.int32)
    res = _gravity_vs_direct(ic, parray, ids, thetas=(0.09, 0.25, 0.49))
    for th in (0.09, 0.25, 0.49):
        print(f"theta^2={th}: mixed rms {res[(1, th)][0]:.3e} max {res[(1, th)][1]:.3e}; "
              f"fp64 rms {res[(0, th)][0]:.3e} max {res[(0, th)][1]:.3e}; "
              f"mixed vs fp64 rms {res[('mixed_vs_fp64', th)]:.3e}")
        # FP32 arithmetic adds nothing visible to the tree's own truncation error
        assert res[("mixed_vs_fp64", th)] < RMS_VS_FP64
        assert abs(res[(1, th)][0] - res[(0, th)][0]) < 0.02 * res[(0, th)][0] + 1e-6
    assert res[(1, 0.09)][0] < RMS_VS_DIRECT
    assert res[(1, 0.25)][0] < RMS_VS_DIRECT


@pytest.mark.parametrize("kind", ["core4m", "disc8m"])
def test_mixed_vs_fp64_and_direct_full_size(kind):
    if kind == "core4m":
        ic = ics.turbulent_core(n=4194304, seed=4, sound=0.2, mach=2.0, h_fac=1.2,
                                thetamaxsqd=0.25)
    else:
        ic = ics.protostellar_disc(n=8388608, seed=5)
    sinks = ic.get("sink")
    sm = _solved_state(ic, 1, sinks)
    sd = _solved_state(ic, 0, sinks)
    assert np.array_equal(sm["perm"], sd["perm"]), "both precisions build the same tree"
    da = rel_rows(sm["a"], sd["a"])
    drho = np.abs(sm["rho"] - sd["rho"]) / sd["rho"]
    print(f"{kind}: mixed vs fp64 |da|/|a| rms {_rms(da):.3e} max {da.max():.3e}; "
          f"|drho|/rho rms {_rms(drho):.3e} max {drho.max():.3e}")
    assert _rms(da) < RMS_VS_FP64
    assert drho.max() < RHO_VS_FP64
    n = sd["parray"].shape[0]
    ids = np.arange(0, n, n // 256, dtype=np.int32)[:256]
    res = _gravity_vs_direct(ic, sd["parray"], ids)
    th = ic["thetamaxsqd"]
    print(f"{kind}: gravity vs direct sum, mixed rms {res[(1, th)][0]:.3e} "
          f"max {res[(1, th)][1]:.3e}, fp64 rms {res[(0, th)][0]:.3e}")
    assert res[("mixed_vs_fp64", th)] < RMS_VS_FP64
    assert res[(1, th)][0] < RMS_VS_DIRECT
