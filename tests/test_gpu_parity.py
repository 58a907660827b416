"""Parity of the CUDA force path with the CPU oracle, stage by stage.

Bars: integer work (tree cells, particle order, neighbour lists at the same h)
bit-exact; stock FP64 values bit-exact (same expressions, no contraction);
FP64 per-particle results within 1e-12 relative; the mixed-precision gravity
within 1e-5 rms / 1e-3 max of the FP64 path.  All calls go through the C ABI.
"""
import numpy as np
import pytest

from seren_b200 import ics
from tests.helpers import case, lists_equal, params, rel_rows, rel_scaled, run_pipeline

pytestmark = pytest.mark.gpu

CASES = ["sphere4k", "sphere32k", "turb20k", "plummer16k", "disc12k", "ragged777", "tiny100"]
TOL = 1e-12


@pytest.fixture(scope="module")
def libs():
    from oracle.oracle import Oracle
    from seren_b200.gpu import GpuHotPath
    return Oracle, GpuHotPath


def _pair(libs, ic, **kw):
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    prm = params(ic, **kw)
    return Oracle(n, prm), Gpu(n, prm)


@pytest.mark.parametrize("name", CASES)
def test_tree_bit_exact(libs, name):
    ic = case(name)
    o, g = _pair(libs, ic)
    po, permo = o.tree_update(ic["parray"])
    pg, permg = g.tree_update(ic["parray"])
    assert np.array_equal(permo, permg)
    assert np.array_equal(po, pg)
    to, tg = o.tree_export(), g.tree_export()
    assert to["ctot"] == tg["ctot"] and to["ltot"] == tg["ltot"]
    for k in ("leaf", "nextcell", "ifopen", "plist", "first_cell", "last_cell"):
        assert np.array_equal(to[k], tg[k]), k
    for k in ("grav_r", "grav_m", "grav_q", "dminsqd", "hydro_r", "rmax"):
        assert np.array_equal(to[k], tg[k]), k


@pytest.mark.parametrize("name", CASES)
def test_full_evaluation_fp64(libs, name):
    ic = case(name)
    o, g = _pair(libs, ic)
    sinks = ic.get("sink")
    ro = run_pipeline(o, ic, sinks=sinks)
    rg = run_pipeline(g, ic, sinks=sinks)
    so, sg = ro["sph"], rg["sph"]
    assert rel_rows(sg["parray"][:, 4], so["parray"][:, 4]).max() < TOL
    for k in ("rho", "omega"):
        assert rel_rows(sg[k], so[k]).max() < TOL, k
    for k in ("div_v", "drhodt"):
        assert rel_scaled(sg[k], so[k]) < TOL, k
    assert rel_scaled(sg["parray"][:, 5], so["parray"][:, 5]) < TOL
    L = g.params.pp_limit
    assert lists_equal(so["pptot"], so["pplist"], sg["pptot"], sg["pplist"], L)
    assert rel_scaled(rg["a_hydro"], ro["a_hydro"]) < TOL
    assert rel_rows(rg["a"], ro["a"]).max() < 1e-11
    assert rel_rows(rg["gpot"], ro["gpot"]).max() < TOL


def test_whole_gpu_gradh_path_matches_oracle(libs):
    """With a tiny redo scratch (redo_cap) the particles that grad-h hands to
    the redo kernel on the first call (h guess) go on to the whole-GPU path:
    counting walks over subtrees, passes over all particles.  The results are
    still the oracle's."""
    ic = case("turb20k")
    o, g = _pair(libs, ic, redo_cap=8)
    ro = run_pipeline(o, ic)
    rg = run_pipeline(g, ic)
    so, sg = ro["sph"], rg["sph"]
    assert rel_rows(sg["parray"][:, 4], so["parray"][:, 4]).max() < TOL
    for k in ("rho", "omega"):
        assert rel_rows(sg[k], so[k]).max() < TOL, k
    for k in ("div_v", "drhodt"):
        assert rel_scaled(sg[k], so[k]) < TOL, k
    L = g.params.pp_limit
    assert lists_equal(so["pptot"], so["pplist"], sg["pptot"], sg["pplist"], L)
    assert rel_rows(rg["a"], ro["a"]).max() < 1e-11
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    g2 = Gpu(n, params(ic, redo_cap=8))
    g2.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g2.force_step(first_call=True)
    assert g2.last_step_stats()[2][8] > 0           # particles on the whole-GPU path


@pytest.mark.parametrize("name,redo_cap,wide", [("clumps12k", 8, True), ("clumps12k", 0, False),
                                                ("disc100k", 0, True)])
def test_gradh_bisection_matches_oracle(libs, name, redo_cap, wide):
    """Cases whose first call (h guess) takes some particles' grad-h iteration
    to the reference's bisection (all_sph_gradh.F90:256-275), which restarts
    from h_upper = rextent: three dense clumps, and the protostellar disc with
    its sink at N = 100,000.  In the clumps the redo kernel's scratch holds
    the whole tree's leaves, so it runs the bisection itself; with redo_cap = 8,
    and in the disc, the walks at h ~ rextent outgrow it and those particles
    continue on the whole-GPU path, where the bisection passes that a lower
    bound on the density decides, and the counting walks whose ball covers a
    whole cell of pp_gather particles, are taken without a walk, and the other
    passes walk at radius 2h.  The results are the oracle's."""
    ic = case(name) if name == "clumps12k" else ics.protostellar_disc(n=100000, seed=5)
    o, g = _pair(libs, ic, redo_cap=redo_cap)
    ro = run_pipeline(o, ic)
    assert o.counts()["gradh_bisections"] > 0          # the case reaches the bisection
    rg = run_pipeline(g, ic)
    so, sg = ro["sph"], rg["sph"]
    assert rel_rows(sg["parray"][:, 4], so["parray"][:, 4]).max() < TOL
    for k in ("rho", "omega"):
        assert rel_rows(sg[k], so[k]).max() < TOL, k
    for k in ("div_v", "drhodt"):
        assert rel_scaled(sg[k], so[k]) < TOL, k
    L = g.params.pp_limit
    assert lists_equal(so["pptot"], so["pplist"], sg["pptot"], sg["pplist"], L)
    assert rel_rows(rg["a"], ro["a"]).max() < 1e-11
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    g2 = Gpu(n, params(ic, redo_cap=redo_cap))
    g2.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    if ic.get("sink") is not None:
        g2.set_sinks(ic["sink"])
    g2.force_step(first_call=True)
    assert (g2.last_step_stats()[2][8] > 0) == wide      # particles on the whole-GPU path
    g2.close()


def test_neighbour_lists_with_overflowing_rows(libs):
    """pp_limit = 40, below the ~56 neighbours of a particle of the core: most
    rows overflow (get_neib keeps no list for them, pptot is the full count,
    sph/get_neib.F90:115-118) and so do the gather sets that the grad-h final
    pass records, whose transposition then walks the tree.  The lists after
    grad-h (sph_update) and the accelerations of the device-resident force
    step, whose hydro forces find an overflowing row's neighbours on the fly
    (get_neib_on_fly.F90), are still the oracle's."""
    ic = case("turb20k")
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    prm = params(ic)
    prm.pp_limit = 40
    o, g = Oracle(n, prm), Gpu(n, prm)
    ro = run_pipeline(o, ic)
    rg = run_pipeline(g, ic)
    so, sg = ro["sph"], rg["sph"]
    assert (so["pptot"] > 40).mean() > 0.5                # most rows overflow
    assert lists_equal(so["pptot"], so["pplist"], sg["pptot"], sg["pplist"], 40)
    assert rel_rows(sg["parray"][:, 4], so["parray"][:, 4]).max() < TOL
    assert rel_scaled(rg["a_hydro"], ro["a_hydro"]) < TOL
    g2 = Gpu(n, prm)
    g2.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g2.force_step(first_call=True)
    st = g2.download()
    g2.close()
    assert np.array_equal(st["perm"], ro["perm"])
    assert rel_rows(st["a"], ro["a"]).max() < 1e-11


@pytest.mark.parametrize("name", ["sphere4k", "plummer16k", "disc12k"])
def test_neighbour_lists_at_oracle_h(libs, name):
    """get_neib at the same h is bit-exact (sph/get_neib.F90:83-118)."""
    ic = case(name)
    o, g = _pair(libs, ic)
    ro = run_pipeline(o, ic)
    g.tree_update(ic["parray"])
    h = ro["sph"]["parray"][:, 4]
    pto, plo = o.get_neib(h=h)
    ptg, plg = g.get_neib(h=h)
    assert lists_equal(pto, plo, ptg, plg, g.params.pp_limit)
    to, tg = o.tree_export(), g.tree_export()
    assert np.array_equal(to["hrangemax"], tg["hrangemax"])


@pytest.mark.parametrize("name", ["sphere4k", "turb20k", "plummer16k"])
def test_gravity_counts_equal_oracle(libs, name):
    """The GPU walk accepts exactly the oracle's cells and pairs (FP64 MAC)."""
    from seren_b200.gpu import library
    import ctypes as C
    ic = case(name)
    for prec in (0, 1):
        o, g = _pair(libs, ic, precision=prec)
        ro = run_pipeline(o, ic)
        run_pipeline(g, ic)
        cnt = (C.c_int64 * 16)()
        library().seren_gpu_last_step_stats(g._ctx, None, None, cnt)
        co = o.counts()
        assert cnt[0] == co["grav_cells"] and cnt[1] == co["grav_pairs"], (prec, list(cnt), co)
        del ro


@pytest.mark.parametrize("name", ["sphere4k", "turb20k", "plummer16k", "disc12k"])
def test_mixed_gravity_vs_fp64(libs, name):
    ic = case(name)
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    g64 = Gpu(n, params(ic, precision=0))
    g32 = Gpu(n, params(ic, precision=1))
    r64 = run_pipeline(g64, ic, sinks=ic.get("sink"))
    r32 = run_pipeline(g32, ic, sinks=ic.get("sink"))
    assert np.array_equal(r64["perm"], r32["perm"])
    err = rel_rows(r32["a"], r64["a"])
    assert np.sqrt(np.mean(err ** 2)) < 1e-5
    assert err.max() < 1e-3
    assert rel_rows(r32["gpot"], r64["gpot"]).max() < 1e-4


def test_gpu_tree_against_direct_sum(libs):
    """The tree with a vanishing opening angle is the direct sum
    (sph/direct_sph_gravity.F90) up to summation order."""
    ic = case("sphere4k")
    o, g = _pair(libs, ic, thetamaxsqd=1e-8)
    rg = run_pipeline(g, ic)
    run_pipeline(o, ic)
    ids = np.arange(0, 4096, 16, dtype=np.int32)
    ad, gd = o.direct_gravity(ids)
    ag = rg["a"] - rg["a_hydro"]
    assert rel_rows(ag[ids], ad).max() < 1e-11
    assert rel_rows(rg["gpot"][ids], gd).max() < 1e-11


def test_index_base_one_and_acclist(libs):
    """Fortran ids (index_base = 1) and an active subset (acclist) give the
    oracle's results for the active rows and leave the others untouched."""
    ic = case("sphere4k")
    n = 4096
    o, g = _pair(libs, ic, index_base=1)
    po, permo = o.tree_update(ic["parray"])
    pg, permg = g.tree_update(ic["parray"])
    assert permg.min() == 1 and np.array_equal(permo, permg)
    v = ic["v"][permg - 1]
    so = o.sph_update(po, v, first_call=True)
    sg = g.sph_update(pg, v, first_call=True)
    assert sg["pplist"][0, 0] >= 1
    assert lists_equal(so["pptot"], so["pplist"], sg["pptot"], sg["pplist"], g.params.pp_limit)
    act = np.arange(1, n + 1, 3, dtype=np.int32)
    sound = ic["sound"][permg - 1]
    press = sound * sound * sg["rho"]
    base = np.full((n, 3), 7.0)
    ao = o.hydro_forces(press, sound, a=base, acclist=act)
    ag = g.hydro_forces(press, sound, a=base, acclist=act)
    idx = act - 1
    mask = np.ones(n, bool)
    mask[idx] = False
    assert np.all(ag[mask] == 7.0)
    assert rel_scaled(ag[idx], ao[idx]) < TOL
    go, gpo = o.grav_forces(ao, acclist=act)
    gg, gpg = g.grav_forces(ag, acclist=act)
    assert rel_rows(gg[idx], go[idx]).max() < 1e-11
    assert np.all(gg[mask] == 7.0)


def test_thomas_couchman_kernel(libs):
    ic = case("sphere4k")
    o, g = _pair(libs, ic, kernel=1)
    ro = run_pipeline(o, ic)
    rg = run_pipeline(g, ic)
    assert rel_scaled(rg["a_hydro"], ro["a_hydro"]) < TOL


def test_sink_forces(libs):
    ic = case("disc12k")
    o, g = _pair(libs, ic)
    run_pipeline(o, ic, sinks=ic["sink"])
    run_pipeline(g, ic, sinks=ic["sink"])
    sinks = np.vstack([ic["sink"], [[0.5, 0.2, 0.0, 0.01, 0.02]]])
    sa_o, sp_o = o.sink_forces(sinks)
    sa_g, sp_g = g.sink_forces(sinks)
    assert rel_rows(sa_g, sa_o).max() < 1e-11
    assert rel_rows(sp_g, sp_o).max() < 1e-11


def test_restock_without_build(libs):
    """tree_update(do_build=0) restocks the existing cells with new h."""
    ic = case("sphere4k")
    o, g = _pair(libs, ic)
    po, _ = o.tree_update(ic["parray"])
    pg, _ = g.tree_update(ic["parray"])
    po[:, 4] *= 1.3
    pg[:, 4] *= 1.3
    o.tree_update(po, do_build=False)
    g.tree_update(pg, do_build=False)
    to, tg = o.tree_export(), g.tree_export()
    assert np.array_equal(to["dminsqd"], tg["dminsqd"])


def test_resident_step_matches_host_calls(libs):
    """seren_gpu_force_step on device-resident data equals the sequence of
    host-buffer calls (with the host doing the isothermal thermal step)."""
    ic = case("turb20k")
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    g1 = Gpu(n, params(ic))
    g2 = Gpu(n, params(ic))
    r = run_pipeline(g1, ic)
    g2.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g2.force_step(first_call=True)
    st = g2.download()
    assert np.array_equal(st["perm"], r["perm"])
    assert np.array_equal(st["parray"][:, 4], r["sph"]["parray"][:, 4])
    assert rel_rows(st["a"], r["a"]).max() < 1e-13
    assert np.array_equal(st["gpot"], r["gpot"])


def test_force_step_io_matches_resident_step(libs):
    """seren_gpu_force_step_io (copies overlapped on a second stream) returns
    what upload + force_step + download return, on two steps in a row (the
    second from the first's tree-ordered outputs, written over its inputs)."""
    ic = case("turb20k")
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    g1 = Gpu(n, params(ic))
    g2 = Gpu(n, params(ic))
    parray, v, csq = ic["parray"].copy(), ic["v"].copy(), ic["sound"] ** 2
    for step in range(2):
        g1.upload(parray, v, csq)
        g1.force_step(first_call=step == 0)
        ref = g1.download()
        got = g2.force_step_io(parray, v, csq, first_call=step == 0)
        for k in ("parray", "v", "rho", "omega", "a", "gpot", "perm"):
            assert np.array_equal(got[k], ref[k]), (step, k)
        assert np.array_equal(got["csq"], csq[got["perm"]])
        assert g2.last_step_stats()[1] > g1.last_step_stats()[1]
        parray, v, csq = got["parray"], got["v"], got["csq"]
        parray[:, 0:3] += 1e-3 * v


def test_force_step_io_pinned_buffers(libs):
    """With page-locked host buffers seren_gpu_force_step_io writes a and gpot
    from the gravity kernel straight into them (mapped) and defers the v, c_s^2
    reorder; the results equal the resident step's."""
    import ctypes as C

    import torch
    ic = case("turb20k")
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    g1 = Gpu(n, params(ic))
    g2 = Gpu(n, params(ic))
    g1.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g1.force_step(first_call=True)
    ref = g1.download()

    def pinned(a, dtype=torch.float64):
        t = torch.empty(a.shape, dtype=dtype, pin_memory=True)
        t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
        return t

    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    P = lambda t: C.cast(t.data_ptr(), dp)  # noqa: E731
    parray, v, csq = pinned(ic["parray"]), pinned(ic["v"]), pinned(ic["sound"] ** 2)
    out = {k: pinned(np.zeros(shape)) for k, shape in
           (("rho", (n,)), ("omega", (n,)), ("a", (n, 3)), ("gpot", (n,)))}
    perm = pinned(np.zeros(n, dtype=np.int32), torch.int32)
    g2._call("force_step_io", g2._ctx, n, P(parray), P(v), P(csq), 1, P(parray), P(v), P(csq),
             P(out["rho"]), P(out["omega"]), P(out["a"]), P(out["gpot"]),
             C.cast(perm.data_ptr(), ip))
    assert np.array_equal(perm.numpy(), ref["perm"])
    assert np.array_equal(parray.numpy(), ref["parray"])
    assert np.array_equal(v.numpy(), ref["v"])
    for k in ("rho", "omega", "a", "gpot"):
        assert np.array_equal(out[k].numpy(), ref[k]), k
    assert np.array_equal(csq.numpy(), (ic["sound"] ** 2)[ref["perm"]])


def test_host_calls_with_pinned_buffers(libs):
    """With page-locked buffers the reference-shaped calls overlap their copies
    (sph_update) or map the buffers (hydro_forces writes a, grav_forces reads
    and writes a and gpot, straight from the kernels); the results equal the
    ones from pageable buffers."""
    import ctypes as C

    import torch
    ic = case("turb20k")
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    prm = params(ic)
    g1 = Gpu(n, prm)
    g2 = Gpu(n, prm)
    r = run_pipeline(g1, ic)

    def pinned(a, dtype=torch.float64):
        t = torch.empty(a.shape, dtype=dtype, pin_memory=True)
        t.copy_(torch.from_numpy(np.ascontiguousarray(a)))
        return t

    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    P = lambda t: C.cast(t.data_ptr(), dp)  # noqa: E731
    I = lambda t: C.cast(t.data_ptr(), ip)  # noqa: E731,E741
    parray = pinned(ic["parray"])
    perm = pinned(np.zeros(n, dtype=np.int32), torch.int32)
    g2._call("tree_update", g2._ctx, n, P(parray), 1, 1, I(perm))
    pm = perm.numpy().copy()
    v = pinned(ic["v"][pm])
    L = prm.pp_limit
    out = {k: pinned(np.zeros(n)) for k in ("rho", "omega", "div_v", "drhodt")}
    pptot = pinned(np.zeros(n, dtype=np.int32), torch.int32)
    pplist = pinned(np.full((n, L), -1, dtype=np.int32), torch.int32)
    g2._call("sph_update", g2._ctx, n, None, 0, P(parray), P(v), P(out["rho"]), P(out["omega"]),
             P(out["div_v"]), P(out["drhodt"]), I(pptot), I(pplist), 1)
    sound = ic["sound"][pm]
    press = pinned(sound * sound * out["rho"].numpy())
    a = pinned(np.zeros((n, 3)))
    g2._call("hydro_forces", g2._ctx, None, 0, P(press), P(pinned(sound)), P(a))
    a_hydro = a.numpy().copy()
    gpot = pinned(np.zeros(n))
    g2._call("grav_forces", g2._ctx, None, 0, P(a), P(gpot), 0, None)
    assert np.array_equal(pm, r["perm"])
    assert np.array_equal(parray.numpy(), r["sph"]["parray"])
    for k in ("rho", "omega", "div_v", "drhodt"):
        assert np.array_equal(out[k].numpy(), r["sph"][k]), k
    assert lists_equal(pptot.numpy(), pplist.numpy(), r["sph"]["pptot"], r["sph"]["pplist"], L)
    assert np.array_equal(a_hydro, r["a_hydro"])
    assert np.array_equal(a.numpy(), r["a"])
    assert np.array_equal(gpot.numpy(), r["gpot"])


def test_resident_step_with_sink_matches_host_calls(libs):
    """seren_gpu_set_sinks puts the sink-gas term of grav_forces into the
    device-resident step."""
    ic = case("disc12k")
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    g1 = Gpu(n, params(ic))
    g2 = Gpu(n, params(ic))
    r = run_pipeline(g1, ic, sinks=ic["sink"])
    g2.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g2.set_sinks(ic["sink"])
    g2.force_step(first_call=True)
    st = g2.download()
    assert np.array_equal(st["perm"], r["perm"])
    assert rel_rows(st["a"], r["a"]).max() < 1e-13
    assert np.array_equal(st["gpot"], r["gpot"])


def test_timestep_and_rk2_step_match_oracle(libs):
    """seren_gpu_timestep equals timestep_size.F90 on the oracle's state, and
    one device-resident second-order Runge-Kutta step (two force evaluations,
    the particles reordered at each tree build) equals the oracle's forces
    driven through the same step with advance_runge_kutta.F90's updates."""
    from oracle.oracle import rk2_full, rk2_half, timestep_sizes
    ic = case("turb20k")
    o, g = _pair(libs, ic)
    n = ic["parray"].shape[0]
    # start: forces and timesteps
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g.force_step(first_call=True)
    dt_min, dt_g = g.timestep(0.2, 0.5, per_particle=True)
    r0 = run_pipeline(o, ic)
    p0, perm0 = r0["sph"]["parray"], r0["perm"]
    dt_o = timestep_sizes(p0[:, 4], r0["a"], r0["sph"]["div_v"], r0["sound"], ic["alpha"])
    assert np.array_equal(g.download()["perm"], perm0)
    assert rel_rows(dt_g, dt_o).max() < 1e-11
    assert dt_min == dt_g.min()
    dt = dt_min
    g.rk2_step(dt)
    st = g.download()
    # the oracle through the same step: half step, forces, full step, forces
    v0 = ic["v"][perm0]
    rh, vh = rk2_half(p0[:, 0:3], v0, r0["a"], 0.5 * dt)
    ph = p0.copy()
    ph[:, 0:3] = rh
    r1 = run_pipeline(o, dict(ic, parray=ph, v=vh, sound=r0["sound"]), first_call=False)
    perm1 = r1["perm"]                                   # tree order 1 -> tree order 0
    x1, v1 = rk2_full(p0[perm1, 0:3], v0[perm1], vh[perm1], r1["a"], dt)
    p1 = r1["sph"]["parray"].copy()
    p1[:, 0:3] = x1
    r2 = run_pipeline(o, dict(ic, parray=p1, v=v1, sound=r1["sound"]), first_call=False)
    perm2 = r2["perm"]
    assert np.array_equal(st["perm"], perm0[perm1[perm2]])
    assert np.abs(st["parray"][:, 0:3] - r2["parray"][:, 0:3]).max() < 1e-12
    assert rel_rows(st["v"], v1[perm2]).max() < 1e-10
    assert rel_rows(st["parray"][:, 4], r2["sph"]["parray"][:, 4]).max() < 1e-10
    assert rel_rows(st["a"], r2["a"]).max() < 1e-9


def test_rk2_step_with_a_moving_sink_matches_oracle(libs):
    """A sink set in motion moves with the gas through the Runge-Kutta step
    (advance_sink_RK.F90), its accelerations from sph_sink_forces on each
    step's tree; the oracle driven through the same step agrees, and the sink
    timestep equals sink_timestep.F90's."""
    from oracle.oracle import rk2_full, rk2_half, sink_timesteps
    ic = case("disc12k")
    o, g = _pair(libs, ic)
    sink0 = np.atleast_2d(ic["sink"]).astype(float)
    sv0, srad = np.array([[0.02, -0.01, 0.0]]), np.array([0.1])
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g.set_sinks(sink0)
    g.set_sink_motion(sv0, srad)
    g.force_step(first_call=True)
    s0 = g.get_sinks()
    r0 = run_pipeline(o, ic, sinks=sink0)
    sa0, _ = o.sink_forces(sink0)
    assert rel_rows(s0["a"], sa0).max() < 1e-11
    dts = g.sink_timestep(0.5)
    assert abs(dts - sink_timesteps(sink0, sv0, sa0, srad).min()) <= 1e-12 * dts
    dt = min(g.timestep(), dts)
    g.rk2_step(dt)
    st, s1 = g.download(), g.get_sinks()
    perm0, p0 = r0["perm"], r0["sph"]["parray"]
    v0 = ic["v"][perm0]
    # half step: gas and sink
    rh, vh = rk2_half(p0[:, 0:3], v0, r0["a"], 0.5 * dt)
    srh, svh = rk2_half(sink0[:, 0:3], sv0, sa0, 0.5 * dt)
    sinkh = sink0.copy()
    sinkh[:, 0:3] = srh
    ph = p0.copy()
    ph[:, 0:3] = rh
    r1 = run_pipeline(o, dict(ic, parray=ph, v=vh, sound=r0["sound"]), first_call=False,
                      sinks=sinkh)
    sah, _ = o.sink_forces(sinkh)
    perm1 = r1["perm"]
    x1, v1 = rk2_full(p0[perm1, 0:3], v0[perm1], vh[perm1], r1["a"], dt)
    sx1, sv1 = rk2_full(sink0[:, 0:3], sv0, svh, sah, dt)
    sink1 = sink0.copy()
    sink1[:, 0:3] = sx1
    p1 = r1["sph"]["parray"].copy()
    p1[:, 0:3] = x1
    r2 = run_pipeline(o, dict(ic, parray=p1, v=v1, sound=r1["sound"]), first_call=False,
                      sinks=sink1)
    sa1, sp1 = o.sink_forces(sink1)
    perm2 = r2["perm"]
    assert np.array_equal(st["perm"], perm0[perm1[perm2]])
    assert np.abs(st["parray"][:, 0:3] - r2["parray"][:, 0:3]).max() < 1e-12
    assert rel_rows(st["v"], v1[perm2]).max() < 1e-10
    assert rel_rows(st["a"], r2["a"]).max() < 1e-9
    assert np.abs(s1["rmh"][:, 0:3] - sx1).max() < 1e-13
    assert rel_rows(s1["v"], sv1).max() < 1e-11
    assert rel_rows(s1["a"], sa1).max() < 1e-9


def test_active_subset_after_a_rebuild(libs):
    """Block-timestep use of the reference-shaped calls: after a first full
    evaluation the particles move, the tree is rebuilt (the host permutes its
    arrays), and only every third particle is updated.  The inactive particles'
    rho, omega (the neighbours' values the active particles' hydro reads) must
    follow the reorder, as main/reorder_array.F90 permutes them."""
    ic = case("turb20k")
    o, g = _pair(libs, ic)
    n = ic["parray"].shape[0]
    r0 = run_pipeline(o, ic)
    rg0 = run_pipeline(g, ic)
    assert np.array_equal(r0["perm"], rg0["perm"])
    p1 = r0["sph"]["parray"].copy()
    v0 = ic["v"][r0["perm"]]
    p1[:, 0:3] += 2e-3 * v0
    po, permo = o.tree_update(p1)
    pg, permg = g.tree_update(p1)
    assert np.array_equal(permo, permg)
    v1 = v0[permo]
    act = np.arange(0, n, 3, dtype=np.int32)
    so = o.sph_update(po, v1, acclist=act)
    sg = g.sph_update(pg, v1, acclist=act)
    for k in ("rho", "omega"):
        assert rel_rows(sg[k][act], so[k][act]).max() < TOL, k
    for k in ("div_v", "drhodt"):                   # they pass through zero
        assert rel_scaled(sg[k][act], so[k][act]) < TOL, k
    assert rel_rows(sg["parray"][act, 4], so["parray"][act, 4]).max() < TOL
    # the host's rho: the previous values, permuted, with the active rows new
    rho = r0["sph"]["rho"][permo].copy()
    rho[act] = so["rho"][act]
    sound = r0["sound"][permo]
    press = sound * sound * rho
    ao = o.hydro_forces(press, sound, acclist=act)
    ag = g.hydro_forces(press, sound, acclist=act)
    assert rel_scaled(ag[act], ao[act]) < TOL
    go, _ = o.grav_forces(ao, acclist=act)
    gg, _ = g.grav_forces(ag, acclist=act)
    assert rel_rows(gg[act], go[act]).max() < 1e-11


@pytest.mark.parametrize("energy,flags", [(True, None), (False, [1, 1, 0])])
def test_accretion_matches_oracle(libs, energy, flags):
    """Sink accretion on the device-resident particles (accrete_particles.F90
    with remove_from_list.F90) against the oracle on the same state: which
    particles go to which sink (nearest of two overlapping sinks, a sink that
    does not accrete, the energy test), the new sink mass, position, velocity,
    acceleration and angular momentum (FP64 sums in particle order: bit-exact),
    and the kept particles in their order; the next force step runs on them."""
    from oracle.oracle import accrete_particles
    ic = case("turb20k")
    _, g = _pair(libs, ic)
    sinks = np.array([[0.0, 0.0, 0.0, 0.05, 0.05], [0.2, 0.0, 0.0, 0.02, 0.04],
                      [0.5, 0.5, 0.0, 0.01, 0.05]])
    sv = np.array([[0.4, 0.0, 0.0], [0.0, -0.1, 0.0], [0.0, 0.0, 0.0]])
    srad = np.array([0.15, 0.12, 0.1])
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g.set_sinks(sinks)
    g.set_sink_motion(sv, srad)
    g.force_step(first_call=True)
    st, s0 = g.download(), g.get_sinks()
    p = st["parray"]
    want = accrete_particles(p[:, 0:3], p[:, 3], p[:, 4], st["v"], st["a"], s0["rmh"], s0["v"],
                             s0["a"], srad, accrete=flags, energy_accrete=energy)
    assert want["count"][0] > 0 and want["count"][1] > 0
    if flags:
        assert want["count"][2] == 0
    if energy:                                            # some candidates are unbound
        within = accrete_particles(p[:, 0:3], p[:, 3], p[:, 4], st["v"], st["a"], s0["rmh"],
                                   s0["v"], s0["a"], srad)
        assert want["count"].sum() < within["count"].sum()
    angmom = np.zeros((3, 3))
    cnt = g.accrete(energy_accrete=energy, accrete=flags, angmom=angmom)
    assert cnt.tolist() == want["count"].tolist()
    s1 = g.get_sinks()
    assert np.array_equal(s1["rmh"], want["rmh"])
    assert np.array_equal(s1["v"], want["v"]) and np.array_equal(s1["a"], want["a"])
    assert np.array_equal(angmom, want["angmom"])
    keep = want["keep"]
    assert g.ptot == keep.size == p.shape[0] - want["count"].sum()
    st1 = g.download()
    assert np.array_equal(st1["perm"], st["perm"][keep])
    assert np.array_equal(st1["parray"], p[keep]) and np.array_equal(st1["v"], st["v"][keep])
    assert np.array_equal(st1["a"], st["a"][keep]) and np.array_equal(st1["rho"], st["rho"][keep])
    g.force_step(first_call=False)
    st2 = g.download()
    assert np.array_equal(np.sort(st2["perm"]), np.sort(st1["perm"]))
    assert np.isfinite(st2["a"]).all()


def test_sink_search_matches_oracle(libs):
    """Sink search and creation on the device (sink_search.F90, create_sink.F90)
    against the oracle on the same state, three dense clumps: first with no
    sink (the densest candidate fails div v / div a, a lighter one passes, and
    the sink is made at the densest, as the reference's loop leaves it), then,
    after a force step that includes the new sink, a second search with it in
    place (overlap, Hill and timescale tests, the radius in units of h).  The
    chosen particle, the new sink's mass, position, velocity, acceleration and
    angular momentum (FP64 sums in index order: bit-exact) and the kept
    particles in their order all match."""
    from oracle.oracle import sink_search
    ic = case("clumps12k")
    _, g = _pair(libs, ic)
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g.force_step(first_call=True)
    st = g.download()
    p = st["parray"]
    rhosink = float(np.percentile(st["rho"], 90))
    none = (np.zeros((0, 5)), np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0))
    want = sink_search(p[:, 0:3], p[:, 3], p[:, 4], st["v"], st["a"], st["rho"], st["gpot"],
                       *none, rhosink=rhosink, sinkrad=0.05)
    assert want["psink"] >= 0 and want["flags"][-1] is False
    got = g.sink_search(rhosink, 0.05)
    assert got["created"] and got["psink_id"] == st["perm"][want["psink"]]
    assert got["nremoved"] == len(want["removed"]) and g.ptot == len(want["keep"])
    assert np.array_equal(got["angmom"], want["angmom"])
    s1 = g.get_sinks()
    assert g.nsink == 1
    assert np.array_equal(s1["rmh"][0], np.r_[want["r"], want["m"], want["h"]])
    assert np.array_equal(s1["v"][0], want["v"]) and np.array_equal(s1["a"][0], want["a"])
    st1 = g.download()
    keep = want["keep"]
    assert np.array_equal(st1["perm"], st["perm"][keep])
    assert np.array_equal(st1["parray"], p[keep]) and np.array_equal(st1["v"], st["v"][keep])
    # a second search with the sink in place (overlap, Hill and timescale loops)
    g.force_step(first_call=False)
    st2, s2 = g.download(), g.get_sinks()
    p2 = st2["parray"]
    args = dict(rhosink=rhosink, sinkrad=0.05, div_a_search=False)
    want2 = sink_search(p2[:, 0:3], p2[:, 3], p2[:, 4], st2["v"], st2["a"], st2["rho"],
                        st2["gpot"], s2["rmh"], s2["v"], s2["a"], np.full(1, 0.05), **args)
    assert want2["psink"] >= 0
    got2 = g.sink_search(**args)
    assert got2["created"] and got2["psink_id"] == st2["perm"][want2["psink"]]
    assert np.array_equal(got2["angmom"], want2["angmom"])
    s3 = g.get_sinks()
    assert g.nsink == 2 and np.array_equal(s3["rmh"][0], s2["rmh"][0])
    assert np.array_equal(s3["rmh"][1], np.r_[want2["r"], want2["m"], want2["h"]])
    assert np.array_equal(g.download()["perm"], st2["perm"][want2["keep"]])
    # the radius in units of h and the timescale test
    g.force_step(first_call=False)
    st3, s3 = g.download(), g.get_sinks()
    p3 = st3["parray"]
    args = dict(rhosink=rhosink, sinkrad=0.6, hmult_sinkrad=True, timescale_search=True)
    want3 = sink_search(p3[:, 0:3], p3[:, 3], p3[:, 4], st3["v"], st3["a"], st3["rho"],
                        st3["gpot"], s3["rmh"], s3["v"], s3["a"], np.full(2, 0.05), **args)
    got3 = g.sink_search(**args)
    assert got3["created"] == (want3["psink"] >= 0)
    if got3["created"]:
        assert got3["psink_id"] == st3["perm"][want3["psink"]]
        assert np.array_equal(got3["angmom"], want3["angmom"])
    else:
        assert g.ptot == p3.shape[0] and np.array_equal(g.download()["perm"], st3["perm"])
    g.force_step(first_call=False)
    assert np.isfinite(g.download()["a"]).all()


def _restock_pipeline(o, parray, v, sound):
    """The oracle's evaluation on the tree it holds, restocked at new
    positions (tree_update without a build: main/tree_update.F90 between
    builds), particles in their current order."""
    p, _ = o.tree_update(parray, do_build=False)
    s = o.sph_update(p, v, first_call=False)
    press = sound * sound * s["rho"]
    a, gpot = o.grav_forces(o.hydro_forces(press, sound))
    return dict(parray=s["parray"], a=a, gpot=gpot, rho=s["rho"])


def test_rk2_step_restocks_between_builds(libs):
    """With nbuildstep = 8 (the reference's default) the two evaluations of a
    Runge-Kutta step after the first build restock the same cells at the new
    positions instead of building: the particle order stays, and positions,
    velocities, rho and accelerations match the oracle driven through the same
    restocks."""
    from oracle.oracle import rk2_full, rk2_half
    ic = case("sphere4k")
    o, g = _pair(libs, ic)
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g.set_build_step(8)
    g.force_step(first_call=True)
    r0 = run_pipeline(o, ic)
    dt = g.timestep()
    g.rk2_step(dt)
    st = g.download()
    assert np.array_equal(st["perm"], r0["perm"])            # no build: same order
    p0, v0, snd = r0["sph"]["parray"], r0["v"], r0["sound"]
    rh, vh = rk2_half(p0[:, 0:3], v0, r0["a"], 0.5 * dt)
    ph = p0.copy()
    ph[:, 0:3] = rh
    r1 = _restock_pipeline(o, ph, vh, snd)
    x1, v1 = rk2_full(p0[:, 0:3], v0, vh, r1["a"], dt)
    p1 = r1["parray"].copy()
    p1[:, 0:3] = x1
    r2 = _restock_pipeline(o, p1, v1, snd)
    assert np.abs(st["parray"][:, 0:3] - x1).max() < 1e-13
    assert rel_rows(st["v"], v1).max() < 1e-10
    assert np.abs(st["parray"][:, 4] / r2["parray"][:, 4] - 1).max() < TOL
    assert np.abs(st["rho"] / r2["rho"] - 1).max() < TOL
    assert rel_rows(st["a"], r2["a"]).max() < 1e-9
    # a build every evaluation again: the next step reorders
    g.set_build_step(1)
    g.rk2_step(g.timestep())
    assert np.isfinite(g.download()["a"]).all()


def test_accretion_full_size_properties(libs):
    """Accretion at the full 4,194,304-particle core, mixed precision (too large
    for the Python oracle): size-independent properties of the result.  Mass and
    momentum are conserved; every removed particle lies inside the radius of an
    accreting sink and the per-sink counts follow the nearest-sink rule; no
    particle outside every radius is removed; the kept particles keep their
    order; a force step runs on them."""
    from seren_b200 import ics
    ic = ics.turbulent_core(n=1 << 22, seed=4, sound=0.2, mach=2.0, h_fac=1.2,
                            thetamaxsqd=0.25)
    g = libs[1](ic["parray"].shape[0], params(ic, precision=1))
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    rng = np.random.default_rng(3)
    pick = rng.choice(ic["parray"].shape[0], 8, replace=False)
    sinks = np.c_[ic["parray"][pick, 0:3], np.full(8, 1e-3), np.full(8, 0.01)]
    sv, srad = np.zeros((8, 3)), np.full(8, 0.03)
    g.set_sinks(sinks)
    g.set_sink_motion(sv, srad)
    g.force_step(first_call=True)
    st, s0 = g.download(), g.get_sinks()
    p, v = st["parray"], st["v"]
    cnt = g.accrete(energy_accrete=True)
    s1, st1 = g.get_sinks(), g.download()
    keep_ids = st1["perm"]
    kept = np.isin(st["perm"], keep_ids)
    assert np.array_equal(st["perm"][kept], keep_ids)           # order kept
    assert cnt.sum() == (~kept).sum() > 0
    m0 = p[:, 3].sum() + s0["rmh"][:, 3].sum()
    m1 = st1["parray"][:, 3].sum() + s1["rmh"][:, 3].sum()
    assert abs(m1 / m0 - 1) < 1e-12
    P0 = (p[:, 3:4] * v).sum(0) + (s0["rmh"][:, 3:4] * s0["v"]).sum(0)
    P1 = (st1["parray"][:, 3:4] * st1["v"]).sum(0) + (s1["rmh"][:, 3:4] * s1["v"]).sum(0)
    assert np.abs(P1 - P0).max() < 1e-12 * (np.abs(p[:, 3:4] * v).sum() + 1e-300)
    d2 = np.stack([((p[:, 0:3] - s0["rmh"][k, 0:3]) ** 2).sum(1) for k in range(8)], axis=1)
    inside = d2 < srad[None, :] ** 2
    near = np.where(inside, d2, np.inf).argmin(1)
    assert inside[~kept].any(1).all() and not (~kept & ~inside.any(1)).any()
    assert np.array_equal(cnt, np.bincount(near[~kept], minlength=8))
    g.force_step(first_call=False)
    assert np.isfinite(g.download()["a"]).all()


@pytest.mark.parametrize("a", [1e-5, 3e-7])
def test_deep_tree_bit_exact_and_full_evaluation(libs, a):
    """Trees of 22-30 levels (the reference's LMAX = 30, headers/macros.h:139):
    a tight clump inside a wide halo.  The GPU builds them from 30-level keys;
    cells, order and stock are bit-exact, and the whole evaluation matches."""
    from tests.helpers import deep_clump
    ic = deep_clump(a)
    o, g = _pair(libs, ic)
    po, permo = o.tree_update(ic["parray"])
    pg, permg = g.tree_update(ic["parray"])
    assert np.array_equal(permo, permg)
    to, tg = o.tree_export(), g.tree_export()
    assert to["ltot"] > 21 and to["ltot"] == tg["ltot"] and to["ctot"] == tg["ctot"]
    for k in ("leaf", "nextcell", "ifopen", "plist", "first_cell", "last_cell"):
        assert np.array_equal(to[k], tg[k]), k
    for k in ("grav_r", "grav_m", "grav_q", "dminsqd", "hydro_r", "rmax"):
        assert np.array_equal(to[k], tg[k]), k
    o, g = _pair(libs, ic)
    ro = run_pipeline(o, ic)
    rg = run_pipeline(g, ic)
    so, sg = ro["sph"], rg["sph"]
    assert rel_rows(sg["parray"][:, 4], so["parray"][:, 4]).max() < TOL
    assert rel_rows(sg["rho"], so["rho"]).max() < TOL
    assert lists_equal(so["pptot"], so["pplist"], sg["pptot"], sg["pplist"], g.params.pp_limit)
    assert rel_scaled(rg["a_hydro"], ro["a_hydro"]) < TOL
    assert rel_rows(rg["a"], ro["a"]).max() < 1e-11
    g32 = libs[1](ic["parray"].shape[0], params(ic, precision=1))
    r32 = run_pipeline(g32, ic)
    assert np.array_equal(r32["perm"], rg["perm"])
    err = rel_rows(r32["a"], rg["a"])
    assert np.sqrt(np.mean(err ** 2)) < 1e-5


def test_tree_beyond_lmax_fails_like_the_reference(libs):
    """A clump that needs more than 30 levels, and a 24-level tree under
    lmax = 22: both the oracle and the GPU stop with ERR_LMAX."""
    from seren_b200.cabi import SerenError
    from tests.helpers import deep_clump
    for a, lmax in ((1e-7, 30), (1e-5, 22)):
        ic = deep_clump(a)
        n = ic["parray"].shape[0]
        prm = params(ic)
        prm.lmax = lmax
        Oracle, Gpu = libs
        for hp in (Oracle(n, prm), Gpu(n, prm)):
            with pytest.raises(SerenError) as e:
                hp.tree_update(ic["parray"])
            assert e.value.code == 3


@pytest.mark.parametrize("name", ["sphere4k", "plummer16k", "disc12k", "ragged777", "tiny100"])
def test_h_gather_bit_exact(libs, name):
    """h_gather (sph/h_gather.F90) for every particle, then for an active
    subset with Fortran ids: h bit-exact with the oracle's restatement, and
    the neighbour lists at that h too."""
    ic = case(name)
    o, g = _pair(libs, ic)
    po, permo = o.tree_update(ic["parray"])
    pg, permg = g.tree_update(ic["parray"])
    assert np.array_equal(permo, permg)
    ho = o.h_gather(po)
    hg = g.h_gather(pg)
    assert np.array_equal(ho[:, 4], hg[:, 4])
    pto, plo = o.get_neib()
    ptg, plg = g.get_neib()
    assert lists_equal(pto, plo, ptg, plg, g.params.pp_limit)
    n = ic["parray"].shape[0]
    o1, g1 = _pair(libs, ic, index_base=1)
    po, _ = o1.tree_update(ic["parray"])
    pg, _ = g1.tree_update(ic["parray"])
    acc = np.arange(1, n + 1, 3, dtype=np.int32)
    ho = o1.h_gather(po, acclist=acc)
    hg = g1.h_gather(pg, acclist=acc)
    assert np.array_equal(ho[:, 4], hg[:, 4])
    rest = np.setdiff1d(np.arange(n), acc - 1)
    assert np.array_equal(hg[rest, 4], pg[rest, 4])       # inactive rows untouched


def test_h_gather_deep_clump_and_too_few_particles(libs):
    """A 24-level tree (h spanning seven decades) is bit-exact too; with
    fewer particles than pp_gather + 1 the reference never ends its search,
    here both stop with ERR_WALK."""
    from seren_b200.cabi import SerenError
    from tests.helpers import deep_clump
    ic = deep_clump(1e-5)
    o, g = _pair(libs, ic)
    po, _ = o.tree_update(ic["parray"])
    pg, _ = g.tree_update(ic["parray"])
    assert np.array_equal(o.h_gather(po)[:, 4], g.h_gather(pg)[:, 4])
    small = ics.uniform_sphere(n=40, seed=8)
    o, g = _pair(libs, small)
    for hp in (o, g):
        p, _ = hp.tree_update(small["parray"])
        with pytest.raises(SerenError) as e:
            hp.h_gather(p)
        assert e.value.code == 5


@pytest.mark.parametrize("nlevels,level_mode,check_neib,nbuildstep,nsteps", [
    (4, 1, 1, 1, 36),        # the reference's default options, a build every step
    (3, 2, 2, 4, 28),        # fixed levels, immediate reduction, restocks between builds
])
def test_block_timesteps_match_oracle(libs, nlevels, level_mode, check_neib, nbuildstep, nsteps):
    """Block timesteps on the device (seren_gpu_block_step: forces of the
    accdo particles, sph_timesteps, check_neighbour_timesteps,
    advance_runge_kutta, reduce_timesteps) against the same loop restated
    in oracle/oracle.py driving the oracle's force path: after every integer
    step the particle order, every level, nlast, nminneib and accdo are
    equal, the time scalars equal, positions within 1e-12 and velocities
    and accelerations within 1e-9."""
    from oracle.oracle import BlockSteps
    ic = case("plummer16k")
    o, g = _pair(libs, ic)
    b = BlockSteps(o, ic, nlevels=nlevels, level_mode=level_mode, check_neib=check_neib,
                   nbuildstep=nbuildstep)
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g.set_build_step(nbuildstep)
    g.force_step(first_call=True)
    g.block_start(nlevels=nlevels, level_mode=level_mode, check_neib=check_neib)
    seen_levels, seen_active = set(), set()
    for k in range(nsteps):
        b.step()
        st = g.block_step()
        assert (st["n"], st["nresync"], st["nsteps"], st["level_max"], st["level_step"]) == \
            (b.n, b.nresync, b.nsteps, b.level_max, b.level_step), k
        assert st["nactive"] == b.nactive, k
        assert st["timestep"] == b.timestep and st["time"] == b.time, k
        d, lv = g.download(), g.block_levels()
        assert np.array_equal(d["perm"], b.perm), k
        assert np.array_equal(lv["nlevel"], b.nlevel), k
        assert np.array_equal(lv["nlast"], b.nlast), k
        assert np.array_equal(lv["accdo"].astype(bool), b.accdo), k
        if check_neib:
            assert np.array_equal(lv["nminneib"], b.nminneib), k
        assert np.abs(d["parray"][:, 0:3] - b.parray[:, 0:3]).max() < 1e-12, k
        assert rel_rows(d["v"], b.v).max() < 1e-9, k
        assert rel_rows(d["a"], b.a).max() < 1e-9, k
        seen_levels.update(np.unique(b.nlevel).tolist())
        seen_active.add(b.nactive)
    assert len(seen_levels) >= 3 and len(seen_active) >= 4     # a real block hierarchy


@pytest.mark.parametrize("precision", [0, 1])
def test_autotune_keeps_results(libs, precision):
    """seren_gpu_autotune times four configurations of the kernel knobs and
    keeps the fastest per stage.  The same inputs under the tuned knobs and
    under the defaults give the same FP64 results bit for bit, and mixed ones
    within the mixed-precision bars.  A second context of the same size takes
    the recorded choice with trials = 0, and bad knobs are refused."""
    from seren_b200.cabi import SerenError
    ic = case("sphere32k")
    n = ic["parray"].shape[0]
    Oracle, Gpu = libs
    g = Gpu(n, params(ic, precision=precision))
    g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g.force_step(first_call=True)
    t = g.autotune(trials=1)
    g.close()
    assert t["hydro_sub"] in (2, 4, 8) and t["grav_cap"] in (64, 96) and t["ms_per_step"] > 0
    knobs = {k: t[k] for k in ("hydro_sub", "grav_cap", "grav_bps", "gradh_bps", "neib_bps")}
    runs = []
    for tuned in (False, True):
        h = Gpu(n, params(ic, precision=precision))
        h.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
        if tuned:
            h.set_tuning(**knobs)
        h.force_step(first_call=True)
        h.drift(1.0e-3)
        h.force_step()
        runs.append(h.download())
        h.close()
    d0, d1 = runs
    assert np.array_equal(d0["perm"], d1["perm"])
    assert np.array_equal(d0["rho"], d1["rho"])               # grad-h is FP64 in both
    if precision == 0:
        assert np.array_equal(d0["a"], d1["a"])
    else:
        err = rel_rows(d1["a"], d0["a"])
        assert np.sqrt(np.mean(err ** 2)) < 1e-5
    g2 = Gpu(n, params(ic, precision=precision))
    g2.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
    g2.force_step(first_call=True)
    t2 = g2.autotune(trials=0)
    assert {k: t2[k] for k in knobs} == knobs
    with pytest.raises(SerenError):
        g2.set_tuning(hydro_sub=3)
    g2.close()


def test_whole_gpu_gradh_path_repeats_bit_for_bit(libs):
    """The whole-GPU grad-h path (particles whose walks outgrow the redo
    kernel's scratch) sums its walk slices and particle tiles in a fixed order:
    two runs give the same h, rho, omega, div v and drho/dt bit for bit."""
    ic = case("turb20k")
    Oracle, Gpu = libs
    n = ic["parray"].shape[0]
    runs = []
    for _ in range(2):
        g = Gpu(n, params(ic, redo_cap=8))
        g.upload(ic["parray"], ic["v"], ic["sound"] ** 2)
        g.force_step(first_call=True)
        assert g.last_step_stats()[2][8] > 0            # particles on the whole-GPU path
        runs.append(g.download())
        g.close()
    for k in ("parray", "rho", "omega", "a", "gpot"):
        assert np.array_equal(runs[0][k], runs[1][k]), k
