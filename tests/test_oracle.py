"""The CPU oracle: kernel tables, tree structure, physical invariants of the
reference's algorithm (the checks the reference's own physics relies on,
since it ships no test vectors), and its error handling."""
import numpy as np
import pytest

from oracle.oracle import KERNTOT, Oracle, kernel_tables
from seren_b200 import ics
from seren_b200.cabi import Params, SerenError
from tests.helpers import case, params, rel_rows, run_pipeline

S = (2.0 * np.arange(KERNTOT + 1) + 1.0) / KERNTOT


def test_kernel_normalisation():
    """Integral of W over 3-D space is 1 (setup/kernel.F90 M4, 3-D norm INVPI)."""
    w0 = kernel_tables(0)[0]
    ds = 2.0 / KERNTOT
    integral = np.sum(4.0 * np.pi * S[:KERNTOT] ** 2 * w0[:KERNTOT]) * ds
    assert abs(integral - 1.0) < 1e-6


def test_kernel_identities():
    t = kernel_tables(0)
    w0, w1, w4, w5, w6, wh = t[0], t[1], t[4], t[5], t[6], t[7]
    assert np.array_equal(w1, w4)                       # M4: gradient table used twice
    # wh = -NDIM*w0 - s*w4 (kernel.F90:84, the commented identity)
    assert np.max(np.abs(wh - (-3.0 * w0 - S * w4))) < 1e-12
    # softened force and potential approach 1/s^2 and 1/s at s >= 2
    assert abs(w5[KERNTOT] - 1.0 / S[KERNTOT] ** 2) < 1e-6
    assert abs(w6[KERNTOT] - 1.0 / S[KERNTOT]) < 1e-6


def test_thomas_couchman_table():
    t0, t1 = kernel_tables(0), kernel_tables(1)
    kerntc = int(KERNTOT / 3.0)
    assert np.all(t1[1, :kerntc] == -1.0 * 0.318309886)
    assert np.array_equal(t1[1, kerntc:], t0[1, kerntc:])
    assert np.array_equal(np.delete(t1, 1, 0), np.delete(t0, 1, 0))


def test_pp_gather():
    assert ics.pp_gather_for(1.2) == 57          # initialize_seren_variables_1.F90:36
    assert ics.pp_gather_for(ics.h_fac_for(50)) in (49, 50)


@pytest.mark.parametrize("name", ["sphere4k", "plummer16k", "ragged777"])
def test_tree_structure(name):
    ic = case(name)
    n = ic["parray"].shape[0]
    o = Oracle(n, params(ic))
    p, perm = o.tree_update(ic["parray"])
    t = o.tree_export()
    assert np.array_equal(np.sort(perm), np.arange(n))
    assert np.array_equal(p, ic["parray"][perm])
    leaf = t["leaf"]
    assert leaf[0] == 0 and leaf.max() <= 8
    # leaves in depth-first order list every particle once, in tree order 0..n-1
    order = []
    c = 0
    while c <= t["ctot"]:
        if leaf[c] > 0:
            order.extend(t["plist"][c, :leaf[c]].tolist())
            c = t["nextcell"][c]
        else:
            c = t["ifopen"][c]
    assert order == list(range(n))
    # levels partition the cell ids
    assert t["first_cell"][0] == 0 and t["last_cell"][-1] == t["ctot"]
    assert np.all(t["first_cell"][1:] == t["last_cell"][:-1] + 1)
    # every cell mass is the sum of its particles; the root holds the total mass
    assert abs(t["grav_m"][0] - ic["parray"][:, 3].sum()) < 1e-12


def test_leaf_lists_keep_input_order():
    """Within a leaf the reference keeps the particles' input order
    (linked lists, BHgrav_build.F90:170-182)."""
    ic = case("sphere4k")
    o = Oracle(4096, params(ic))
    _, perm = o.tree_update(ic["parray"])
    t = o.tree_export()
    for c in np.nonzero(t["leaf"] > 1)[0]:
        ids = perm[t["plist"][c, :t["leaf"][c]]]
        assert np.all(np.diff(ids) > 0)


def test_hydro_conserves_momentum():
    ic = case("turb20k")
    o = Oracle(20000, params(ic))
    r = run_pipeline(o, ic)
    m = r["parray"][:, 3]
    mom = np.abs((m[:, None] * r["a_hydro"]).sum(0))
    scale = np.sum(m[:, None] * np.abs(r["a_hydro"]))
    assert np.all(mom < 1e-13 * scale)


def test_tree_tends_to_direct_sum():
    """theta -> 0 opens every cell: the walk becomes direct_sph_gravity."""
    ic = case("sphere4k")
    o = Oracle(4096, params(ic, thetamaxsqd=1e-8))
    r = run_pipeline(o, ic)
    ids = np.arange(0, 4096, 7, dtype=np.int32)
    ad, gd = o.direct_gravity(ids)
    ag = r["a"] - r["a_hydro"]
    assert rel_rows(ag[ids], ad).max() < 1e-12
    assert rel_rows(r["gpot"][ids], gd).max() < 1e-12


def test_tree_error_at_theta_half():
    ic = case("sphere32k")
    o = Oracle(32768, params(ic))
    r = run_pipeline(o, ic)
    ids = np.arange(0, 32768, 64, dtype=np.int32)
    ad, _ = o.direct_gravity(ids)
    err = rel_rows((r["a"] - r["a_hydro"])[ids], ad)
    assert np.sqrt(np.mean(err ** 2)) < 5e-3


def test_direct_sum_plummer_analytic():
    """Direct-sum gravity of a Plummer sphere follows -M r / (r^2 + a^2)^1.5."""
    ic = ics.plummer(n=8192, seed=21)
    ic["sound"] = np.full(8192, 0.1)
    o = Oracle(8192, params(ic))
    r = run_pipeline(o, ic)
    ids = np.arange(0, 8192, 8, dtype=np.int32)
    ad, _ = o.direct_gravity(ids)
    x = r["parray"][ids, :3]
    rr = np.linalg.norm(x, axis=1)
    sel = (rr > 0.3) & (rr < 3.0)
    ana = rr[sel] / (rr[sel] ** 2 + 1.0) ** 1.5
    ratio = np.linalg.norm(ad[sel], axis=1) / ana
    assert abs(np.median(ratio) - 1.0) < 0.05


def test_uniform_density():
    """SPH density inside a uniform sphere is near 3M/(4 pi R^3); the Poisson
    sampling and the self term bias it high by tens of per cent, not more."""
    ic = case("sphere32k")
    o = Oracle(32768, params(ic))
    r = run_pipeline(o, ic)
    rr = np.linalg.norm(r["parray"][:, :3], axis=1)
    rho = r["sph"]["rho"][rr < 0.6]
    ratio = np.median(rho) / (3.0 / (4.0 * np.pi))
    assert 1.0 < ratio < 1.5
    nn = r["sph"]["pptot"][rr < 0.6]
    assert 40 < np.median(nn) < 80


def test_error_codes():
    ic = case("tiny100")
    o = Oracle(50, params(ic))
    with pytest.raises(SerenError) as e:
        o.tree_update(ic["parray"])
    assert e.value.code == 2                  # ptot > pmax: capacity
    o = Oracle(100, params(ic))
    bad = ic["parray"].copy()
    bad[5, 1] = np.nan
    with pytest.raises(SerenError) as e:
        o.tree_update(bad)
    assert e.value.code == 4                  # non-finite input
    same = ic["parray"].copy()
    same[:20, :3] = 0.25                      # 20 coincident particles: the tree cannot split them
    with pytest.raises(SerenError) as e:
        o.tree_update(same)
    assert e.value.code == 3
    with pytest.raises(SerenError):
        Oracle(100, Params.make(h_fac=1.2, index_base=2))


def test_too_few_particles_is_an_error():
    """With fewer particles than pp_gather the reference grows h forever; the
    restatement stops with ERR_WALK."""
    ic = ics.uniform_sphere(n=40, seed=1)
    o = Oracle(40, params(ic))
    p, perm = o.tree_update(ic["parray"])
    with pytest.raises(SerenError) as e:
        o.sph_update(p, ic["v"][perm], first_call=True)
    assert e.value.code == 5


def test_timestep_sizes_formula():
    """timestep_size.F90:95-105 on hand numbers: h = 0.1, a = (3, 4, 0), c = 1,
    div v = -2, alpha = 1 (beta = 2): tacc = 0.5 sqrt(0.1/5), tcour =
    0.2*0.1/((1 + 0.2) + 0.6 (1 + 0.4)) = 0.02/2.04, dt = the smaller."""
    from oracle.oracle import timestep_sizes
    dt = timestep_sizes([0.1, 0.1], [[3.0, 4.0, 0.0], [0.0, 0.0, 1e-8]], [-2.0, 0.0], [1.0, 1.0],
                        1.0)
    assert abs(dt[0] - 0.02 / 2.04) < 1e-15
    # with |a| tiny and div v = 0 the Courant limit 0.2*0.1/(1 + 0.6) holds
    assert abs(dt[1] - 0.02 / 1.6) < 1e-15


def test_rk2_steps():
    """advance_runge_kutta.F90:40-69: half step with the start forces, full
    step from the start with the half-step velocity and forces."""
    from oracle.oracle import rk2_full, rk2_half
    r, v, a = np.array([[1.0, 0.0, 0.0]]), np.array([[0.0, 1.0, 0.0]]), np.array([[-1.0, 0.0, 0.0]])
    rh, vh = rk2_half(r, v, a, 0.05)
    assert np.allclose(rh, [[1.0, 0.05, 0.0]]) and np.allclose(vh, [[-0.05, 1.0, 0.0]])
    r1, v1 = rk2_full(r, v, vh, -rh, 0.1)
    assert np.allclose(r1, [[1.0 - 0.005, 0.1, 0.0]]) and np.allclose(v1, [[-0.1, 0.995, 0.0]])


def test_accretion_conserves_mass_momentum_and_angular_momentum():
    """The accretion restatement (accrete_particles.F90) against invariants that
    do not depend on its loops: each accreted particle lies inside its sink's
    radius and no accreting sink is nearer; mass, momentum, mass-weighted
    acceleration and angular momentum about the origin (sink orbital part plus
    the spin added) are conserved; a sink that does not accrete takes nothing;
    without the energy test every particle inside a radius is taken."""
    from oracle.oracle import accrete_particles
    rng = np.random.default_rng(11)
    n = 3000
    r = rng.uniform(-1, 1, (n, 3))
    v = rng.normal(0, 0.5, (n, 3))
    a = rng.normal(0, 1.0, (n, 3))
    m = rng.uniform(0.5, 1.5, n) / n
    h = rng.uniform(0.05, 0.1, n)
    rmh = np.array([[0.0, 0.0, 0.0, 0.05, 0.05], [0.25, 0.0, 0.0, 0.03, 0.04],
                    [-0.5, 0.5, 0.2, 0.02, 0.05]])
    sv = np.array([[0.1, 0.0, 0.0], [0.0, -0.2, 0.1], [0.0, 0.0, 0.3]])
    sa = rng.normal(0, 1.0, (3, 3))
    rad = np.array([0.3, 0.2, 0.25])
    flags = [1, 1, 0]
    w = accrete_particles(r, m, h, v, a, rmh, sv, sa, rad, accrete=flags, energy_accrete=True)
    allin = accrete_particles(r, m, h, v, a, rmh, sv, sa, rad, accrete=flags)
    d2 = ((r[:, None, :] - rmh[None, :, 0:3]) ** 2).sum(-1)
    inside = (d2 < rad[None, :] ** 2) & (np.array(flags, bool)[None, :])
    assert (allin["dead"] >= 0).sum() == inside.any(1).sum()
    assert 0 < (w["dead"] >= 0).sum() < (allin["dead"] >= 0).sum()
    for q in np.flatnonzero(w["dead"] >= 0):
        s = w["dead"][q]
        assert inside[q, s] and d2[q, s] == d2[q, inside[q]].min()
    assert w["count"][2] == 0 and np.array_equal(w["rmh"][2], rmh[2])
    for s in (0, 1):
        mine = w["dead"] == s
        mt = rmh[s, 3] + m[mine].sum()
        assert np.isclose(w["rmh"][s, 3], mt, rtol=1e-14)
        p0 = rmh[s, 3] * sv[s] + (m[mine, None] * v[mine]).sum(0)
        assert np.allclose(w["rmh"][s, 3] * w["v"][s], p0, rtol=1e-12, atol=1e-15)
        f0 = rmh[s, 3] * sa[s] + (m[mine, None] * a[mine]).sum(0)
        assert np.allclose(w["rmh"][s, 3] * w["a"][s], f0, rtol=1e-12, atol=1e-15)
        L0 = rmh[s, 3] * np.cross(rmh[s, 0:3], sv[s]) + (m[mine, None] *
                                                          np.cross(r[mine], v[mine])).sum(0)
        L1 = w["rmh"][s, 3] * np.cross(w["rmh"][s, 0:3], w["v"][s]) + w["angmom"][s]
        assert np.allclose(L1, L0, rtol=1e-10, atol=1e-15)
    assert np.array_equal(w["keep"], np.flatnonzero(w["dead"] < 0))


def test_sink_search_picks_as_the_reference_does():
    """The sink search restatement (sink_search.F90, create_sink.F90) on three
    dense clumps: the three potential minima are the candidates; with the
    div v / div a tests the densest fails and a lighter one passes, and the
    sink is made at the densest all the same (the last loop leaves psink at
    the densest candidate it visited); the new sink holds the mass, centre of
    mass and momentum of the particles it removes, and the angular momentum
    about its centre."""
    from oracle.oracle import sink_search
    ic = case("clumps12k")
    n = ic["parray"].shape[0]
    o = Oracle(n, params(ic))
    r = run_pipeline(o, ic)
    p, rho, g = r["sph"]["parray"], r["sph"]["rho"], r["gpot"]
    none = (np.zeros((0, 5)), np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0))
    s = sink_search(p[:, 0:3], p[:, 3], p[:, 4], r["v"], r["a"], rho, g, *none,
                    rhosink=np.percentile(rho, 90), sinkrad=0.05)
    cand = s["candidates"]
    assert len(cand) == 3 and list(np.argsort(rho[cand])) == [0, 1, 2]
    assert s["flags"][2] is False and any(s["flags"])
    assert s["psink"] == cand[2]
    gone = s["removed"]
    assert s["psink"] in gone and len(gone) > 100
    d = np.sqrt(np.sum((p[gone, 0:3] - p[s["psink"], 0:3]) ** 2, axis=1))
    assert d.max() <= 0.05 * (1 + 1e-12)
    m = p[gone, 3]
    assert np.isclose(s["m"], m.sum(), rtol=1e-14)
    assert np.allclose(s["r"], (m[:, None] * p[gone, 0:3]).sum(0) / m.sum(), rtol=1e-12)
    assert np.allclose(s["v"], (m[:, None] * r["v"][gone]).sum(0) / m.sum(), rtol=1e-12, atol=1e-15)
    L = (m[:, None] * np.cross(p[gone, 0:3] - s["r"], r["v"][gone] - s["v"])).sum(0)
    assert np.allclose(s["angmom"], L, rtol=1e-9, atol=1e-18)
    assert s["h"] == 0.025 and s["radius"] == 0.05
    assert np.array_equal(np.sort(np.concatenate([s["keep"], gone])), np.arange(n))
    # no density or divergence tests: the densest candidate passes and is taken
    s2 = sink_search(p[:, 0:3], p[:, 3], p[:, 4], r["v"], r["a"], rho, g, *none,
                     rhosink=np.percentile(rho, 90), sinkrad=0.05, div_v_search=False,
                     div_a_search=False)
    assert s2["psink"] == cand[2] and all(s2["flags"])


@pytest.mark.parametrize("name", ["sphere4k", "plummer16k", "disc12k", "ragged777"])
def test_h_gather_is_the_pp_gather_th_neighbour_distance(name):
    """The oracle's h_gather (a statement-by-statement restatement of
    sph/h_gather.F90, insertion sort included) against an independent brute
    force: h = 0.5 sqrt of the pp_gather-th smallest squared distance to any
    other particle, bit for bit (the same FP64 expression per pair)."""
    ic = case(name)
    n = ic["parray"].shape[0]
    prm = params(ic)
    o = Oracle(n, prm)
    p, _ = o.tree_update(ic["parray"])
    h = o.h_gather(p)[:, 4]
    x = p[:, :3]
    k = prm.pp_gather
    for i in range(0, n, max(1, n // 300)):
        d = x - x[i]
        d2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        d2[i] = np.inf
        assert h[i] == 0.5 * np.sqrt(np.partition(d2, k - 1)[k - 1]), i
    o.close()


def test_gradh_bisection_cases():
    """The cases the GPU's bisection parity test relies on: on the first call
    (h guess) some particles of three dense clumps reach the reference's
    bisection (all_sph_gradh.F90:256-275), none of the uniform sphere's do,
    and every h ends finite and positive."""
    for name, expect in (("clumps12k", True), ("sphere4k", False)):
        ic = case(name)
        n = ic["parray"].shape[0]
        o = Oracle(n, params(ic))
        r = run_pipeline(o, ic)
        nb = o.counts()["gradh_bisections"]
        o.close()
        assert (nb > 0) == expect, (name, nb)
        h = r["sph"]["parray"][:, 4]
        assert np.all(np.isfinite(h)) and np.all(h > 0.0)
