// sph.cu - grad-h smoothing length / density solve, neighbour lists, grad-h
// hydro forces with MON97 viscosity, and the isothermal equation of state.
//
// One thread owns one active particle and follows its reference routine step
// by step.  The candidate lists of the reference (BHhydrowalk_hgather,
// BHhydro_walk) are never materialised: the stackless walk is re-run and each
// opened leaf's particles are consumed as they come, which visits candidates
// in exactly the reference's list order (depth-first leaf order, particles in
// leaf order), so every sum is accumulated in the reference's order.
#include "ctx.cuh"

namespace seren {

namespace {

struct HydroTree {
  const int4* link;     // {leaf, nextcell, ifopen, pstart}
  const double4* hA;    // bbox centre, rmax
  const double* hrm;    // hrangemax
  int ctot;
};

// BHtree/BHhydrowalk_hgather.F90:11-77 (gather test only).  f(q) is called
// for every particle of every opened leaf.  Returns false when the walk
// exceeded its cap (a corrupt tree), after flagging the error.
template <class F>
__device__ __forceinline__ bool walk_gather(const HydroTree& t, double rx, double ry, double rz,
                                            double hrange, DevError* err, int who, F&& f) {
  int c = 0;
  int visits = 0;
  const int cap = t.ctot + 2;
  while (true) {
    if (++visits > cap) {
      set_error(err, SEREN_GPU_ERR_WALK, KID_GRADH, who, c);
      return false;
    }
    const double4 h = t.hA[c];
    const int4 lk = t.link[c];
    const double d0 = h.x - rx, d1 = h.y - ry, d2 = h.z - rz;
    const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
    const double tt = hrange + h.w;
    if (drsqd <= tt * tt) {
      if (lk.x > 0) {
        for (int i = 0; i < lk.x; ++i) f(lk.w + i);
        c = lk.y;
      } else if (lk.x == 0) {
        c = lk.z;
      } else {
        c = lk.y;
      }
    } else {
      c = lk.y;
    }
    if (c > t.ctot) break;
  }
  return true;
}

// BHtree/BHhydro_walk.F90:9-80 (gather or scatter test)
template <class F>
__device__ __forceinline__ bool walk_gather_scatter(const HydroTree& t, double rx, double ry,
                                                    double rz, double hrange, DevError* err,
                                                    int who, F&& f) {
  int c = 0;
  int visits = 0;
  const int cap = t.ctot + 2;
  while (true) {
    if (++visits > cap) {
      set_error(err, SEREN_GPU_ERR_WALK, KID_NEIB, who, c);
      return false;
    }
    const double4 h = t.hA[c];
    const int4 lk = t.link[c];
    const double d0 = h.x - rx, d1 = h.y - ry, d2 = h.z - rz;
    const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
    const double t1 = hrange + h.w;
    const double t2 = t.hrm[c] + h.w;
    if (drsqd <= t1 * t1 || drsqd <= t2 * t2) {
      if (lk.x > 0) {
        for (int i = 0; i < lk.x; ++i) f(lk.w + i);
        c = lk.y;
      } else if (lk.x == 0) {
        c = lk.z;
      } else {
        c = lk.y;
      }
    } else {
      c = lk.y;
    }
    if (c > t.ctot) break;
  }
  return true;
}

// sph/all_sph_gradh.F90:11-492 (GRAD_H_SPH, BH_TREE, GRAVITY)
__global__ void __launch_bounds__(128) k_gradh(int nact, const int* __restrict__ act,
                                               const double4* __restrict__ pm, double2* __restrict__ hz,
                                               const double4* __restrict__ vel, double* __restrict__ rho,
                                               double* __restrict__ omega, double* __restrict__ divv,
                                               double* __restrict__ drhodt, HydroTree t,
                                               const double4* __restrict__ tabA, double h_fac,
                                               int pp_gather, double rextent, DevError* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nact) return;
  const int p = act ? act[i] : i;
  const double4 P = pm[p];
  const double rx = P.x, ry = P.y, rz = P.z, mp = P.w;
  double hp = hz[p].x;
  const double4 vp = vel[p];
  const double4 t0 = tabA[0];
  double invhp, hfactor_p, hrangesqd;
  int iteration = 0;
  const double h_old = hp;
  double h_new = hp;
  double h_high = 0.0, h_upper = rextent, h_lower = 0.0;
  int pp_pot = 0, ngrow = 0;
  double rhotemp = 0.0, omega_p = 0.0;
  while (true) {
    while (true) {                                                     // :154-191
      if (hp > h_high) {
        h_high = hp * HMULT;
        int cnt = 0;
        if (!walk_gather(t, rx, ry, rz, KERNRANGE * h_high, err, p, [&](int) { ++cnt; })) return;
        pp_pot = cnt;
      }
      if (pp_pot < pp_gather) {
        h_high = 0.0;
        pp_pot = 0;
        hp = hp * HMULT;
        if (++ngrow > HGROW_CAP) {
          set_error(err, SEREN_GPU_ERR_WALK, KID_GRADH, p, -1);
          return;
        }
      }
      if (pp_pot > 0) break;
    }
    h_new = hp;                                                        // :199-210
    invhp = 1.0 / hp;
    hfactor_p = pow(invhp, NDIMPR);
    hrangesqd = (KERNRANGESQD * hp) * hp;
    rhotemp = (mp * t0.x) * hfactor_p;
    omega_p = ((mp * hfactor_p) * invhp) * t0.y;
    const double hs = hrangesqd, ih = invhp, hf = hfactor_p;
    double rt = rhotemp, om = omega_p;
    walk_gather(t, rx, ry, rz, KERNRANGE * h_high, err, p, [&](int q) {  // :214-235
      if (q == p) return;
      const double4 Q = pm[q];
      const double d0 = Q.x - rx, d1 = Q.y - ry, d2 = Q.z - rz;
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      if (drsqd >= hs) return;
      const double drmag = sqrt(drsqd) + SMALL_NUMBER;
      const int kern = (int)((HALFKERNTOT * drmag) * ih);
      if (kern >= KERNTOT) return;
      const double4 w = tabA[kern];
      rt = rt + (Q.w * hf) * w.x;
      om = om + ((Q.w * hf) * ih) * w.y;
    });
    rhotemp = rt;
    omega_p = 1.0 + ((hp * om) / (NDIMPR * rhotemp));                  // :238
    const double hcand = h_fac * pow(mp / rhotemp, ONETHIRD);
    if (fabs(hp - hcand) / hp < H_CON && iteration >= 1) break;        // :246
    if (iteration < GRADH_ITERATION_MAX) {
      h_new = hcand;
    } else if (iteration == GRADH_ITERATION_MAX) {
      h_upper = rextent;
      h_lower = 0.0;
      h_new = 0.5 * (h_lower + h_upper);
    } else if (iteration < 2 * GRADH_ITERATION_MAX) {
      double fb;
      if (rhotemp > SMALL_NUMBER) fb = pow(hp, NDIMPR) - (pow(h_fac, NDIMPR) * mp) / rhotemp;
      else fb = 1.0;
      if (fb > 0.0) h_upper = hp;
      else h_lower = hp;
      h_new = 0.5 * (h_lower + h_upper);
    } else {
      h_new = h_old;
      hp = h_new;
      break;
    }
    hp = h_new;
    iteration = iteration + 1;
  }
  hp = h_fac * pow(mp / rhotemp, ONETHIRD);                           // :317
  invhp = 1.0 / hp;
  hfactor_p = pow(invhp, NDIMPR);
  hrangesqd = (KERNRANGESQD * hp) * hp;
  double rt = (mp * t0.x) * hfactor_p;
  double om = ((mp * hfactor_p) * invhp) * t0.y;
  double dv_sum = 0.0;
  double zt = ((mp * invhp) * invhp) * t0.w;
  const double hs = hrangesqd, ih = invhp, hf = hfactor_p;
  walk_gather(t, rx, ry, rz, KERNRANGE * h_high, err, p, [&](int q) {  // :360-425
    if (q == p) return;
    const double4 Q = pm[q];
    const double d0 = Q.x - rx, d1 = Q.y - ry, d2 = Q.z - rz;
    double drmag = (d0 * d0 + d1 * d1) + d2 * d2;
    if (drmag > hs) return;
    drmag = sqrt(drmag) + SMALL_NUMBER;
    const int kern = (int)((HALFKERNTOT * drmag) * ih);
    if (kern > KERNTOT) return;
    const double4 V = vel[q];
    const double dv0 = V.x - vp.x, dv1 = V.y - vp.y, dv2 = V.z - vp.z;
    const double dvdr = (dv0 * d0 + dv1 * d1) + dv2 * d2;
    const double4 w = tabA[kern];
    rt = rt + (Q.w * hf) * w.x;
    om = om + ((Q.w * hf) * ih) * w.y;
    dv_sum = dv_sum - ((((Q.w * dvdr) * w.z) * hf) * ih) / drmag;
    zt = zt + ((Q.w * ih) * ih) * w.w;
  });
  const double omega_f = 1.0 + ((hp * om) / (NDIMPR * rt));            // :428
  const double div_v_p = dv_sum / rt;
  rho[p] = rt;                                                         // :436-442
  omega[p] = omega_f;
  divv[p] = div_v_p;
  drhodt[p] = -((rt * div_v_p) / omega_f);
  hz[p] = make_double2(hp, -((hp * zt) / ((NDIMPR * rt) * omega_f)));
  if (hp < 0.0) set_error(err, SEREN_GPU_ERR_NEGATIVE_H, KID_GRADH, p, 0);
}

// sph/get_neib.F90:10-140
__global__ void __launch_bounds__(128) k_neib(int nact, const int* __restrict__ act,
                                              const double4* __restrict__ pm,
                                              const double2* __restrict__ hz, HydroTree t, int L,
                                              int* __restrict__ pptot, int* __restrict__ pplist,
                                              DevError* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nact) return;
  const int p = act ? act[i] : i;
  const double4 P = pm[p];
  const double hp = hz[p].x;
  const double hsp = (KERNRANGESQD * hp) * hp;
  int cnt = 0;
  int* row = pplist + (size_t)p * L;
  walk_gather_scatter(t, P.x, P.y, P.z, KERNRANGE * hp, err, p, [&](int q) {
    if (q == p) return;
    const double hq = hz[q].x;
    const double hsq = (KERNRANGESQD * hq) * hq;
    const double4 Q = pm[q];
    const double d0 = Q.x - P.x, d1 = Q.y - P.y, d2 = Q.z - P.z;
    const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
    if (drsqd <= hsp || drsqd <= hsq) {
      if (cnt < L) row[cnt] = q;
      ++cnt;
    }
  });
  pptot[p] = cnt;
}

// sph/hydro_gradh.F90:9-339 (NEIGHBOUR_LISTS, ARTIFICIAL_VISCOSITY=MON97)
__global__ void __launch_bounds__(128) k_hydro(int nact, const int* __restrict__ act,
                                               const double4* __restrict__ pm,
                                               const double2* __restrict__ hz,
                                               const double4* __restrict__ vel,
                                               const double* __restrict__ rho,
                                               const double* __restrict__ omega,
                                               const double* __restrict__ press,
                                               const double* __restrict__ sound,
                                               const int* __restrict__ pptot,
                                               const int* __restrict__ pplist, int L, HydroTree t,
                                               const double4* __restrict__ tabG, double alpha,
                                               double* __restrict__ acc, DevError* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nact) return;
  const int p = act ? act[i] : i;
  const double4 P = pm[p];
  const double hp = hz[p].x;
  const double invhp = 1.0 / hp;
  const double hfactor_p = pow(invhp, NDIMPLUS1);
  const double4 vp = vel[p];
  const double sound_p = sound[p];
  const double rho_p = rho[p];
  const double pfactor_p = ((press[p] / rho_p) / rho_p) / omega[p];
  const double beta = 2.0 * alpha;
  double at0 = 0.0, at1 = 0.0, at2 = 0.0, ad0 = 0.0, ad1 = 0.0, ad2 = 0.0;
  auto pair = [&](int q) {
    double wmean = 0.0;
    const double rho_q = rho[q];
    const double4 Q = pm[q];
    const double hq = hz[q].x;
    double u0 = Q.x - P.x, u1 = Q.y - P.y, u2 = Q.z - P.z;
    double drmag = (u0 * u0 + u1 * u1) + u2 * u2;
    if (drmag >= (KERNRANGESQD * hp) * hp && drmag >= (KERNRANGESQD * hq) * hq) return;
    drmag = sqrt(drmag) + SMALL_NUMBER;
    const double4 V = vel[q];
    const double dv0 = V.x - vp.x, dv1 = V.y - vp.y, dv2 = V.z - vp.z;
    const double dvdr = (dv0 * u0 + dv1 * u1) + dv2 * u2;
    const double invdrmag = 1.0 / drmag;
    u0 = u0 * invdrmag; u1 = u1 * invdrmag; u2 = u2 * invdrmag;
    const double pfactor_q = ((press[q] / rho_q) / rho_q) / omega[q];
    if (drmag < KERNRANGE * hp) {
      int kern = (int)((HALFKERNTOT * drmag) * invhp);
      kern = min(kern, KERNTOT);
      const double w1 = tabG[kern].w;
      wmean = (0.5 * hfactor_p) * w1;
      const double f = ((Q.w * pfactor_p) * hfactor_p) * w1;
      at0 = at0 + f * u0; at1 = at1 + f * u1; at2 = at2 + f * u2;
    }
    if (drmag < KERNRANGE * hq) {
      const double invhq = 1.0 / hq;
      const double hfq = pow(invhq, NDIMPLUS1);
      int kern = (int)((HALFKERNTOT * drmag) * invhq);
      kern = min(kern, KERNTOT);
      const double w1 = tabG[kern].w;
      wmean = wmean + (0.5 * hfq) * w1;
      const double f = ((Q.w * pfactor_q) * hfq) * w1;
      at0 = at0 + f * u0; at1 = at1 + f * u1; at2 = at2 + f * u2;
    }
    const double rhomean = 0.5 * (rho_p + rho_q);
    if (dvdr < 0.0) {
      const double vsignal = (sound_p + sound[q]) - ((beta * dvdr) * invdrmag);
      const double g = (((Q.w * alpha) * vsignal) * dvdr) * invdrmag;
      ad0 = ad0 - ((g * u0) * wmean) / rhomean;
      ad1 = ad1 - ((g * u1) * wmean) / rhomean;
      ad2 = ad2 - ((g * u2) * wmean) / rhomean;
    }
  };
  const int nn = pptot[p];
  if (nn <= L) {
    const int* row = pplist + (size_t)p * L;
    for (int k = 0; k < nn; ++k) pair(row[k]);
  } else {
    // get_neib_on_fly (sph/get_neib_on_fly.F90:11-130): same test as get_neib
    const double hsp = (KERNRANGESQD * hp) * hp;
    walk_gather_scatter(t, P.x, P.y, P.z, KERNRANGE * hp, err, p, [&](int q) {
      if (q == p) return;
      const double hq = hz[q].x;
      const double hsq = (KERNRANGESQD * hq) * hq;
      const double4 Q = pm[q];
      const double d0 = Q.x - P.x, d1 = Q.y - P.y, d2 = Q.z - P.z;
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      if (drsqd <= hsp || drsqd <= hsq) pair(q);
    });
  }
  double* a = acc + (size_t)p * 3;
  a[0] = at0 + ad0;
  a[1] = at1 + ad1;
  a[2] = at2 + ad2;
}

// sph/thermal.F90:52-59 (ISOTHERMAL): press = Pconst*T*rho, sound = sqrt(press/rho)
__global__ void k_thermal(int n, const double* __restrict__ csq, const double* __restrict__ rho,
                          double* __restrict__ press, double* __restrict__ sound) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double r = rho[p];
  const double pr = csq[p] * r;
  press[p] = pr;
  sound[p] = sqrt(pr / r);
}

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

HydroTree hydro_tree(const Ctx& c) { return HydroTree{c.link, c.hA, c.hrm, c.info.ctot}; }

}  // namespace

void launch_gradh(Ctx& c, int nact) {
  if (nact <= 0) return;
  k_gradh<<<nb(nact, 128), 128, 0, c.st>>>(nact, c.act, c.pm, c.hz, c.vel, c.rho, c.omega, c.div_v,
                                           c.drhodt, hydro_tree(c), c.tabA, c.prm.h_fac,
                                           c.prm.pp_gather, c.info.rextent, c.d_err); ++c.nlaunch;
}

void launch_neib(Ctx& c, int nact) {
  if (nact <= 0) return;
  k_neib<<<nb(nact, 128), 128, 0, c.st>>>(nact, c.act, c.pm, c.hz, hydro_tree(c), c.prm.pp_limit,
                                          c.pptot, c.pplist, c.d_err); ++c.nlaunch;
}

void launch_hydro(Ctx& c, int nact) {
  if (nact <= 0) return;
  k_hydro<<<nb(nact, 128), 128, 0, c.st>>>(nact, c.act, c.pm, c.hz, c.vel, c.rho, c.omega, c.press,
                                           c.sound, c.pptot, c.pplist, c.prm.pp_limit,
                                           hydro_tree(c), c.tabG, c.prm.alpha, c.acc, c.d_err); ++c.nlaunch;
}

void launch_thermal(Ctx& c) {
  k_thermal<<<nb(c.ptot, 256), 256, 0, c.st>>>(c.ptot, c.csq, c.rho, c.press, c.sound); ++c.nlaunch;
}

}  // namespace seren
