// Sink accretion on the device-resident particles: sinks/accrete_particles.F90:16-365
// (each gas particle inside the radius of an accreting sink is given to the nearest
// such sink; when bound to it, or always without the energy test, its mass, momentum
// and mass-weighted acceleration go to the sink, which moves to the new centre of mass
// and takes the angular momentum about it), then main/remove_from_list.F90:10-96 (the
// accreted particles leave the arrays; the rest keep their order).
//
// Layout: Ctx::acc_sinks holds ACC_STRIDE doubles per sink, {x, y, z, m, h, radius,
// accrete (1 or 0), vx, vy, vz, ax, ay, az}; Ctx::acc_out the same stride per sink,
// {m, x, y, z, vx, vy, vz, ax, ay, az, Lx, Ly, Lz, -, -, accreted count}; Ctx::acc_ws
// four int arrays of pmax: the sink each particle goes to (-1: none), the exclusive
// scan of the accreted flags, the accreted particles in index order and the kept ones.
//
// Arithmetic is FP64 in the reference's operation order (no contraction), so the sink
// sums, the energy test and the new sink state are those of the reference's serial
// loops: the per-sink sums run in particle index order, one warp per sink.
#include "ctx.cuh"

namespace seren {

namespace {

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

constexpr double SINK_PI = 3.1415926536;   // the reference's PI (headers/macros.h)

// gravity/gravity_gradh.F90:11-95, the potential only, with zeta/omega = 0, as
// accrete_particles.F90:186-188 calls it: the sink's 1/h is passed where the
// routine takes the second body's h (hq below is that value)
__device__ __forceinline__ double accrete_pot(double d0, double d1, double d2, double invhp,
                                              double hq, double mq,
                                              const double4* __restrict__ tabG) {
  const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
  const double drmag = sqrt(drsqd) + SMALL_NUMBER;
  const double invdrmag = 1.0 / drmag;
  double dpot;
  if (invdrmag > INVKERNRANGE * invhp) {
    int kern = (int)((HALFKERNTOT * drmag) * invhp);
    kern = max(0, min(kern, KERNTOT));
    dpot = invhp * tabG[kern].z;
  } else {
    dpot = invdrmag;
  }
  if (drmag < KERNRANGE * hq) {
    const double invhq = 1.0 / hq;
    int kern = (int)((HALFKERNTOT * drmag) * invhq);
    kern = max(0, min(kern, KERNTOT));
    dpot = dpot + invhq * tabG[kern].z;
  } else {
    dpot = dpot + invdrmag;
  }
  return (0.5 * mq) * dpot;
}

// accrete_particles.F90:82-106 (nearest accreting sink whose radius holds the
// particle; a later sink wins only when strictly nearer) and :165-205 (the
// energy test); dead[p] = that sink when the particle is accreted, else -1
__global__ void k_acc_flag(int n, int ns, int energy, const double4* __restrict__ pm,
                           const double2* __restrict__ hz, const double4* __restrict__ vel,
                           const double* __restrict__ sk, const double4* __restrict__ tabG,
                           int* __restrict__ dead, int* __restrict__ mark) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double4 P = pm[p];
  int flag = -1;
  double best = 0.0;
  for (int s = 0; s < ns; ++s) {
    const double* S = sk + (size_t)s * ACC_STRIDE;
    if (S[6] == 0.0) continue;
    const double d0 = P.x - S[0], d1 = P.y - S[1], d2 = P.z - S[2];
    const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
    const double rads = S[5];
    if (drsqd < rads * rads && (flag == -1 || drsqd < best)) {
      flag = s;
      best = drsqd;
    }
  }
  int d = -1;
  if (flag >= 0) {
    bool bound = true;
    if (energy) {
      const double* S = sk + (size_t)flag * ACC_STRIDE;
      const double ms = S[3];
      const double mp = P.w;
      const double invhp = 1.0 / hz[p].x;
      const double invhs = 1.0 / S[4];
      const double4 V = vel[p];
      const double e0 = S[7] - V.x, e1 = S[8] - V.y, e2 = S[9] - V.z;
      const double reduced_mass = (ms * mp) / (ms + mp);
      const double dpotp = accrete_pot(S[0] - P.x, S[1] - P.y, S[2] - P.z, invhp, invhs, ms, tabG);
      const double total_energy =
          ((0.5 * reduced_mass) * ((e0 * e0 + e1 * e1) + e2 * e2)) - dpotp * mp;
      bound = total_energy < 0.0;
    }
    if (bound) d = flag;
  }
  dead[p] = d;
  mark[p] = d >= 0 ? 1 : 0;
}

// the accreted particles in index order and the kept ones in index order
// (remove_from_list.F90:46-61); pos is the exclusive scan of the flags
__global__ void k_acc_lists(int n, const int* __restrict__ dead, const int* __restrict__ pos,
                            int* __restrict__ dlist, int* __restrict__ live) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  if (dead[p] >= 0)
    dlist[pos[p]] = p;
  else
    live[p - pos[p]] = p;
}

// accrete_particles.F90:128-281 for one sink per warp: the sums over its
// accreted particles in index order, the new centre of mass, velocity and
// acceleration, and the angular momentum about the new centre of mass of the
// old sink and of each accreted particle
__global__ void k_acc_sinks(int ns, const double* __restrict__ sk, const int* __restrict__ dlist,
                            int nd, const int* __restrict__ dead, const double4* __restrict__ pm,
                            const double4* __restrict__ vel, const double* __restrict__ acc,
                            double* __restrict__ out) {
  const int s = blockIdx.x;
  const int lane = threadIdx.x;
  if (s >= ns) return;
  const double* S = sk + (size_t)s * ACC_STRIDE;
  double* O = out + (size_t)s * ACC_STRIDE;
  if (S[6] == 0.0) {
    if (lane == 0) O[15] = 0.0;
    return;
  }
  const double ms = S[3];
  const double rs0 = S[0], rs1 = S[1], rs2 = S[2];
  const double vs0 = S[7], vs1 = S[8], vs2 = S[9];
  double mt = ms;
  double r0 = ms * rs0, r1 = ms * rs1, r2 = ms * rs2;
  double v0 = ms * vs0, v1 = ms * vs1, v2 = ms * vs2;
  double a0 = ms * S[10], a1 = ms * S[11], a2 = ms * S[12];
  int cnt = 0;
  for (int base = 0; base < nd; base += 32) {
    const int i = base + lane;
    const int p = i < nd ? dlist[i] : -1;
    unsigned m = __ballot_sync(0xffffffffu, p >= 0 && dead[p] == s);
    while (m) {
      const int j = __ffs(m) - 1;
      m &= m - 1;
      const int q = __shfl_sync(0xffffffffu, p, j);
      const double4 Q = pm[q];
      const double4 V = vel[q];
      const double* A = acc + 3 * (size_t)q;
      const double mp = Q.w;
      mt = mt + mp;
      r0 = r0 + mp * Q.x; r1 = r1 + mp * Q.y; r2 = r2 + mp * Q.z;
      v0 = v0 + mp * V.x; v1 = v1 + mp * V.y; v2 = v2 + mp * V.z;
      a0 = a0 + mp * A[0]; a1 = a1 + mp * A[1]; a2 = a2 + mp * A[2];
      ++cnt;
    }
  }
  double L0 = 0.0, L1 = 0.0, L2 = 0.0;
  if (cnt > 0) {
    r0 = r0 / mt; r1 = r1 / mt; r2 = r2 / mt;
    v0 = v0 / mt; v1 = v1 / mt; v2 = v2 / mt;
    a0 = a0 / mt; a1 = a1 / mt; a2 = a2 / mt;
    {
      // the old sink: dr = r_sink - r_com, dv = v_sink - v_com
      const double d0 = rs0 - r0, d1 = rs1 - r1, d2 = rs2 - r2;
      const double e0 = vs0 - v0, e1 = vs1 - v1, e2 = vs2 - v2;
      L0 = (L0 + (ms * d1) * e2) - (ms * d2) * e1;
      L1 = (L1 + (ms * d2) * e0) - (ms * d0) * e2;
      L2 = (L2 + (ms * d0) * e1) - (ms * d1) * e0;
    }
    for (int base = 0; base < nd; base += 32) {
      const int i = base + lane;
      const int p = i < nd ? dlist[i] : -1;
      unsigned m = __ballot_sync(0xffffffffu, p >= 0 && dead[p] == s);
      while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1;
        const int q = __shfl_sync(0xffffffffu, p, j);
        const double4 Q = pm[q];
        const double4 V = vel[q];
        const double mp = Q.w;
        // dr = r_com - r_p, dv = v_com - v_p
        const double d0 = r0 - Q.x, d1 = r1 - Q.y, d2 = r2 - Q.z;
        const double e0 = v0 - V.x, e1 = v1 - V.y, e2 = v2 - V.z;
        L0 = (L0 + (mp * d1) * e2) - (mp * d2) * e1;
        L1 = (L1 + (mp * d2) * e0) - (mp * d0) * e2;
        L2 = (L2 + (mp * d0) * e1) - (mp * d1) * e0;
      }
    }
  }
  if (lane == 0) {
    O[0] = mt;
    O[1] = r0; O[2] = r1; O[3] = r2;
    O[4] = v0; O[5] = v1; O[6] = v2;
    O[7] = a0; O[8] = a1; O[9] = a2;
    O[10] = L0; O[11] = L1; O[12] = L2;
    O[15] = (double)cnt;
  }
}

// remove_from_list.F90:46-62 with reorder_particle_arrays: every per-particle
// array gathered over the kept particles (the Runge-Kutta state when it exists)
__global__ void k_acc_compact(const int* __restrict__ live, int n, const double4* __restrict__ pm,
                              const double2* __restrict__ hz, const double4* __restrict__ vel,
                              const double* __restrict__ csq, const int* __restrict__ orig,
                              double4* __restrict__ pm2, double2* __restrict__ hz2,
                              double4* __restrict__ vel2, double* __restrict__ csq2,
                              int* __restrict__ orig2, const double* __restrict__ rho,
                              const double* __restrict__ omega, const double* __restrict__ divv,
                              const double* __restrict__ drdt, double* __restrict__ rho2,
                              double* __restrict__ omega2, double* __restrict__ divv2,
                              double* __restrict__ drdt2, const double* __restrict__ acc,
                              const double* __restrict__ gpot, double* __restrict__ acc2,
                              double* __restrict__ gpot2, const double4* __restrict__ ro,
                              const double4* __restrict__ vo, const double4* __restrict__ vh,
                              double4* __restrict__ ro2, double4* __restrict__ vo2,
                              double4* __restrict__ vh2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = live[i];
  pm2[i] = pm[p];
  hz2[i] = hz[p];
  vel2[i] = vel[p];
  csq2[i] = csq[p];
  orig2[i] = orig[p];
  rho2[i] = rho[p];
  omega2[i] = omega[p];
  divv2[i] = divv[p];
  drdt2[i] = drdt[p];
  acc2[3 * (size_t)i] = acc[3 * (size_t)p];
  acc2[3 * (size_t)i + 1] = acc[3 * (size_t)p + 1];
  acc2[3 * (size_t)i + 2] = acc[3 * (size_t)p + 2];
  gpot2[i] = gpot[p];
  if (ro) {
    ro2[i] = ro[p];
    vo2[i] = vo[p];
    vh2[i] = vh[p];
  }
}

// ---------------------------------------------------------------------------
// Sink search (sinks/sink_search.F90:25-433) and creation (sinks/create_sink.F90:11-268)

// BHtree/BHhydrowalk_hgather.F90:11-77: the depth-first walk over the cells
// whose hydro sphere (bbox centre, rmax) comes within hrange of r, calling f on
// every particle of each opened leaf.  The tree build numbers particles depth
// first, so f sees them in increasing index order, the order of the
// reference's potential-neighbour list.  At most 2 (ctot + 1) steps; more
// means broken links and sets the error flag.
template <class F>
__device__ void hgather_walk(double rx, double ry, double rz, double hrange, int ctot,
                             const int4* __restrict__ link, const double4* __restrict__ hA,
                             DevError* err, F&& f) {
  int c = 0;
  long steps = 0;
  const long cap = 2L * (ctot + 1) + 2;
  while (c >= 0 && c <= ctot) {
    if (++steps > cap) {
      set_error(err, SEREN_GPU_ERR_WALK, KID_SINK_SEARCH, c, ctot);
      return;
    }
    const double4 H = hA[c];
    const int4 L = link[c];                 // leaf, nextcell, ifopen, pstart
    const double d0 = H.x - rx, d1 = H.y - ry, d2 = H.z - rz;
    const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
    const double maxdistsqd = (hrange + H.w) * (hrange + H.w);
    if (drsqd <= maxdistsqd) {
      if (L.x > 0) {
        for (int i = 0; i < L.x; ++i) f(L.w + i);
        c = L.y;
      } else if (L.x == 0) {
        c = L.z;
      } else {
        c = L.y;
      }
    } else {
      c = L.y;
    }
  }
}

// candidates by density (sink_search.F90:106-131): flag[p] = 1 unless rho_search
// and rho < rhosink
__global__ void k_ss_mark(int n, int rho_search, double rhosink, const double* __restrict__ rho,
                          int* __restrict__ flag, int* __restrict__ mark) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int f = (rho_search && rho[p] < rhosink) ? 0 : 1;
  flag[p] = f;
  mark[p] = f;
}

__global__ void k_ss_list(int n, const int* __restrict__ flag, const int* __restrict__ pos,
                          int* __restrict__ list) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && flag[p]) list[pos[p]] = p;
}

// Every test of sink_search.F90 for one candidate per thread: the potential
// minimum (all_sph_gradh.F90:355-471 over the gather neighbours within 2h),
// the existing sinks (:155-200; the Hill test reads a_grav and the sinks'
// agrav, which only DEBUG_FORCES builds fill: zero, so it rejects nothing),
// the smoothed density, div v, div a and curl v over the neighbours within
// max(sinkrad, 2h) (:221-300, the reference's expressions in order; div a
// divides by the relative acceleration along the separation, as there), and
// the timescale test (:328-400).  entry[i]: the candidate is still flagged when
// the last of those loops reaches it (the loop that leaves psink = p); fin[i]:
// it passed every test.
__global__ void k_ss_test(int n1, const int* __restrict__ list, const double4* __restrict__ pm,
                          const double2* __restrict__ hz, const double4* __restrict__ vel,
                          const double* __restrict__ acc, const double* __restrict__ rho,
                          const double* __restrict__ gpot, int ctot,
                          const int4* __restrict__ link, const double4* __restrict__ hA,
                          const double4* __restrict__ tabA, const double4* __restrict__ tabG,
                          int nsink, const double* __restrict__ sk, SinkSearchArgs sa,
                          int* __restrict__ entry, int* __restrict__ fin, DevError* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n1) return;
  const int p = list[i];
  const double4 P = pm[p];
  const double hp = hz[p].x;
  if (sa.potmin_search) {
    const double invhp = 1.0 / hp;
    const double hrangesqd = (KERNRANGESQD * hp) * hp;
    double gpotmin = 0.0;
    hgather_walk(P.x, P.y, P.z, KERNRANGE * hp, ctot, link, hA, err, [&](int pp) {
      if (pp == p) return;
      const double4 Q = pm[pp];
      const double d0 = Q.x - P.x, d1 = Q.y - P.y, d2 = Q.z - P.z;
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      if (drsqd > hrangesqd) return;
      const double drmag = sqrt(drsqd) + SMALL_NUMBER;
      const int kern = (int)((HALFKERNTOT * drmag) * invhp);
      if (kern > KERNTOT) return;
      gpotmin = fmin(-gpot[pp], gpotmin);
    });
    if (!(gpotmin > -gpot[p])) {
      entry[i] = 0;
      fin[i] = 0;
      return;
    }
  }
  bool flag = true;
  if (nsink > 0) {
    const double rhop = rho[p];
    for (int s = 0; s < nsink; ++s) {
      const double* S = sk + (size_t)s * ACC_STRIDE;
      const double d0 = S[0] - P.x, d1 = S[1] - P.y, d2 = S[2] - P.z;
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      const double rr = 2.0 * S[5];
      if (drsqd < rr * rr) flag = false;
      if (sa.hill_sphere_search) {
        const double e0 = 0.0, e1 = 0.0, e2 = 0.0;        // sink agrav - particle a_grav
        const double dadr = (e0 * d0 + e1 * d1) + e2 * d2;
        const double rho_hill = -(3.0 * dadr) / ((4.0 * SINK_PI) * drsqd);
        if (rhop < 3.0 * rho_hill) flag = false;
      }
    }
  }
  bool at_last = flag;                                   // entering the hydro loop
  double div_v = 0.0;
  if (flag) {
    const double4 V = vel[p];
    const double ax = acc[3 * (size_t)p], ay = acc[3 * (size_t)p + 1], az = acc[3 * (size_t)p + 2];
    const double hrange = sa.hmult_sinkrad ? fmax(sa.sinkrad * hp, KERNRANGE * hp)
                                           : fmax(sa.sinkrad, KERNRANGE * hp);
    const double hrangesqd = hrange * hrange;
    const double invhp = KERNRANGE / hrange;
    const double hfactor = pow(invhp, NDIMPR);
    double rhotemp = (P.w * tabA[0].x) * hfactor;
    double dvp = 0.0, dap = 0.0, c0 = 0.0, c1 = 0.0, c2 = 0.0;
    hgather_walk(P.x, P.y, P.z, hrange, ctot, link, hA, err, [&](int pp) {
      if (pp == p) return;
      const double4 Q = pm[pp];
      const double d0 = Q.x - P.x, d1 = Q.y - P.y, d2 = Q.z - P.z;
      double drmag = (d0 * d0 + d1 * d1) + d2 * d2;
      if (drmag > hrangesqd) return;
      drmag = sqrt(drmag) + SMALL_NUMBER;
      const double invdrmag = 1.0 / drmag;
      const int kern = (int)((HALFKERNTOT * drmag) * invhp);
      if (kern > KERNTOT) return;
      const double mpp = Q.w;
      const double4 W = vel[pp];
      const double v0 = W.x - V.x, v1 = W.y - V.y, v2 = W.z - V.z;
      const double dvdr = (v0 * d0 + v1 * d1) + v2 * d2;
      const double4 TA = tabA[kern];                   // w0, wh, w4, wg
      const double w1 = tabG[kern].w;
      rhotemp = rhotemp + (mpp * hfactor) * TA.x;
      dvp = dvp - ((((mpp * dvdr) * TA.z) * hfactor) * invhp) * invdrmag;
      const double dadr = ((acc[3 * (size_t)pp] - ax) * d0 + (acc[3 * (size_t)pp + 1] - ay) * d1) +
                          (acc[3 * (size_t)pp + 2] - az) * d2;
      dap = dap - ((((mpp * TA.z) * hfactor) * invhp) / dadr) * invdrmag;
      const double x0 = v1 * d2 - v2 * d1, x1 = v2 * d0 - v0 * d2, x2 = v0 * d1 - v1 * d0;
      c0 = c0 - ((((mpp * x0) * invdrmag) * w1) * hfactor) * invhp;
      c1 = c1 - ((((mpp * x1) * invdrmag) * w1) * hfactor) * invhp;
      c2 = c2 - ((((mpp * x2) * invdrmag) * w1) * hfactor) * invhp;
    });
    div_v = dvp / rhotemp;
    const double div_a = dap / rhotemp;
    if (sa.div_a_search && div_a > 0.0) flag = false;
    if (sa.div_v_search && div_v > 0.0) flag = false;
  }
  if (nsink > 0) {
    at_last = flag;                                      // entering the timescale loop
    if (flag) {
      const double4 V = vel[p];
      for (int s = 0; s < nsink; ++s) {
        const double* S = sk + (size_t)s * ACC_STRIDE;
        const double d0 = S[0] - P.x, d1 = S[1] - P.y, d2 = S[2] - P.z;
        const double drmag = sqrt((d0 * d0 + d1 * d1) + d2 * d2) + SMALL_NUMBER;
        const double u0 = d0 / drmag, u1 = d1 / drmag, u2 = d2 / drmag;
        const double e0 = S[7] - V.x, e1 = S[8] - V.y, e2 = S[9] - V.z;
        const double drad = drmag - 2.0 * S[5];
        const double vrad = (e0 * u0 + e1 * u1) + e2 * u2;
        const double tacc1 = -drad / vrad;
        const double tcond1 = -1.0 / div_v;
        if (sa.timescale_search && tcond1 > tacc1) flag = false;
      }
    }
  }
  entry[i] = at_last ? 1 : 0;
  fin[i] = flag ? 1 : 0;
}

// sink_search.F90:405-423: the candidates were sorted by density (stable) and
// the last loop left p at the densest candidate it visited (ties: the highest
// index); a sink is made there when any candidate passed every test
__global__ void k_ss_select(int n1, const int* __restrict__ list, const double* __restrict__ rho,
                            const int* __restrict__ entry, const int* __restrict__ fin,
                            int* __restrict__ out) {
  __shared__ double br[1024];
  __shared__ int bp[1024];
  __shared__ int any;
  const int t = threadIdx.x;
  if (t == 0) any = 0;
  __syncthreads();
  double best = 0.0;
  int bestp = -1;
  int anyf = 0;
  for (int i = t; i < n1; i += blockDim.x) {
    anyf |= fin[i];
    if (!entry[i]) continue;
    const int p = list[i];
    const double r = rho[p];
    if (bestp < 0 || r > best || (r == best && p > bestp)) {
      best = r;
      bestp = p;
    }
  }
  if (anyf) atomicOr(&any, 1);
  br[t] = best;
  bp[t] = bestp;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (t < w) {
      const int q = bp[t + w];
      if (q >= 0 && (bp[t] < 0 || br[t + w] > br[t] || (br[t + w] == br[t] && q > bp[t]))) {
        br[t] = br[t + w];
        bp[t] = q;
      }
    }
    __syncthreads();
  }
  if (t == 0) out[0] = any ? bp[0] : -1;
}

// create_sink.F90:88 and sph/gather_neib_on_fly.F90: psink and the particles within the new sink's
// radius of it (gather_neib_on_fly with h = rads/2: within (2h)^2 inclusive)
__global__ void k_cs_mark(int n, int psink, double hrangesqd, const double4* __restrict__ pm,
                          int* __restrict__ dead, int* __restrict__ mark) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double4 S = pm[psink];
  const double4 Q = pm[p];
  const double d0 = Q.x - S.x, d1 = Q.y - S.y, d2 = Q.z - S.z;
  const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
  const int d = (p == psink || drsqd <= hrangesqd) ? 0 : -1;
  dead[p] = d;
  mark[p] = d >= 0 ? 1 : 0;
}

// create_sink.F90:64-150 in one warp: the new sink's mass, centre of mass,
// velocity and acceleration from psink then its neighbours in index order, and
// the angular momentum about the centre of mass; out = {m, x, y, z, vx, vy,
// vz, ax, ay, az, Lx, Ly, Lz}
__global__ void k_cs_sink(int psink, const int* __restrict__ dlist, int nd,
                          const double4* __restrict__ pm, const double4* __restrict__ vel,
                          const double* __restrict__ acc, double* __restrict__ out) {
  const int lane = threadIdx.x;
  const double4 P = pm[psink];
  const double4 V = vel[psink];
  const double mp = P.w;
  double ms = mp;
  double r0 = mp * P.x, r1 = mp * P.y, r2 = mp * P.z;
  double v0 = mp * V.x, v1 = mp * V.y, v2 = mp * V.z;
  double a0 = mp * acc[3 * (size_t)psink], a1 = mp * acc[3 * (size_t)psink + 1],
         a2 = mp * acc[3 * (size_t)psink + 2];
  for (int base = 0; base < nd; base += 32) {
    const int i = base + lane;
    const int q0 = i < nd ? dlist[i] : -1;
    unsigned m = __ballot_sync(0xffffffffu, q0 >= 0 && q0 != psink);
    while (m) {
      const int j = __ffs(m) - 1;
      m &= m - 1;
      const int q = __shfl_sync(0xffffffffu, q0, j);
      const double4 Q = pm[q];
      const double4 W = vel[q];
      const double* A = acc + 3 * (size_t)q;
      const double mq = Q.w;
      ms = ms + mq;
      r0 = r0 + mq * Q.x; r1 = r1 + mq * Q.y; r2 = r2 + mq * Q.z;
      v0 = v0 + mq * W.x; v1 = v1 + mq * W.y; v2 = v2 + mq * W.z;
      a0 = a0 + mq * A[0]; a1 = a1 + mq * A[1]; a2 = a2 + mq * A[2];
    }
  }
  r0 = r0 / ms; r1 = r1 / ms; r2 = r2 / ms;
  v0 = v0 / ms; v1 = v1 / ms; v2 = v2 / ms;
  a0 = a0 / ms; a1 = a1 / ms; a2 = a2 / ms;
  // psink: dr = r_sink - r_p, dv = v_sink - v_p
  double L0, L1, L2;
  {
    const double d0 = r0 - P.x, d1 = r1 - P.y, d2 = r2 - P.z;
    const double e0 = v0 - V.x, e1 = v1 - V.y, e2 = v2 - V.z;
    L0 = (mp * d1) * e2 - (mp * d2) * e1;
    L1 = (mp * d2) * e0 - (mp * d0) * e2;
    L2 = (mp * d0) * e1 - (mp * d1) * e0;
  }
  for (int base = 0; base < nd; base += 32) {
    const int i = base + lane;
    const int q0 = i < nd ? dlist[i] : -1;
    unsigned m = __ballot_sync(0xffffffffu, q0 >= 0 && q0 != psink);
    while (m) {
      const int j = __ffs(m) - 1;
      m &= m - 1;
      const int q = __shfl_sync(0xffffffffu, q0, j);
      const double4 Q = pm[q];
      const double4 W = vel[q];
      const double mq = Q.w;
      const double d0 = r0 - Q.x, d1 = r1 - Q.y, d2 = r2 - Q.z;
      const double e0 = v0 - W.x, e1 = v1 - W.y, e2 = v2 - W.z;
      L0 = (L0 + (mq * d1) * e2) - (mq * d2) * e1;
      L1 = (L1 + (mq * d2) * e0) - (mq * d0) * e2;
      L2 = (L2 + (mq * d0) * e1) - (mq * d1) * e0;
    }
  }
  if (lane == 0) {
    out[0] = ms;
    out[1] = r0; out[2] = r1; out[3] = r2;
    out[4] = v0; out[5] = v1; out[6] = v2;
    out[7] = a0; out[8] = a1; out[9] = a2;
    out[10] = L0; out[11] = L1; out[12] = L2;
  }
}

}  // namespace

// remove_from_list.F90:46-62 on the device: the kept particles (live, in
// index order) gathered into the spare buffers, which become the arrays; a and
// gpot go through the staging buffer
void remove_dead(Ctx& c, const int* live, int nlive) {
  const size_t P = (size_t)c.pmax;
  double* acc2 = c.stage;
  double* gpot2 = c.stage + 3 * P;
  if (nlive > 0) {
    k_acc_compact<<<nb(nlive, 256), 256, 0, c.st>>>(
        live, nlive, c.pm, c.hz, c.vel, c.csq, c.orig, c.pm_alt, c.hz_alt, c.vel_alt, c.csq_alt,
        c.orig_alt, c.rho, c.omega, c.div_v, c.drhodt, c.rho_alt, c.omega_alt, c.div_v_alt,
        c.drhodt_alt, c.acc, c.gpot, acc2, gpot2, c.r_old, c.v_old, c.v_half, c.r_old_alt,
        c.v_old_alt, c.v_half_alt); ++c.nlaunch;
    cudaMemcpyAsync(c.acc, acc2, sizeof(double) * 3 * (size_t)nlive, cudaMemcpyDeviceToDevice, c.st);
    cudaMemcpyAsync(c.gpot, gpot2, sizeof(double) * (size_t)nlive, cudaMemcpyDeviceToDevice, c.st);
  }
  std::swap(c.pm, c.pm_alt);
  std::swap(c.hz, c.hz_alt);
  std::swap(c.vel, c.vel_alt);
  std::swap(c.csq, c.csq_alt);
  std::swap(c.orig, c.orig_alt);
  std::swap(c.rho, c.rho_alt);
  std::swap(c.omega, c.omega_alt);
  std::swap(c.div_v, c.div_v_alt);
  std::swap(c.drhodt, c.drhodt_alt);
  if (c.r_old) {
    std::swap(c.r_old, c.r_old_alt);
    std::swap(c.v_old, c.v_old_alt);
    std::swap(c.v_half, c.v_half_alt);
  }
  c.ptot = nlive;
}

int launch_accrete(Ctx& c, int nsink, int energy, std::vector<double>& out, int& ndead) {
  const int n = c.ptot;
  const size_t P = (size_t)c.pmax;
  int* dead = c.acc_ws;
  int* mark = c.acc_ws + P;
  int* dlist = c.acc_ws + 2 * P;
  int* live = c.acc_ws + 3 * P;
  ndead = 0;
  k_acc_flag<<<nb(n, 256), 256, 0, c.st>>>(n, nsink, energy, c.pm, c.hz, c.vel, c.acc_sinks,
                                            c.tabG, dead, mark); ++c.nlaunch;
  scan_exclusive(c, mark, mark, n);
  int rc = read_dev(c, c.scan.total, &ndead, sizeof(int));
  if (rc) return rc;
  if (ndead <= 0) return SEREN_GPU_OK;
  k_acc_lists<<<nb(n, 256), 256, 0, c.st>>>(n, dead, mark, dlist, live); ++c.nlaunch;
  k_acc_sinks<<<nsink, 32, 0, c.st>>>(nsink, c.acc_sinks, dlist, ndead, dead, c.pm, c.vel, c.acc,
                                       c.acc_out); ++c.nlaunch;
  out.assign((size_t)nsink * ACC_STRIDE, 0.0);
  cudaMemcpyAsync(out.data(), c.acc_out, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, c.st);
  remove_dead(c, live, n - ndead);
  return SEREN_GPU_OK;
}

int launch_sink_search(Ctx& c, int nsink, const SinkSearchArgs& sa, int& psink, int& psink_id,
                       std::vector<double>& out, int& nremoved) {
  const int n = c.ptot;
  const size_t P = (size_t)c.pmax;
  int* flag = c.acc_ws;
  int* mark = c.acc_ws + P;
  int* list = c.acc_ws + 2 * P;
  int* live = c.acc_ws + 3 * P;
  psink = -1;
  nremoved = 0;
  k_ss_mark<<<nb(n, 256), 256, 0, c.st>>>(n, sa.rho_search, sa.rhosink, c.rho, flag, mark);
  ++c.nlaunch;
  scan_exclusive(c, mark, mark, n);
  int n1 = 0;
  int rc = read_dev(c, c.scan.total, &n1, sizeof(int));
  if (rc) return rc;
  if (n1 <= 0) return SEREN_GPU_OK;
  k_ss_list<<<nb(n, 256), 256, 0, c.st>>>(n, flag, mark, list); ++c.nlaunch;
  // per-candidate results in the first two scratch arrays (their flags are used up)
  int* entry = flag;
  int* fin = mark;
  k_ss_test<<<nb(n1, 64), 64, 0, c.st>>>(n1, list, c.pm, c.hz, c.vel, c.acc, c.rho, c.gpot,
                                          c.info.ctot, c.link, c.hA, c.tabA, c.tabG, nsink,
                                          c.acc_sinks, sa, entry, fin, c.d_err); ++c.nlaunch;
  k_ss_select<<<1, 1024, 0, c.st>>>(n1, list, c.rho, entry, fin, c.acc_ws + 4 * P); ++c.nlaunch;
  rc = read_dev(c, c.acc_ws + 4 * P, &psink, sizeof(int));
  if (rc) return rc;
  if (psink < 0) return SEREN_GPU_OK;
  // create_sink: psink and its neighbours within the sink radius leave
  rc = read_dev(c, c.orig + psink, &psink_id, sizeof(int));
  if (rc) return rc;
  double2 hzp{0.0, 0.0};
  if (sa.hmult_sinkrad && (rc = read_dev(c, c.hz + psink, &hzp, sizeof(double2)))) return rc;
  const double rads = sa.hmult_sinkrad ? sa.sinkrad * hzp.x : sa.sinkrad;
  const double hh = INVKERNRANGE * rads;
  int* dead = c.acc_ws;
  int* dlist = c.acc_ws + 2 * P;
  k_cs_mark<<<nb(n, 256), 256, 0, c.st>>>(n, psink, (KERNRANGESQD * hh) * hh, c.pm, dead, mark);
  ++c.nlaunch;
  scan_exclusive(c, mark, mark, n);
  rc = read_dev(c, c.scan.total, &nremoved, sizeof(int));
  if (rc) return rc;
  k_acc_lists<<<nb(n, 256), 256, 0, c.st>>>(n, dead, mark, dlist, live); ++c.nlaunch;
  k_cs_sink<<<1, 32, 0, c.st>>>(psink, dlist, nremoved, c.pm, c.vel, c.acc, c.acc_out);
  ++c.nlaunch;
  out.assign(ACC_STRIDE, 0.0);
  cudaMemcpyAsync(out.data(), c.acc_out, sizeof(double) * ACC_STRIDE, cudaMemcpyDeviceToHost, c.st);
  out[13] = rads;
  remove_dead(c, live, n - nremoved);
  return SEREN_GPU_OK;
}

}  // namespace seren
