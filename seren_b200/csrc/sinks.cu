// Sink accretion on the device-resident particles: sinks/accrete_particles.F90:14-365
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

}  // namespace

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
  // the kept particles, gathered into the spare buffers; a and gpot through the staging buffer
  const int nlive = n - ndead;
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
  return SEREN_GPU_OK;
}

}  // namespace seren
