// blockstep.cu - block timesteps of the device-resident step loop.
//
// The reference's main loop (sph_sim/sph_integrate.F90:27-136, RUNGE_KUTTA)
// with nlevels > 1: every call evaluates the forces of the accdo particles
// only, then sph_timesteps (sph_sim/sph_timesteps.F90:11-341) sets the
// timestep level of each particle that finished its step, resynchronising
// every nresync integer steps; check_neighbour_timesteps
// (timestep/check_neighbour_timesteps.F90:11-85) lets each active particle's
// level reach its neighbours; advance_runge_kutta (advance/
// advance_runge_kutta.F90:9-111) predicts every particle to the new integer
// time and flags those at their half or full step; reduce_timesteps
// (timestep/reduce_timesteps.F90) restarts, with IMMEDIATE_TIMESTEP_REDUCTION,
// the steps of particles whose neighbours moved to much shorter ones.
//
// The per-particle state (level, start of the current step, least neighbour
// level, accdo, last step length) lives on the device in tree order and is
// permuted at every build with a and gpot; the scalars (integer time n,
// nresync, level_max, level_step, the integer-step length) are the host's.
// Integer decisions use the reference's integer arithmetic; the level of a
// timestep is int(INVLOGETWO*log(dt_max/dt)) + 1 (:105, :169).
#include <cmath>
#include <cstring>
#include <utility>

#include "ctx.cuh"

namespace seren {

namespace {

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

constexpr double INVLOGETWO = 1.442695041;     // headers/macros.h:15
constexpr int TIMESTEP_LEVEL_DIFF_MAX = 2;     // headers/macros.h:185

__device__ __forceinline__ long long dt_level(double dt_max, double dt) {
  return (long long)(INVLOGETWO * log(dt_max / dt)) + 1ll;
}

// initialize_sph_variables_2.F90:72-73 and :157: the start of the first step
// is the state after the first evaluation; nobody is active
__global__ void k_blk_init(int n, const double4* __restrict__ pm, const double4* __restrict__ vel,
                           double4* __restrict__ r_old, double4* __restrict__ v_old,
                           double4* __restrict__ v_half, int* __restrict__ accdo,
                           long long* __restrict__ nlast, int* __restrict__ nlevel,
                           int* __restrict__ nminneib, double* __restrict__ laststep) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  r_old[i] = pm[i];
  v_old[i] = vel[i];
  v_half[i] = make_double4(0.0, 0.0, 0.0, 0.0);
  accdo[i] = 0;
  nlast[i] = 0;
  nlevel[i] = 0;
  nminneib[i] = 0;
  laststep[i] = 0.0;
}

__global__ void k_blk_reorder(const int* __restrict__ perm, int n, const int* __restrict__ nlevel,
                              const long long* __restrict__ nlast, const int* __restrict__ nmin,
                              const int* __restrict__ accdo, const double* __restrict__ last,
                              const double* __restrict__ acc, const double* __restrict__ gpot,
                              int* __restrict__ nlevel2, long long* __restrict__ nlast2,
                              int* __restrict__ nmin2, int* __restrict__ accdo2,
                              double* __restrict__ last2, double* __restrict__ acc2,
                              double* __restrict__ gpot2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  nlevel2[i] = nlevel[p];
  nlast2[i] = nlast[p];
  nmin2[i] = nmin[p];
  accdo2[i] = accdo[p];
  last2[i] = last[p];
  acc2[3 * i] = acc[3 * p];
  acc2[3 * i + 1] = acc[3 * p + 1];
  acc2[3 * i + 2] = acc[3 * p + 2];
  gpot2[i] = gpot[p];
}

// the active list in tree order: act[scan[i]] = i for accdo[i]
__global__ void k_blk_compact(int n, const int* __restrict__ accdo, const int* __restrict__ scan,
                              int* __restrict__ act) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && accdo[i]) act[scan[i]] = (int)i;
}

// timestep/timestep_size.F90:52-120 for every particle (as k_timestep in the
// C ABI) and their least, as the bit pattern of a positive double
__global__ void k_blk_dt(int n, const double2* __restrict__ hz, const double* __restrict__ acc,
                         const double* __restrict__ div_v, const double* __restrict__ sound,
                         double alpha, double beta, double courant_mult, double accel_mult,
                         double* __restrict__ dt_out, unsigned long long* __restrict__ dt_min) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double dt = 1.0e300;
  if (i < n) {
    const double a0 = acc[3 * i], a1 = acc[3 * i + 1], a2 = acc[3 * i + 2];
    const double hp = hz[i].x;
    const double dv = fabs(div_v[i]);
    const double vsignal = sound[i];
    const double amag = sqrt((a0 * a0 + a1 * a1) + a2 * a2);
    const double tacc = accel_mult * sqrt(hp / (amag + 1.0e-20));
    const double tcour = (courant_mult * hp) /
                         ((vsignal + hp * dv) + 0.6 * (alpha * vsignal + (beta * hp) * dv));
    dt = fmin(tacc, tcour);
    dt_out[i] = dt;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dt = fmin(dt, __shfl_xor_sync(0xffffffffu, dt, o));
  if ((threadIdx.x & 31) == 0) atomicMin(dt_min, (unsigned long long)__double_as_longlong(dt));
}

// sph_timesteps.F90:56-60, :100-110: resynchronisation, every particle's level
__global__ void k_blk_resync(int n, const double* __restrict__ dt, double dt_max, int level_max,
                             int check, int* __restrict__ nlevel, int* __restrict__ nminneib,
                             long long* __restrict__ nlast) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  nlast[i] = 0;
  long long level = dt_level(dt_max, dt[i]);
  level = level < level_max ? level : level_max;
  level = level > 0 ? level : 0;
  nlevel[i] = (int)level;
  if (check) nminneib[i] = (int)level;
}

// sph_timesteps.F90:161-183: the particles at the end of their step (n ==
// nlast) take a new level; red[0] counts them, red[1] the highest level of all
__global__ void k_blk_update(int n, long long nn, int level_step, double dt_max,
                             const double* __restrict__ dt, const long long* __restrict__ nlast,
                             int* __restrict__ nlevel, unsigned long long* __restrict__ red) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int lev = -1;
  bool upd = false;
  if (i < n) {
    lev = nlevel[i];
    if (nn == nlast[i]) {
      upd = true;
      const int last = lev;
      long long level = dt_level(dt_max, dt[i]);
      level = level > 0 ? level : 0;
      if (level < last && last > 1 && nn % (1ll << (level_step - (last - 1))) == 0)
        lev = last - 1;
      else if (level > last)
        lev = (int)level;
      else
        lev = last;
      nlevel[i] = lev;
    }
  }
  const unsigned cnt = __popc(__ballot_sync(0xffffffffu, upd));
  int m = lev;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) {
    if (cnt) atomicAdd(red, (unsigned long long)cnt);
    if (m >= 0) atomicMax(red + 1, (unsigned long long)m);
  }
}

// sph_timesteps.F90:236-249 (CHECK_NEIGHBOUR_TIMESTEPS, no sinks)
__global__ void k_blk_nminneib(int n, long long nn, int level_step, int level_max,
                               const long long* __restrict__ nlast, int* __restrict__ nlevel,
                               int* __restrict__ nminneib) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int mn = nminneib[i];
  mn = mn < level_max ? mn : level_max;
  const int lv = nlevel[i];
  if (mn - lv > TIMESTEP_LEVEL_DIFF_MAX && nlast[i] == nn &&
      nn % (1ll << (level_step - mn + TIMESTEP_LEVEL_DIFF_MAX)) == 0) {
    const int l = mn - TIMESTEP_LEVEL_DIFF_MAX;
    nlevel[i] = l < level_max ? l : level_max;
    mn = nlevel[i];
  } else if (nlast[i] == nn) {
    mn = lv;
  }
  nminneib[i] = mn;
}

// sph_timesteps.F90:259-273: integer times follow a change of level_max
__global__ void k_blk_rescale(int n, long long* __restrict__ nlast, int up, int shift) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long f = 1ll << shift;
  nlast[i] = up ? nlast[i] * f : nlast[i] / f;
}

// advance/advance_runge_kutta.F90:20-97 for every particle at integer time nn
__global__ void k_blk_advance(int n, long long nn, int level_step, double timestep,
                              double4* __restrict__ pm, double4* __restrict__ vel,
                              const double* __restrict__ acc, double4* __restrict__ r_old,
                              double4* __restrict__ v_old, double4* __restrict__ v_half,
                              const int* __restrict__ nlevel, long long* __restrict__ nlast,
                              int* __restrict__ accdo, double* __restrict__ laststep) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int act = 0;
  const long long dn = nn - nlast[i];
  const long long nfull = 1ll << (level_step - nlevel[i]);
  const long long nhalf = nfull / 2;
  const double dt = timestep * (double)dn;
  const double4 ro = r_old[i], vo = v_old[i];
  const double a0 = acc[3 * i], a1 = acc[3 * i + 1], a2 = acc[3 * i + 2];
  double4 rp, vp;
  if (dn <= nhalf) {                                                  // :38-54
    rp = make_double4(ro.x + vo.x * dt, ro.y + vo.y * dt, ro.z + vo.z * dt, 0.0);
    vp = make_double4(vo.x + a0 * dt, vo.y + a1 * dt, vo.z + a2 * dt, 0.0);
    if (dn == nhalf) {
      v_half[i] = vp;
      act = 1;
    }
  } else {                                                            // :58-67
    const double4 vh = v_half[i];
    rp = make_double4(ro.x + vh.x * dt, ro.y + vh.y * dt, ro.z + vh.z * dt, 0.0);
    vp = make_double4(vo.x + a0 * dt, vo.y + a1 * dt, vo.z + a2 * dt, 0.0);
  }
  rp.w = pm[i].w;                                                     // the mass stays
  pm[i] = rp;
  vel[i] = vp;
  if (dn == nfull) {                                                  // :86-97
    act = 1;
    nlast[i] = nn;
    laststep[i] = timestep * (double)nfull;
    r_old[i] = rp;
    v_old[i] = vp;
  }
  accdo[i] = act;
}

// timestep/reduce_timesteps.F90:20-40 with reduce_particle_timestep.F90:25-70
__global__ void k_blk_reduce(int n, long long nn, int level_step, int level_max, double timestep,
                             const double4* __restrict__ pm, const double4* __restrict__ vel,
                             double4* __restrict__ r_old, double4* __restrict__ v_old,
                             int* __restrict__ nlevel, long long* __restrict__ nlast,
                             int* __restrict__ nminneib, int* __restrict__ accdo,
                             double* __restrict__ laststep, DevError* err) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int mn = nminneib[i];
  if (mn > level_max) {                       // the reference stops here
    set_error(err, SEREN_GPU_ERR_STATE, KID_GRADH, (int)i, mn);
    return;
  }
  if (mn - nlevel[i] > TIMESTEP_LEVEL_DIFF_MAX && mn != -1 && nlast[i] != nn &&
      nn % (1ll << (level_step - mn + TIMESTEP_LEVEL_DIFF_MAX)) == 0) {
    const int lnew = mn - TIMESTEP_LEVEL_DIFF_MAX;
    r_old[i] = pm[i];
    v_old[i] = vel[i];
    laststep[i] = timestep * (double)(nn - nlast[i]);
    nlevel[i] = lnew;
    nlast[i] = nn;
    nminneib[i] = lnew;
    accdo[i] = 1;
  }
}

template <typename T>
int alloc_n(T*& p, size_t n) {
  if (p) return 0;
  if (cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    return -1;
  }
  return 0;
}

}  // namespace

int rk_alloc(Ctx& c) {
  if (c.r_old) return 0;
  const size_t P = (size_t)c.pmax;
  for (double4** p : {&c.r_old, &c.v_old, &c.v_half, &c.r_old_alt, &c.v_old_alt, &c.v_half_alt})
    if (cudaMalloc(p, sizeof(double4) * P) != cudaSuccess) {
      *p = nullptr;
      cudaGetLastError();
      for (double4** q : {&c.r_old, &c.v_old, &c.v_half, &c.r_old_alt, &c.v_old_alt, &c.v_half_alt})
        if (*q) {
          cudaFree(*q);
          *q = nullptr;
        }
      return -1;
    }
  return 0;
}

void block_free(Ctx& c) {
  BlockState& b = c.blk;
  void* ps[] = {b.nlevel, b.nlast, b.nminneib, b.accdo, b.laststep, b.nlevel_alt, b.nlast_alt,
                b.nminneib_alt, b.accdo_alt, b.laststep_alt, b.acc_alt, b.gpot_alt, b.dt, b.red};
  for (void* p : ps)
    if (p) cudaFree(p);
  b = BlockState{};
}

void reorder_block(Ctx& c) {
  BlockState& b = c.blk;
  const int n = c.ptot;
  k_blk_reorder<<<nb(n, 256), 256, 0, c.st>>>(c.idx, n, b.nlevel, b.nlast, b.nminneib, b.accdo,
                                               b.laststep, c.acc, c.gpot, b.nlevel_alt,
                                               b.nlast_alt, b.nminneib_alt, b.accdo_alt,
                                               b.laststep_alt, b.acc_alt, b.gpot_alt);
  ++c.nlaunch;
  std::swap(b.nlevel, b.nlevel_alt);
  std::swap(b.nlast, b.nlast_alt);
  std::swap(b.nminneib, b.nminneib_alt);
  std::swap(b.accdo, b.accdo_alt);
  std::swap(b.laststep, b.laststep_alt);
  std::swap(c.acc, b.acc_alt);
  std::swap(c.gpot, b.gpot_alt);
}

int block_active(Ctx& c, int& nact) {
  BlockState& b = c.blk;
  const int n = c.ptot;
  scan_exclusive(c, b.accdo, c.bscan, n);
  int* act = c.istage;
  k_blk_compact<<<nb(n, 256), 256, 0, c.st>>>(n, b.accdo, c.bscan, act);
  ++c.nlaunch;
  // the count: the exclusive scan's total
  int total = 0;
  if (read_dev(c, c.scan.total, &total, sizeof(int))) return SEREN_GPU_ERR_CUDA;
  nact = total;
  b.nactive = total;
  c.act = act;
  return SEREN_GPU_OK;
}

int block_start(Ctx& c) {
  BlockState& b = c.blk;
  const size_t P = (size_t)c.pmax;
  if (rk_alloc(c)) return SEREN_GPU_ERR_CUDA;
  int bad = 0;
  bad |= alloc_n(b.nlevel, P) | alloc_n(b.nlast, P) | alloc_n(b.nminneib, P) |
         alloc_n(b.accdo, P) | alloc_n(b.laststep, P);
  bad |= alloc_n(b.nlevel_alt, P) | alloc_n(b.nlast_alt, P) | alloc_n(b.nminneib_alt, P) |
         alloc_n(b.accdo_alt, P) | alloc_n(b.laststep_alt, P);
  bad |= alloc_n(b.acc_alt, 3 * P) | alloc_n(b.gpot_alt, P) | alloc_n(b.dt, P) |
         alloc_n(b.red, (size_t)4);
  if (bad) return SEREN_GPU_ERR_CUDA;
  const int n = c.ptot;
  k_blk_init<<<nb(n, 256), 256, 0, c.st>>>(n, c.pm, c.vel, c.r_old, c.v_old, c.v_half, b.accdo,
                                            b.nlast, b.nlevel, b.nminneib, b.laststep);
  ++c.nlaunch;
  b.on = true;
  b.n = b.nresync = b.nsteps = 0;                     // initialize_seren_variables_2.F90:60-61
  b.level_max = b.level_step = 0;
  b.timestep = b.dt_max = b.time = 0.0;
  b.nactive = 0;
  return SEREN_GPU_OK;
}

// sph_timesteps.F90:11-341 without sinks
static int block_timesteps(Ctx& c) {
  BlockState& b = c.blk;
  const int n = c.ptot;
  static const unsigned long long init[4] = {0x7ff0000000000000ull, 0ull, 0ull, 0ull};
  cudaMemcpyAsync(b.red, init, sizeof(init), cudaMemcpyHostToDevice, c.st);
  k_blk_dt<<<nb(n, 256), 256, 0, c.st>>>(n, c.hz, c.acc, c.div_v, c.sound, c.prm.alpha,
                                          2.0 * c.prm.alpha, b.courant, b.accel, b.dt, b.red);
  ++c.nlaunch;
  if (b.n == b.nresync) {                                              // :47-147
    b.n = 0;
    unsigned long long bits = 0;
    if (read_dev(c, b.red, &bits, sizeof(bits))) return SEREN_GPU_ERR_CUDA;
    double dt_min = 0.0;
    std::memcpy(&dt_min, &bits, sizeof(double));
    const int level_max = b.nlevels - 1;
    if (b.level_mode == 1) {                                           // :75-77
      const long long level = (long long)(INVLOGETWO * std::log(b.dt_fixed / dt_min)) + 1ll;
      dt_min = b.dt_fixed / std::pow(2.0, (double)level);
    } else if (b.level_mode == 2) {
      dt_min = b.dt_fixed / std::pow(2.0, (double)level_max);
    }
    const double dt_max = dt_min * std::pow(2.0, (double)level_max);
    k_blk_resync<<<nb(n, 256), 256, 0, c.st>>>(n, b.dt, dt_max, level_max, b.check_neib >= 1,
                                                b.nlevel, b.nminneib, b.nlast);
    ++c.nlaunch;
    b.level_max = level_max;
    b.dt_max = dt_max;
    b.level_step = level_max + 1;                                      // :130-139
    b.nresync = 1ll << b.level_step;
    b.timestep = dt_max / (double)b.nresync;
  } else {                                                             // :152-296
    const int level_old = b.level_max;
    k_blk_update<<<nb(n, 256), 256, 0, c.st>>>(n, b.n, b.level_step, b.dt_max, b.dt, b.nlast,
                                                b.nlevel, b.red + 1);
    ++c.nlaunch;
    unsigned long long r[2] = {0, 0};
    if (read_dev(c, b.red + 1, r, sizeof(r))) return SEREN_GPU_ERR_CUDA;
    if (r[0] > 0) {
      int level_max = (int)r[1];
      if (level_max <= level_old - 1 && level_old > 1 &&
          b.n % (1ll << (b.level_step - (level_old - 1))) == 0)
        level_max = level_old - 1;
      else if (level_max < level_old)
        level_max = level_old;
      if (b.check_neib >= 1) {
        k_blk_nminneib<<<nb(n, 256), 256, 0, c.st>>>(n, b.n, b.level_step, level_max, b.nlast,
                                                       b.nlevel, b.nminneib);
        ++c.nlaunch;
      }
      if (level_max != level_old) {
        const bool up = level_max > level_old;
        const int d = up ? level_max - level_old : level_old - level_max;
        k_blk_rescale<<<nb(n, 256), 256, 0, c.st>>>(n, b.nlast, up ? 1 : 0, d);
        ++c.nlaunch;
        if (up) {
          b.n *= (1ll << d);
          b.nresync *= (1ll << d);
        } else {
          b.n /= (1ll << d);
          b.nresync /= (1ll << d);
        }
      }
      b.level_max = level_max;
      b.level_step = level_max + 1;
      b.timestep = b.dt_max / (double)b.nresync;
    }
  }
  b.n += 1;                                                            // :333-336
  b.nsteps += 1;
  b.time += b.timestep;
  return SEREN_GPU_OK;
}

int block_after_forces(Ctx& c) {
  BlockState& b = c.blk;
  const int n = c.ptot;
  const int nact = b.nactive;
  int rc = block_timesteps(c);
  if (rc) return rc;
  if (b.check_neib >= 1 && nact > 0) launch_neib_levels(c, nact, b.nlevel, b.nminneib);
  k_blk_advance<<<nb(n, 256), 256, 0, c.st>>>(n, b.n, b.level_step, b.timestep, c.pm, c.vel,
                                               c.acc, c.r_old, c.v_old, c.v_half, b.nlevel,
                                               b.nlast, b.accdo, b.laststep);
  ++c.nlaunch;
  if (b.check_neib == 2) {
    k_blk_reduce<<<nb(n, 256), 256, 0, c.st>>>(n, b.n, b.level_step, b.level_max, b.timestep,
                                                c.pm, c.vel, c.r_old, c.v_old, b.nlevel, b.nlast,
                                                b.nminneib, b.accdo, b.laststep, c.d_err);
    ++c.nlaunch;
  }
  return SEREN_GPU_OK;
}

}  // namespace seren
