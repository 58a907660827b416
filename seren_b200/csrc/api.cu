// api.cu - the C ABI of include/seren_gpu.h: context management, host <->
// device transfers and the order of the stages inside each call, which
// follows the Fortran drivers the calls replace (sph_sim/sph_setup.F90:42-66,
// main/tree_update.F90:27-60, sph_sim/sph_update.F90:57-100,
// sph_sim/sph_hydro_forces.F90:41-85, sph_sim/sph_grav_forces.F90:94-157).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <map>
#include <mutex>
#include <tuple>
#include <array>
#include "ctx.cuh"

struct seren_gpu_ctx {
  seren::Ctx c;
};

namespace seren {
namespace {

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

int fail(Ctx& c, int code, const char* msg) {
  c.err = msg;
  return code;
}

int cuda_fail(Ctx& c, cudaError_t e, const char* where) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
  c.err = buf;
  return SEREN_GPU_ERR_CUDA;
}

// Wait for the stream, then turn a device error record into a status.
int finish(Ctx& c, const char* where) {
  cudaError_t e = cudaStreamSynchronize(c.st);
  if (e != cudaSuccess) return cuda_fail(c, e, where);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(c, e, where);
  DevError de;
  e = cudaMemcpy(&de, c.d_err, sizeof(DevError), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(c, e, where);
  if (de.code != 0) {
    char buf[256];
    static const char* kn[] = {"?", "bbox", "keys", "sort", "split", "emit", "reorder", "stock",
                               "hguess", "gradh", "hmax", "neib", "hydro", "grav", "grav_mixed",
                               "sink", "thermal"};
    const char* k = (de.where >= 0 && de.where <= 16) ? kn[de.where] : "?";
    const char* what = de.code == SEREN_GPU_ERR_NONFINITE ? "non-finite input"
                       : de.code == SEREN_GPU_ERR_WALK     ? "walk or search cap reached"
                       : de.code == SEREN_GPU_ERR_NEGATIVE_H ? "negative smoothing length"
                                                             : "device error";
    std::snprintf(buf, sizeof(buf), "%s: %s in kernel %s (index %d, aux %d)", where, what, k,
                  de.index, de.aux);
    c.err = buf;
    cudaMemset(c.d_err, 0, sizeof(DevError));
    return de.code;
  }
  return SEREN_GPU_OK;
}

template <class T>
int alloc(T*& p, size_t n) {
  return cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)) == cudaSuccess ? 0 : -1;
}

__global__ void k_unpack_v(const double* __restrict__ st, int n, double4* __restrict__ vel) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  vel[i] = make_double4(st[i * 3 + 0], st[i * 3 + 1], st[i * 3 + 2], 0.0);
}

__global__ void k_pack_v(double* __restrict__ st, int n, const double4* __restrict__ vel) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 v = vel[i];
  st[i * 3 + 0] = v.x; st[i * 3 + 1] = v.y; st[i * 3 + 2] = v.z;
}

__global__ void k_iota(int* __restrict__ a, int n) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = (int)i;
}

__global__ void k_set_h(const double* __restrict__ h, int n, double2* __restrict__ hz) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) hz[i].x = h[i];
}

__global__ void k_pack_hz(const double2* __restrict__ hz, int n, double* __restrict__ st) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  st[i * 2 + 0] = hz[i].x;
  st[i * 2 + 1] = hz[i].y;
}

__global__ void k_add_base(const int* __restrict__ src, int* __restrict__ dst, long n, int base) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[i] + base;
}

// independent FMA chains for the pipe-throughput microbenchmark
constexpr int FMA_CHAINS = 8;
template <typename T>
__global__ void k_fma_peak(T* out, int iters, T a, T b) {
  T x[FMA_CHAINS];
#pragma unroll
  for (int k = 0; k < FMA_CHAINS; ++k) x[k] = (T)(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < FMA_CHAINS; ++k) x[k] = fma(x[k], a, b);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < FMA_CHAINS; ++k) s += x[k];
  if (s == (T)-1.2345) out[0] = s;
}

// timestep/timestep_size.F90:52-120 (HYDRO, ARTIFICIAL_VISCOSITY, no internal
// energy): dt = min(accel_mult sqrt(h / (|a| + 1e-20)),
// courant_mult h / (c + h|div v| + 0.6 (alpha c + beta h|div v|))), and the
// least over the particles (positive doubles order as their bit patterns)
__global__ void k_timestep(int n, const double2* __restrict__ hz, const double* __restrict__ acc,
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

// advance/advance_runge_kutta.F90:40-72, one timestep level: the first half
// (dt = step/2) keeps r_old, v_old and v_half; the second (dt = step) uses them
__global__ void k_rk_half(int n, double4* __restrict__ pm, double4* __restrict__ vel,
                          const double* __restrict__ acc, double4* __restrict__ r_old,
                          double4* __restrict__ v_old, double4* __restrict__ v_half, double dt) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 r = pm[i], v = vel[i];
  r_old[i] = r;
  v_old[i] = v;
  const double4 rp = make_double4(r.x + v.x * dt, r.y + v.y * dt, r.z + v.z * dt, r.w);
  const double4 vp = make_double4(v.x + acc[3 * i] * dt, v.y + acc[3 * i + 1] * dt,
                                  v.z + acc[3 * i + 2] * dt, 0.0);
  pm[i] = rp;
  vel[i] = vp;
  v_half[i] = vp;
}

__global__ void k_rk_full(int n, double4* __restrict__ pm, double4* __restrict__ vel,
                          const double* __restrict__ acc, const double4* __restrict__ r_old,
                          const double4* __restrict__ v_old, const double4* __restrict__ v_half,
                          double dt) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 r = r_old[i], v = v_old[i], vh = v_half[i];
  pm[i] = make_double4(r.x + vh.x * dt, r.y + vh.y * dt, r.z + vh.z * dt, pm[i].w);
  vel[i] = make_double4(v.x + acc[3 * i] * dt, v.y + acc[3 * i + 1] * dt,
                        v.z + acc[3 * i + 2] * dt, 0.0);
}

__global__ void k_drift(int n, double4* __restrict__ pm, const double4* __restrict__ vel, double dt) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double4 p = pm[i];
  const double4 v = vel[i];
  p.x = p.x + v.x * dt;
  p.y = p.y + v.y * dt;
  p.z = p.z + v.z * dt;
  pm[i] = p;
}

// Active list: NULL means all particles (returns nact = ptot and c.act unset).
int set_active(Ctx& c, const int32_t* acclist, int32_t nacc, int& nact) {
  c.act = nullptr;
  if (acclist == nullptr) {
    nact = c.ptot;
    return SEREN_GPU_OK;
  }
  if (c.ncloud > 1) return fail(c, SEREN_GPU_ERR_ARG, "no active lists with several clouds");
  if (nacc < 0 || nacc > c.ptot) return fail(c, SEREN_GPU_ERR_ARG, "nacc out of range");
  std::vector<int> a(nacc);
  for (int i = 0; i < nacc; ++i) {
    a[i] = acclist[i] - c.prm.index_base;
    if (a[i] < 0 || a[i] >= c.ptot) return fail(c, SEREN_GPU_ERR_ARG, "acclist id out of range");
  }
  // the active buffer lives after the staging area
  int* d = c.istage;
  if (nacc > 0) cudaMemcpyAsync(d, a.data(), sizeof(int) * nacc, cudaMemcpyHostToDevice, c.st);
  c.act = d;
  nact = nacc;
  return SEREN_GPU_OK;
}

// host staging buffer (pinned), grown on demand
double* pinned(Ctx& c, size_t ndouble) {
  static_assert(sizeof(double) == 8, "");
  if (c.h_pin == nullptr) {
    if (cudaMallocHost(&c.h_pin, sizeof(double) * (size_t)c.pmax * 6) != cudaSuccess) {
      c.h_pin = nullptr;
      return nullptr;
    }
  }
  return ndouble <= (size_t)c.pmax * 6 ? c.h_pin : nullptr;
}

// copy rows of a device [ptot][w] double array to the host array, all rows
// when every particle is active, else only the active rows
int d2h_rows(Ctx& c, double* host, const double* dev, int w, const int32_t* acclist, int nact) {
  const size_t n = (size_t)c.ptot * w;
  if (acclist == nullptr) {
    cudaMemcpyAsync(host, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, c.st);
    return SEREN_GPU_OK;
  }
  double* pin = pinned(c, n);
  if (!pin) return fail(c, SEREN_GPU_ERR_CUDA, "pinned staging allocation failed");
  cudaMemcpyAsync(pin, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, c.st);
  cudaError_t e = cudaStreamSynchronize(c.st);
  if (e != cudaSuccess) return cuda_fail(c, e, "d2h_rows");
  for (int i = 0; i < nact; ++i) {
    const size_t p = (size_t)(acclist[i] - c.prm.index_base);
    for (int k = 0; k < w; ++k) host[p * w + k] = pin[p * w + k];
  }
  return SEREN_GPU_OK;
}

int check_tree(Ctx& c, int32_t ptot) {
  if (!c.have_tree) return fail(c, SEREN_GPU_ERR_STATE, "no tree: call seren_gpu_tree_update first");
  if (ptot != c.ptot) return fail(c, SEREN_GPU_ERR_STATE, "ptot differs from the last tree_update");
  return SEREN_GPU_OK;
}

void free_all(Ctx& c) {
  block_free(c);
  if (c.d_clouds) cudaFree(c.d_clouds);
  if (c.gact) cudaFree(c.gact);
  void* ps[] = {c.pm, c.hz, c.vel, c.csq, c.orig, c.pm_alt, c.hz_alt, c.vel_alt, c.csq_alt,
                c.orig_alt, c.rho, c.omega, c.div_v, c.drhodt, c.rho_alt, c.omega_alt, c.div_v_alt,
                c.drhodt_alt, c.press, c.sound, c.acc, c.gpot,
                c.pf, c.hf4,
                c.pptot, c.pplist, c.stage, c.istage, c.keys, c.keys_alt, c.keys_hi, c.keys_lo, c.idx, c.idx_alt,
                c.rs_hist, c.bbox_part, c.branch, c.branch_next, c.nchild, c.choff, c.cstart,
                c.bflag, c.bscan, c.leaf, c.nextcell, c.ifopen, c.pstart, c.pcount, c.parent,
                c.level, c.nkids, c.work, c.sinks, c.wstack, c.leaves, c.nleaf, c.npot, c.redo, c.wide, c.wst, c.wacc, c.link, c.gA, c.gB, c.gC, c.wA, c.hN, c.hA, c.hrm, c.hA32, c.hrm32, c.hmax, c.bbmin, c.bbmax, c.d_info,
                c.d_err, c.d_counts, c.sink_out, c.tabA, c.tabG, c.tabG32, c.scan.total, c.scan.level_buf[0],
                c.scan.level_buf[1], c.scan.level_buf[2], c.scan.level_buf[3]};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (c.h_pin) cudaFreeHost(c.h_pin);
  if (c.h_map) cudaFreeHost(c.h_map);
  if (c.stage_io) cudaFree(c.stage_io);
  if (c.wpart) cudaFree(c.wpart);
  if (c.wpart_brute) cudaFree(c.wpart_brute);
  if (c.wcover) cudaFree(c.wcover);
  if (c.hrec) cudaFree(c.hrec);
  for (double4* p : {c.r_old, c.v_old, c.v_half, c.r_old_alt, c.v_old_alt, c.v_half_alt})
    if (p) cudaFree(p);
  for (void* p : {(void*)c.acc_sinks, (void*)c.acc_out, (void*)c.acc_ws})
    if (p) cudaFree(p);
  for (auto& e : c.ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : c.ev_io)
    if (e) cudaEventDestroy(e);
  if (c.st_io) cudaStreamDestroy(c.st_io);
  if (c.st) cudaStreamDestroy(c.st);
}

int alloc_all(Ctx& c) {
  const size_t P = (size_t)c.pmax;
  const size_t C = (size_t)c.cmax + 1;
  const size_t L = (size_t)c.prm.pp_limit;
  const size_t nbr = P / 9 + 2;
  const size_t rsblk = (P + 4095) / 4096;
  int bad = 0;
  bad |= alloc(c.pm, P) | alloc(c.hz, P) | alloc(c.vel, P) | alloc(c.csq, P) | alloc(c.orig, P);
  bad |= alloc(c.pm_alt, P) | alloc(c.hz_alt, P) | alloc(c.vel_alt, P) | alloc(c.csq_alt, P) |
         alloc(c.orig_alt, P);
  bad |= alloc(c.rho_alt, P) | alloc(c.omega_alt, P) | alloc(c.div_v_alt, P) |
         alloc(c.drhodt_alt, P);
  bad |= alloc(c.rho, P) | alloc(c.omega, P) | alloc(c.div_v, P) | alloc(c.drhodt, P) |
         alloc(c.press, P) | alloc(c.sound, P) | alloc(c.acc, 3 * P) | alloc(c.gpot, P) |
         alloc(c.pf, P) | alloc(c.hf4, P);
  // stage: host-layout arrays and up to 1024 sinks; istage: active list + id arrays
  bad |= alloc(c.pptot, P) | alloc(c.pplist, P * L) | alloc(c.stage, std::max<size_t>(6 * P, 16384)) |
         alloc(c.istage, P * L + P);
  bad |= alloc(c.keys, P) | alloc(c.keys_alt, P) | alloc(c.keys_hi, P) | alloc(c.keys_lo, P) |
         alloc(c.idx, P) | alloc(c.idx_alt, P) |
         alloc(c.rs_hist, 256 * rsblk) | alloc(c.bbox_part, 6 * 1184);
  bad |= alloc(c.branch, nbr) | alloc(c.branch_next, nbr) | alloc(c.nchild, nbr) |
         alloc(c.choff, nbr) | alloc(c.cstart, 9 * nbr) | alloc(c.bflag, C) | alloc(c.bscan, C);
  bad |= alloc(c.leaf, C) | alloc(c.nextcell, C) | alloc(c.ifopen, C) | alloc(c.pstart, C) |
         alloc(c.pcount, C) | alloc(c.parent, C) | alloc(c.level, C) | alloc(c.link, C);
  bad |= alloc(c.hA32, C) | alloc(c.hrm32, C) | alloc(c.nkids, C) | alloc(c.work, 4);
  bad |= alloc(c.leaves, P * 256) | alloc(c.nleaf, P) | alloc(c.npot, P) | alloc(c.redo, P) | alloc(c.wide, P);
  bad |= wide_scratch_alloc(c);
  bad |= alloc(c.gA, C) | alloc(c.gB, C) | alloc(c.gC, C) | alloc(c.wA, 2 * C) | alloc(c.hN, 2 * C) |
         alloc(c.hA, C) | alloc(c.hrm, C) |
         alloc(c.hmax, C) | alloc(c.bbmin, C) | alloc(c.bbmax, C);
  bad |= alloc(c.d_info, 1) | alloc(c.d_err, 1) | alloc(c.d_counts, 32) | alloc(c.sinks, 5 * 1024) |
         alloc(c.sink_out, 4 * 1024);
  bad |= alloc(c.tabA, KERNTOT + 1) | alloc(c.tabG, KERNTOT + 1) | alloc(c.tabG32, KERNTOT + 1);
  c.wstack_slots = std::max(grav_walk_slots(c), hydro_walk_slots(c));
  c.wstack_cap = grav_walk_stack_cap(c);
  bad |= alloc(c.wstack, (size_t)c.wstack_slots * c.wstack_cap);
  if (bad) return -1;
  const size_t scan_n = std::max(std::max(256 * rsblk, C), P) + 16;
  if (scan_scratch_alloc(c.scan, (int)scan_n)) return -1;
  cudaMemset(c.d_err, 0, sizeof(DevError));
  cudaMemset(c.d_counts, 0, sizeof(int) * 32);
  cudaMemset(c.hrm, 0, sizeof(double) * C);
  cudaMemset(c.hrm32, 0, sizeof(float) * C);
  for (auto& e : c.ev)
    if (cudaEventCreate(&e) != cudaSuccess) return -1;
  // kernel tables
  std::vector<double> w0, w1, w4, w5, w6, wh, wg;
  make_kernel_tables(c.prm.kernel, w0, w1, w4, w5, w6, wh, wg);
  std::vector<double4> ta(KERNTOT + 1), tg(KERNTOT + 1);
  for (int i = 0; i <= KERNTOT; ++i) {
    ta[i] = make_double4(w0[i], wh[i], w4[i], wg[i]);
    tg[i] = make_double4(w5[i], w4[i], w6[i], w1[i]);
  }
  if (cudaMemcpy(c.tabA, ta.data(), sizeof(double4) * ta.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return -1;
  if (cudaMemcpy(c.tabG, tg.data(), sizeof(double4) * tg.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return -1;
  std::vector<float4> t32(KERNTOT + 1);
  for (int i = 0; i <= KERNTOT; ++i)
    t32[i] = make_float4((float)w5[i], (float)w4[i], (float)w6[i], 0.0f);
  if (cudaMemcpy(c.tabG32, t32.data(), sizeof(float4) * t32.size(), cudaMemcpyHostToDevice) !=
      cudaSuccess)
    return -1;
  return 0;
}

// new particle set: identity order, clear per-particle state
void reset_particles(Ctx& c, int ptot) {
  c.ptot = ptot;
  c.blk.on = false;                          // block timesteps start again after a new upload
  c.ncloud = 1;                              // and the particles are one cloud again
  c.have_tree = c.have_sph = c.have_v = c.have_csq = false;
  k_iota<<<nb(ptot, 256), 256, 0, c.st>>>(c.orig, ptot); ++c.nlaunch;
  cudaMemsetAsync(c.vel, 0, sizeof(double4) * ptot, c.st);
  cudaMemsetAsync(c.csq, 0, sizeof(double) * ptot, c.st);
  cudaMemsetAsync(c.pptot, 0, sizeof(int) * ptot, c.st);
}

// the device address of a host buffer that is page-locked and mapped (as
// pinned allocations are under unified addressing), else nullptr
double* mapped_host(double* p) {
  if (!p) return nullptr;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return at.type == cudaMemoryTypeHost ? static_cast<double*>(at.devicePointer) : nullptr;
}

int io_init(Ctx& c) {
  if (c.st_io) return 0;
  if (cudaStreamCreateWithFlags(&c.st_io, cudaStreamNonBlocking) != cudaSuccess) {
    c.st_io = nullptr;
    return -1;
  }
  for (auto& e : c.ev_io)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return -1;
  if (cudaMalloc(&c.stage_io, sizeof(double) * 6 * (size_t)c.pmax) != cudaSuccess) {
    c.stage_io = nullptr;
    return -1;
  }
  return 0;
}

}  // namespace
}  // namespace seren

using seren::Ctx;
using seren::fail;
using seren::finish;
using seren::nb;

extern "C" {

int seren_gpu_create(seren_gpu_ctx** out, int64_t pmax, const seren_gpu_params* prm) {
  if (!out || !prm) return SEREN_GPU_ERR_ARG;
  *out = nullptr;
  if (pmax < 1 || pmax > (int64_t)1 << 28) return SEREN_GPU_ERR_ARG;
  if (prm->ndim != 3 || prm->leafmax != seren::LEAFMAX || prm->lmax < 1 || prm->lmax > 30 ||
      (prm->kernel != 0 && prm->kernel != 1) || prm->visc != 0 ||
      (prm->precision != 0 && prm->precision != 1) || prm->pp_gather < 1 || prm->pp_limit < 1 ||
      (prm->index_base != 0 && prm->index_base != 1) || !(prm->h_fac > 0.0) ||
      !(prm->thetamaxsqd >= 0.0))
    return SEREN_GPU_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return SEREN_GPU_ERR_CUDA;
  seren_gpu_ctx* h = new seren_gpu_ctx();
  Ctx& c = h->c;
  c.prm = *prm;
  c.pmax = pmax;
  c.cmax = (int)(2 * pmax);
  cudaGetDevice(&c.dev);
  if (cudaStreamCreateWithFlags(&c.st, cudaStreamNonBlocking) != cudaSuccess || seren::alloc_all(c)) {
    seren::free_all(c);
    delete h;
    cudaGetLastError();
    return SEREN_GPU_ERR_CUDA;
  }
  *out = h;
  return SEREN_GPU_OK;
}

void seren_gpu_destroy(seren_gpu_ctx* h) {
  if (!h) return;
  cudaStreamSynchronize(h->c.st);
  if (h->c.st_io) cudaStreamSynchronize(h->c.st_io);
  seren::free_all(h->c);
  delete h;
}

int seren_gpu_last_error(seren_gpu_ctx* h, char* buf, int32_t len) {
  if (!h || !buf || len <= 0) return SEREN_GPU_ERR_ARG;
  std::snprintf(buf, (size_t)len, "%s", h->c.err.c_str());
  return SEREN_GPU_OK;
}

int seren_gpu_tree_update(seren_gpu_ctx* h, int32_t ptot, double* parray, int32_t do_build,
                          int32_t do_reorder, int32_t* perm_out) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!parray || ptot < 1) return fail(c, SEREN_GPU_ERR_ARG, "parray NULL or ptot < 1");
  if (ptot > c.pmax) return fail(c, SEREN_GPU_ERR_CAPACITY, "ptot > pmax");
  if (!do_build && (!c.have_tree || ptot != c.ptot))
    return fail(c, SEREN_GPU_ERR_STATE, "restock without a tree of this size");
  if (do_build && !do_reorder)
    return fail(c, SEREN_GPU_ERR_ARG, "a build requires the particle reorder (REORDER=PARTICLES)");
  if (ptot != c.ptot) seren::reset_particles(c, ptot);
  else if (do_build) {
    seren::k_iota<<<nb(ptot, 256), 256, 0, c.st>>>(c.orig, ptot);
    ++c.nlaunch;
  }
  cudaMemcpyAsync(c.stage, parray, sizeof(double) * 6 * (size_t)ptot, cudaMemcpyHostToDevice, c.st);
  seren::launch_unpack_parray(c, c.stage, ptot);
  int rc = finish(c, "tree_update(upload)");
  if (rc) return rc;
  if (do_build) {
    rc = seren::build_tree(c);
    if (rc) return rc;
  }
  seren::launch_stock(c);
  if (do_build) {
    seren::launch_pack_parray(c, c.stage, ptot);
    cudaMemcpyAsync(parray, c.stage, sizeof(double) * 6 * (size_t)ptot, cudaMemcpyDeviceToHost, c.st);
  }
  if (perm_out) {
    if (do_build)
      cudaMemcpyAsync(perm_out, c.idx, sizeof(int) * ptot, cudaMemcpyDeviceToHost, c.st);
  }
  rc = finish(c, "tree_update");
  if (rc) return rc;
  if (perm_out) {
    if (do_build) {
      if (c.prm.index_base)
        for (int i = 0; i < ptot; ++i) perm_out[i] += c.prm.index_base;
    } else {
      for (int i = 0; i < ptot; ++i) perm_out[i] = i + c.prm.index_base;
    }
  }
  return SEREN_GPU_OK;
}

int seren_gpu_sph_update(seren_gpu_ctx* h, int32_t ptot, const int32_t* acclist, int32_t nacc,
                         double* parray, const double* v, double* rho, double* omega,
                         double* div_v, double* drhodt, int32_t* pptot, int32_t* pplist,
                         int32_t first_call) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  int rc = seren::check_tree(c, ptot);
  if (rc) return rc;
  if (!v) return fail(c, SEREN_GPU_ERR_ARG, "v is NULL");
  const size_t N = (size_t)ptot;
  // every particle active: v comes in on the copy stream while the grad-h
  // walk runs (its passes wait for it), and the results of grad-h go back on
  // it while the neighbour lists are built
  const bool overlap = acclist == nullptr && seren::io_init(c) == 0;
  cudaGetLastError();
  if (overlap) {
    cudaEventRecord(c.ev_io[0], c.st);
    cudaStreamWaitEvent(c.st_io, c.ev_io[0], 0);
    cudaMemcpyAsync(c.stage_io, v, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, c.st_io);
    seren::k_unpack_v<<<nb(ptot, 256), 256, 0, c.st_io>>>(c.stage_io, ptot, c.vel); ++c.nlaunch;
    cudaEventRecord(c.ev_io[1], c.st_io);
    c.vel_wait = c.ev_io[1];
  } else {
    cudaMemcpyAsync(c.stage, v, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, c.st);
    seren::k_unpack_v<<<nb(ptot, 256), 256, 0, c.st>>>(c.stage, ptot, c.vel); ++c.nlaunch;
  }
  c.have_v = true;
  auto drain = [&](int code) {                // no copy left in flight on an error
    if (overlap) cudaStreamSynchronize(c.st_io);
    c.vel_wait = nullptr;
    return code;
  };
  int nact = 0;
  rc = seren::set_active(c, acclist, nacc, nact);
  if (rc) return drain(rc);
  if (first_call) seren::launch_hguess(c);
  seren::launch_gradh(c, nact);
  seren::finish_reorder(c);
  if (overlap) {
    cudaEventRecord(c.ev_io[2], c.st);
    cudaStreamWaitEvent(c.st_io, c.ev_io[2], 0);
    if (parray) {
      // every row changes: copy whole rows (positions and masses are the ones
      // uploaded by the last tree_update) instead of scattering two columns
      seren::launch_pack_parray(c, c.stage_io, ptot, c.st_io);
      cudaMemcpyAsync(parray, c.stage_io, sizeof(double) * 6 * N, cudaMemcpyDeviceToHost, c.st_io);
    }
    if (rho) cudaMemcpyAsync(rho, c.rho, sizeof(double) * N, cudaMemcpyDeviceToHost, c.st_io);
    if (omega) cudaMemcpyAsync(omega, c.omega, sizeof(double) * N, cudaMemcpyDeviceToHost, c.st_io);
    if (div_v) cudaMemcpyAsync(div_v, c.div_v, sizeof(double) * N, cudaMemcpyDeviceToHost, c.st_io);
    if (drhodt)
      cudaMemcpyAsync(drhodt, c.drhodt, sizeof(double) * N, cudaMemcpyDeviceToHost, c.st_io);
  }
  seren::launch_update_hmax(c);
  seren::launch_neib(c, nact, pplist != nullptr);  // the reference's order when the caller reads them
  rc = finish(c, "sph_update");
  if (rc) return drain(rc);
  if (overlap) {
    const cudaError_t e = cudaStreamSynchronize(c.st_io);
    if (e != cudaSuccess) return seren::cuda_fail(c, e, "sph_update(copies)");
  }
  c.have_sph = true;
  // results back to the host arrays (the overlapped path has sent them)
  if (overlap) {
  } else if (parray && acclist == nullptr) {
    seren::launch_pack_parray(c, c.stage, ptot);
    cudaMemcpyAsync(parray, c.stage, sizeof(double) * 6 * N, cudaMemcpyDeviceToHost, c.st);
  } else if (parray) {
    double* pin = seren::pinned(c, (size_t)2 * ptot);
    if (!pin) return fail(c, SEREN_GPU_ERR_CUDA, "pinned staging allocation failed");
    seren::k_pack_hz<<<nb(ptot, 256), 256, 0, c.st>>>(c.hz, ptot, c.stage); ++c.nlaunch;
    cudaMemcpyAsync(pin, c.stage, sizeof(double) * 2 * (size_t)ptot, cudaMemcpyDeviceToHost, c.st);
    cudaError_t e = cudaStreamSynchronize(c.st);
    if (e != cudaSuccess) return seren::cuda_fail(c, e, "sph_update(h)");
    if (acclist == nullptr || first_call) {
      for (int p = 0; p < ptot; ++p) parray[(size_t)p * 6 + 4] = pin[(size_t)p * 2];
    }
    const int na = acclist ? nact : ptot;
    for (int i = 0; i < na; ++i) {
      const size_t p = acclist ? (size_t)(acclist[i] - c.prm.index_base) : (size_t)i;
      parray[p * 6 + 4] = pin[p * 2];
      parray[p * 6 + 5] = pin[p * 2 + 1];
    }
  }
  if (!overlap) {
    if (rho && (rc = seren::d2h_rows(c, rho, c.rho, 1, acclist, nact))) return rc;
    if (omega && (rc = seren::d2h_rows(c, omega, c.omega, 1, acclist, nact))) return rc;
    if (div_v && (rc = seren::d2h_rows(c, div_v, c.div_v, 1, acclist, nact))) return rc;
    if (drhodt && (rc = seren::d2h_rows(c, drhodt, c.drhodt, 1, acclist, nact))) return rc;
  }
  if (pptot || pplist) {
    const int L = c.prm.pp_limit;
    std::vector<int> tot(ptot);
    cudaMemcpyAsync(tot.data(), c.pptot, sizeof(int) * ptot, cudaMemcpyDeviceToHost, c.st);
    cudaStreamSynchronize(c.st);
    if (pptot) {
      if (!acclist) std::memcpy(pptot, tot.data(), sizeof(int) * ptot);
      else
        for (int i = 0; i < nact; ++i) {
          const int p = acclist[i] - c.prm.index_base;
          pptot[p] = tot[p];
        }
    }
    if (pplist) {
      int* src = c.pplist;
      if (c.prm.index_base) {
        const long n = (long)ptot * L;
        seren::k_add_base<<<nb(n, 256), 256, 0, c.st>>>(c.pplist, c.istage + ptot, n, c.prm.index_base); ++c.nlaunch;
        src = c.istage + ptot;
      }
      if (!acclist) {
        cudaMemcpyAsync(pplist, src, sizeof(int) * (size_t)ptot * L, cudaMemcpyDeviceToHost, c.st);
      } else {
        for (int i = 0; i < nact; ++i) {
          const int p = acclist[i] - c.prm.index_base;
          if (tot[p] <= L)
            cudaMemcpyAsync(pplist + (size_t)p * L, src + (size_t)p * L, sizeof(int) * tot[p],
                            cudaMemcpyDeviceToHost, c.st);
        }
      }
    }
  }
  return finish(c, "sph_update(copy back)");
}

int seren_gpu_get_neib(seren_gpu_ctx* h, int32_t ptot, const int32_t* acclist, int32_t nacc,
                       const double* hh, int32_t* pptot, int32_t* pplist) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  int rc = seren::check_tree(c, ptot);
  if (rc) return rc;
  if (hh) {
    cudaMemcpyAsync(c.stage, hh, sizeof(double) * (size_t)ptot, cudaMemcpyHostToDevice, c.st);
    seren::k_set_h<<<nb(ptot, 256), 256, 0, c.st>>>(c.stage, ptot, c.hz); ++c.nlaunch;
  }
  int nact = 0;
  rc = seren::set_active(c, acclist, nacc, nact);
  if (rc) return rc;
  seren::launch_update_hmax(c);
  seren::launch_neib(c, nact);
  rc = finish(c, "get_neib");
  if (rc) return rc;
  const int L = c.prm.pp_limit;
  std::vector<int> tot(ptot);
  cudaMemcpy(tot.data(), c.pptot, sizeof(int) * ptot, cudaMemcpyDeviceToHost);
  std::vector<int> lst;
  if (pplist) {
    lst.resize((size_t)ptot * L);
    cudaMemcpy(lst.data(), c.pplist, sizeof(int) * lst.size(), cudaMemcpyDeviceToHost);
  }
  const int na = acclist ? nact : ptot;
  for (int i = 0; i < na; ++i) {
    const int p = acclist ? acclist[i] - c.prm.index_base : i;
    if (pptot) pptot[p] = tot[p];
    if (pplist && tot[p] <= L)
      for (int k = 0; k < tot[p]; ++k) pplist[(size_t)p * L + k] = lst[(size_t)p * L + k] + c.prm.index_base;
  }
  return SEREN_GPU_OK;
}

int seren_gpu_h_gather(seren_gpu_ctx* h, int32_t ptot, const int32_t* acclist, int32_t nacc,
                       double* parray) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!parray) return fail(c, SEREN_GPU_ERR_ARG, "parray is NULL");
  int rc = seren::check_tree(c, ptot);
  if (rc) return rc;
  int nact = 0;
  rc = seren::set_active(c, acclist, nacc, nact);
  if (rc) return rc;
  seren::launch_hgather(c, nact);
  seren::launch_update_hmax(c);            // sph_sim/sph_update.F90:121-124
  rc = finish(c, "h_gather");
  if (rc) return rc;
  // the new h of the active rows (hz = (h, zeta) per particle, tree order)
  std::vector<double> hzh((size_t)ptot * 2);
  cudaError_t e = cudaMemcpy(hzh.data(), c.hz, sizeof(double) * hzh.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return seren::cuda_fail(c, e, "h_gather");
  const int na = acclist ? nact : ptot;
  for (int i = 0; i < na; ++i) {
    const int p = acclist ? acclist[i] - c.prm.index_base : i;
    parray[(size_t)p * 6 + 4] = hzh[(size_t)p * 2];
  }
  return SEREN_GPU_OK;
}

int seren_gpu_hydro_forces(seren_gpu_ctx* h, const int32_t* acclist, int32_t nacc,
                           const double* press, const double* sound, double* a) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!c.have_sph || !c.have_tree)
    return fail(c, SEREN_GPU_ERR_STATE, "call seren_gpu_sph_update first");
  if (!press || !sound || !a) return fail(c, SEREN_GPU_ERR_ARG, "NULL array");
  const int ptot = c.ptot;
  cudaMemcpyAsync(c.press, press, sizeof(double) * ptot, cudaMemcpyHostToDevice, c.st);
  cudaMemcpyAsync(c.sound, sound, sizeof(double) * ptot, cudaMemcpyHostToDevice, c.st);
  int nact = 0;
  int rc = seren::set_active(c, acclist, nacc, nact);
  if (rc) return rc;
  // every particle active and a page-locked: the kernel writes a straight to it
  double* amap = acclist == nullptr ? seren::mapped_host(a) : nullptr;
  seren::launch_hydro(c, nact, amap);
  rc = finish(c, "hydro_forces");
  if (rc || amap) return rc;
  if ((rc = seren::d2h_rows(c, a, c.acc, 3, acclist, nact))) return rc;
  return finish(c, "hydro_forces(copy back)");
}

int seren_gpu_grav_forces(seren_gpu_ctx* h, const int32_t* acclist, int32_t nacc, double* a,
                          double* gpot, int32_t nsink, const double* sink_rmh) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!c.have_tree || c.ptot < 1) return fail(c, SEREN_GPU_ERR_STATE, "no tree");
  if (!a || !gpot || nsink < 0 || (nsink > 0 && !sink_rmh))
    return fail(c, SEREN_GPU_ERR_ARG, "bad arguments");
  if (nsink > 1024) return fail(c, SEREN_GPU_ERR_ARG, "nsink > 1024");
  const int ptot = c.ptot;
  // every particle active and a, gpot page-locked: the kernel reads the
  // acceleration to add to from a and writes a and gpot straight back
  double* amap = acclist == nullptr ? seren::mapped_host(a) : nullptr;
  double* gmap = amap ? seren::mapped_host(gpot) : nullptr;
  if (!gmap) amap = nullptr;
  if (!amap)
    cudaMemcpyAsync(c.acc, a, sizeof(double) * 3 * (size_t)ptot, cudaMemcpyHostToDevice, c.st);
  double* d_sinks = c.stage;
  if (nsink > 0)
    cudaMemcpyAsync(d_sinks, sink_rmh, sizeof(double) * 5 * nsink, cudaMemcpyHostToDevice, c.st);
  int nact = 0;
  int rc = seren::set_active(c, acclist, nacc, nact);
  if (rc) return rc;
  cudaMemsetAsync(c.d_counts, 0, sizeof(int) * 32, c.st);
  seren::launch_grav(c, nact, nsink, d_sinks, amap, gmap, amap);
  rc = finish(c, "grav_forces");
  if (rc || amap) return rc;
  if ((rc = seren::d2h_rows(c, a, c.acc, 3, acclist, nact))) return rc;
  if ((rc = seren::d2h_rows(c, gpot, c.gpot, 1, acclist, nact))) return rc;
  return finish(c, "grav_forces(copy back)");
}

int seren_gpu_sink_forces(seren_gpu_ctx* h, int32_t nsink, const double* sink_rmh, double* sink_a,
                          double* sink_gpot) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!c.have_tree) return fail(c, SEREN_GPU_ERR_STATE, "no tree");
  if (nsink < 1 || nsink > 1024 || !sink_rmh || !sink_a || !sink_gpot)
    return fail(c, SEREN_GPU_ERR_ARG, "bad arguments");
  double* d_sinks = c.stage;
  double* d_out = c.stage + 5 * 1024;
  cudaMemcpyAsync(d_sinks, sink_rmh, sizeof(double) * 5 * nsink, cudaMemcpyHostToDevice, c.st);
  seren::launch_sink_walk(c, nsink, d_sinks, d_out);
  std::vector<double> out((size_t)nsink * 4);
  cudaMemcpyAsync(out.data(), d_out, sizeof(double) * 4 * nsink, cudaMemcpyDeviceToHost, c.st);
  int rc = finish(c, "sink_forces");
  if (rc) return rc;
  for (int s = 0; s < nsink; ++s) {
    for (int k = 0; k < 3; ++k) sink_a[s * 3 + k] = out[s * 4 + k];
    sink_gpot[s] = out[s * 4 + 3];
  }
  return SEREN_GPU_OK;
}

int seren_gpu_upload(seren_gpu_ctx* h, int32_t ptot, const double* parray, const double* v,
                     const double* csq) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!parray || !v || !csq || ptot < 1) return fail(c, SEREN_GPU_ERR_ARG, "NULL array or ptot < 1");
  if (ptot > c.pmax) return fail(c, SEREN_GPU_ERR_CAPACITY, "ptot > pmax");
  seren::reset_particles(c, ptot);
  cudaMemcpyAsync(c.stage, parray, sizeof(double) * 6 * (size_t)ptot, cudaMemcpyHostToDevice, c.st);
  seren::launch_unpack_parray(c, c.stage, ptot);
  int rc = finish(c, "upload(parray)");
  if (rc) return rc;
  cudaMemcpyAsync(c.stage, v, sizeof(double) * 3 * (size_t)ptot, cudaMemcpyHostToDevice, c.st);
  seren::k_unpack_v<<<nb(ptot, 256), 256, 0, c.st>>>(c.stage, ptot, c.vel); ++c.nlaunch;
  cudaMemcpyAsync(c.csq, csq, sizeof(double) * (size_t)ptot, cudaMemcpyHostToDevice, c.st);
  c.have_v = c.have_csq = true;
  return finish(c, "upload");
}

namespace seren {
namespace {

// Host buffers of seren_gpu_force_step_io (NULL ones are skipped)
struct IoPlan {
  const double* v_in;      // velocities and c_s^2 to copy in after the tree build
  const double* csq_in;
  double* parray;
  double* v;
  double* csq;
  double* rho;
  double* omega;
  double* a;
  double* gpot;
  int32_t* perm;
};

// The device-resident force step.  With io, each result leaves on the copy
// stream once the stage that makes it has run: v, c_s^2 and the permutation
// after the tree build, parray (h), rho and omega after grad-h; a and gpot
// follow gravity on the compute stream.
int force_step_body(Ctx& c, int first_call, const IoPlan* io, bool block = false) {
  const int n = c.ptot;
  const size_t N = (size_t)n;
  c.act = nullptr;
  c.sink_a_valid = false;                    // a new tree: the sinks' accelerations are stale
  cudaMemsetAsync(c.d_counts, 0, sizeof(int) * 32, c.st);
  cudaEventRecord(c.ev[0], c.st);
  // main/tree_update.F90:26-88: a build every nbuildstep evaluations (and
  // whenever there is no tree, on a first call, or from host buffers), a
  // restock of the same cells in between
  int rc = SEREN_GPU_OK;
  if (io || first_call || !c.have_tree || c.since_build >= c.nbuildstep) {
    rc = build_tree(c);
    if (rc) return rc;
    launch_stock(c);
    c.since_build = 0;
  } else {
    bool rebuilt = false;
    rc = restock(c, rebuilt);
    if (rc) return rc;
    if (rebuilt) c.since_build = 0;
  }
  ++c.since_build;
  // block timesteps: the forces of the accdo particles only (in tree order,
  // listed after the build's reorder)
  int nact = n;
  if (block && (rc = block_active(c, nact))) return rc;
  cudaEventRecord(c.ev[1], c.st);
  if (io) {
    // v and c_s^2 come in on the copy stream while the grad-h walk runs (the
    // tree build has the device to itself); the passes wait for them
    cudaStreamWaitEvent(c.st_io, c.ev[1], 0);
    cudaMemcpyAsync(c.stage_io, io->v_in, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, c.st_io);
    k_unpack_v<<<nb(n, 256), 256, 0, c.st_io>>>(c.stage_io, n, c.vel); ++c.nlaunch;
    cudaMemcpyAsync(c.csq, io->csq_in, sizeof(double) * N, cudaMemcpyHostToDevice, c.st_io);
    cudaEventRecord(c.ev_io[1], c.st_io);
    if (io->perm) cudaMemcpyAsync(io->perm, c.orig, sizeof(int) * N, cudaMemcpyDeviceToHost, c.st_io);
  }
  if (first_call) launch_hguess(c);
  launch_gradh(c, nact);                      // runs finish_reorder before its passes
  finish_reorder(c);
  cudaEventRecord(c.ev[2], c.st);
  if (io) {
    cudaStreamWaitEvent(c.st_io, c.ev[2], 0);
    if (io->v) {
      k_pack_v<<<nb(n, 256), 256, 0, c.st_io>>>(c.stage_io, n, c.vel); ++c.nlaunch;
      cudaMemcpyAsync(io->v, c.stage_io, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, c.st_io);
    }
    if (io->csq) cudaMemcpyAsync(io->csq, c.csq, sizeof(double) * N, cudaMemcpyDeviceToHost, c.st_io);
    if (io->parray) {
      launch_pack_parray(c, c.stage_io, n, c.st_io);
      cudaMemcpyAsync(io->parray, c.stage_io, sizeof(double) * 6 * N, cudaMemcpyDeviceToHost,
                      c.st_io);
    }
    if (io->rho) cudaMemcpyAsync(io->rho, c.rho, sizeof(double) * N, cudaMemcpyDeviceToHost, c.st_io);
    if (io->omega)
      cudaMemcpyAsync(io->omega, c.omega, sizeof(double) * N, cudaMemcpyDeviceToHost, c.st_io);
  }
  launch_update_hmax(c);
  launch_neib(c, nact, false);                // the lists stay on the device
  cudaEventRecord(c.ev[3], c.st);
  launch_thermal(c);
  launch_hydro(c, nact);
  cudaEventRecord(c.ev[4], c.st);
  // a and gpot go straight to mapped (pinned) host buffers from the gravity
  // kernel, else they are copied after it
  double* amap = io ? mapped_host(io->a) : nullptr;
  double* gmap = io ? mapped_host(io->gpot) : nullptr;
  launch_grav(c, nact, c.nsink, c.nsink > 0 ? c.sinks : nullptr, amap, gmap);
  cudaEventRecord(c.ev[5], c.st);
  if (io) {
    if (io->a && !amap)
      cudaMemcpyAsync(io->a, c.acc, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, c.st);
    if (io->gpot && !gmap)
      cudaMemcpyAsync(io->gpot, c.gpot, sizeof(double) * N, cudaMemcpyDeviceToHost, c.st);
  }
  rc = finish(c, "force_step");
  if (rc) return rc;
  if (io) {
    const cudaError_t e = cudaStreamSynchronize(c.st_io);
    if (e != cudaSuccess) return cuda_fail(c, e, "force_step_io(copies)");
  }
  c.step_launches = c.nlaunch;
  c.have_sph = true;
  for (int k = 0; k < 5; ++k) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c.ev[k], c.ev[k + 1]);
    c.stage_ms[k] = ms;
  }
  float tot = 0.f;
  cudaEventElapsedTime(&tot, c.ev[0], c.ev[5]);
  c.stage_ms[5] = tot;
  return SEREN_GPU_OK;
}

}  // namespace
}  // namespace seren

int seren_gpu_force_step(seren_gpu_ctx* h, int32_t first_call) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!c.have_v || !c.have_csq || c.ptot < 1)
    return fail(c, SEREN_GPU_ERR_STATE, "call seren_gpu_upload first");
  c.nlaunch = 0;
  return seren::force_step_body(c, first_call, nullptr);
}

int seren_gpu_force_step_io(seren_gpu_ctx* h, int32_t ptot, const double* parray, const double* v,
                            const double* csq, int32_t first_call, double* parray_out,
                            double* v_out, double* csq_out, double* rho, double* omega, double* a,
                            double* gpot, int32_t* perm_total) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!parray || !v || !csq || ptot < 1) return fail(c, SEREN_GPU_ERR_ARG, "NULL array or ptot < 1");
  if (ptot > c.pmax) return fail(c, SEREN_GPU_ERR_CAPACITY, "ptot > pmax");
  if (seren::io_init(c)) {
    cudaGetLastError();
    return fail(c, SEREN_GPU_ERR_CUDA, "force_step_io: copy stream or staging buffer");
  }
  const size_t N = (size_t)ptot;
  c.nlaunch = 0;
  seren::reset_particles(c, ptot);
  cudaMemcpyAsync(c.stage, parray, sizeof(double) * 6 * N, cudaMemcpyHostToDevice, c.st);
  seren::launch_unpack_parray(c, c.stage, ptot);
  // velocities and c_s^2 arrive after the tree build (force_step_body), in
  // upload order in vel / csq; the tree build reorders the rest and leaves
  // them to finish_reorder, which waits for the copy
  c.reorder_wait = c.ev_io[1];
  c.have_v = c.have_csq = true;
  int rc = finish(c, "force_step_io(upload)");
  if (rc == SEREN_GPU_OK) {
    const seren::IoPlan io{v, csq, parray_out, v_out, csq_out, rho, omega, a, gpot, perm_total};
    rc = seren::force_step_body(c, first_call, &io);
  }
  if (rc != SEREN_GPU_OK) {                                // leave no copy in flight
    cudaStreamSynchronize(c.st_io);
    c.reorder_wait = nullptr;
    c.reorder_late = false;
    c.have_v = c.have_csq = false;
    return rc;
  }
  if (perm_total && c.prm.index_base)
    for (size_t i = 0; i < N; ++i) perm_total[i] += c.prm.index_base;
  return SEREN_GPU_OK;
}

int seren_gpu_set_sinks(seren_gpu_ctx* h, int32_t nsink, const double* sink_rmh) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (nsink < 0 || nsink > 1024 || (nsink > 0 && !sink_rmh))
    return fail(c, SEREN_GPU_ERR_ARG, "set_sinks: 0 <= nsink <= 1024 with sink_rmh given");
  if (nsink > 0 && c.ncloud > 1)
    return fail(c, SEREN_GPU_ERR_STATE, "set_sinks: not available with several clouds");
  if (nsink > 0)
    cudaMemcpyAsync(c.sinks, sink_rmh, sizeof(double) * 5 * nsink, cudaMemcpyHostToDevice, c.st);
  c.nsink = nsink;
  c.sink_rmh.assign(sink_rmh, sink_rmh + 5 * (size_t)nsink);
  c.sink_move = false;                       // velocities again with seren_gpu_set_sink_motion
  c.sink_a_valid = false;
  return finish(c, "set_sinks");
}

namespace seren {
namespace {

// the sinks' accelerations and potentials (sph_sink_forces.F90:49-110) on the
// current tree, into the host copies
int sink_accels(Ctx& c) {
  launch_sink_walk(c, c.nsink, c.sinks, c.sink_out);
  std::vector<double> out((size_t)c.nsink * 4);
  cudaMemcpyAsync(out.data(), c.sink_out, sizeof(double) * out.size(), cudaMemcpyDeviceToHost, c.st);
  const int rc = finish(c, "sink accelerations");
  if (rc) return rc;
  c.sink_a.resize((size_t)c.nsink * 3);
  c.sink_pot.resize((size_t)c.nsink);
  for (int s = 0; s < c.nsink; ++s) {
    for (int k = 0; k < 3; ++k) c.sink_a[s * 3 + k] = out[s * 4 + k];
    c.sink_pot[s] = out[s * 4 + 3];
  }
  c.sink_a_valid = true;
  return SEREN_GPU_OK;
}

// the scratch of accretion and sink search, made on first use; 0 or -1
int sink_scratch(Ctx& c) {
  if (c.acc_ws) return 0;
  const size_t P = (size_t)c.pmax;
  if (cudaMalloc(&c.acc_sinks, sizeof(double) * ACC_STRIDE * 1024) != cudaSuccess ||
      cudaMalloc(&c.acc_out, sizeof(double) * ACC_STRIDE * 1024) != cudaSuccess ||
      cudaMalloc(&c.acc_ws, sizeof(int) * (4 * P + 16)) != cudaSuccess) {
    cudaGetLastError();
    for (void** p : {(void**)&c.acc_sinks, (void**)&c.acc_out, (void**)&c.acc_ws})
      if (*p) { cudaFree(*p); *p = nullptr; }
    return -1;
  }
  return 0;
}

// the sinks' records for the accretion and search kernels: x, y, z, m, h,
// radius, accrete (1/0; accrete NULL: every sink), v, a
void sink_records(Ctx& c, const int32_t* accrete) {
  const int ns = c.nsink;
  if (ns < 1) return;
  const int S = ACC_STRIDE;
  std::vector<double> rec((size_t)ns * S, 0.0);
  for (int s = 0; s < ns; ++s) {
    double* R = &rec[(size_t)s * S];
    for (int k = 0; k < 5; ++k) R[k] = c.sink_rmh[s * 5 + k];
    R[5] = c.sink_radius[s];
    R[6] = (!accrete || accrete[s]) ? 1.0 : 0.0;
    for (int k = 0; k < 3; ++k) {
      R[7 + k] = c.sink_v[s * 3 + k];
      R[10 + k] = c.sink_a[s * 3 + k];
    }
  }
  cudaMemcpyAsync(c.acc_sinks, rec.data(), sizeof(double) * rec.size(), cudaMemcpyHostToDevice, c.st);
  cudaStreamSynchronize(c.st);              // rec is a local vector
}

int sink_upload(Ctx& c) {
  cudaMemcpyAsync(c.sinks, c.sink_rmh.data(), sizeof(double) * 5 * (size_t)c.nsink,
                  cudaMemcpyHostToDevice, c.st);
  return SEREN_GPU_OK;
}

}  // namespace
}  // namespace seren

int seren_gpu_set_sink_motion(seren_gpu_ctx* h, int32_t nsink, const double* sink_v,
                              const double* sink_radius) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (c.blk.on) return fail(c, SEREN_GPU_ERR_STATE, "set_sink_motion: not available with block timesteps");
  if (nsink < 1 || nsink != c.nsink || !sink_v || !sink_radius)
    return fail(c, SEREN_GPU_ERR_ARG, "set_sink_motion: nsink as in seren_gpu_set_sinks, arrays given");
  c.sink_v.assign(sink_v, sink_v + 3 * (size_t)nsink);
  c.sink_radius.assign(sink_radius, sink_radius + (size_t)nsink);
  c.sink_move = true;
  return SEREN_GPU_OK;
}

int seren_gpu_get_sinks(seren_gpu_ctx* h, int32_t nsink, double* sink_rmh, double* sink_v,
                        double* sink_a, double* sink_gpot) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (nsink < 1 || nsink != c.nsink) return fail(c, SEREN_GPU_ERR_ARG, "get_sinks: nsink differs");
  if ((sink_a || sink_gpot) && !c.sink_a_valid) {
    if (!c.have_tree) return fail(c, SEREN_GPU_ERR_STATE, "get_sinks: no tree for the accelerations");
    const int rc = seren::sink_accels(c);
    if (rc) return rc;
  }
  const size_t n = (size_t)nsink;
  if (sink_rmh) std::memcpy(sink_rmh, c.sink_rmh.data(), sizeof(double) * 5 * n);
  if (sink_v) {
    if (c.sink_v.size() < 3 * n) return fail(c, SEREN_GPU_ERR_STATE, "get_sinks: no sink velocities");
    std::memcpy(sink_v, c.sink_v.data(), sizeof(double) * 3 * n);
  }
  if (sink_a) std::memcpy(sink_a, c.sink_a.data(), sizeof(double) * 3 * n);
  if (sink_gpot) std::memcpy(sink_gpot, c.sink_pot.data(), sizeof(double) * n);
  return SEREN_GPU_OK;
}

int seren_gpu_sink_timestep(seren_gpu_ctx* h, double sink_mult, double* dt_min) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!dt_min || !(sink_mult > 0.0)) return fail(c, SEREN_GPU_ERR_ARG, "sink_timestep: bad arguments");
  if (!c.sink_move) return fail(c, SEREN_GPU_ERR_STATE, "sink_timestep: call seren_gpu_set_sink_motion");
  if (!c.sink_a_valid) {
    if (!c.have_tree) return fail(c, SEREN_GPU_ERR_STATE, "sink_timestep: no tree");
    const int rc = seren::sink_accels(c);
    if (rc) return rc;
  }
  // sinks/sink_timestep.F90:28-52, the least over the sinks (sph_timesteps.F90:69-74)
  double best = 1.0e300;
  for (int s = 0; s < c.nsink; ++s) {
    const double rads = c.sink_radius[s];
    const double* as = &c.sink_a[s * 3];
    const double* vs = &c.sink_v[s * 3];
    const double* rs = &c.sink_rmh[s * 5];
    const double acc_mag = std::sqrt((as[0] * as[0] + as[1] * as[1]) + as[2] * as[2]);
    double vel_mag = std::sqrt((vs[0] * vs[0] + vs[1] * vs[1]) + vs[2] * vs[2]);
    const double dt1 = sink_mult * std::sqrt(rads / (acc_mag + 1.0e-20));
    double dt2 = (sink_mult * rads) / (vel_mag + 1.0e-20);
    double dt = std::min(dt1, dt2);
    if (c.nsink > 1) {
      for (int ss = 0; ss < c.nsink; ++ss) {
        if (ss == s) continue;
        const double* rss = &c.sink_rmh[ss * 5];
        const double d0 = rss[0] - rs[0], d1 = rss[1] - rs[1], d2 = rss[2] - rs[2];
        const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
        const double dist = std::max(0.5 * (rads + c.sink_radius[ss]), std::sqrt(drsqd));
        const double* vss = &c.sink_v[ss * 3];
        const double e0 = vs[0] - vss[0], e1 = vs[1] - vss[1], e2 = vs[2] - vss[2];
        vel_mag = std::sqrt((e0 * e0 + e1 * e1) + e2 * e2);
        dt2 = (sink_mult * dist) / (vel_mag + 1.0e-20);
        dt = std::min(dt, dt2);
      }
    }
    best = std::min(best, dt);
  }
  *dt_min = best;
  return SEREN_GPU_OK;
}

int seren_gpu_timestep(seren_gpu_ctx* h, double courant_mult, double accel_mult, double* dt_min,
                       double* dt) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!dt_min || !(courant_mult > 0.0) || !(accel_mult > 0.0))
    return fail(c, SEREN_GPU_ERR_ARG, "timestep: dt_min NULL or a multiplier not positive");
  if (!c.have_sph || c.ptot < 1) return fail(c, SEREN_GPU_ERR_STATE, "no forces yet");
  const int n = c.ptot;
  double* d_dt = c.stage;                                  // [n] steps, then the least
  unsigned long long* d_min = reinterpret_cast<unsigned long long*>(c.stage + n);
  static const unsigned long long inf_bits = 0x7ff0000000000000ull;
  cudaMemcpyAsync(d_min, &inf_bits, sizeof(inf_bits), cudaMemcpyHostToDevice, c.st);
  seren::k_timestep<<<nb(n, 256), 256, 0, c.st>>>(n, c.hz, c.acc, c.div_v, c.sound, c.prm.alpha,
                                                   2.0 * c.prm.alpha, courant_mult, accel_mult,
                                                   d_dt, d_min);
  ++c.nlaunch;
  if (seren::read_dev(c, d_min, dt_min, sizeof(double))) return finish(c, "timestep");
  if (dt) cudaMemcpyAsync(dt, d_dt, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, c.st);
  return finish(c, "timestep");
}

int seren_gpu_rk2_step(seren_gpu_ctx* h, double dt) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!(dt > 0.0) || !std::isfinite(dt)) return fail(c, SEREN_GPU_ERR_ARG, "rk2_step: dt not positive");
  if (!c.have_v || !c.have_csq || !c.have_sph || c.ptot < 1)
    return fail(c, SEREN_GPU_ERR_STATE, "rk2_step: call seren_gpu_upload and seren_gpu_force_step first");
  if (c.blk.on) return fail(c, SEREN_GPU_ERR_STATE, "rk2_step: block timesteps are on (upload again)");
  if (seren::rk_alloc(c)) return fail(c, SEREN_GPU_ERR_CUDA, "rk2_step: state allocation failed");
  const int n = c.ptot;
  c.nlaunch = 0;
  // sinks set in motion move with the same scheme (sinks/advance_sink_RK.F90:22-51)
  const bool sinks = c.sink_move && c.nsink > 0;
  int rc = SEREN_GPU_OK;
  if (sinks && !c.sink_a_valid && (rc = seren::sink_accels(c))) return rc;
  const size_t ns = (size_t)c.nsink;
  // first half (advance_runge_kutta.F90:40-54) with the forces at the start
  seren::k_rk_half<<<nb(n, 256), 256, 0, c.st>>>(n, c.pm, c.vel, c.acc, c.r_old, c.v_old,
                                                  c.v_half, 0.5 * dt);
  ++c.nlaunch;
  if (sinks) {
    c.sink_rold.resize(3 * ns);
    c.sink_vold.resize(3 * ns);
    c.sink_vhalf.resize(3 * ns);
    const double hdt = 0.5 * dt;
    for (size_t s = 0; s < ns; ++s)
      for (int k = 0; k < 3; ++k) {
        c.sink_rold[s * 3 + k] = c.sink_rmh[s * 5 + k];
        c.sink_vold[s * 3 + k] = c.sink_v[s * 3 + k];
        c.sink_rmh[s * 5 + k] = c.sink_rold[s * 3 + k] + c.sink_vold[s * 3 + k] * hdt;
        c.sink_v[s * 3 + k] = c.sink_vold[s * 3 + k] + c.sink_a[s * 3 + k] * hdt;
        c.sink_vhalf[s * 3 + k] = c.sink_v[s * 3 + k];
      }
    seren::sink_upload(c);
  }
  rc = seren::force_step_body(c, 0, nullptr);                 // forces at the half step
  if (rc) return rc;
  if (sinks && (rc = seren::sink_accels(c))) return rc;
  // second half (:56-69) from the start with v_half and the half-step forces
  seren::k_rk_full<<<nb(n, 256), 256, 0, c.st>>>(n, c.pm, c.vel, c.acc, c.r_old, c.v_old,
                                                  c.v_half, dt);
  ++c.nlaunch;
  if (sinks) {
    for (size_t s = 0; s < ns; ++s)
      for (int k = 0; k < 3; ++k) {
        c.sink_rmh[s * 5 + k] = c.sink_rold[s * 3 + k] + c.sink_vhalf[s * 3 + k] * dt;
        c.sink_v[s * 3 + k] = c.sink_vold[s * 3 + k] + c.sink_a[s * 3 + k] * dt;
      }
    seren::sink_upload(c);
  }
  rc = seren::force_step_body(c, 0, nullptr);                 // forces at the end
  if (rc) return rc;
  return sinks ? seren::sink_accels(c) : SEREN_GPU_OK;
}

int seren_gpu_set_clouds(seren_gpu_ctx* h, int32_t ncloud, const int32_t* counts) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (ncloud < 1 || (ncloud > 1 && !counts)) return fail(c, SEREN_GPU_ERR_ARG, "set_clouds: ncloud < 1 or counts NULL");
  if (c.ptot < 1) return fail(c, SEREN_GPU_ERR_STATE, "set_clouds: upload the particles first");
  c.have_tree = false;                               // the next force step builds
  if (ncloud == 1) {
    c.ncloud = 1;
    return SEREN_GPU_OK;
  }
  if (c.nsink > 0 || c.blk.on)
    return fail(c, SEREN_GPU_ERR_STATE, "set_clouds: not available with sinks or block timesteps");
  std::vector<seren::CloudInfo> cl(ncloud);
  long long sum = 0;
  for (int k = 0; k < ncloud; ++k) {
    if (counts[k] < 1) return fail(c, SEREN_GPU_ERR_ARG, "set_clouds: a cloud without particles");
    cl[k] = seren::CloudInfo{};
    cl[k].pstart = (int)sum;
    cl[k].n = counts[k];
    cl[k].cell = k;
    sum += counts[k];
  }
  if (sum != c.ptot) return fail(c, SEREN_GPU_ERR_ARG, "set_clouds: counts do not add up to ptot");
  // the group kernels' list: each cloud's particles, padded to a multiple of 32
  std::vector<int> gl;
  gl.reserve((size_t)c.ptot + 32 * (size_t)ncloud);
  for (int k = 0; k < ncloud; ++k) {
    for (int i = 0; i < cl[k].n; ++i) gl.push_back(cl[k].pstart + i);
    while (gl.size() % 32) gl.push_back(-1);
  }
  if (c.d_clouds) cudaFree(c.d_clouds);
  if (c.gact) cudaFree(c.gact);
  c.d_clouds = nullptr;
  c.gact = nullptr;
  if (cudaMalloc(&c.d_clouds, sizeof(seren::CloudInfo) * ncloud) != cudaSuccess ||
      cudaMalloc(&c.gact, sizeof(int) * gl.size()) != cudaSuccess) {
    cudaGetLastError();
    return fail(c, SEREN_GPU_ERR_CUDA, "set_clouds: allocation failed");
  }
  cudaMemcpyAsync(c.d_clouds, cl.data(), sizeof(seren::CloudInfo) * ncloud, cudaMemcpyHostToDevice, c.st);
  cudaMemcpyAsync(c.gact, gl.data(), sizeof(int) * gl.size(), cudaMemcpyHostToDevice, c.st);
  c.clouds = cl;
  c.ngact = (int)gl.size();
  c.ncloud = ncloud;
  return finish(c, "set_clouds");
}

namespace {
// tuned knobs per (device, precision, ceil(log2 N)), shared by the contexts of
// the process (seren_gpu_autotune with trials = 0 reuses them)
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int>, seren::Tuning> g_tune_cache;

int tune_key_bits(int n) {
  int b = 0;
  while ((1ll << b) < (long long)n) ++b;
  return b;
}

bool tune_valid(const seren::Tuning& t) {
  return (t.hydro_sub == 2 || t.hydro_sub == 4 || t.hydro_sub == 8) &&
         (t.grav_cap == 64 || t.grav_cap == 96) && t.grav_bps >= 0 && t.gradh_bps >= 0 &&
         t.neib_bps >= 0;
}

void tune_out(const seren::Tuning& t, double ms, seren_gpu_tuning* out) {
  if (!out) return;
  out->hydro_sub = t.hydro_sub;
  out->grav_cap = t.grav_cap;
  out->grav_bps = t.grav_bps;
  out->gradh_bps = t.gradh_bps;
  out->neib_bps = t.neib_bps;
  out->reserved = 0;
  out->ms_per_step = ms;
}
}  // namespace

int seren_gpu_set_tuning(seren_gpu_ctx* h, const seren_gpu_tuning* t) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!t) return fail(c, SEREN_GPU_ERR_ARG, "set_tuning: NULL");
  seren::Tuning k;
  k.hydro_sub = t->hydro_sub;
  k.grav_cap = t->grav_cap;
  k.grav_bps = t->grav_bps;
  k.gradh_bps = t->gradh_bps;
  k.neib_bps = t->neib_bps;
  if (!tune_valid(k)) return fail(c, SEREN_GPU_ERR_ARG, "set_tuning: a knob out of range");
  c.tune = k;
  return SEREN_GPU_OK;
}

int seren_gpu_autotune(seren_gpu_ctx* h, int32_t trials, seren_gpu_tuning* out) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!c.have_v || !c.have_csq || !c.have_sph || c.ptot < 1 || c.blk.on)
    return fail(c, SEREN_GPU_ERR_STATE, "autotune: upload and a first force step come first");
  const auto key = std::make_tuple(c.dev, c.prm.precision, tune_key_bits(c.ptot));
  if (trials <= 0) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it == g_tune_cache.end())
      return fail(c, SEREN_GPU_ERR_STATE, "autotune: nothing tuned yet for this size");
    c.tune = it->second;
    tune_out(c.tune, 0.0, out);
    return SEREN_GPU_OK;
  }
  const bool mixed = c.prm.precision != 0;
  // candidates per knob; round r takes candidate r of the gravity pairs and
  // candidate r mod n of the others, and each stage keeps its best round
  struct GravKnob { int cap, bps; };
  std::vector<GravKnob> grav = mixed
      ? std::vector<GravKnob>{{64, 0}, {96, 0}, {64, 3}, {96, 4}}
      : std::vector<GravKnob>{{64, 0}, {64, 3}, {64, 2}, {64, 0}};
  const int hsub[3] = {4, 2, 8};
  const int gbps[3] = {0, 4, 2};
  const int nbps[3] = {0, 4, 2};
  const int rounds = 4;
  std::vector<std::array<double, 5>> ms(rounds);
  const seren::Tuning keep = c.tune;
  for (int r = 0; r < rounds; ++r) {
    seren::Tuning t;
    t.grav_cap = grav[r].cap;
    t.grav_bps = grav[r].bps;
    t.hydro_sub = mixed ? hsub[r % 3] : 4;
    t.gradh_bps = gbps[r % 3];
    t.neib_bps = nbps[r % 3];
    c.tune = t;
    ms[r].fill(0.0);
    for (int k = 0; k < trials; ++k) {
      c.nlaunch = 0;
      int rc = seren::force_step_body(c, 0, nullptr);
      if (rc) {
        c.tune = keep;
        return rc;
      }
      for (int st = 0; st < 5; ++st) ms[r][st] += c.stage_ms[st];
    }
  }
  auto best = [&](int stage) {
    int b = 0;
    for (int r = 1; r < rounds; ++r)
      if (ms[r][stage] < ms[b][stage]) b = r;
    return b;
  };
  seren::Tuning t;
  const int bg = best(4), bh = best(3), bgr = best(1), bn = best(2);
  t.grav_cap = grav[bg].cap;
  t.grav_bps = grav[bg].bps;
  t.hydro_sub = mixed ? hsub[bh % 3] : 4;
  t.gradh_bps = gbps[bgr % 3];
  t.neib_bps = nbps[bn % 3];
  c.tune = t;
  const double chosen = (ms[0][0] + ms[bgr][1] + ms[bn][2] + ms[bh][3] + ms[bg][4]) / trials;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = t;
  }
  tune_out(t, chosen, out);
  return SEREN_GPU_OK;
}

int seren_gpu_block_start(seren_gpu_ctx* h, const seren_gpu_block_params* prm) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!prm || prm->nlevels < 1 || prm->nlevels > 24 || prm->level_mode < 0 ||
      prm->level_mode > 2 || prm->check_neib < 0 || prm->check_neib > 2 ||
      !(prm->dt_fixed > 0.0) || !(prm->courant_mult > 0.0) || !(prm->accel_mult > 0.0))
    return fail(c, SEREN_GPU_ERR_ARG, "block_start: bad parameters");
  if (!c.have_v || !c.have_csq || !c.have_sph || c.ptot < 1)
    return fail(c, SEREN_GPU_ERR_STATE, "block_start: call seren_gpu_upload and seren_gpu_force_step first");
  if (c.sink_move) return fail(c, SEREN_GPU_ERR_ARG, "block_start: moving sinks are not supported");
  if (c.ncloud > 1) return fail(c, SEREN_GPU_ERR_STATE, "block_start: not available with several clouds");
  c.nlaunch = 0;
  seren::BlockState& b = c.blk;
  b.nlevels = prm->nlevels;
  b.level_mode = prm->level_mode;
  b.check_neib = prm->check_neib;
  b.dt_fixed = prm->dt_fixed;
  b.courant = prm->courant_mult;
  b.accel = prm->accel_mult;
  int rc = seren::block_start(c);
  if (rc) return fail(c, rc, "block_start: state allocation failed");
  return finish(c, "block_start");
}

int seren_gpu_block_step(seren_gpu_ctx* h, seren_gpu_block_state* out) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!c.blk.on) return fail(c, SEREN_GPU_ERR_STATE, "block_step: call seren_gpu_block_start first");
  c.nlaunch = 0;
  int rc = seren::force_step_body(c, 0, nullptr, true);      // sph_integrate.F90:36-66
  if (rc) return rc;
  rc = seren::block_after_forces(c);                         // :79-113
  if (rc) return fail(c, rc, "block_step: device result read failed");
  rc = finish(c, "block_step");
  if (rc) return rc;
  c.step_launches = c.nlaunch;
  if (out) {
    const seren::BlockState& b = c.blk;
    out->n = b.n;
    out->nresync = b.nresync;
    out->nsteps = b.nsteps;
    out->level_max = b.level_max;
    out->level_step = b.level_step;
    out->nactive = b.nactive;
    out->reserved = 0;
    out->timestep = b.timestep;
    out->dt_max = b.dt_max;
    out->time = b.time;
  }
  return SEREN_GPU_OK;
}

int seren_gpu_block_levels(seren_gpu_ctx* h, int32_t* nlevel, int64_t* nlast, int32_t* nminneib,
                           int32_t* accdo) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!c.blk.on) return fail(c, SEREN_GPU_ERR_STATE, "block_levels: block timesteps are off");
  const size_t N = (size_t)c.ptot;
  const seren::BlockState& b = c.blk;
  if (nlevel) cudaMemcpyAsync(nlevel, b.nlevel, sizeof(int) * N, cudaMemcpyDeviceToHost, c.st);
  if (nlast) cudaMemcpyAsync(nlast, b.nlast, sizeof(long long) * N, cudaMemcpyDeviceToHost, c.st);
  if (nminneib) cudaMemcpyAsync(nminneib, b.nminneib, sizeof(int) * N, cudaMemcpyDeviceToHost, c.st);
  if (accdo) cudaMemcpyAsync(accdo, b.accdo, sizeof(int) * N, cudaMemcpyDeviceToHost, c.st);
  return finish(c, "block_levels");
}

int seren_gpu_accrete(seren_gpu_ctx* h, int32_t nsink, const int32_t* accrete,
                      int32_t energy_accrete, double* sink_angmom, int32_t* naccreted,
                      int32_t* ptot_out) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (c.blk.on) return fail(c, SEREN_GPU_ERR_STATE, "accrete: not available with block timesteps");
  if (nsink < 1 || nsink != c.nsink)
    return fail(c, SEREN_GPU_ERR_ARG, "accrete: nsink as in seren_gpu_set_sinks");
  if (!c.sink_move)
    return fail(c, SEREN_GPU_ERR_STATE, "accrete: call seren_gpu_set_sink_motion");
  if (!c.have_v || !c.have_sph || c.ptot < 1)
    return fail(c, SEREN_GPU_ERR_STATE, "accrete: call seren_gpu_force_step first");
  if (!c.sink_a_valid) {
    if (!c.have_tree) return fail(c, SEREN_GPU_ERR_STATE, "accrete: no tree for the sinks' accelerations");
    const int rc = seren::sink_accels(c);
    if (rc) return rc;
  }
  if (seren::sink_scratch(c)) return fail(c, SEREN_GPU_ERR_CUDA, "accrete: scratch allocation failed");
  const int ns = nsink;
  const int S = seren::ACC_STRIDE;
  seren::sink_records(c, accrete);
  c.nlaunch = 0;
  std::vector<double> out;
  int ndead = 0;
  int rc = seren::launch_accrete(c, ns, energy_accrete ? 1 : 0, out, ndead);
  if (rc) return finish(c, "accrete");
  rc = finish(c, "accrete");
  if (rc) return rc;
  if (naccreted)
    for (int s = 0; s < ns; ++s) naccreted[s] = 0;
  if (ndead > 0) {
    // accrete_particles.F90:264-285: the new sink state; rold and vold (the
    // Runge-Kutta start values) are the new position and velocity
    for (int s = 0; s < ns; ++s) {
      const double* O = &out[(size_t)s * S];
      const int cnt = (int)O[15];
      if (naccreted) naccreted[s] = cnt;
      if (cnt <= 0) continue;
      c.sink_rmh[s * 5 + 3] = O[0];
      for (int k = 0; k < 3; ++k) {
        c.sink_rmh[s * 5 + k] = O[1 + k];
        c.sink_v[s * 3 + k] = O[4 + k];
        c.sink_a[s * 3 + k] = O[7 + k];
        if (c.sink_rold.size() == 3 * (size_t)ns) c.sink_rold[s * 3 + k] = O[1 + k];
        if (c.sink_vold.size() == 3 * (size_t)ns) c.sink_vold[s * 3 + k] = O[4 + k];
        if (sink_angmom) sink_angmom[s * 3 + k] = sink_angmom[s * 3 + k] + O[10 + k];
      }
    }
    rc = seren::sink_upload(c);
    if (rc) return rc;
    // the tree and neighbour lists index the old arrays: the next force step
    // builds a new tree (accrete_particles.F90:330, nstock = nsteps)
    c.have_tree = false;
  }
  if (ptot_out) *ptot_out = c.ptot;
  return SEREN_GPU_OK;
}

int seren_gpu_sink_search(seren_gpu_ctx* h, const seren_gpu_sink_search_params* prm,
                          int32_t* created, int32_t* psink_id, double* sink_angmom,
                          int32_t* nremoved, int32_t* ptot_out) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (c.blk.on) return fail(c, SEREN_GPU_ERR_STATE, "sink_search: not available with block timesteps");
  if (!prm || !(prm->sinkrad > 0.0))
    return fail(c, SEREN_GPU_ERR_ARG, "sink_search: parameters with sinkrad > 0");
  if (!c.have_tree || !c.have_v || !c.have_sph || c.ptot < 1)
    return fail(c, SEREN_GPU_ERR_STATE, "sink_search: call seren_gpu_force_step first");
  if (c.nsink >= 1024) return fail(c, SEREN_GPU_ERR_CAPACITY, "sink_search: 1024 sinks already");
  if (c.nsink > 0 && !c.sink_move)
    return fail(c, SEREN_GPU_ERR_STATE, "sink_search: call seren_gpu_set_sink_motion");
  if (c.nsink > 0 && !c.sink_a_valid) {
    const int rc = seren::sink_accels(c);
    if (rc) return rc;
  }
  if (seren::sink_scratch(c)) return fail(c, SEREN_GPU_ERR_CUDA, "sink_search: scratch allocation failed");
  seren::sink_records(c, nullptr);
  const seren::SinkSearchArgs sa{prm->rhosink, prm->sinkrad, prm->hmult_sinkrad != 0,
                                 prm->rho_search != 0, prm->potmin_search != 0,
                                 prm->hill_sphere_search != 0, prm->div_v_search != 0,
                                 prm->div_a_search != 0, prm->timescale_search != 0};
  c.nlaunch = 0;
  int psink = -1, pid = -1, nrem = 0;
  std::vector<double> out;
  int rc = seren::launch_sink_search(c, c.nsink, sa, psink, pid, out, nrem);
  if (rc) return finish(c, "sink_search");
  rc = finish(c, "sink_search");
  if (rc) return rc;
  if (created) *created = psink >= 0 ? 1 : 0;
  if (psink_id) *psink_id = psink >= 0 ? pid + c.prm.index_base : -1;
  if (nremoved) *nremoved = nrem;
  if (psink >= 0) {
    // create_sink.F90:160-201: the new sink (accreting, h = radius / 2)
    const double rads = out[13];
    const bool first = c.nsink == 0;
    const size_t ns = (size_t)c.nsink;
    c.sink_rmh.resize(5 * ns);
    c.sink_v.resize(3 * ns);
    c.sink_a.resize(3 * ns);
    c.sink_radius.resize(ns);
    for (int k = 0; k < 3; ++k) c.sink_rmh.push_back(out[1 + k]);
    c.sink_rmh.push_back(out[0]);
    c.sink_rmh.push_back(seren::INVKERNRANGE * rads);
    for (int k = 0; k < 3; ++k) c.sink_v.push_back(out[4 + k]);
    for (int k = 0; k < 3; ++k) c.sink_a.push_back(out[7 + k]);
    c.sink_radius.push_back(rads);
    c.sink_pot.resize((size_t)c.nsink + 1, 0.0);
    c.nsink += 1;
    c.sink_move = true;
    if (first) c.sink_a_valid = true;
    if (sink_angmom)
      for (int k = 0; k < 3; ++k) sink_angmom[k] = out[10 + k];
    rc = seren::sink_upload(c);
    if (rc) return rc;
    c.have_tree = false;                     // create_sink.F90:250-251: nbuild = nstock = nsteps
  }
  if (ptot_out) *ptot_out = c.ptot;
  return SEREN_GPU_OK;
}

int seren_gpu_set_build_step(seren_gpu_ctx* h, int32_t nbuildstep) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (nbuildstep < 1) return fail(c, SEREN_GPU_ERR_ARG, "set_build_step: nbuildstep >= 1");
  c.nbuildstep = nbuildstep;
  c.since_build = nbuildstep;                // the next evaluation builds
  return SEREN_GPU_OK;
}

int seren_gpu_drift(seren_gpu_ctx* h, double dt) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!c.have_v) return fail(c, SEREN_GPU_ERR_STATE, "no velocities");
  seren::k_drift<<<nb(c.ptot, 256), 256, 0, c.st>>>(c.ptot, c.pm, c.vel, dt); ++c.nlaunch;
  return finish(c, "drift");
}

int seren_gpu_download(seren_gpu_ctx* h, double* parray, double* v, double* rho, double* omega,
                       double* a, double* gpot, int32_t* perm_total) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  const int n = c.ptot;
  if (n < 1) return fail(c, SEREN_GPU_ERR_STATE, "nothing uploaded");
  if (parray) {
    seren::launch_pack_parray(c, c.stage, n);
    cudaMemcpyAsync(parray, c.stage, sizeof(double) * 6 * (size_t)n, cudaMemcpyDeviceToHost, c.st);
    int rc = finish(c, "download(parray)");
    if (rc) return rc;
  }
  if (v) {
    seren::k_pack_v<<<nb(n, 256), 256, 0, c.st>>>(c.stage, n, c.vel); ++c.nlaunch;
    cudaMemcpyAsync(v, c.stage, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, c.st);
    int rc = finish(c, "download(v)");
    if (rc) return rc;
  }
  if (rho) cudaMemcpyAsync(rho, c.rho, sizeof(double) * n, cudaMemcpyDeviceToHost, c.st);
  if (omega) cudaMemcpyAsync(omega, c.omega, sizeof(double) * n, cudaMemcpyDeviceToHost, c.st);
  if (a) cudaMemcpyAsync(a, c.acc, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, c.st);
  if (gpot) cudaMemcpyAsync(gpot, c.gpot, sizeof(double) * n, cudaMemcpyDeviceToHost, c.st);
  if (perm_total) cudaMemcpyAsync(perm_total, c.orig, sizeof(int) * n, cudaMemcpyDeviceToHost, c.st);
  int rc = finish(c, "download");
  if (rc) return rc;
  if (perm_total && c.prm.index_base)
    for (int i = 0; i < n; ++i) perm_total[i] += c.prm.index_base;
  return SEREN_GPU_OK;
}

int seren_gpu_tree_export(seren_gpu_ctx* h, int32_t* ctot, int32_t* ltot, int32_t* leaf,
                          int32_t* nextcell, int32_t* ifopen, int32_t* plist, int32_t* first_cell,
                          int32_t* last_cell, double* grav_r, double* grav_m, double* grav_q,
                          double* dminsqd, double* hydro_r, double* rmax, double* hrangemax) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (!c.have_tree) return fail(c, SEREN_GPU_ERR_STATE, "no tree");
  const int nc = c.info.ctot + 1;
  if (ctot) *ctot = c.info.ctot;
  if (ltot) *ltot = c.info.ltot;
  std::vector<int4> lk(nc);
  std::vector<double4> a(nc), b(nc), ha(nc);
  std::vector<double2> cc(nc);
  std::vector<double> hr(nc);
  cudaMemcpy(lk.data(), c.link, sizeof(int4) * nc, cudaMemcpyDeviceToHost);
  cudaMemcpy(a.data(), c.gA, sizeof(double4) * nc, cudaMemcpyDeviceToHost);
  cudaMemcpy(b.data(), c.gB, sizeof(double4) * nc, cudaMemcpyDeviceToHost);
  cudaMemcpy(cc.data(), c.gC, sizeof(double2) * nc, cudaMemcpyDeviceToHost);
  cudaMemcpy(ha.data(), c.hA, sizeof(double4) * nc, cudaMemcpyDeviceToHost);
  cudaMemcpy(hr.data(), c.hrm, sizeof(double) * nc, cudaMemcpyDeviceToHost);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return seren::cuda_fail(c, e, "tree_export");
  const int base = c.prm.index_base;
  for (int i = 0; i < nc; ++i) {
    if (leaf) leaf[i] = lk[i].x;
    if (nextcell) nextcell[i] = lk[i].y;
    if (ifopen) ifopen[i] = lk[i].x > 0 ? -1 : lk[i].z;
    if (plist)
      for (int k = 0; k < 8; ++k) plist[i * 8 + k] = (lk[i].x > 0 && k < lk[i].x) ? lk[i].w + k + base : -1;
    if (grav_r) { grav_r[i * 3] = a[i].x; grav_r[i * 3 + 1] = a[i].y; grav_r[i * 3 + 2] = a[i].z; }
    if (grav_m) grav_m[i] = a[i].w;
    if (grav_q) {
      grav_q[i * 5] = b[i].x; grav_q[i * 5 + 1] = b[i].y; grav_q[i * 5 + 2] = b[i].z;
      grav_q[i * 5 + 3] = b[i].w; grav_q[i * 5 + 4] = cc[i].x;
    }
    if (dminsqd) dminsqd[i] = cc[i].y;
    if (hydro_r) { hydro_r[i * 3] = ha[i].x; hydro_r[i * 3 + 1] = ha[i].y; hydro_r[i * 3 + 2] = ha[i].z; }
    if (rmax) rmax[i] = ha[i].w;
    if (hrangemax) hrangemax[i] = hr[i];
  }
  for (int l = 0; l <= c.info.ltot; ++l) {
    if (first_cell) first_cell[l] = c.info.first_cell[l];
    if (last_cell) last_cell[l] = c.info.last_cell[l];
  }
  return SEREN_GPU_OK;
}

int seren_gpu_last_step_stats(seren_gpu_ctx* h, double* stage_ms, int32_t* nlaunch,
                              int64_t* counts) {
  if (!h) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  if (stage_ms)
    for (int k = 0; k < 8; ++k) stage_ms[k] = c.stage_ms[k];
  if (nlaunch) *nlaunch = c.step_launches;
  if (counts) {
    unsigned long long cc[16] = {};
    cudaMemcpy(cc, c.d_counts, sizeof(cc), cudaMemcpyDeviceToHost);
    for (int k = 0; k < 16; ++k) counts[k] = (int64_t)cc[k];
  }
  return SEREN_GPU_OK;
}

int seren_gpu_get_stream(seren_gpu_ctx* h, void** stream) {
  if (!h || !stream) return SEREN_GPU_ERR_ARG;
  *stream = (void*)h->c.st;
  return SEREN_GPU_OK;
}

int seren_gpu_fma_peak(seren_gpu_ctx* h, int32_t precision, double* tflops) {
  if (!h || !tflops || (precision != 0 && precision != 1)) return SEREN_GPU_ERR_ARG;
  Ctx& c = h->c;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.dev);
  const int blocks = nsm * 4, threads = 256, iters = 2048;
  float best = 1e30f;
  for (int rep = 0; rep < 3; ++rep) {
    cudaEventRecord(c.ev[8], c.st);
    if (precision == 1)
      seren::k_fma_peak<float><<<blocks, threads, 0, c.st>>>(reinterpret_cast<float*>(c.stage), iters, 0.999f, 1.0e-3f);
    else
      seren::k_fma_peak<double><<<blocks, threads, 0, c.st>>>(c.stage, iters, 0.999, 1.0e-3);
    cudaEventRecord(c.ev[9], c.st);
    int rc = finish(c, "fma_peak");
    if (rc) return rc;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c.ev[8], c.ev[9]);
    best = ms < best ? ms : best;
  }
  const double flops = 2.0 * seren::FMA_CHAINS * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return SEREN_GPU_OK;
}

}  // extern "C"
