// sph.cu - grad-h smoothing length / density solve, neighbour lists, grad-h
// hydro forces with MON97 viscosity, and the isothermal equation of state.
//
// grad-h and the neighbour lists run on group walks: a warp walks the tree
// for 32 neighbouring particles at once with each lane's own test, so every
// lane opens exactly the leaves of its own reference walk (BHhydrowalk_hgather,
// BHhydro_walk); the lanes then run their reference routines over the shared
// list of opened leaves.  Neighbour lists come out in the reference's order
// (depth-first leaf order, particles in leaf order); density sums only differ
// from the reference's in the order of their terms.  The hydro force kernel
// gives one thread to one particle and follows hydro_gradh step by step.
#include <algorithm>
#include <climits>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

#include "ctx.cuh"
#include "kernel_fns.h"

namespace seren {

namespace {

struct HydroTree {
  const int4* link;     // {leaf, nextcell, ifopen, pstart}
  const double4* hA;    // bbox centre, rmax
  const double* hrm;    // hrangemax
  const float4* hA32;   // FP32 centre - root centre, rmax rounded up
  const float* hrm32;   // hrangemax rounded up
  const int* nkids;     // children per cell (ids ifopen .. ifopen + nkids - 1)
  const float4* hN;     // two per cell: hA32; hrm32, first particle / first child,
                        // leaf count / -children (int bits)
  int ctot;
  double rootx, rooty, rootz;
  float delta;          // bound on the FP32 rounding of a root-relative coordinate
  int root;             // root cell of the walks
  double rextent;       // root box extent (the grad-h bisection's first h_upper)
  const CloudInfo* cl;  // a forest of ncl trees (NULL: one tree)
  int ncl;
};

// The tree particle p walks: its root cell, root box, rounding bound and
// extent - in a forest those of its cloud, else the one tree's.  (A local
// value, so the tree's pointers stay kernel parameters.)
struct TreeFrame {
  int root;
  double rootx, rooty, rootz;
  float delta;
  double rextent;
};

__device__ __forceinline__ TreeFrame frame_for(const HydroTree& t, int p) {
  if (!t.cl) return TreeFrame{t.root, t.rootx, t.rooty, t.rootz, t.delta, t.rextent};
  const CloudInfo& C = t.cl[cloud_of(t.cl, t.ncl, p)];
  return TreeFrame{C.cell, C.root[0], C.root[1], C.root[2], C.delta, C.rextent};
}

// Lane i of a group of 32 in an active list: act[i] < 0 pads a cloud's last
// group in a forest (the groups of each cloud start at its first particle);
// dead lanes take lane 0's particle (lane 0 is always live).
__device__ __forceinline__ int group_particle(int i, int nact, const int* act, bool& live) {
  int p = i < nact ? (act ? act[i] : i) : -1;
  live = p >= 0;
  const int p0 = __shfl_sync(0xffffffffu, p, 0);
  return live ? p : p0;
}

// BHtree/BHhydro_walk.F90:9-80 (gather or scatter test)
template <class F>
__device__ __forceinline__ bool walk_gather_scatter(const HydroTree& t, int root, double rx,
                                                    double ry,
                                                    double rz, double hrange, DevError* err,
                                                    int who, F&& f) {
  int c = root;
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

// ---------------------------------------------------------------------------
// grad-h solve, sph/all_sph_gradh.F90:11-492 (GRAD_H_SPH, BH_TREE, GRAVITY).
//
// Per-particle state of the iteration (:132-145) and its update after a
// density pass (:238-285).  The omega sum of the iteration passes (:230, :238)
// is never used after the loop (the final pass recomputes it), so the passes
// accumulate the density only.
struct GhState {
  double hp, h_old, h_high, h_upper, h_lower, rho;
  int iteration, pp_pot, ngrow;
};

__device__ __forceinline__ void gh_init(GhState& s, double h, double rextent) {
  s.hp = h; s.h_old = h; s.h_high = 0.0; s.h_upper = rextent; s.h_lower = 0.0; s.rho = 0.0;
  s.iteration = 0; s.pp_pot = 0; s.ngrow = 0;
}

// returns true when the iteration has ended (converged or given up)
__device__ __forceinline__ bool gh_after_pass(GhState& s, double mp, double h_fac, double rextent,
                                              double rt) {
  s.rho = rt;
  const double hcand = h_fac * pow(mp / rt, ONETHIRD);
  if (fabs(s.hp - hcand) / s.hp < H_CON && s.iteration >= 1) return true;   // :246
  double h_new;
  if (s.iteration < GRADH_ITERATION_MAX) {
    h_new = hcand;
  } else if (s.iteration == GRADH_ITERATION_MAX) {
    s.h_upper = rextent;
    s.h_lower = 0.0;
    h_new = 0.5 * (s.h_lower + s.h_upper);
  } else if (s.iteration < 2 * GRADH_ITERATION_MAX) {
    double fb;
    if (rt > SMALL_NUMBER) fb = pow(s.hp, NDIMPR) - (pow(h_fac, NDIMPR) * mp) / rt;
    else fb = 1.0;
    if (fb > 0.0) s.h_upper = s.hp;
    else s.h_lower = s.hp;
    h_new = 0.5 * (s.h_lower + s.h_upper);
  } else {
    s.hp = s.h_old;
    return true;
  }
  s.hp = h_new;
  s.iteration = s.iteration + 1;
  return false;
}

// the final-pass sums (:360-425)
struct GhFinal {
  double rt, om, dv, zt;
};

__device__ __forceinline__ void gh_store(int p, double mp, double hp, const GhFinal& f,
                                         double2* __restrict__ hz, double* __restrict__ rho,
                                         double* __restrict__ omega, double* __restrict__ divv,
                                         double* __restrict__ drhodt, DevError* err) {
  const double omega_f = 1.0 + ((hp * f.om) / (NDIMPR * f.rt));        // :428
  const double div_v_p = f.dv / f.rt;
  rho[p] = f.rt;                                                       // :436-442
  omega[p] = omega_f;
  divv[p] = div_v_p;
  drhodt[p] = -((f.rt * div_v_p) / omega_f);
  hz[p] = make_double2(hp, -((hp * f.zt) / ((NDIMPR * f.rt) * omega_f)));
  if (hp < 0.0) set_error(err, SEREN_GPU_ERR_NEGATIVE_H, KID_GRADH, p, 0);
}

__device__ __forceinline__ void gh_final_init(GhFinal& f, double mp, double ih, double hf,
                                              const double4& t0) {
  f.rt = (mp * t0.x) * hf;                                             // :323-346
  f.om = ((mp * hf) * ih) * t0.y;
  f.dv = 0.0;
  f.zt = ((mp * ih) * ih) * t0.w;
}

// ---------------------------------------------------------------------------
// Cell tests run first in FP32 on coordinates relative to the root centre:
// test32() decides when the FP32 distance is outside a margin around the
// threshold that covers every FP32 rounding involved (coordinates within
// delta, the difference, the squares, the sum and the threshold itself), and
// the test is redone in FP64 exactly as the reference writes it otherwise.
constexpr unsigned FULL = 0xffffffffu;

// 1: d2 <= T^2 for sure, 0: d2 > T^2 for sure, -1: too close to tell in FP32
__device__ __forceinline__ int test32(float d2, float T, float delta) {
  const float T2 = T * T;
  const float marg = fmaf(8.0f * delta, T, fmaf(16.0f * delta, delta, 1.0e-6f * T2));
  if (d2 < T2 - marg) return 1;
  if (d2 > T2 + marg) return 0;
  return -1;
}

__device__ __forceinline__ int warp_iscan(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, v, o);
    if (lane >= o) v += y;
  }
  return v;
}

// ---------------------------------------------------------------------------
// get_neib (sph/get_neib.F90:10-140): gather-or-scatter candidates
// (BHhydro_walk.F90:37-43), kept if r^2 <= 4h_p^2 or r^2 <= 4h_pp^2, in order.
__device__ void neib_one(int p, const double4* __restrict__ pm, const double2* __restrict__ hz,
                         const HydroTree& t, int L, int* __restrict__ pptot,
                         int* __restrict__ pplist, DevError* err) {
  const double4 P = pm[p];
  const double hp = hz[p].x;
  const double hsp = (KERNRANGESQD * hp) * hp;
  int cnt = 0;
  int* row = pplist + (size_t)p * L;
  walk_gather_scatter(t, frame_for(t, p).root, P.x, P.y, P.z, KERNRANGE * hp, err, p, [&](int q) {
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

// ---------------------------------------------------------------------------
// Group search.  A warp takes 32 consecutive active particles (tree order:
// spatially adjacent) and walks the tree for all of them at once: the walk
// state is a per-warp stack of (cell, mask) entries, the mask holding the
// lanes whose own walk reaches the cell; each step pops up to 32 entries,
// loads those cells in parallel, and every lane in an entry's mask runs its
// own particle's test on it (test32 in FP32, exact FP64 otherwise).  A cell
// that passes for some lanes is opened for exactly those lanes, so the leaves
// each lane opens are exactly those of its own reference walk.  Opened leaves
// go to a per-warp list of (leaf, mask) entries, from which each particle's
// own leaves are written to its row in global memory for the pass kernels.
constexpr int GR_THREADS = 128;
constexpr int GR_WARPS = GR_THREADS / 32;
constexpr int GR_LCAP = 512;     // (leaf, mask) entries per warp

struct GrShared {
  int code[GR_LCAP];       // leaf: pstart*8 + count-1
  unsigned mask[GR_LCAP];  // lanes whose walk opened the leaf
  float4 fa[32];           // popped cells: hA32
  float fh[32];            // hrm32
  unsigned fm[32];         // lanes whose walk reaches the cell
  int fc[32];
  int fu[32];              // popped cells the group test leaves undecided
};

// A group's bounding sphere in the walks' FP32 root-relative coordinates:
// centre the middle of the live lanes' bounding box, radius the farthest live
// lane's distance from it (rounded up), and
// the least and largest search radius over its live lanes.
struct GrGroup {
  float x, y, z, r, rmin, rmax;
};

__device__ __forceinline__ GrGroup gr_group(float px, float py, float pz, float R, bool live) {
  GrGroup g;
  {
    // centre: the middle of the live lanes' bounding box (lane 0 is live)
    const float x0 = __shfl_sync(0xffffffffu, px, 0), y0 = __shfl_sync(0xffffffffu, py, 0),
                z0 = __shfl_sync(0xffffffffu, pz, 0);
    float lox = live ? px : x0, loy = live ? py : y0, loz = live ? pz : z0;
    float hix = lox, hiy = loy, hiz = loz;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lox = fminf(lox, __shfl_xor_sync(0xffffffffu, lox, o));
      loy = fminf(loy, __shfl_xor_sync(0xffffffffu, loy, o));
      loz = fminf(loz, __shfl_xor_sync(0xffffffffu, loz, o));
      hix = fmaxf(hix, __shfl_xor_sync(0xffffffffu, hix, o));
      hiy = fmaxf(hiy, __shfl_xor_sync(0xffffffffu, hiy, o));
      hiz = fmaxf(hiz, __shfl_xor_sync(0xffffffffu, hiz, o));
    }
    g.x = 0.5f * (lox + hix);
    g.y = 0.5f * (loy + hiy);
    g.z = 0.5f * (loz + hiz);
  }
  const float e0 = px - g.x, e1 = py - g.y, e2 = pz - g.z;
  float r2 = live ? fmaf(e2, e2, fmaf(e1, e1, e0 * e0)) : 0.0f;
  float lo = live ? R : 3.0e38f, hi = live ? R : 0.0f;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    r2 = fmaxf(r2, __shfl_xor_sync(0xffffffffu, r2, o));
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  g.r = sqrtf(r2) * 1.00001f;
  g.rmin = lo;
  g.rmax = hi;
  return g;
}

// Group test of a popped cell (FP32 centre c.xyz, rmax c.w rounded up) for
// searches where a lane passes when its distance is at most its radius + c.w:
// 1 when the group's farthest possible point is within rlo + c.w (rlo: the
// least radius of any lane), 2 when its nearest possible point is beyond
// rhi + c.w (rhi: the largest), else 0.  The margin covers the FP32 rounding
// of coordinates (delta each), radii and arithmetic, so a decision is the
// exact FP64 one of every lane.
__device__ __forceinline__ int gr_decide(const GrGroup& g, const float4& c, float rlo, float rhi,
                                         float delta) {
  const float e0 = c.x - g.x, e1 = c.y - g.y, e2 = c.z - g.z;
  const float D = sqrtf(fmaf(e2, e2, fmaf(e1, e1, e0 * e0)));
  const float mg = fmaf(1.0e-5f, D + g.r + rhi + c.w, 4.0f * delta);
  if (D + g.r + mg < rlo + c.w) return 1;
  if (D - g.r - mg > rhi + c.w) return 2;
  return 0;
}

// Walk for the lanes in `lanes`, appending the opened leaves to R.code/R.mask
// from nent on.  gtest(hA32, hrm32) is the group test of a popped cell (1: it
// passes for every lane, 2: for none, 0: undecided); test(e) is this lane's
// test of undecided popped cell e (R.fa[e], R.fh[e], R.fc[e]).  Returns the
// new entry count, or -1 when the list or the stack would overflow (nothing
// beyond the old count is then valid).
template <class GTest, class Test>
__device__ int gr_walk(const HydroTree& t, int root, unsigned lanes, int2* S, int scap, GrShared& R,
                       int lane, int nent, unsigned long long& nvisit, GTest&& gtest,
                       Test&& test) {
  const unsigned lt = (1u << lane) - 1u;
  __syncwarp();
  if (lane == 0) S[0] = make_int2(root, (int)lanes);
  int sp = 1;
  long long gent = 0;
  while (sp > 0) {
    __syncwarp();
    const int k = min(32, sp);
    sp -= k;
    gent += k;
    int cnt = 0, base = 0;           // cnt: leaf particles, or -children of a branch
    unsigned m = 0;
    int dec = 0;
    if (lane < k) {
      const int2 ent = S[sp + lane];
      const int cc = ent.x;
      m = (unsigned)ent.y;
      const float4 na = t.hN[2 * cc], nb2 = t.hN[2 * cc + 1];
      cnt = __float_as_int(nb2.z);
      base = __float_as_int(nb2.y);
      R.fa[lane] = na;
      R.fh[lane] = nb2.x;
      R.fm[lane] = m;
      R.fc[lane] = cc;
      dec = gtest(na, nb2.x);
    }
    unsigned mpass = dec == 1 ? m : 0u;
    const unsigned und = __ballot_sync(FULL, lane < k && dec == 0);
    if (lane < k && dec == 0) R.fu[__popc(und & lt)] = lane;
    __syncwarp();
    for (unsigned u = und; u != 0u; u &= u - 1u) {         // the undecided cells, lane by lane
      const int e = __ffs(u) - 1;
      const bool pass = ((R.fm[e] >> lane) & 1u) && test(e);
      const unsigned b = __ballot_sync(FULL, pass);
      if (lane == e) mpass = b;
    }
    nvisit += k;
    const bool isleaf = cnt > 0 && mpass != 0u;               // candidates of the lanes in mpass
    const unsigned bl = __ballot_sync(FULL, isleaf);
    if (nent + __popc(bl) > GR_LCAP) return -1;
    if (isleaf) {
      const int o = nent + __popc(bl & lt);
      R.code[o] = base * 8 + (cnt - 1);
      R.mask[o] = mpass;
    }
    nent += __popc(bl);
    const int nch = (cnt < 0 && mpass != 0u) ? -cnt : 0;      // opened for the lanes in mpass
    const int cin = warp_iscan(nch, lane);
    const int ctotal = __shfl_sync(FULL, cin, 31);
    if (sp + ctotal > scap || gent > (long long)t.ctot + 1) return -1;
    for (int q = 0; q < nch; ++q) S[sp + cin - nch + q] = make_int2(base + q, (int)mpass);
    sp += ctotal;
  }
  __syncwarp();
  return nent;
}

// ascending bitonic sort of the entries by leaf (depth-first leaf order, the
// order of the reference's candidate lists), masks carried along
__device__ void gr_sort(GrShared& R, int n, int lane) {
  int N = 1;
  while (N < n) N <<= 1;
  for (int k = n + lane; k < N; k += 32) {
    R.code[k] = 0x7fffffff;
    R.mask[k] = 0u;
  }
  __syncwarp();
  for (int size = 2; size <= N; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < (N >> 1); i += 32) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const int x = R.code[lo], y = R.code[hi];
        if ((x > y) == up) {
          const unsigned mx = R.mask[lo], my = R.mask[hi];
          R.code[lo] = y; R.code[hi] = x;
          R.mask[lo] = my; R.mask[hi] = mx;
        }
      }
      __syncwarp();
    }
  }
}

// sum over the warp, the same value on every lane
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
  return __shfl_sync(FULL, v, 0);
}

__device__ __forceinline__ int gr_next(int* work, int lane) {
  int g = 0;
  if (lane == 0) g = atomicAdd(work, 1);
  return __shfl_sync(FULL, g, 0);
}

// sph/all_sph_gradh.F90:11-492 in two kernels.
//
// k_gradh_walk: the first neighbour walk of every active particle
// (:154-170, BHhydrowalk_hgather at h_high = h*HMULT), 32 particles per warp
// on a group walk; each particle's opened leaves go to its own row of
// c.leaves (GH_LEAVES codes pstart*8 + count-1, in walk order) and their
// number to c.nleaf (-1 when the row or the walk overflows).
//
// k_gradh_pass: 32 particles per warp, each lane holding its particle's state;
// the reference's iteration (:154-285) and final pass (:317-425) run with the
// candidates of one particle at a time (its row flattened) shared out over the
// lanes and the sums reduced across the warp.  The reference leaves this path
// only to grow h (pp_pot < pp_gather) or to walk again (h > h_high); a
// particle that needs either, or whose row overflowed, is redone from the
// start with walks of its own, which take the reference's steps in the same
// order: k_gradh_redo (one warp per particle, walk buffers in global scratch)
// and, for walks too large for those buffers, k_gradh_wide (one block per
// particle, walks split over subtrees).
constexpr int GH_LEAVES = 256;   // opened leaves kept per particle

__global__ void __launch_bounds__(GR_THREADS) k_gradh_walk(
    int nact, const int* __restrict__ act, const double4* __restrict__ pm,
    const double2* __restrict__ hz, HydroTree t, int* __restrict__ leaves,
    int* __restrict__ nleaf, int* __restrict__ npot, int2* __restrict__ stacks, int scap,
    unsigned long long* counts, int* work) {
  extern __shared__ __align__(16) unsigned char gr_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  GrShared& R = reinterpret_cast<GrShared*>(gr_smem)[w];
  int2* const S = stacks + (size_t)(blockIdx.x * GR_WARPS + w) * scap;
  const unsigned bit = 1u << lane;
  unsigned long long nvisit = 0;
  unsigned nwalk = 0;
  for (int g = gr_next(work, lane); (long long)g * 32 < nact; g = gr_next(work, lane)) {
    const int i = g * 32 + lane;
    bool live;
    const int p = group_particle(i, nact, act, live);
    const TreeFrame fr = frame_for(t, p);             // lanes share one cloud
    const double4 P = pm[p];
    const double rx = P.x, ry = P.y, rz = P.z;
    const float px = (float)(rx - fr.rootx), py = (float)(ry - fr.rooty), pz = (float)(rz - fr.rootz);
    const double Rw = KERNRANGE * (hz[p].x * HMULT);                  // :157-158
    const float R32 = (float)Rw;
    const unsigned lanes = __ballot_sync(FULL, live);
    nwalk += live ? 1u : 0u;
    const GrGroup grp = gr_group(px, py, pz, R32, live);
    const int nent = gr_walk(t, fr.root, lanes, S, scap, R, lane, 0, nvisit, [&](const float4& c, float) {
      return gr_decide(grp, c, grp.rmin, grp.rmax, fr.delta);
    }, [&](int e) {
      const float4 h32 = R.fa[e];                      // BHhydrowalk_hgather.F90:36-40
      const float d0 = h32.x - px, d1 = h32.y - py, d2 = h32.z - pz;
      const int r = test32((d0 * d0 + d1 * d1) + d2 * d2, R32 + h32.w, fr.delta);
      if (r >= 0) return r == 1;
      const double4 h = t.hA[R.fc[e]];
      const double e0 = h.x - rx, e1 = h.y - ry, e2 = h.z - rz;
      const double tt = Rw + h.w;
      return ((e0 * e0 + e1 * e1) + e2 * e2) <= tt * tt;
    });
    int n = -1, pot = 0;
    if (nent >= 0) {
      n = 0;
      int* row = leaves + (size_t)p * GH_LEAVES;
      for (int e = 0; e < nent; ++e) {
        if (R.mask[e] & bit) {
          const int code = R.code[e];
          if (n < GH_LEAVES) row[n] = code;
          ++n;
          pot += (code & 7) + 1;                        // pp_pot, :168
        }
      }
      if (n > GH_LEAVES) n = -1;
    }
    if (live) {
      nleaf[p] = n;
      npot[p] = pot;
    }
    __syncwarp();
  }
  atomicAdd(counts + 3, (unsigned long long)nwalk);
  if (lane == 0) atomicAdd(counts + 4, nvisit);
}

constexpr int GP_THREADS = 128;
constexpr int GP_WARPS = GP_THREADS / 32;
constexpr int GP_SEG = 64;       // leaves of a row flattened at a time

// The density term (:218-230) and the final-pass terms (:360-425) of one
// candidate inside 2h, from its r^2, mass and dv.dr, with the reference's
// operations in its order; the kernel bin is int(5000 r/h) with
// r = sqrt(r^2) + 1e-20, its value evaluated in place (kernel_fns.h, equal to
// the table entry).
__device__ __forceinline__ void gh_density_in(double d2, double m, double ih, double hf,
                                              double& rt) {
  const double drmag = sqrt(d2) + SMALL_NUMBER;
  const int kern = (int)((HALFKERNTOT * drmag) * ih);
  if (kern >= KERNTOT) return;
  rt = rt + (m * hf) * kfn::w0(kern);
}

__device__ __forceinline__ void gh_final_in(double d2, double m, double dvdr, double ih,
                                            double hf, GhFinal& f) {
  const double drmag = sqrt(d2) + SMALL_NUMBER;
  const int kern = (int)((HALFKERNTOT * drmag) * ih);
  if (kern > KERNTOT) return;
  f.rt = f.rt + (m * hf) * kfn::w0(kern);
  f.om = f.om + ((m * hf) * ih) * kfn::wh(kern);
  f.dv = f.dv - ((((m * dvdr) * kfn::w4(kern)) * hf) * ih) / drmag;
  f.zt = f.zt + ((m * ih) * ih) * kfn::wg(kern);
}

// A particle's row of opened leaves flattened into its candidates, in order;
// returns the count.
__device__ __forceinline__ int gp_flatten(const int* __restrict__ row, int n, int* cand,
                                          int lane) {
  int total = 0;
  __syncwarp();
  for (int base = 0; base < n; base += 32) {
    const int k = base + lane;
    int code = 0, c = 0;
    if (k < n) {
      code = row[k];
      c = (code & 7) + 1;
    }
    const int inc = warp_iscan(c, lane);
    const int o = total + inc - c;
    for (int j = 0; j < c; ++j) cand[o + j] = (code >> 3) + j;
    total += __shfl_sync(FULL, inc, 31);
  }
  __syncwarp();
  return total;
}

constexpr int GP_PSEG = 32;      // k_gradh_pass: leaves of a row flattened at a time
constexpr int GP_PINB = 128;     // k_gradh_pass: packed in-range candidates per warp

template <int N>
using ICst = std::integral_constant<int, N>;

// k_gradh_pass's per-warp shared state: the group's per-particle values that
// the candidate loops read for one particle at a time (broadcast loads), a
// flattened row segment, and the packed in-range candidates.
struct GpWarp {
  double x[32], y[32], z[32];
  double hs[32], ih[32], hf[32];   // (2h)^2, 1/h, 1/h^3 of the pass in progress
  double hh[32];                   // (2 h_high)^2: radius of the recorded candidates
  int p[32], n[32], npr[32];       // particle, leaves in its row, recorded candidates (-1: none)
  unsigned cpl;                    // lanes whose final-pass candidates hold every particle within 2h
  int cand[GP_PSEG * LEAFMAX];
  double d2[GP_PINB], m[GP_PINB], dv[GP_PINB];
};

// 32 consecutive particles per warp: each lane holds its particle's iteration
// state, so the per-particle arithmetic of a pass (h, its powers, the update
// of :238-285) runs once per lane for all 32; each particle's candidates are
// shared out over the 32 lanes in turn, 32*U at a time with all their loads
// issued together (U = 4 for the recorded candidates of the density passes).
__global__ void __launch_bounds__(GP_THREADS, 8) k_gradh_pass(
    int nact, const int* __restrict__ act, const double4* __restrict__ pm, double2* __restrict__ hz,
    const double4* __restrict__ vel, double* __restrict__ rho, double* __restrict__ omega,
    double* __restrict__ divv, double* __restrict__ drhodt, const double4* __restrict__ tabA,
    double h_fac, int pp_gather, double rextent0, const int* __restrict__ leaves,
    const int* __restrict__ nleaf, int* __restrict__ npot, int* __restrict__ redo,
    int* __restrict__ nredo, int* __restrict__ prune, int L, DevError* err,
    unsigned long long* counts, int* work, const CloudInfo* __restrict__ cl, int ncl, int rec,
    int* __restrict__ pptot) {
  __shared__ GpWarp gpw[GP_WARPS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  GpWarp& W = gpw[w];
  const unsigned lt = (1u << lane) - 1u;
  unsigned npass = 0, ncands = 0, niter = 0, nsingle = 0;

  // Density sum (:211-235) of particle j over the candidates getq(0..nc): r^2
  // of each; those inside 2h (:218) are packed into the buffer and their terms
  // summed 32 at a time.  KEEP (first pass): the candidates within 2 h_high
  // are recorded, in order, in j's row of `prune`.
  auto dscan = [&](int j, int nc, auto getq, auto u_, auto keep_, int& kept, double& part) {
    constexpr int U = decltype(u_)::value;
    constexpr bool KEEP = decltype(keep_)::value;
    const double xj = W.x[j], yj = W.y[j], zj = W.z[j], hsj = W.hs[j];
    const int pj = W.p[j];
    int nin = 0;
    for (int b = 0; b < nc; b += 32 * U) {
      int q[U];
      double4 Q[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = b + 32 * u + lane;
        q[u] = k < nc ? getq(k) : pj;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) Q[u] = pm[q[u]];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const double d0 = Q[u].x - xj, d1 = Q[u].y - yj, d2 = Q[u].z - zj;
        const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
        const bool in = q[u] != pj && drsqd < hsj;
        const unsigned mi = __ballot_sync(FULL, in);
        if (in) {
          const int o = nin + __popc(mi & lt);
          W.d2[o] = drsqd;
          W.m[o] = Q[u].w;
        }
        nin += __popc(mi);
        if constexpr (KEEP) {
          const bool keep = q[u] != pj && drsqd < W.hh[j];
          const unsigned mk = __ballot_sync(FULL, keep);
          const int pos = kept + __popc(mk & lt);
          if (keep && pos < L) prune[(size_t)pj * L + pos] = q[u];
          kept += __popc(mk);
        }
      }
      if (nin > GP_PINB - 32 * U || b + 32 * U >= nc) {
        __syncwarp();
        const double ihj = W.ih[j], hfj = W.hf[j];
        for (int t = lane; t < nin; t += 32) gh_density_in(W.d2[t], W.m[t], ihj, hfj, part);
        nin = 0;
        __syncwarp();
      }
    }
    niter += (nc + 31) >> 5;
  };

  // Final-pass sums (:360-425) of particle j over the candidates getq(0..nc),
  // its velocity vj
  auto fscan = [&](int j, int nc, auto getq, auto u_, double vxj, double vyj, double vzj,
                   GhFinal& part, int& gcnt) {
    constexpr int U = decltype(u_)::value;
    const double xj = W.x[j], yj = W.y[j], zj = W.z[j], hsj = W.hs[j];
    const int pj = W.p[j];
    int nin = 0;
    for (int b = 0; b < nc; b += 32 * U) {
      int q[U];
      double4 Q[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int k = b + 32 * u + lane;
        q[u] = k < nc ? getq(k) : pj;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) Q[u] = pm[q[u]];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const double d0 = Q[u].x - xj, d1 = Q[u].y - yj, d2 = Q[u].z - zj;
        const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
        const bool in = q[u] != pj && drsqd <= hsj;                   // :360
        const unsigned mi = __ballot_sync(FULL, in);
        if (in) {
          const double4 V = vel[q[u]];
          const double dv0 = V.x - vxj, dv1 = V.y - vyj, dv2 = V.z - vzj;
          const int o = nin + __popc(mi & lt);
          W.d2[o] = drsqd;
          W.m[o] = Q[u].w;
          W.dv[o] = (dv0 * d0 + dv1 * d1) + dv2 * d2;
          // the gather neighbours r^2 <= 4h^2 of the neighbour lists, in
          // order, into the particle's own row of prune: each goes to a slot
          // at or before the candidate it came from, whose read is done (the
          // ballot above waits for every lane's candidate), so no candidate
          // still to be read is overwritten
          if (rec && gcnt + o < L) prune[(size_t)pj * L + gcnt + o] = q[u];
        }
        nin += __popc(mi);
      }
      if (nin > GP_PINB - 32 * U || b + 32 * U >= nc) {
        __syncwarp();
        gcnt += nin;
        const double ihj = W.ih[j], hfj = W.hf[j];
        for (int t = lane; t < nin; t += 32)
          gh_final_in(W.d2[t], W.m[t], W.dv[t], ihj, hfj, part);
        nin = 0;
        __syncwarp();
      }
    }
    niter += (nc + 31) >> 5;
  };

  for (int g = gr_next(work, lane); (long long)g * 32 < nact; g = gr_next(work, lane)) {
    const int i = g * 32 + lane;
    bool live;
    const int p = group_particle(i, nact, act, live);
    const double rextent = cl ? cl[cloud_of(cl, ncl, p)].rextent : rextent0;
    const int n = live ? nleaf[p] : 0;
    const double4 P = pm[p];
    const double mp = P.w;
    GhState s;
    gh_init(s, hz[p].x, rextent);
    s.h_high = s.hp * HMULT;                                           // :157-170
    s.pp_pot = n >= 0 ? npot[p] : 0;
    bool single = live && (n < 0 || s.pp_pot < pp_gather);             // :175-181 would grow h
    bool active = live && !single;
    __syncwarp();                                      // the previous group's reads are done
    W.x[lane] = P.x;
    W.y[lane] = P.y;
    W.z[lane] = P.z;
    // The candidates within 2 h_high of the particle, recorded in its row of
    // `prune` by the first pass: every later pass has h <= h_high (else the
    // particle walks again), so they hold all the candidates it can count.
    W.hh[lane] = (KERNRANGESQD * s.h_high) * s.h_high;
    W.p[lane] = p;
    W.n[lane] = n;
    W.npr[lane] = -1;
    bool first = true;
    double rt = 0.0;
    while (true) {
      const unsigned A = __ballot_sync(FULL, active);
      if (A == 0u) break;
      const double ih = 1.0 / s.hp;                                    // :199-235
      const double hf = pow(ih, NDIMPR);
      W.ih[lane] = ih;
      W.hf[lane] = hf;
      W.hs[lane] = (KERNRANGESQD * s.hp) * s.hp;
      __syncwarp();
      for (unsigned todo = A; todo != 0u; todo &= todo - 1u) {
        const int j = __ffs(todo) - 1;
        double part = 0.0;
        int kept = 0;
        const int nprj = W.npr[j];
        if (first || nprj < 0) {
          const int nj = W.n[j];
          const int* row = leaves + (size_t)W.p[j] * GH_LEAVES;
          for (int s0 = 0; s0 < nj; s0 += GP_PSEG) {   // the row, GP_PSEG leaves at a time
            const int nc = gp_flatten(row + s0, min(GP_PSEG, nj - s0), W.cand, lane);
            auto fromrow = [&](int k) { return W.cand[k]; };
            if (first) dscan(j, nc, fromrow, ICst<2>{}, std::true_type{}, kept, part);
            else dscan(j, nc, fromrow, ICst<2>{}, std::false_type{}, kept, part);
          }
          if (first && lane == 0) W.npr[j] = kept <= L ? kept : -1;
        } else {
          const int* prj = prune + (size_t)W.p[j] * L;
          dscan(j, nprj, [&](int k) { return prj[k]; }, ICst<4>{}, std::false_type{}, kept,
                part);
        }
        const double sum = warp_sum(part);
        if (lane == j) rt = sum;
      }
      first = false;
      if (active) {
        ++npass;
        ncands += s.pp_pot;
        if (gh_after_pass(s, mp, h_fac, rextent, (mp * tabA[0].x) * hf + rt)) active = false;
        else if (s.hp > s.h_high) {                                    // :154-170 would walk again
          single = true;
          active = false;
        }
      }
      __syncwarp();
    }
    // final pass (:317-425)
    const bool ok = live && !single;
    const unsigned F = __ballot_sync(FULL, ok);
    const double hp = h_fac * pow(mp / s.rho, ONETHIRD);
    const double ih = 1.0 / hp;
    const double hf = pow(ih, NDIMPR);
    const double4 vp = vel[p];
    W.ih[lane] = ih;
    W.hf[lane] = hf;
    W.hs[lane] = (KERNRANGESQD * hp) * hp;
    // the recorded candidates serve when 2h < 2 h_high (those within 2h of the
    // final h are among them)
    if (!(hp < s.h_high)) W.npr[lane] = -1;
    const unsigned cplm = __ballot_sync(FULL, hp < s.h_high);
    __syncwarp();
    GhFinal f;
    gh_final_init(f, mp, ih, hf, tabA[0]);
    for (unsigned todo = F; todo != 0u; todo &= todo - 1u) {
      const int j = __ffs(todo) - 1;
      const double vxj = __shfl_sync(FULL, vp.x, j), vyj = __shfl_sync(FULL, vp.y, j),
                   vzj = __shfl_sync(FULL, vp.z, j);
      const int nprj = W.npr[j];
      GhFinal part;
      part.rt = 0.0; part.om = 0.0; part.dv = 0.0; part.zt = 0.0;
      int gcnt = 0;
      if (nprj < 0) {
        const int nj = W.n[j];
        const int* row = leaves + (size_t)W.p[j] * GH_LEAVES;
        for (int s0 = 0; s0 < nj; s0 += GP_PSEG) {     // the row, GP_PSEG leaves at a time
          const int nc = gp_flatten(row + s0, min(GP_PSEG, nj - s0), W.cand, lane);
          fscan(j, nc, [&](int k) { return W.cand[k]; }, ICst<1>{}, vxj, vyj, vzj, part, gcnt);
        }
      } else {
        const int* prj = prune + (size_t)W.p[j] * L;
        fscan(j, nprj, [&](int k) { return prj[k]; }, ICst<2>{}, vxj, vyj, vzj, part, gcnt);
      }
      // the gather count (the row's first entries; pptot grows with the
      // scatter neighbours later), or -1 when the candidates may miss some
      // particle within 2h (h >= h_high: the neighbour walk completes the row)
      if (rec && lane == 0) {
        const int pj = W.p[j];
        if ((cplm >> j) & 1u) {
          npot[pj] = gcnt;
          pptot[pj] = gcnt;
        } else {
          npot[pj] = -1;
        }
      }
      const double srt = warp_sum(part.rt), som = warp_sum(part.om), sdv = warp_sum(part.dv),
                   szt = warp_sum(part.zt);
      if (lane == j) {
        f.rt = f.rt + srt;
        f.om = f.om + som;
        f.dv = f.dv + sdv;
        f.zt = f.zt + szt;
      }
    }
    if (ok) {
      ++npass;
      ncands += s.pp_pot;
      gh_store(p, mp, hp, f, hz, rho, omega, divv, drhodt, err);
    }
    if (single) {
      ++nsingle;
      redo[atomicAdd(nredo, 1)] = p;
      if (rec) npot[p] = -1;                       // its neighbour list: from a walk
    }
  }
  atomicAdd(counts + 5, (unsigned long long)npass);
  atomicAdd(counts + 6, (unsigned long long)ncands);
  atomicAdd(counts + 15, (unsigned long long)nsingle);
  if (lane == 0) atomicAdd(counts + 13, (unsigned long long)niter);
}

// ---------------------------------------------------------------------------
// grad-h for the particles k_gradh_pass hands back (redo[0..*nredo)): one warp
// per particle runs the reference's loop (:132-425) with walks of its own.  A
// walk runs breadth-first with the lanes spread over the cells of a level; its
// two frontiers and the opened leaves live in global scratch (three walk-stack
// slots per warp, idle while this kernel runs), and the passes flatten the
// leaves GP_SEG at a time and share the candidates out over the lanes.
constexpr int RD_THREADS = 128;
constexpr int RD_WARPS = RD_THREADS / 32;

// Breadth-first walk of one particle's search (BHhydrowalk_hgather); returns
// the number of opened leaves (codes pstart*8 + count-1 in leaves, in no
// particular order) or -1 when a buffer of cap entries would overflow; cnt =
// the particles in the opened leaves (pp_pot).
template <class Test>
__device__ int rd_walk(const HydroTree& t, int root, int lane, int* fa, int* fb, int* leaves, int cap,
                       int& cnt, unsigned long long& nvisit, Test&& test) {
  __syncwarp();
  if (lane == 0) fa[0] = root;
  __syncwarp();
  int nf = 1, nleaf = 0, mine = 0;
  while (nf > 0) {
    int nnext = 0;
    for (int base = 0; base < nf; base += 32) {
      const int idx = base + lane;
      const bool valid = idx < nf;
      const int c = valid ? fa[idx] : 0;
      const bool pass = valid && test(c);
      const int4 lk = t.link[c];
      const bool isleaf = pass && lk.x > 0;
      const bool isbr = pass && lk.x == 0;
      const unsigned ml = __ballot_sync(FULL, isleaf);
      if (isleaf) {
        const int pos = nleaf + __popc(ml & ((1u << lane) - 1u));
        if (pos < cap) leaves[pos] = lk.w * 8 + (lk.x - 1);
        mine += lk.x;
      }
      nleaf += __popc(ml);
      const int nk = isbr ? t.nkids[c] : 0;
      const int sc = warp_iscan(nk, lane);
      if (isbr) {
        const int o = nnext + sc - nk;
        for (int j = 0; j < nk; ++j)
          if (o + j < cap) fb[o + j] = lk.z + j;
      }
      nnext += __shfl_sync(FULL, sc, 31);
    }
    nvisit += nf;
    __syncwarp();
    if (nnext > cap || nleaf > cap) return -1;
    int* tmp = fa;
    fa = fb;
    fb = tmp;
    nf = nnext;
  }
  cnt = __shfl_sync(FULL, warp_iscan(mine, lane), 31);
  return nleaf;
}

__global__ void __launch_bounds__(RD_THREADS) k_gradh_redo(
    const int* __restrict__ redo, const int* __restrict__ nredo, const double4* __restrict__ pm,
    double2* __restrict__ hz, const double4* __restrict__ vel, double* __restrict__ rho,
    double* __restrict__ omega, double* __restrict__ divv, double* __restrict__ drhodt,
    HydroTree t, const double4* __restrict__ tabA, double h_fac, int pp_gather, double rextent0,
    int* __restrict__ scratch, int cap, int* __restrict__ wide, int* __restrict__ nwide,
    int* __restrict__ leaves, DevError* err, unsigned long long* counts) {
  __shared__ int cand_all[RD_WARPS][GP_SEG * LEAFMAX];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int* cand = cand_all[w];
  const int gw = blockIdx.x * RD_WARPS + w;
  int* fa = scratch + (size_t)gw * 3 * cap;
  int* fb = fa + cap;
  int* lv = fb + cap;
  const double4 t0 = tabA[0];
  unsigned long long nwalk = 0, nvisit = 0, npass = 0, ncands = 0;
  const int nr = *nredo;
  for (int i = gw; i < nr; i += gridDim.x * RD_WARPS) {
    const int p = redo[i];
    const TreeFrame fr = frame_for(t, p);
    const double rextent = t.cl ? fr.rextent : rextent0;
    const double4 P = pm[p];
    const double rx = P.x, ry = P.y, rz = P.z, mp = P.w;
    const float px = (float)(rx - fr.rootx), py = (float)(ry - fr.rooty), pz = (float)(rz - fr.rootz);
    GhState s;
    gh_init(s, hz[p].x, rextent);
    double Rw = 0.0;
    float R32 = 0.0f;
    auto gather_test = [&](int c) {                    // BHhydrowalk_hgather.F90:36-40
      const float4 h32 = t.hA32[c];
      const float d0 = h32.x - px, d1 = h32.y - py, d2 = h32.z - pz;
      const int r = test32((d0 * d0 + d1 * d1) + d2 * d2, R32 + h32.w, fr.delta);
      if (r >= 0) return r == 1;
      const double4 h = t.hA[c];
      const double e0 = h.x - rx, e1 = h.y - ry, e2 = h.z - rz;
      const double tt = Rw + h.w;
      return ((e0 * e0 + e1 * e1) + e2 * e2) <= tt * tt;
    };
    int nl = 0;
    bool over = false, bad = false;
    while (true) {
      while (true) {                                                   // :154-191
        if (s.hp > s.h_high) {
          s.h_high = s.hp * HMULT;
          Rw = KERNRANGE * s.h_high;
          R32 = (float)Rw;
          int cnt = 0;
          ++nwalk;
          nl = rd_walk(t, fr.root, lane, fa, fb, lv, cap, cnt, nvisit, gather_test);
          if (nl < 0) { over = true; break; }
          s.pp_pot = cnt;
        }
        if (s.pp_pot < pp_gather) {
          s.h_high = 0.0;
          s.pp_pot = 0;
          s.hp = s.hp * HMULT;
          if (++s.ngrow > HGROW_CAP) { bad = true; break; }
        }
        if (s.pp_pot > 0) break;
      }
      if (over || bad) break;
      const double ih = 1.0 / s.hp;                                    // :199-235
      const double hf = pow(ih, NDIMPR);
      const double hs = (KERNRANGESQD * s.hp) * s.hp;
      double part = 0.0;
      for (int s0 = 0; s0 < nl; s0 += GP_SEG) {
        const int nc = gp_flatten(lv + s0, min(GP_SEG, nl - s0), cand, lane);
        for (int k = lane; k < nc; k += 32) {
          const int q = cand[k];
          const double4 Q = pm[q];
          const double d0 = Q.x - rx, d1 = Q.y - ry, d2 = Q.z - rz;
          const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
          if (q != p && drsqd < hs) gh_density_in(drsqd, Q.w, ih, hf, part);
        }
      }
      ++npass;
      ncands += s.pp_pot;
      if (gh_after_pass(s, mp, h_fac, rextent, (mp * t0.x) * hf + warp_sum(part))) break;
    }
    if (bad) {
      if (lane == 0) set_error(err, SEREN_GPU_ERR_WALK, KID_GRADH, p, -1);
      continue;
    }
    if (over) {                                        // more than cap leaves or cells a level
      // the whole-GPU path takes the particle from here: its state goes to
      // its leaf row (no longer read once the particle is redone), and its
      // next step is the counting walk at s.h_high that outgrew the scratch
      if (lane == 0) {
        *reinterpret_cast<GhState*>(leaves + (size_t)p * GH_LEAVES) = s;
        wide[atomicAdd(nwide, 1)] = p;
      }
      continue;
    }
    const double hp = h_fac * pow(mp / s.rho, ONETHIRD);              // :317-425
    const double ih = 1.0 / hp;
    const double hf = pow(ih, NDIMPR);
    const double hs = (KERNRANGESQD * hp) * hp;
    const double4 vp = vel[p];
    GhFinal f;
    f.rt = 0.0; f.om = 0.0; f.dv = 0.0; f.zt = 0.0;
    for (int s0 = 0; s0 < nl; s0 += GP_SEG) {
      const int nc = gp_flatten(lv + s0, min(GP_SEG, nl - s0), cand, lane);
      for (int k = lane; k < nc; k += 32) {
        const int q = cand[k];
        const double4 Q = pm[q];
        const double d0 = Q.x - rx, d1 = Q.y - ry, d2 = Q.z - rz;
        const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
        if (q == p || drsqd > hs) continue;
        const double4 V = vel[q];
        const double dv0 = V.x - vp.x, dv1 = V.y - vp.y, dv2 = V.z - vp.z;
        gh_final_in(drsqd, Q.w, (dv0 * d0 + dv1 * d1) + dv2 * d2, ih, hf, f);
      }
    }
    ++npass;
    ncands += s.pp_pot;
    GhFinal g;
    gh_final_init(g, mp, ih, hf, t0);
    g.rt = g.rt + warp_sum(f.rt);
    g.om = g.om + warp_sum(f.om);
    g.dv = g.dv + warp_sum(f.dv);
    g.zt = g.zt + warp_sum(f.zt);
    if (lane == 0) gh_store(p, mp, hp, g, hz, rho, omega, divv, drhodt, err);
  }
  if (lane == 0) {
    atomicAdd(counts + 3, nwalk);
    atomicAdd(counts + 4, nvisit);
    atomicAdd(counts + 5, npass);
    atomicAdd(counts + 6, ncands);
  }
}

// ---------------------------------------------------------------------------
// sph/h_gather.F90:14-203 (standard SPH: h from exactly pp_gather neighbours).
// The reference narrows [h_low, h_high] until 2h_low holds fewer than
// pp_gather other particles and 2h_high at least pp_gather (:143-162), then
// sorts the squared distances of the annulus between them and takes the
// (pp_gather - pp_low)-th (:179-183).  The pp_low particles inside 2h_low are
// all nearer, so the result is h = INVKERNRANGE*sqrt(d2), d2 the pp_gather-th
// smallest squared distance (r_pp - r_p, distance2.F90's order of terms) from
// p to any other particle: it does not depend on the guess or on the path the
// limits take.  One warp per particle finds that value directly: walks with
// BHhydrowalk_hgather's test (the redo kernel's breadth-first walk) at a
// radius R that grows until the ball r < R holds at least pp_gather others
// (shrinking when it holds more than the selection buffer), then a bitonic
// sort in shared memory of the squared distances inside the ball.
constexpr int HG_THREADS = 128;
constexpr int HG_WARPS = HG_THREADS / 32;
constexpr int HG_SEL = 1024;       // squared distances sorted per particle at most
constexpr int HG_ROUNDS = 400;     // radius changes per particle at most

__device__ void hg_sort(double* v, int n, int lane) {
  int N = 32;
  while (N < n) N <<= 1;
  for (int k = n + lane; k < N; k += 32) v[k] = INFINITY;
  __syncwarp();
  for (int size = 2; size <= N; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < (N >> 1); i += 32) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const double x = v[lo], y = v[hi];
        if ((x > y) == up) {
          v[lo] = y;
          v[hi] = x;
        }
      }
      __syncwarp();
    }
  }
}

__global__ void __launch_bounds__(HG_THREADS) k_hgather(
    int nact, const int* __restrict__ act, const double4* __restrict__ pm,
    double2* __restrict__ hz, HydroTree t, int pp_gather, double rextent0,
    int* __restrict__ scratch, int cap, DevError* err, unsigned long long* counts) {
  __shared__ double sel_all[HG_WARPS][HG_SEL];
  __shared__ int cand_all[HG_WARPS][GP_SEG * LEAFMAX];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* sel = sel_all[w];
  int* cand = cand_all[w];
  const int gw = blockIdx.x * HG_WARPS + w;
  int* fa = scratch + (size_t)gw * 3 * cap;
  int* fb = fa + cap;
  int* lv = fb + cap;
  const unsigned lt = (1u << lane) - 1u;
  unsigned long long nwalk = 0, nvisit = 0;
  for (int i = gw; i < nact; i += gridDim.x * HG_WARPS) {
    const int p = act ? act[i] : i;
    const TreeFrame fr = frame_for(t, p);
    const double rextent = t.cl ? fr.rextent : rextent0;
    const double rcap = 4.0 * (rextent > 0.0 ? rextent : 1.0);   // a ball that holds every particle
    const double4 P = pm[p];
    const double rx = P.x, ry = P.y, rz = P.z;
    const float px = (float)(rx - fr.rootx), py = (float)(ry - fr.rooty), pz = (float)(rz - fr.rootz);
    double Rw = KERNRANGE * (HMULT * (HMULT * hz[p].x));    // the reference's first search radius
    if (!(Rw > 0.0) || !isfinite(Rw)) Rw = ldexp(rcap, -12);  // the guess does not change h
    float R32 = 0.0f;
    auto gather_test = [&](int c) {                     // BHhydrowalk_hgather.F90:36-40
      const float4 h32 = t.hA32[c];
      const float d0 = h32.x - px, d1 = h32.y - py, d2 = h32.z - pz;
      const int r = test32((d0 * d0 + d1 * d1) + d2 * d2, R32 + h32.w, fr.delta);
      if (r >= 0) return r == 1;
      const double4 h = t.hA[c];
      const double e0 = h.x - rx, e1 = h.y - ry, e2 = h.z - rz;
      const double tt = Rw + h.w;
      return ((e0 * e0 + e1 * e1) + e2 * e2) <= tt * tt;
    };
    double Rlo = 0.0;            // a radius known to hold fewer than pp_gather others
    double Rhi = INFINITY;       // a radius known to hold more than HG_SEL others (or to overflow)
    bool done = false;
    for (int round = 0; round < HG_ROUNDS && !done; ++round) {
      if (!(Rw > 0.0) || !isfinite(Rw)) break;
      R32 = (float)Rw;
      int cnt = 0;
      ++nwalk;
      const int nl = rd_walk(t, fr.root, lane, fa, fb, lv, cap, cnt, nvisit, gather_test);
      // the opened leaves hold every particle with r <= Rw; count those well
      // inside (r^2 below Rw^2 (1 - 2^-40), clear of the walk's rounding)
      const double rc2 = (Rw * Rw) * (1.0 - 0x1p-40);
      int nin = 0;
      if (nl >= 0) {
        for (int s0 = 0; s0 < nl; s0 += GP_SEG) {
          const int nc = gp_flatten(lv + s0, min(GP_SEG, nl - s0), cand, lane);
          for (int b = 0; b < nc; b += 32) {
            const int k = b + lane;
            double drsqd = 0.0;
            bool in = false;
            if (k < nc) {
              const int q = cand[k];
              const double4 Q = pm[q];
              const double d0 = Q.x - rx, d1 = Q.y - ry, d2 = Q.z - rz;   // distance2.F90
              drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
              in = q != p && drsqd < rc2;
            }
            const unsigned mi = __ballot_sync(FULL, in);
            const int o = nin + __popc(mi & lt);
            if (in && o < HG_SEL) sel[o] = drsqd;
            nin += __popc(mi);
          }
        }
      }
      double Rn;
      if (nl >= 0 && nin >= pp_gather && nin <= HG_SEL) {
        hg_sort(sel, nin, lane);
        if (lane == 0) hz[p].x = INVKERNRANGE * sqrt(sel[pp_gather - 1]);   // :182-183
        done = true;
        __syncwarp();
        break;
      } else if (nl >= 0 && nin < pp_gather) {
        Rlo = Rw;
        if (Rw > rcap) break;                          // fewer than pp_gather others exist
        Rn = isfinite(Rhi) ? 0.5 * (Rw + Rhi) : 2.0 * Rw;
      } else {                                         // too many inside, or the walk overflowed
        Rhi = Rw;
        Rn = Rlo > 0.0 ? 0.5 * (Rlo + Rw) : 0.5 * Rw;
      }
      __syncwarp();
      if (!(Rn > Rlo) || !(Rn < Rhi)) break;           // the bracket cannot narrow further
      Rw = Rn;
    }
    if (!done && lane == 0) set_error(err, SEREN_GPU_ERR_WALK, KID_GRADH, p, -2);
  }
  if (lane == 0) {
    atomicAdd(counts + 3, nwalk);
    atomicAdd(counts + 4, nvisit);
  }
}

// timestep/check_neighbour_timesteps.F90:41-68, thread per active particle:
// its level reaches the nminneib of each neighbour on its list (get_neib's
// pptot/pplist of this step) or, for an overflowed list, of each particle that
// passes get_neib_on_fly's test.  The reference raises nminneib(pp) to levelp
// when it is larger, never touching -1 entries; that is a maximum over the
// active neighbours, the same in any order.
__global__ void k_neib_levels(int nact, const int* __restrict__ act, const double4* __restrict__ pm,
                              const double2* __restrict__ hz, HydroTree t,
                              const int* __restrict__ pptot, const int* __restrict__ pplist, int L,
                              const int* __restrict__ nlevel, int* __restrict__ nminneib,
                              DevError* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nact) return;
  const int p = act ? act[i] : i;
  const int lev = nlevel[p];
  auto raise = [&](int pp) {
    const int cur = nminneib[pp];
    if (cur != -1 && lev > cur) atomicMax(nminneib + pp, lev);
  };
  const int nn = pptot[p];
  if (nn <= L) {
    const int* row = pplist + (size_t)p * L;
    for (int k = 0; k < nn; ++k) raise(row[k]);
    return;
  }
  const double4 P = pm[p];
  const double hp = hz[p].x;
  const double hsp = (KERNRANGESQD * hp) * hp;
  walk_gather_scatter(t, frame_for(t, p).root, P.x, P.y, P.z, KERNRANGE * hp, err, p, [&](int q) {
    if (q == p) return;
    const double hq = hz[q].x;
    const double hsq = (KERNRANGESQD * hq) * hq;
    const double4 Q = pm[q];
    const double d0 = Q.x - P.x, d1 = Q.y - P.y, d2 = Q.z - P.z;
    const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
    if (drsqd <= hsp || drsqd <= hsq) raise(q);
  });
}

// sum over the block, the same value on every thread
__device__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sh[k];
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------------------
// grad-h for the particles whose walks outgrow the redo kernel's scratch (the
// reference's bisection, :262-275, starts from h_upper = rextent, so its first
// walks can cover most of the domain).  They are few, so every walk of every
// such particle is spread over the whole GPU.  Each continues from the state
// the redo kernel reached (its next step: the counting walk that outgrew the
// scratch), and the host runs rounds of
//   k_wide_settle - the steps whose outcome a bound decides, without a walk:
//                   a counting walk whose ball holds a whole cell of at least
//                   pp_gather particles, and bisection passes whose density
//                   is certainly too high (a lower bound from the particle's
//                   tree-order neighbours);
//   k_wide_walk   - each (particle, slice) block walks a slice of a cover of
//                   the tree (the cells of one level and the leaves above it):
//                   a cover cell counts only when each ancestor passes the
//                   particle's test (the reference reaches a cell only through
//                   opened cells), its subtree is walked with the reference's
//                   stackless loop, and the candidates' count or terms are
//                   summed into the particle's accumulators;
//   k_wide_brute  - passes at a large h: the terms of all particles, in tiles;
//   k_wide_update - each particle takes the reference's next step from them
//                   (:154-191 walk / grow, :238-285 density update, :317-425
//                   final pass) and says what its next walk must compute;
// until no particle has a walk left.  Nothing is stored per candidate: a pass
// at h <= h_high sums exactly the particles within 2h (see wide_within), and
// the final pass at h >= h_high walks at the radius of the last counting
// walk, so each sees the reference's candidates.
constexpr int WD_THREADS = 256;

__global__ void k_flag_error(DevError* err, int code, int where) {
  set_error(err, code, where, -1, -1);
}

constexpr int WD_SLICES = 64;    // blocks per particle and round
constexpr int WD_BATCH = 1024;   // particles per batch of rounds

enum WideJob : int { WJ_COUNT = 1, WJ_PASS = 2, WJ_FINAL = 3, WJ_DONE = 0 };

struct WideState {
  GhState s;
  double4 P;        // position, mass
  double4 v;        // velocity
  double ih, hf, hs, hp;   // of the pass in progress
  double rextent;   // of the particle's tree
  int p;
  int job;          // WideJob
  int q0, q1;       // the particles of its cloud (all of them for one tree)
};

// ids: the particles the redo kernel handed over, each with its iteration
// state in its row of `stash` (the grad-h leaf rows)
__global__ void k_wide_init(int n, const int* __restrict__ ids, const double4* __restrict__ pm,
                            const int* __restrict__ stash, const double4* __restrict__ vel,
                            double rextent, int ptot, const CloudInfo* __restrict__ cl, int ncl,
                            WideState* __restrict__ ws, double* __restrict__ acc,
                            unsigned long long* counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  atomicAdd(counts + 8, 1ull);
  WideState& w = ws[i];
  w.p = ids[i];
  w.P = pm[w.p];
  w.v = vel[w.p];
  w.rextent = rextent;
  w.q0 = 0;
  w.q1 = ptot;
  if (cl) {
    const CloudInfo& C = cl[cloud_of(cl, ncl, w.p)];
    w.rextent = C.rextent;
    w.q0 = C.pstart;
    w.q1 = C.pstart + C.n;
  }
  w.s = *reinterpret_cast<const GhState*>(stash + (size_t)w.p * GH_LEAVES);
  w.job = WJ_COUNT;                 // the walk at s.h_high (:154-170)
  for (int k = 0; k < 4; ++k) acc[4 * i + k] = 0.0;
}

// A pass at h <= h_high (every density pass; the final pass when its h is
// below h_high) sums exactly the particles within 2h, all of which the
// reference's candidates (the leaves the walk at h_high opened) hold, since
// the bounding sphere of every cell that holds one holds it.  Such a pass
// walks at radius 2h (1 + 2^-20): every leaf holding a particle within 2h
// passes that walk's test with room to spare for the rounding of the test.
// At a large h (2h above an eighth of the tree's extent) the terms of all
// particles are summed instead (k_wide_brute), which then costs less than the
// walk.  The counting walks and the final pass at h >= h_high walk at 2h_high.
__device__ __forceinline__ double wide_h(const WideState& w) {
  return w.job == WJ_PASS ? w.s.hp : w.hp;
}
__device__ __forceinline__ bool wide_within(const WideState& w) {
  return w.job == WJ_PASS || (w.job == WJ_FINAL && w.hp < w.s.h_high);
}
__device__ __forceinline__ bool wide_brute(const WideState& w) {
  return wide_within(w) && KERNRANGE * wide_h(w) >= 0.125 * w.rextent;
}
__device__ __forceinline__ double wide_radius(const WideState& w) {
  return wide_within(w) ? (KERNRANGE * wide_h(w)) * (1.0 + 0x1p-20) : KERNRANGE * w.s.h_high;
}

// The highest cell on the path from the root to particle p whose every
// particle lies within R of P with room for the rounding of the walk's test
// (|P - centre| + rmax <= R (1 - 2^-30)); returns its particle count, 0 if no
// cell on the path qualifies.  A walk at radius R opens every leaf of such a
// cell: each cell d that holds one of its particles q passes the test
// |centre_d - P| <= |centre_d - q| + |q - P| <= rmax_d + R.
__device__ int wide_cover(const HydroTree& t, const int* __restrict__ pcount, int root, int p,
                          const double4& P, double R) {
  const double Rm = R * (1.0 - 0x1p-30);
  int c = root;
  for (int depth = 0; depth <= 2 * DEEP_LEVELS + 2; ++depth) {
    const double4 h = t.hA[c];
    const double d0 = h.x - P.x, d1 = h.y - P.y, d2 = h.z - P.z;
    if (sqrt((d0 * d0 + d1 * d1) + d2 * d2) + h.w <= Rm) return pcount[c];
    const int4 lk = t.link[c];
    if (lk.x != 0) return 0;                           // a leaf: nothing below
    const int first = lk.z, nk = t.nkids[c];
    int next = -1;
    for (int k = 0; k < nk; ++k) {                     // the child whose range holds p
      const int ch = first + k;
      const int s = t.link[ch].w;
      if (p >= s && p < s + pcount[ch]) {
        next = ch;
        break;
      }
    }
    if (next < 0) return 0;
    c = next;
  }
  return 0;
}

// The steps of each pending particle that a bound decides, taken here without
// a walk (one block per particle):
//  * a counting walk (:154-170) whose ball covers a whole cell of at least
//    pp_gather particles: pp_pot is at least that count, so the reference's
//    next step is the pass at the same h (:175-191);
//  * a bisection pass (GRADH_ITERATION_MAX < iteration < 2 GRADH_ITERATION_MAX)
//    whose density is certainly large: every term of the sum (:211-235) is
//    non-negative, so the self term plus the terms of the WS_THREADS particles
//    nearest in tree order (those of them within 2h) bound it from below, up
//    to the rounding of either sum (covered by a factor 1 - 1e-6).  When that
//    bound already puts h_fac (m/rho)^(1/3) below h (1 - H_CON) (no
//    convergence, :246) and makes h^3 - h_fac^3 m/rho positive (:263-268),
//    the pass's outcome is h_upper = h, h = (h_lower + h_upper)/2 whatever
//    the full sum; such passes are taken one after another until one is not
//    decided.  The density of a decided pass is never read: the loop ends
//    only after a full pass.
constexpr int WS_THREADS = 256;
__global__ void __launch_bounds__(WS_THREADS) k_wide_settle(
    int n, WideState* __restrict__ ws, const double4* __restrict__ pm, HydroTree t,
    const int* __restrict__ pcount, const double4* __restrict__ tabA, double h_fac,
    int pp_gather, unsigned long long* counts) {
  __shared__ double red[WS_THREADS / 32];
  __shared__ int cover;
  const int i = blockIdx.x;
  if (i >= n) return;
  WideState& w = ws[i];
  int job = w.job;
  GhState s = w.s;
  const bool bisecting = s.iteration > GRADH_ITERATION_MAX && s.iteration < 2 * GRADH_ITERATION_MAX;
  if (job != WJ_COUNT && !(job == WJ_PASS && bisecting)) return;  // block-uniform
  const int p = w.p;
  const double4 P = w.P;
  const double mp = P.w;
  bool changed = false;
  if (job == WJ_COUNT) {
    if (threadIdx.x == 0)
      cover = wide_cover(t, pcount, frame_for(t, p).root, p, P, KERNRANGE * s.h_high);
    __syncthreads();
    if (cover < pp_gather) return;                                 // the walk counts
    s.pp_pot = cover;
    job = WJ_PASS;
    changed = true;
  }
  const int q = p - WS_THREADS / 2 + (int)threadIdx.x;
  const bool use = q >= w.q0 && q < w.q1 && q != p;
  double d2 = 0.0, m = 0.0;
  if (use) {
    const double4 Q = pm[q];
    const double d0 = Q.x - P.x, d1 = Q.y - P.y, e2 = Q.z - P.z;   // as the passes form it
    d2 = (d0 * d0 + d1 * d1) + e2 * e2;
    m = Q.w;
  }
  const double w00 = tabA[0].x;
  const double hfac3 = pow(h_fac, NDIMPR);
  unsigned long long nset = 0;
  while (s.iteration > GRADH_ITERATION_MAX && s.iteration < 2 * GRADH_ITERATION_MAX) {
    const double ih = 1.0 / s.hp;
    const double hf = pow(ih, NDIMPR);
    const double hs = (KERNRANGESQD * s.hp) * s.hp;
    double part = 0.0;
    if (use && d2 < hs) gh_density_in(d2, m, ih, hf, part);
    const double lb = ((mp * w00) * hf + block_sum(part, red)) * (1.0 - 1e-6);
    if (!(lb > SMALL_NUMBER)) break;
    const bool noconv = h_fac * pow(mp / lb, ONETHIRD) * (1.0 + 1e-6) <
                        (s.hp * (1.0 - H_CON)) * (1.0 - 1e-6);
    const bool fbpos = lb > ((hfac3 * mp) / pow(s.hp, NDIMPR)) * (1.0 + 1e-6);
    if (!(noconv && fbpos)) break;
    s.rho = lb;
    s.h_upper = s.hp;
    s.hp = 0.5 * (s.h_lower + s.h_upper);
    s.iteration = s.iteration + 1;
    ++nset;
    changed = true;
  }
  if (threadIdx.x == 0 && changed) {
    w.s = s;
    w.job = job;
    w.ih = 1.0 / s.hp;                                             // :199-210
    w.hf = pow(w.ih, NDIMPR);
    w.hs = (KERNRANGESQD * s.hp) * s.hp;
    if (nset) atomicAdd(counts + 5, nset);
  }
}

// The cover the walks are spread over: the cells of at most WD_COVER
// particles whose parent holds more (or that are a root).  Every particle lies
// in exactly one of them (the first cell of at most WD_COVER particles on the
// path from its root), and no thread walks a subtree of more than WD_COVER
// particles, however unevenly the particles fill the tree.
constexpr int WD_COVER = 256;
__global__ void k_wide_cover_mark(int ctot, const int* __restrict__ pcount,
                                  const int* __restrict__ parent, int* __restrict__ flag) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ctot) return;
  const int a = parent[c];
  flag[c] = pcount[c] <= WD_COVER && (a < 0 || pcount[a] > WD_COVER) ? 1 : 0;
}

// the flagged cells in cell order: out[scan[c]] = c
__global__ void k_wide_cover_list(int ctot, const int* __restrict__ flag,
                                  const int* __restrict__ scan, int* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c <= ctot && flag[c]) out[scan[c]] = c;
}

// one walk per pending particle, WD_SLICES blocks each
__global__ void __launch_bounds__(WD_THREADS) k_wide_walk(
    int n, const WideState* __restrict__ ws, const double4* __restrict__ pm,
    const double4* __restrict__ vel, HydroTree t, const int* __restrict__ parent,
    const int* __restrict__ cover, int ncover, double* __restrict__ part, DevError* err) {
  __shared__ double red[WD_THREADS / 32];
  const int i = blockIdx.x / WD_SLICES, slice = blockIdx.x % WD_SLICES;
  if (i >= n) return;
  const WideState& w = ws[i];
  const int job = w.job;
  if (job == WJ_DONE || wide_brute(w)) return;                   // block-uniform
  const int p = w.p;
  const double rx = w.P.x, ry = w.P.y, rz = w.P.z;
  const double hrange = wide_radius(w);
  const double hs = w.hs, ih = w.ih, hf = w.hf;
  const double4 vp = w.v;
  auto pass = [&](int c) {                             // BHhydrowalk_hgather.F90:36-40
    const double4 h = t.hA[c];
    const double d0 = h.x - rx, d1 = h.y - ry, d2 = h.z - rz;
    const double tt = hrange + h.w;
    return ((d0 * d0 + d1 * d1) + d2 * d2) <= tt * tt;
  };
  double s0 = 0.0;
  GhFinal f;
  f.rt = 0.0; f.om = 0.0; f.dv = 0.0; f.zt = 0.0;
  const int stride = WD_SLICES * WD_THREADS;
  for (int k = slice * WD_THREADS + threadIdx.x; k < ncover; k += stride) {
    const int c = cover[k];
    const int4 lk = t.link[c];
    if (lk.w < w.q0 || lk.w >= w.q1) continue;                  // another cloud's tree
    bool reach = true;
    for (int a = parent[c]; a >= 0 && reach; a = parent[a]) reach = pass(a);
    if (!reach) continue;
    const int stop = lk.y;
    int cur = c, visits = 0;
    while (true) {
      if (++visits > t.ctot + 2) {
        set_error(err, SEREN_GPU_ERR_WALK, KID_GRADH, p, cur);
        break;
      }
      const int4 l2 = t.link[cur];
      const bool ok = pass(cur);
      if (ok && l2.x > 0) {
        for (int k = 0; k < l2.x; ++k) {
          const int q = l2.w + k;
          if (job == WJ_COUNT) {
            s0 += 1.0;                                   // pp_pot counts every particle
            continue;
          }
          if (q == p) continue;
          const double4 Q = pm[q];
          const double d0 = Q.x - rx, d1 = Q.y - ry, d2 = Q.z - rz;
          const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
          if (job == WJ_PASS) {
            if (drsqd < hs) gh_density_in(drsqd, Q.w, ih, hf, s0);
          } else if (drsqd <= hs) {
            const double4 V = vel[q];
            const double dv0 = V.x - vp.x, dv1 = V.y - vp.y, dv2 = V.z - vp.z;
            gh_final_in(drsqd, Q.w, (dv0 * d0 + dv1 * d1) + dv2 * d2, ih, hf, f);
          }
        }
        cur = l2.y;
      } else if (ok && l2.x == 0) {
        cur = l2.z;
      } else {
        cur = l2.y;
      }
      if (cur == stop || cur > t.ctot) break;
    }
  }
  // this slice's partial sums; k_wide_reduce adds the slices in order
  const double r0 = block_sum(job == WJ_FINAL ? f.rt : s0, red);
  double r1 = 0.0, r2 = 0.0, r3 = 0.0;
  if (job == WJ_FINAL) {
    r1 = block_sum(f.om, red);
    r2 = block_sum(f.dv, red);
    r3 = block_sum(f.zt, red);
  }
  if (threadIdx.x == 0) {
    double* o = part + ((size_t)i * WD_SLICES + slice) * 4;
    o[0] = r0; o[1] = r1; o[2] = r2; o[3] = r3;
  }
}

// the passes wide_brute() selects: each block takes WD_THREADS * BR_Q
// particles and adds their terms of every such pass (same terms and tests as
// the walk's candidates give)
constexpr int BR_Q = 4;          // particles per thread
__global__ void __launch_bounds__(WD_THREADS) k_wide_brute(int n, const WideState* __restrict__ ws,
                                                           int ptot, const double4* __restrict__ pm,
                                                           const double4* __restrict__ vel,
                                                           double* __restrict__ part) {
  __shared__ double red[WD_THREADS / 32];
  int qi[BR_Q];
  double4 Q[BR_Q];
  bool loaded = false;
  for (int i = 0; i < n; ++i) {
    const WideState& w = ws[i];
    if (!wide_brute(w)) continue;                                 // block-uniform
    if (!loaded) {                       // the tile, once a particle needs it
#pragma unroll
      for (int k = 0; k < BR_Q; ++k) {
        const long q = (long)blockIdx.x * (WD_THREADS * BR_Q) + k * WD_THREADS + threadIdx.x;
        qi[k] = q < ptot ? (int)q : -1;
        Q[k] = q < ptot ? pm[q] : make_double4(0.0, 0.0, 0.0, 0.0);
      }
      loaded = true;
    }
    const int p = w.p;
    const int q0 = w.q0, q1 = w.q1;
    const double rx = w.P.x, ry = w.P.y, rz = w.P.z;
    const double hs = w.hs, ih = w.ih, hf = w.hf;
    if (w.job == WJ_PASS) {                                       // :211-235
      double s0 = 0.0;
#pragma unroll
      for (int k = 0; k < BR_Q; ++k) {
        if (qi[k] < q0 || qi[k] >= q1 || qi[k] == p) continue;
        const double d0 = Q[k].x - rx, d1 = Q[k].y - ry, d2 = Q[k].z - rz;
        const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
        if (drsqd < hs) gh_density_in(drsqd, Q[k].w, ih, hf, s0);
      }
      const double r0 = block_sum(s0, red);
      if (threadIdx.x == 0) {
        double* o = part + ((size_t)i * gridDim.x + blockIdx.x) * 4;
        o[0] = r0; o[1] = 0.0; o[2] = 0.0; o[3] = 0.0;
      }
    } else {                                                      // :360-425
      const double4 vp = w.v;
      GhFinal f;
      f.rt = 0.0; f.om = 0.0; f.dv = 0.0; f.zt = 0.0;
#pragma unroll
      for (int k = 0; k < BR_Q; ++k) {
        if (qi[k] < q0 || qi[k] >= q1 || qi[k] == p) continue;
        const double d0 = Q[k].x - rx, d1 = Q[k].y - ry, d2 = Q[k].z - rz;
        const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
        if (drsqd > hs) continue;
        const double4 V = vel[qi[k]];
        const double dv0 = V.x - vp.x, dv1 = V.y - vp.y, dv2 = V.z - vp.z;
        gh_final_in(drsqd, Q[k].w, (dv0 * d0 + dv1 * d1) + dv2 * d2, ih, hf, f);
      }
      const double r0 = block_sum(f.rt, red), r1 = block_sum(f.om, red),
                   r2 = block_sum(f.dv, red), r3 = block_sum(f.zt, red);
      if (threadIdx.x == 0) {
        double* o = part + ((size_t)i * gridDim.x + blockIdx.x) * 4;
        o[0] = r0; o[1] = r1; o[2] = r2; o[3] = r3;
      }
    }
  }
}

// The sums of each pending particle's walk or passes of this round: its
// partials (one per walk slice, or one per particle tile of the passes) added
// in slice or tile order by one warp - a fixed order, so the results repeat
// from run to run.
__global__ void k_wide_reduce(int n, const WideState* __restrict__ ws,
                              const double* __restrict__ part_walk,
                              const double* __restrict__ part_brute, int nbrute,
                              double* __restrict__ acc) {
  const int i = blockIdx.x;
  const int lane = threadIdx.x;
  if (i >= n) return;
  const WideState& w = ws[i];
  if (w.job == WJ_DONE) return;
  const bool brute = wide_brute(w);
  const int np = brute ? nbrute : WD_SLICES;
  const double* src = brute ? part_brute + (size_t)i * nbrute * 4 : part_walk + (size_t)i * WD_SLICES * 4;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int b = lane; b < np; b += 32)
    for (int k = 0; k < 4; ++k) s[k] = s[k] + src[(size_t)b * 4 + k];
  for (int k = 0; k < 4; ++k) {
    const double v = warp_sum(s[k]);
    if (lane == 0) acc[4 * i + k] = v;
  }
}

// the reference's next step for each particle; *more = 1 while walks remain
__global__ void k_wide_update(int n, WideState* __restrict__ ws, double* __restrict__ acc,
                              const double4* __restrict__ tabA, double h_fac, int pp_gather,
                              double rextent, double2* __restrict__ hz, double* __restrict__ rho,
                              double* __restrict__ omega, double* __restrict__ divv,
                              double* __restrict__ drhodt, int* __restrict__ more,
                              DevError* err, unsigned long long* counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  WideState& w = ws[i];
  if (w.job == WJ_DONE) return;
  GhState& s = w.s;
  const double mp = w.P.w;
  const double4 t0 = tabA[0];
  double* a = acc + 4 * i;
  if (w.job == WJ_FINAL) {                                          // :426-442
    GhFinal g;
    gh_final_init(g, mp, w.ih, w.hf, t0);
    g.rt = g.rt + a[0];
    g.om = g.om + a[1];
    g.dv = g.dv + a[2];
    g.zt = g.zt + a[3];
    gh_store(w.p, mp, w.hp, g, hz, rho, omega, divv, drhodt, err);
    w.job = WJ_DONE;
    atomicAdd(counts + 5, 1ull);
    return;
  }
  if (w.job == WJ_COUNT) {
    s.pp_pot = (int)a[0];
    atomicAdd(counts + 3, 1ull);
  } else {                                                          // WJ_PASS
    atomicAdd(counts + 5, 1ull);
    if (gh_after_pass(s, mp, h_fac, w.rextent, (mp * t0.x) * w.hf + a[0])) {
      w.hp = h_fac * pow(mp / s.rho, ONETHIRD);                      // :317
      w.ih = 1.0 / w.hp;
      w.hf = pow(w.ih, NDIMPR);
      w.hs = (KERNRANGESQD * w.hp) * w.hp;
      w.job = WJ_FINAL;
      a[0] = a[1] = a[2] = a[3] = 0.0;
      *more = 1;
      return;
    }
  }
  a[0] = a[1] = a[2] = a[3] = 0.0;
  while (true) {                                                    // :154-191
    if (s.hp > s.h_high) {
      s.h_high = s.hp * HMULT;
      w.job = WJ_COUNT;
      *more = 1;
      return;
    }
    if (s.pp_pot < pp_gather) {
      s.h_high = 0.0;
      s.pp_pot = 0;
      s.hp = s.hp * HMULT;
      if (++s.ngrow > HGROW_CAP) {
        set_error(err, SEREN_GPU_ERR_WALK, KID_GRADH, w.p, -1);
        w.job = WJ_DONE;
        return;
      }
    }
    if (s.pp_pot > 0) break;
  }
  w.ih = 1.0 / s.hp;                                                // :199-210
  w.hf = pow(w.ih, NDIMPR);
  w.hs = (KERNRANGESQD * s.hp) * s.hp;
  w.job = WJ_PASS;
  *more = 1;
}

// get_neib (sph/get_neib.F90:10-140) in two kernels.
//
// k_neib_walk: 32 particles per warp on one group walk with each lane's
// gather-or-scatter test (BHhydro_walk.F90:37-43); the opened leaves are sorted
// into depth-first order (the order of the reference's candidate lists) and
// each particle's go to its own row of c.leaves, their number to c.nleaf (-1
// when the row or the walk overflows).
//
// k_neib_rows: 32 particles per warp; for each particle in turn the warp
// flattens its row, keeps the candidates with r^2 <= 4h_p^2 or r^2 <= 4h_pp^2
// in that order and writes them with coalesced stores.  A particle whose row
// overflowed gets its list from neib_one.
__global__ void __launch_bounds__(GR_THREADS) k_neib_walk(
    int nact, const int* __restrict__ act, const double4* __restrict__ pm,
    const double2* __restrict__ hz, HydroTree t, int* __restrict__ leaves,
    int* __restrict__ nleaf, int2* __restrict__ stacks, int scap, unsigned long long* counts,
    int* work) {
  extern __shared__ __align__(16) unsigned char gr_smem[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  GrShared& R = reinterpret_cast<GrShared*>(gr_smem)[w];
  int2* const S = stacks + (size_t)(blockIdx.x * GR_WARPS + w) * scap;
  const unsigned bit = 1u << lane;
  unsigned long long nvisit = 0;
  for (int g = gr_next(work, lane); (long long)g * 32 < nact; g = gr_next(work, lane)) {
    const int i = g * 32 + lane;
    bool live;
    const int p = group_particle(i, nact, act, live);
    const TreeFrame fr = frame_for(t, p);             // lanes share one cloud
    const double4 P = pm[p];
    const float px = (float)(P.x - fr.rootx), py = (float)(P.y - fr.rooty),
                pz = (float)(P.z - fr.rootz);
    const double Rw = KERNRANGE * hz[p].x;
    const float R32 = (float)Rw;
    const unsigned lanes = __ballot_sync(FULL, live);
    const GrGroup grp = gr_group(px, py, pz, R32, live);
    const int nent = gr_walk(t, fr.root, lanes, S, scap, R, lane, 0, nvisit, [&](const float4& c, float fh) {
      // gather or scatter (BHhydro_walk.F90:37-43): a lane passes within
      // max(its 2h, hrangemax) + rmax
      return gr_decide(grp, c, fmaxf(grp.rmin, fh), fmaxf(grp.rmax, fh), fr.delta);
    }, [&](int e) {
      const float4 h32 = R.fa[e];
      const float d0 = h32.x - px, d1 = h32.y - py, d2 = h32.z - pz;
      const float d2s = (d0 * d0 + d1 * d1) + d2 * d2;
      const int r1 = test32(d2s, R32 + h32.w, fr.delta);
      const int r2 = test32(d2s, R.fh[e] + h32.w, fr.delta);
      if (r1 == 1 || r2 == 1) return true;
      if (r1 == 0 && r2 == 0) return false;
      const int c = R.fc[e];
      const double4 h = t.hA[c];
      const double e0 = h.x - P.x, e1 = h.y - P.y, e2 = h.z - P.z;
      const double drsqd = (e0 * e0 + e1 * e1) + e2 * e2;
      const double t1 = Rw + h.w;
      const double t2 = t.hrm[c] + h.w;
      return drsqd <= t1 * t1 || drsqd <= t2 * t2;
    });
    int n = -1;
    if (nent >= 0) {
      gr_sort(R, nent, lane);
      n = 0;
      int* row = leaves + (size_t)p * GH_LEAVES;
      for (int e = 0; e < nent; ++e) {
        if (R.mask[e] & bit) {
          if (n < GH_LEAVES) row[n] = R.code[e];
          ++n;
        }
      }
      if (n > GH_LEAVES) n = -1;
    }
    if (live) nleaf[p] = n;
    __syncwarp();
  }
  if (lane == 0) atomicAdd(counts + 4, nvisit);
}

__global__ void __launch_bounds__(GP_THREADS) k_neib_rows(
    int nact, const int* __restrict__ act, const double4* __restrict__ pm,
    const double2* __restrict__ hz, HydroTree t, int L, const int* __restrict__ leaves,
    const int* __restrict__ nleaf, int* __restrict__ pptot, int* __restrict__ pplist,
    DevError* err, unsigned long long* counts, int* work) {
  __shared__ int cand_all[GP_WARPS][GP_SEG * LEAFMAX];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int* cand = cand_all[w];
  const unsigned lt = (1u << lane) - 1u;
  unsigned long long ncands = 0, niter = 0, nsingle = 0;
  for (int g = gr_next(work, lane); (long long)g * 32 < nact; g = gr_next(work, lane)) {
    const int i = g * 32 + lane;
    bool live;
    const int p = group_particle(i, nact, act, live);
    const int n = live ? nleaf[p] : 0;
    const double4 P = pm[p];
    const double hp = hz[p].x;
    const double hsp = (KERNRANGESQD * hp) * hp;
    const unsigned G = __ballot_sync(FULL, live && n >= 0);
    for (unsigned todo = G; todo != 0u; todo &= todo - 1u) {
      const int j = __ffs(todo) - 1;
      const double xj = __shfl_sync(FULL, P.x, j), yj = __shfl_sync(FULL, P.y, j),
                   zj = __shfl_sync(FULL, P.z, j), hsj = __shfl_sync(FULL, hsp, j);
      const int pj = __shfl_sync(FULL, p, j);
      const int nj = __shfl_sync(FULL, n, j);
      int* row = pplist + (size_t)pj * L;
      int kept = 0;
      for (int s0 = 0; s0 < nj; s0 += GP_SEG) {       // the row, GP_SEG leaves at a time
      const int nc = gp_flatten(leaves + (size_t)pj * GH_LEAVES + s0, min(GP_SEG, nj - s0),
                                cand, lane);
      for (int b = 0; b < nc; b += 32) {
        const int k = b + lane;
        const int q = k < nc ? cand[k] : pj;
        bool keep = false;
        if (q != pj) {
          const double4 Q = pm[q];
          const double hq = hz[q].x;
          const double hsq = (KERNRANGESQD * hq) * hq;
          const double d0 = Q.x - xj, d1 = Q.y - yj, d2 = Q.z - zj;
          const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
          keep = drsqd <= hsj || drsqd <= hsq;
        }
        const unsigned m = __ballot_sync(FULL, keep);
        const int pos = kept + __popc(m & lt);
        if (keep && pos < L) row[pos] = q;
        kept += __popc(m);
      }
      niter += (nc + 31) >> 5;
      ncands += nc;
      }
      if (lane == 0) pptot[pj] = kept;
    }
    if (live && n < 0) {
      ++nsingle;
      neib_one(p, pm, hz, t, L, pptot, pplist, err);
    }
    __syncwarp();
  }
  atomicAdd(counts + 15, nsingle);
  if (lane == 0) {
    atomicAdd(counts + 7, ncands);
    atomicAdd(counts + 14, niter);
  }
}

// sph/hydro_gradh.F90:9-339 (NEIGHBOUR_LISTS, ARTIFICIAL_VISCOSITY=MON97).
// The per-particle factors press/rho/rho/omega (:96, :178) and
// (1/h)**(NDIM+1) (:91, :196) are computed once per particle by k_hydro_prep
// with the reference's expressions, so every pair reads them instead of
// recomputing them (same values).
__global__ void k_hydro_prep(int n, const double2* __restrict__ hz, const double* __restrict__ rho,
                             const double* __restrict__ omega, const double* __restrict__ press,
                             double* __restrict__ pf, double* __restrict__ hf4) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double r = rho[p];
  pf[p] = ((press[p] / r) / r) / omega[p];
  hf4[p] = pow(1.0 / hz[p].x, NDIMPLUS1);
}

// M4 (or M4 Thomas-Couchman) gradient w1 (setup/kernel.F90:66-73, :93) at the
// centre of table bin int(5000 r/h) in FP32, for the mixed form of the hydro
// pair arithmetic.
__device__ __forceinline__ float m4_w1_bin(float x, bool tc) {
  const float kf = fminf(floorf(5000.0f * x), (float)KERNTOT);
  const float s = fmaf(kf, 2.0e-4f, 1.0e-4f);
  const float inner = (tc && kf < 3333.0f) ? -1.0f : s * fmaf(2.25f, s, -3.0f);
  const float sa = 2.0f - s;
  const float outer = -0.75f * sa * sa;
  return 0.318309886f * (kf < 0.5f * (float)KERNTOT ? inner : outer);
}

constexpr int HY_SUB = 4;        // threads per particle in the mixed hydro kernel

// SUB consecutive threads share one particle, each taking every SUB-th entry
// of its neighbour list, and their sums are added at the end (SUB = 1 keeps the
// reference's order of terms).
// k_hydro_prep for the mixed kernel, which also writes the neighbours' values
// as one 96-byte record per particle (three 32-byte sectors: x, y, z, m |
// vx, vy, vz, h | pf, hf4, c_s, rho), so that a pair gathers two or three
// adjacent sectors instead of one per array
__global__ void k_hydro_prep_pack(int n, const double4* __restrict__ pm,
                                  const double2* __restrict__ hz, const double4* __restrict__ vel,
                                  const double* __restrict__ rho, const double* __restrict__ omega,
                                  const double* __restrict__ press, const double* __restrict__ sound,
                                  double* __restrict__ pf, double* __restrict__ hf4,
                                  double4* __restrict__ rec) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double r = rho[p];
  const double pfv = ((press[p] / r) / r) / omega[p];
  const double h = hz[p].x;
  const double hfv = pow(1.0 / h, NDIMPLUS1);
  pf[p] = pfv;
  hf4[p] = hfv;
  const double4 v = vel[p];
  rec[3 * (size_t)p] = pm[p];
  rec[3 * (size_t)p + 1] = make_double4(v.x, v.y, v.z, h);
  rec[3 * (size_t)p + 2] = make_double4(pfv, hfv, sound[p], r);
}

// PACKED: the neighbours' values come from k_hydro_prep_pack's records (rec), else
// from the separate arrays (the form without a context keeps those)
template <bool MIXED, int SUB, bool PACKED = false>
__global__ void __launch_bounds__(128, 8) k_hydro(int nact, const int* __restrict__ act,
                                               const double4* __restrict__ pm,
                                               const double2* __restrict__ hz,
                                               const double4* __restrict__ vel,
                                               const double* __restrict__ rho,
                                               const double* __restrict__ pf,
                                               const double* __restrict__ hf4,
                                               const double* __restrict__ sound,
                                               const int* __restrict__ pptot,
                                               const int* __restrict__ pplist, int L, HydroTree t,
                                               const double4* __restrict__ tabG, double alpha,
                                               bool tc, double* __restrict__ acc,
                                               double* __restrict__ amap, DevError* err,
                                               const double4* __restrict__ rec = nullptr) {
  auto ld_pm = [&](int q) { if constexpr (PACKED) return rec[3 * (size_t)q]; else return pm[q]; };
  auto ld_h = [&](int q) {
    if constexpr (PACKED) return rec[3 * (size_t)q + 1].w; else return hz[q].x;
  };
  auto ld_v = [&](int q) {
    if constexpr (PACKED) return rec[3 * (size_t)q + 1]; else return vel[q];
  };
  auto ld_pf = [&](int q) { if constexpr (PACKED) return rec[3 * (size_t)q + 2].x; else return pf[q]; };
  auto ld_hf4 = [&](int q) {
    if constexpr (PACKED) return rec[3 * (size_t)q + 2].y; else return hf4[q];
  };
  auto ld_c = [&](int q) {
    if constexpr (PACKED) return rec[3 * (size_t)q + 2].z; else return sound[q];
  };
  auto ld_rho = [&](int q) {
    if constexpr (PACKED) return rec[3 * (size_t)q + 2].w; else return rho[q];
  };
  const int gi = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = gi / SUB, sub = gi % SUB;
  if (SUB == 1 && i >= nact) return;
  const bool valid = i < nact;
  const int p = valid ? (act ? act[i] : i) : 0;
  const double4 P = pm[p];
  const double hp = hz[p].x;
  const double invhp = 1.0 / hp;
  const double hfactor_p = hf4[p];
  const double4 vp = vel[p];
  const double sound_p = sound[p];
  const double rho_p = rho[p];
  const double pfactor_p = pf[p];
  const double beta = 2.0 * alpha;
  double at0 = 0.0, at1 = 0.0, at2 = 0.0, ad0 = 0.0, ad1 = 0.0, ad2 = 0.0;
  // FP32 form
  const float hp32 = (float)hp, invhp32 = (float)invhp, hf32 = (float)hfactor_p;
  const float pf32 = (float)pfactor_p, c32 = (float)sound_p, rho32 = (float)rho_p;
  const float alpha32 = (float)alpha, beta32 = (float)beta;
  float f0 = 0.f, f1 = 0.f, f2 = 0.f, g0 = 0.f, g1 = 0.f, g2 = 0.f;
  auto pair = [&](int q) {
    const double4 Q = ld_pm(q);
    const double hq = ld_h(q);
    if (MIXED) {
      const float u0 = (float)(Q.x - P.x), u1 = (float)(Q.y - P.y), u2 = (float)(Q.z - P.z);
      const float hq32 = (float)hq;
      const float r2 = fmaf(u2, u2, fmaf(u1, u1, u0 * u0));
      if (r2 >= 4.0f * hp32 * hp32 && r2 >= 4.0f * hq32 * hq32) return;
      const double4 V = ld_v(q);
      const float dv0 = (float)(V.x - vp.x), dv1 = (float)(V.y - vp.y), dv2 = (float)(V.z - vp.z);
      const float inv = rsqrtf(fmaxf(r2, 1.0e-30f));
      const float drmag = r2 * inv;
      const float dvdr = fmaf(dv2, u2, fmaf(dv1, u1, dv0 * u0));
      const float e0 = u0 * inv, e1 = u1 * inv, e2 = u2 * inv;
      const float invhq32 = __frcp_rn(hq32);
      const float mq = (float)Q.w;
      float wmean = 0.f, fsum = 0.f;
      const float xp = drmag * invhp32;
      if (xp < KERNRANGE) {
        const float w1 = m4_w1_bin(xp, tc);
        wmean = 0.5f * hf32 * w1;
        fsum = mq * pf32 * hf32 * w1;
      }
      const float xq = drmag * invhq32;
      if (xq < KERNRANGE) {
        const float w1 = m4_w1_bin(xq, tc);
        const float hfq = (float)ld_hf4(q);
        wmean = fmaf(0.5f * hfq, w1, wmean);
        fsum = fmaf(mq * (float)ld_pf(q) * hfq, w1, fsum);
      }
      f0 = fmaf(fsum, e0, f0); f1 = fmaf(fsum, e1, f1); f2 = fmaf(fsum, e2, f2);
      if (dvdr < 0.0f) {
        const float vsignal = c32 + (float)ld_c(q) - beta32 * dvdr * inv;
        const float g = mq * alpha32 * vsignal * dvdr * inv * wmean *
                        __frcp_rn(0.5f * (rho32 + (float)ld_rho(q)));
        g0 = fmaf(-g, e0, g0); g1 = fmaf(-g, e1, g1); g2 = fmaf(-g, e2, g2);
      }
      return;
    }
    double wmean = 0.0;
    const double rho_q = ld_rho(q);
    double u0 = Q.x - P.x, u1 = Q.y - P.y, u2 = Q.z - P.z;
    double drmag = (u0 * u0 + u1 * u1) + u2 * u2;
    if (drmag >= (KERNRANGESQD * hp) * hp && drmag >= (KERNRANGESQD * hq) * hq) return;  // :154
    drmag = sqrt(drmag) + SMALL_NUMBER;
    const double4 V = ld_v(q);
    const double dv0 = V.x - vp.x, dv1 = V.y - vp.y, dv2 = V.z - vp.z;
    const double dvdr = (dv0 * u0 + dv1 * u1) + dv2 * u2;                         // :157
    const double invdrmag = 1.0 / drmag;
    u0 = u0 * invdrmag; u1 = u1 * invdrmag; u2 = u2 * invdrmag;
    const double pfactor_q = ld_pf(q);
    if (drmag < KERNRANGE * hp) {                                                 // :181-192
      int kern = (int)((HALFKERNTOT * drmag) * invhp);
      kern = min(kern, KERNTOT);
      const double w1 = tabG[kern].w;
      wmean = (0.5 * hfactor_p) * w1;
      const double f = ((Q.w * pfactor_p) * hfactor_p) * w1;
      at0 = at0 + f * u0; at1 = at1 + f * u1; at2 = at2 + f * u2;
    }
    if (drmag < KERNRANGE * hq) {                                                 // :194-207
      const double invhq = 1.0 / hq;
      const double hfq = ld_hf4(q);
      int kern = (int)((HALFKERNTOT * drmag) * invhq);
      kern = min(kern, KERNTOT);
      const double w1 = tabG[kern].w;
      wmean = wmean + (0.5 * hfq) * w1;
      const double f = ((Q.w * pfactor_q) * hfq) * w1;
      at0 = at0 + f * u0; at1 = at1 + f * u1; at2 = at2 + f * u2;
    }
    const double rhomean = 0.5 * (rho_p + rho_q);                                 // :213
    if (dvdr < 0.0) {                                                             // :225-255
      const double vsignal = (sound_p + ld_c(q)) - ((beta * dvdr) * invdrmag);
      const double g = (((Q.w * alpha) * vsignal) * dvdr) * invdrmag;
      ad0 = ad0 - ((g * u0) * wmean) / rhomean;
      ad1 = ad1 - ((g * u1) * wmean) / rhomean;
      ad2 = ad2 - ((g * u2) * wmean) / rhomean;
    }
  };
  const int nn = valid ? pptot[p] : 0;
  if (nn <= L) {
    const int* row = pplist + (size_t)p * L;
    for (int k = sub; k < nn; k += SUB) pair(row[k]);
  } else if (sub == 0) {
    // get_neib_on_fly (sph/get_neib_on_fly.F90:11-130): same test as get_neib
    const double hsp = (KERNRANGESQD * hp) * hp;
    walk_gather_scatter(t, frame_for(t, p).root, P.x, P.y, P.z, KERNRANGE * hp, err, p, [&](int q) {
      if (q == p) return;
      const double hq = ld_h(q);
      const double hsq = (KERNRANGESQD * hq) * hq;
      const double4 Q = ld_pm(q);
      const double d0 = Q.x - P.x, d1 = Q.y - P.y, d2 = Q.z - P.z;
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      if (drsqd <= hsp || drsqd <= hsq) pair(q);
    });
  }
  if (SUB > 1) {
#pragma unroll
    for (int o = SUB / 2; o > 0; o >>= 1) {
      f0 += __shfl_xor_sync(0xffffffffu, f0, o);
      f1 += __shfl_xor_sync(0xffffffffu, f1, o);
      f2 += __shfl_xor_sync(0xffffffffu, f2, o);
      g0 += __shfl_xor_sync(0xffffffffu, g0, o);
      g1 += __shfl_xor_sync(0xffffffffu, g1, o);
      g2 += __shfl_xor_sync(0xffffffffu, g2, o);
    }
    if (!valid || sub != 0) return;
  }
  double r0, r1, r2;
  if (MIXED) {
    r0 = (double)f0 + (double)g0;
    r1 = (double)f1 + (double)g1;
    r2 = (double)f2 + (double)g2;
  } else {
    r0 = at0 + ad0;                                                              // :287, :297
    r1 = at1 + ad1;
    r2 = at2 + ad2;
  }
  double* a = acc + (size_t)p * 3;
  a[0] = r0;
  a[1] = r1;
  a[2] = r2;
  if (amap) {                                  // a mapped host buffer: straight over PCIe
    amap[(size_t)p * 3] = r0;
    amap[(size_t)p * 3 + 1] = r1;
    amap[(size_t)p * 3 + 2] = r2;
  }
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

HydroTree hydro_tree(const Ctx& c) {
  const double delta = ldexp(1.0, -22) * (c.info.cellsize > 0.0 ? c.info.cellsize : 1.0);
  return HydroTree{c.link, c.hA, c.hrm, c.hA32, c.hrm32, c.nkids, c.hN, c.info.ctot, c.info.root[0],
                   c.info.root[1], c.info.root[2], (float)delta, 0, c.info.rextent,
                   c.ncloud > 1 ? c.d_clouds : nullptr, c.ncloud};
}

}  // namespace

constexpr size_t GR_SMEM = sizeof(GrShared) * GR_WARPS;

// Resident blocks per SM of the group-walk kernels on device dev (their
// dynamic shared-memory limit is raised on first use per device).
static int gr_blocks_per_sm(int dev, int which) {
  static int occ[16][2] = {};
  int dummy[2] = {0, 0};
  int* o = dev >= 0 && dev < 16 ? occ[dev] : dummy;
  int& r = o[which];
  if (r == 0) {
    if (which == 0) {
      cudaFuncSetAttribute(k_gradh_walk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GR_SMEM);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_gradh_walk, GR_THREADS, GR_SMEM);
    } else {
      cudaFuncSetAttribute(k_neib_walk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GR_SMEM);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_neib_walk, GR_THREADS, GR_SMEM);
    }
    if (r < 1) r = 1;
  }
  return r;
}

static int sm_count(const Ctx& c) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.dev);
  return nsm;
}

int hydro_walk_slots(const Ctx& c) {
  return sm_count(c) * std::max(gr_blocks_per_sm(c.dev, 0), gr_blocks_per_sm(c.dev, 1)) *
         GR_WARPS;
}

// persistent grid of warps taking 32-particle groups from a counter, no more
// warps than there are walk stacks
static int gr_grid(const Ctx& c, int nact, int which) {
  const int groups = nb(nact, 32);
  int blocks = std::min(sm_count(c) * gr_blocks_per_sm(c.dev, which), nb(groups, GR_WARPS));
  return std::max(1, std::min(blocks, c.wstack_slots / GR_WARPS));
}

int wide_scratch_alloc(Ctx& c) {
  if (cudaMalloc(&c.wst, sizeof(WideState) * WD_BATCH) != cudaSuccess) return -1;
  if (cudaMalloc(&c.wacc, sizeof(double) * 4 * WD_BATCH) != cudaSuccess) return -1;
  return 0;
}

// the active list of the group kernels: in a forest with every particle
// active, the particles cloud by cloud with each cloud padded to a multiple of 32
static const int* group_list(const Ctx& c, int& nact) {
  if (c.act || c.ncloud <= 1) return c.act;
  nact = c.ngact;
  return c.gact;
}

void launch_gradh(Ctx& c, int nact) {
  c.gsets = false;
  if (nact <= 0) return;
  unsigned long long* counts = reinterpret_cast<unsigned long long*>(c.d_counts);
  const HydroTree t = hydro_tree(c);
  // with every particle active, the final passes record each particle's
  // gather neighbours for the neighbour lists that follow (launch_neib)
  const bool rec = c.act == nullptr;
  int ngrp = nact;
  const int* gl = group_list(c, ngrp);
  cudaMemsetAsync(c.work, 0, sizeof(int), c.st);
  k_gradh_walk<<<gr_grid(c, ngrp, 0), GR_THREADS, GR_SMEM, c.st>>>(
      ngrp, gl, c.pm, c.hz, t, c.leaves, c.nleaf, c.npot, c.wstack, c.wstack_cap, counts,
      c.work);
  finish_reorder(c);            // velocities still arriving: the passes need them from here on
  static int occ[16] = {};
  int& o = occ[c.dev >= 0 && c.dev < 16 ? c.dev : 0];
  if (o == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_gradh_pass, GP_THREADS, 0);
    if (o < 1) o = 1;
  }
  const int bps = c.tune.gradh_bps > 0 ? std::min(o, c.tune.gradh_bps) : o;
  const int blocks = std::min(sm_count(c) * bps, nb(nb(ngrp, 32), GP_WARPS));
  cudaMemsetAsync(c.work, 0, 3 * sizeof(int), c.st);     // group counter, nredo, nwide
  k_gradh_pass<<<blocks, GP_THREADS, 0, c.st>>>(
      ngrp, gl, c.pm, c.hz, c.vel, c.rho, c.omega, c.div_v, c.drhodt, c.tabA, c.prm.h_fac,
      c.prm.pp_gather, c.info.rextent, c.leaves, c.nleaf, c.npot, c.redo, c.work + 1,
      c.pplist, c.prm.pp_limit, c.d_err, counts, c.work, t.cl, t.ncl, rec ? 1 : 0, c.pptot);
  // three walk-stack slots of scratch per redo warp
  k_gradh_redo<<<std::max(1, (c.wstack_slots / 3) / RD_WARPS), RD_THREADS, 0, c.st>>>(
      c.redo, c.work + 1, c.pm, c.hz, c.vel, c.rho, c.omega, c.div_v, c.drhodt, t, c.tabA,
      c.prm.h_fac, c.prm.pp_gather, c.info.rextent, reinterpret_cast<int*>(c.wstack),
      c.prm.redo_cap > 0 ? std::min(c.prm.redo_cap, 2 * c.wstack_cap) : 2 * c.wstack_cap,
      c.wide, c.work + 2, c.leaves, c.d_err, counts);
  // the particles whose walks outgrew the redo kernel's scratch: rounds of
  // whole-GPU walks until each has taken its last step
  int nwide = 0;
  read_dev(c, c.work + 2, &nwide, sizeof(int));
  if (nwide > 0) {
    const int round_cap = 4 * GRADH_ITERATION_MAX + 2 * HGROW_CAP + 16;
    const int nbrute = nb(c.ptot, WD_THREADS * BR_Q);
    // the partial sums of a batch (made on first use, grown with ptot)
    const size_t need_walk = (size_t)WD_BATCH * WD_SLICES * 4;
    const size_t need_brute = (size_t)WD_BATCH * nbrute * 4;
    if (!c.wpart || c.wpart_brute_cap < need_brute) {
      if (c.wpart) cudaFree(c.wpart);
      if (c.wpart_brute) cudaFree(c.wpart_brute);
      c.wpart = c.wpart_brute = nullptr;
      c.wpart_brute_cap = 0;
      if (cudaMalloc(&c.wpart, sizeof(double) * need_walk) != cudaSuccess ||
          cudaMalloc(&c.wpart_brute, sizeof(double) * need_brute) != cudaSuccess) {
        cudaGetLastError();
        k_flag_error<<<1, 1, 0, c.st>>>(c.d_err, SEREN_GPU_ERR_CUDA, KID_GRADH);
        return;
      }
      c.wpart_brute_cap = need_brute;
    }
    // the cover of the tree the walks are spread over (k_wide_cover_mark),
    // listed in cell order through the build's flag and scan scratch
    const int ncell = c.info.ctot + 1;
    if (c.wcover_cap < ncell) {
      if (c.wcover) cudaFree(c.wcover);
      c.wcover = nullptr;
      c.wcover_cap = 0;
      if (cudaMalloc(&c.wcover, sizeof(int) * ((size_t)c.cmax + 1)) != cudaSuccess) {
        cudaGetLastError();
        k_flag_error<<<1, 1, 0, c.st>>>(c.d_err, SEREN_GPU_ERR_CUDA, KID_GRADH);
        return;
      }
      c.wcover_cap = c.cmax + 1;
    }
    k_wide_cover_mark<<<nb(ncell, 256), 256, 0, c.st>>>(c.info.ctot, c.pcount, c.parent, c.bflag);
    scan_exclusive(c, c.bflag, c.bscan, ncell);
    k_wide_cover_list<<<nb(ncell, 256), 256, 0, c.st>>>(c.info.ctot, c.bflag, c.bscan, c.wcover);
    c.nlaunch += 2;
    int ncover = 0;
    read_dev(c, c.scan.total, &ncover, sizeof(int));
    for (int b0 = 0; b0 < nwide; b0 += WD_BATCH) {
      const int n = std::min(WD_BATCH, nwide - b0);
      k_wide_init<<<nb(n, 128), 128, 0, c.st>>>(n, c.wide + b0, c.pm, c.leaves, c.vel,
                                                  c.info.rextent, c.ptot, t.cl, t.ncl,
                                                  static_cast<WideState*>(c.wst), c.wacc, counts);
      ++c.nlaunch;
      for (int round = 0;; ++round) {
        k_wide_settle<<<n, WS_THREADS, 0, c.st>>>(n, static_cast<WideState*>(c.wst), c.pm, t,
                                                   c.pcount, c.tabA, c.prm.h_fac,
                                                   c.prm.pp_gather, counts);
        ++c.nlaunch;
        k_wide_walk<<<n * WD_SLICES, WD_THREADS, 0, c.st>>>(
            n, static_cast<WideState*>(c.wst), c.pm, c.vel, t, c.parent, c.wcover, ncover,
            c.wpart, c.d_err);
        k_wide_brute<<<nbrute, WD_THREADS, 0, c.st>>>(
            n, static_cast<WideState*>(c.wst), c.ptot, c.pm, c.vel, c.wpart_brute);
        k_wide_reduce<<<n, 32, 0, c.st>>>(n, static_cast<WideState*>(c.wst), c.wpart,
                                          c.wpart_brute, nbrute, c.wacc);
        c.nlaunch += 2;
        cudaMemsetAsync(c.work + 3, 0, sizeof(int), c.st);
        k_wide_update<<<nb(n, 128), 128, 0, c.st>>>(
            n, static_cast<WideState*>(c.wst), c.wacc, c.tabA, c.prm.h_fac, c.prm.pp_gather, c.info.rextent, c.hz, c.rho,
            c.omega, c.div_v, c.drhodt, c.work + 3, c.d_err, counts);
        c.nlaunch += 2;
        int more = 0;
        read_dev(c, c.work + 3, &more, sizeof(int));
        if (!more) break;
        if (round > round_cap) {               // cannot happen: each step is bounded
          k_flag_error<<<1, 1, 0, c.st>>>(c.d_err, SEREN_GPU_ERR_WALK, KID_GRADH);
          break;
        }
      }
    }
  }
  c.nlaunch += 3;
  c.gsets = rec;
}

static void launch_neib_gsets(Ctx& c, bool sorted);

void launch_neib(Ctx& c, int nact, bool sorted) {
  if (nact <= 0) return;
  const bool gsets = c.gsets;
  c.gsets = false;
  if (gsets) {                   // every particle active, right after grad-h
    launch_neib_gsets(c, sorted);
    return;
  }
  unsigned long long* counts = reinterpret_cast<unsigned long long*>(c.d_counts);
  const HydroTree t = hydro_tree(c);
  int ngrp = nact;
  const int* gl = group_list(c, ngrp);
  cudaMemsetAsync(c.work, 0, sizeof(int), c.st);
  k_neib_walk<<<gr_grid(c, ngrp, 1), GR_THREADS, GR_SMEM, c.st>>>(
      ngrp, gl, c.pm, c.hz, t, c.leaves, c.nleaf, c.wstack, c.wstack_cap, counts, c.work);
  static int occ[16] = {};
  int& o = occ[c.dev >= 0 && c.dev < 16 ? c.dev : 0];
  if (o == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_neib_rows, GP_THREADS, 0);
    if (o < 1) o = 1;
  }
  const int bps = c.tune.neib_bps > 0 ? std::min(o, c.tune.neib_bps) : o;
  const int blocks = std::min(sm_count(c) * bps, nb(nb(ngrp, 32), GP_WARPS));
  cudaMemsetAsync(c.work, 0, sizeof(int), c.st);          // group counter
  k_neib_rows<<<blocks, GP_THREADS, 0, c.st>>>(ngrp, gl, c.pm, c.hz, t, c.prm.pp_limit,
                                               c.leaves, c.nleaf, c.pptot, c.pplist, c.d_err,
                                               counts, c.work);
  c.nlaunch += 2;
}

// get_neib (sph/get_neib.F90:10-140) for every particle right after grad-h,
// without the walks.  The list of p is the set of q != p with r^2 <= 4h_p^2
// (gather) or r^2 <= 4h_q^2 (scatter), in increasing particle order: the
// reference walks the tree depth first (BHhydro_walk.F90), which visits the
// leaves, and so the particles (numbered in tree order), in increasing order,
// and its walk reaches every such q (a cell holding q lies within
// hrangemax + rmax of p).  r^2 is the same in both rows of a pair (the
// components only change sign).  So the lists follow from the gather sets:
//  * the grad-h final pass has already applied the test r^2 <= 4h_p^2 with
//    the final h to candidates that hold every particle within 2h (h <
//    h_high) and written the gather set to p's row, its size to pptot and npot;
//    the particles it did not finish (npot = -1), listed in order, get their
//    whole rows from a walk of their own (k_neib_walked);
//  * k_neib_transpose adds p to the row of each q in p's gather set that does
//    not have p in its own (r^2 > 4h_q^2): the scatter neighbours;
//  * k_neib_sort puts each such row in increasing order when the caller reads
//    the lists, and otherwise only its scatter part (a fixed order from run
//    to run: the gather part in the final pass's order, then the scatter part).
// pptot ends as the full count in every row (the reference's pp_tot), and a
// row of more than pp_limit neighbours keeps no list, as in the reference.
__global__ void k_neib_flag(int n, const int* __restrict__ npot, int* __restrict__ flag) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) flag[p] = npot[p] < 0 ? 1 : 0;
}

__global__ void k_neib_list(int n, const int* __restrict__ flag, const int* __restrict__ scan,
                            int* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && flag[p]) out[scan[p]] = p;
}

// position and h of every particle, h negated for a walked row (npot = -1),
// so that the transposition gathers one 32-byte record per neighbour
__global__ void k_neib_hflag(int n, const double4* __restrict__ pm, const double2* __restrict__ hz,
                             const int* __restrict__ npot, double4* __restrict__ ph) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double4 P = pm[p];
  const double h = hz[p].x;
  ph[p] = make_double4(P.x, P.y, P.z, npot[p] < 0 ? -h : h);
}

// one warp per particle p: its gather neighbours q, from its row (the first
// npot[p] entries; the gather part of a walked row), or from a walk when the
// row has more than L; p joins q's row when q's own gather set lacks it
constexpr int NT_THREADS = 256;
__global__ void __launch_bounds__(NT_THREADS) k_neib_transpose(
    int n, const double4* __restrict__ ph, const int* __restrict__ npot, int* __restrict__ pptot,
    int* __restrict__ pplist, int L, HydroTree t, DevError* err, unsigned long long* counts) {
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (NT_THREADS / 32);
  unsigned long long ntest = 0;
  for (int p = blockIdx.x * (NT_THREADS / 32) + (threadIdx.x >> 5); p < n; p += nw) {
    const int g0 = npot[p];
    // a walked row is complete and final; a recorded row grows from g0 on
    const int ng = g0 >= 0 ? g0 : pptot[p];
    const double4 P = ph[p];
    const double hp = fabs(P.w);
    const double hsp = (KERNRANGESQD * hp) * hp;
    auto visit = [&](int q, bool test_gather) {
      const double4 Q = ph[q];
      const double hq = Q.w;
      const double d0 = Q.x - P.x, d1 = Q.y - P.y, d2 = Q.z - P.z;
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      if (test_gather && !(drsqd <= hsp)) return;
      if (hq < 0.0) return;                          // q's row came from a walk
      if (drsqd <= (KERNRANGESQD * hq) * hq) return; // p is in q's gather set
      const int slot = atomicAdd(pptot + q, 1);
      if (slot < L) pplist[(size_t)q * L + slot] = p;
    };
    if (ng <= L) {
      const int* row = pplist + (size_t)p * L;
      for (int k = lane; k < ng; k += 64) {          // two entries per lane in flight
        const int q0 = row[k];
        const int q1 = k + 32 < ng ? row[k + 32] : -1;
        visit(q0, g0 < 0);
        if (q1 >= 0) visit(q1, g0 < 0);
      }
      ntest += ng;
    } else if (lane == 0) {                          // more than L: the gather set from a walk
      walk_gather_scatter(t, frame_for(t, p).root, P.x, P.y, P.z, KERNRANGE * hp, err, p,
                          [&](int q) {
                            if (q != p) visit(q, true);
                          });
    }
  }
  if (lane == 0) atomicAdd(counts + 7, ntest);
}

// bitonic sort of N = 32 R values per warp, value r*32 + lane in e[r] (or,
// with R = 1, of the first N <= 32 lanes' values, each block of N lanes on
// its own, the first one ascending)
template <int R, int N = 32 * R>
__device__ __forceinline__ void warp_bitonic(int (&e)[R], int lane) {
#pragma unroll
  for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int rs = stride >> 5;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if ((r & rs) == 0) {
            const int r2 = r | rs;
            const bool up = ((r * 32 + lane) & size) == 0;
            const int a = e[r], b = e[r2];
            const bool sw = up ? (a > b) : (a < b);
            e[r] = sw ? b : a;
            e[r2] = sw ? a : b;
          }
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const bool up = ((r * 32 + lane) & size) == 0;
          const int o = __shfl_xor_sync(FULL, e[r], stride);
          const bool lower = (lane & stride) == 0;
          e[r] = (lower == up) ? min(e[r], o) : max(e[r], o);
        }
      }
    }
  }
}

template <int R, int N = 32 * R>
__device__ __forceinline__ void sort_row(int* row, int m, int lane) {
  int e[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int k = r * 32 + lane;
    e[r] = k < m ? row[k] : INT_MAX;
  }
  warp_bitonic<R, N>(e, lane);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int k = r * 32 + lane;
    if (k < m) row[k] = e[r];
  }
}

// one warp per recorded row that holds its whole list: the row in increasing
// order (full), or only its scatter part (the entries the transposition
// appended, in an order that depends on the atomics), so that the row's order
// is the same from run to run
__global__ void __launch_bounds__(NT_THREADS) k_neib_sort(int n, const int* __restrict__ npot,
                                                         const int* __restrict__ pptot,
                                                         int* __restrict__ pplist, int L,
                                                         int full) {
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (NT_THREADS / 32);
  for (int p = blockIdx.x * (NT_THREADS / 32) + (threadIdx.x >> 5); p < n; p += nw) {
    const int g0 = npot[p];
    if (g0 < 0) continue;                            // a walked row: in order already
    const int tot = pptot[p];
    if (tot > L) continue;
    const int b = full ? 0 : g0;
    const int m = tot - b;
    if (m < 2) continue;
    int* row = pplist + (size_t)p * L + b;
    if (m <= 8) sort_row<1, 8>(row, m, lane);
    else if (m <= 16) sort_row<1, 16>(row, m, lane);
    else if (m <= 32) sort_row<1>(row, m, lane);
    else if (m <= 64) sort_row<2>(row, m, lane);
    else if (m <= 128) sort_row<4>(row, m, lane);
    else if (m <= 256) sort_row<8>(row, m, lane);
    else if (lane == 0) {                            // pp_limit above 256: insertion sort
      for (int i = 1; i < m; ++i) {
        const int x = row[i];
        int j = i - 1;
        while (j >= 0 && row[j] > x) {
          row[j + 1] = row[j];
          --j;
        }
        row[j + 1] = x;
      }
    }
    __syncwarp();
  }
}

// The rows of the particles grad-h left to a walk (npot = -1: redone, or
// h >= h_high at the final pass): one warp per particle, the reference's
// gather-or-scatter walk (BHhydro_walk.F90:37-43, FP64 test) breadth first
// through the redo kernel's scratch, the neighbours kept as get_neib keeps
// them (sph/get_neib.F90:83-118) and put in increasing order; a walk beyond
// the scratch falls back to the stackless walk of one thread.
__global__ void __launch_bounds__(RD_THREADS) k_neib_walked(
    int nw, const int* __restrict__ list, const double4* __restrict__ pm,
    const double2* __restrict__ hz, HydroTree t, int L, int* __restrict__ pptot,
    int* __restrict__ pplist, int* __restrict__ scratch, int cap, DevError* err,
    unsigned long long* counts) {
  __shared__ int cand_all[RD_WARPS][GP_SEG * LEAFMAX];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int* cand = cand_all[w];
  const int gw = blockIdx.x * RD_WARPS + w;
  int* fa = scratch + (size_t)gw * 3 * cap;
  int* fb = fa + cap;
  int* lv = fb + cap;
  const unsigned lt = (1u << lane) - 1u;
  unsigned long long nvisit = 0, ncands = 0;
  for (int i = gw; i < nw; i += gridDim.x * RD_WARPS) {
    const int p = list[i];
    const double4 P = pm[p];
    const double hp = hz[p].x;
    const double hsp = (KERNRANGESQD * hp) * hp;
    const double R = KERNRANGE * hp;
    auto test = [&](int c) {
      const double4 h = t.hA[c];
      const double d0 = h.x - P.x, d1 = h.y - P.y, d2 = h.z - P.z;
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      const double t1 = R + h.w;
      const double t2 = t.hrm[c] + h.w;
      return drsqd <= t1 * t1 || drsqd <= t2 * t2;
    };
    int cnt = 0;
    const int nl = rd_walk(t, frame_for(t, p).root, lane, fa, fb, lv, cap, cnt, nvisit, test);
    if (nl < 0) {
      if (lane == 0) neib_one(p, pm, hz, t, L, pptot, pplist, err);
      __syncwarp();
      continue;
    }
    int* row = pplist + (size_t)p * L;
    int kept = 0;
    for (int s0 = 0; s0 < nl; s0 += GP_SEG) {
      const int nc = gp_flatten(lv + s0, min(GP_SEG, nl - s0), cand, lane);
      for (int b = 0; b < nc; b += 32) {
        const int k = b + lane;
        const int q = k < nc ? cand[k] : p;
        bool keep = false;
        if (q != p) {
          const double4 Q = pm[q];
          const double hq = hz[q].x;
          const double hsq = (KERNRANGESQD * hq) * hq;
          const double d0 = Q.x - P.x, d1 = Q.y - P.y, d2 = Q.z - P.z;
          const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
          keep = drsqd <= hsp || drsqd <= hsq;
        }
        const unsigned m = __ballot_sync(FULL, keep);
        const int pos = kept + __popc(m & lt);
        if (keep && pos < L) row[pos] = q;
        kept += __popc(m);
      }
      ncands += nc;
    }
    if (lane == 0) pptot[p] = kept;
    __syncwarp();
    if (kept <= L && kept >= 2) {
      if (kept <= 32) sort_row<1>(row, kept, lane);
      else if (kept <= 64) sort_row<2>(row, kept, lane);
      else if (kept <= 128) sort_row<4>(row, kept, lane);
      else if (kept <= 256) sort_row<8>(row, kept, lane);
      else if (lane == 0) {
        for (int a = 1; a < kept; ++a) {
          const int x = row[a];
          int j = a - 1;
          while (j >= 0 && row[j] > x) {
            row[j + 1] = row[j];
            --j;
          }
          row[j + 1] = x;
        }
      }
    }
    __syncwarp();
  }
  if (lane == 0) {
    atomicAdd(counts + 4, nvisit);
    atomicAdd(counts + 7, ncands);
  }
}

static void launch_neib_gsets(Ctx& c, bool sorted) {
  unsigned long long* counts = reinterpret_cast<unsigned long long*>(c.d_counts);
  const HydroTree t = hydro_tree(c);
  const int n = c.ptot;
  const int L = c.prm.pp_limit;
  // the particles grad-h left to a walk, in order (c.redo is free after grad-h)
  k_neib_flag<<<nb(n, 256), 256, 0, c.st>>>(n, c.npot, c.bflag);
  scan_exclusive(c, c.bflag, c.bscan, n);
  k_neib_list<<<nb(n, 256), 256, 0, c.st>>>(n, c.bflag, c.bscan, c.redo);
  c.nlaunch += 2;
  int nw = 0;
  read_dev(c, c.scan.total, &nw, sizeof(int));
  if (nw > 0) {
    // three walk-stack slots of scratch per warp, as the redo kernel
    const int blocks = std::min((c.wstack_slots / 3) / RD_WARPS, nb(nw, RD_WARPS));
    k_neib_walked<<<std::max(1, blocks), RD_THREADS, 0, c.st>>>(
        nw, c.redo, c.pm, c.hz, t, L, c.pptot, c.pplist, reinterpret_cast<int*>(c.wstack),
        2 * c.wstack_cap, c.d_err, counts);
    ++c.nlaunch;
  }
  // positions with h and the walked flag, one record per particle, in the
  // pm_alt reorder target (free between reorders: the next one overwrites it)
  double4* ph = c.pm_alt;
  k_neib_hflag<<<nb(n, 256), 256, 0, c.st>>>(n, c.pm, c.hz, c.npot, ph);
  const int blocks = std::min(sm_count(c) * 8, nb((long)n * 32, NT_THREADS));
  k_neib_transpose<<<blocks, NT_THREADS, 0, c.st>>>(n, ph, c.npot, c.pptot, c.pplist, L, t,
                                                    c.d_err, counts);
  ++c.nlaunch;
  k_neib_sort<<<blocks, NT_THREADS, 0, c.st>>>(n, c.npot, c.pptot, c.pplist, L, sorted ? 1 : 0);
  c.nlaunch += 2;
}

void launch_hydro(Ctx& c, int nact, double* amap) {
  if (nact <= 0) return;
  if (c.prm.precision != 0 && !c.hrec) {        // made on first use
    if (cudaMalloc(&c.hrec, sizeof(double4) * 3 * (size_t)c.pmax) != cudaSuccess) {
      cudaGetLastError();
      c.hrec = nullptr;
      k_flag_error<<<1, 1, 0, c.st>>>(c.d_err, SEREN_GPU_ERR_CUDA, KID_HYDRO);
      return;
    }
  }
  if (c.prm.precision != 0)
    k_hydro_prep_pack<<<nb(c.ptot, 256), 256, 0, c.st>>>(c.ptot, c.pm, c.hz, c.vel, c.rho,
                                                         c.omega, c.press, c.sound, c.pf, c.hf4,
                                                         c.hrec);
  else
    k_hydro_prep<<<nb(c.ptot, 256), 256, 0, c.st>>>(c.ptot, c.hz, c.rho, c.omega, c.press, c.pf,
                                                    c.hf4);
  ++c.nlaunch;
  const HydroTree t = hydro_tree(c);
  const bool tc = c.prm.kernel == 1;
  auto go = [&](auto kern, int sub) {
    kern<<<nb((long)nact * sub, 128), 128, 0, c.st>>>(
        nact, c.act, c.pm, c.hz, c.vel, c.rho, c.pf, c.hf4, c.sound, c.pptot, c.pplist,
        c.prm.pp_limit, t, c.tabG, c.prm.alpha, tc, c.acc, amap, c.d_err, c.hrec);
  };
  // the records pay for the mixed kernel's threads; the FP64 kernel (one
  // thread per particle) runs faster on the separate arrays (6.9 against 7.4 ms
  // on the 4M core)
  if (c.prm.precision == 0) go(k_hydro<false, 1, false>, 1);
  else if (c.tune.hydro_sub == 2) go(k_hydro<true, 2, true>, 2);
  else if (c.tune.hydro_sub == 8) go(k_hydro<true, 8, true>, 8);
  else go(k_hydro<true, HY_SUB, true>, HY_SUB);
  ++c.nlaunch;
}

void launch_hgather(Ctx& c, int nact) {
  if (nact <= 0) return;
  unsigned long long* counts = reinterpret_cast<unsigned long long*>(c.d_counts);
  // three walk-stack slots of scratch per warp, as the redo kernel
  k_hgather<<<std::max(1, (c.wstack_slots / 3) / HG_WARPS), HG_THREADS, 0, c.st>>>(
      nact, c.act, c.pm, c.hz, hydro_tree(c), c.prm.pp_gather, c.info.rextent,
      reinterpret_cast<int*>(c.wstack), 2 * c.wstack_cap, c.d_err, counts);
  ++c.nlaunch;
}

void launch_neib_levels(Ctx& c, int nact, const int* nlevel, int* nminneib) {
  if (nact <= 0) return;
  k_neib_levels<<<nb(nact, 128), 128, 0, c.st>>>(nact, c.act, c.pm, c.hz, hydro_tree(c), c.pptot,
                                                 c.pplist, c.prm.pp_limit, nlevel, nminneib,
                                                 c.d_err);
  ++c.nlaunch;
}

void launch_thermal(Ctx& c) {
  k_thermal<<<nb(c.ptot, 256), 256, 0, c.st>>>(c.ptot, c.csq, c.rho, c.press, c.sound); ++c.nlaunch;
}

}  // namespace seren

// ---------------------------------------------------------------------------
// Hydro forces without a context and without allocation.
//
// Some callers cannot call cudaMalloc: an application whose device memory is
// owned by its own pool allocator (a framework's caching allocator, or a
// Fortran/OpenACC runtime that reserves the GPU's memory up front) or that runs
// under a fixed device-memory budget.  Such a caller cannot create a context
// (seren_gpu_create allocates the tree, lists and staging buffers), but it does
// hold the particle arrays and neighbour lists in device buffers of its own.
// seren_gpu_hydro_forces_noalloc runs the hydro kernel of
// seren_gpu_hydro_forces on those buffers.  The kernel's scratch (the particle
// arrays in the kernel's layout, the per-particle factors, the kernel tables
// and the error block) lives in one file-scope device array of fixed size,
// which every GPU that loads this library holds until the process exits.
namespace seren {
namespace {

constexpr int NOALLOC_PMAX = SEREN_GPU_NOALLOC_PMAX;
constexpr size_t NA_ERR = 0;                                     // DevError
constexpr size_t NA_TAB = 32;                                    // 2 kernel tables (M4, M4TC)
constexpr size_t NA_TABLEN = (size_t)(KERNTOT + 1) * 4;          // doubles per table
constexpr size_t NA_PART = NA_TAB + ((2 * NA_TABLEN + 31) / 32) * 32;
constexpr size_t NA_PM = NA_PART;                                // double4 per particle
constexpr size_t NA_HZ = NA_PM + 4 * (size_t)NOALLOC_PMAX;       // double2
constexpr size_t NA_VEL = NA_HZ + 2 * (size_t)NOALLOC_PMAX;      // double4
constexpr size_t NA_PF = NA_VEL + 4 * (size_t)NOALLOC_PMAX;      // double
constexpr size_t NA_HF4 = NA_PF + (size_t)NOALLOC_PMAX;          // double
constexpr size_t NA_TOTAL = NA_HF4 + (size_t)NOALLOC_PMAX;       // 3.6 MiB in all

static __device__ __align__(256) double g_noalloc_scratch[NA_TOTAL];

// Copies the caller's rows into the kernel's layout and checks the lists:
// 0 <= pptot <= pp_limit (rows the context entry point would complete with a
// tree walk are refused here) and every listed id in 0..n-1.
__global__ void k_noalloc_pack(int n, const double* __restrict__ parray,
                               const double* __restrict__ v, const int* __restrict__ pptot,
                               const int* __restrict__ pplist, int L, double4* __restrict__ pm,
                               double2* __restrict__ hz, double4* __restrict__ vel,
                               DevError* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* r = parray + (size_t)i * 6;
  pm[i] = make_double4(r[0], r[1], r[2], r[3]);
  hz[i] = make_double2(r[4], r[5]);
  const double* u = v + (size_t)i * 3;
  vel[i] = make_double4(u[0], u[1], u[2], 0.0);
  const int nn = pptot[i];
  if (nn < 0 || nn > L) {
    set_error(err, SEREN_GPU_ERR_CAPACITY, KID_HYDRO, i, nn);
    return;
  }
  const int* row = pplist + (size_t)i * L;
  for (int k = 0; k < nn; ++k) {
    const int q = row[k];
    if (q < 0 || q >= n) {
      set_error(err, SEREN_GPU_ERR_ARG, KID_HYDRO, i, q);
      return;
    }
  }
}

struct NoallocDevice {
  bool ready = false;
  double* base = nullptr;   // device address of g_noalloc_scratch
};

std::mutex g_noalloc_mutex;
NoallocDevice g_noalloc_dev[64];

// Once per device, with that device current: the device address of the
// scratch array (the host-side name is only a stand-in) and the two kernel
// tables, which stay in the array from then on.
int noalloc_setup(int dev, double** base) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  NoallocDevice& d = g_noalloc_dev[dev];
  if (d.ready) {
    *base = d.base;
    return SEREN_GPU_OK;
  }
  double* ptr = nullptr;
  if (cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch) != cudaSuccess || !ptr)
    return SEREN_GPU_ERR_CUDA;
  for (int kernel = 0; kernel < 2; ++kernel) {
    std::vector<double> w0, w1, w4, w5, w6, wh, wg;
    make_kernel_tables(kernel, w0, w1, w4, w5, w6, wh, wg);
    std::vector<double4> tg(KERNTOT + 1);
    for (int i = 0; i <= KERNTOT; ++i) tg[i] = make_double4(w5[i], w4[i], w6[i], w1[i]);
    if (cudaMemcpy(ptr + NA_TAB + kernel * NA_TABLEN, tg.data(), sizeof(double4) * tg.size(),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return SEREN_GPU_ERR_CUDA;
  }
  d.base = ptr;
  d.ready = true;
  *base = ptr;
  return SEREN_GPU_OK;
}

// Reads the error block after the stream has drained.  Only this call's own
// return codes are looked at: an error the caller's earlier work left pending
// stays pending (no cudaGetLastError here), and is not reported as ours.
int noalloc_status(cudaStream_t st, const DevError* d_err) {
  DevError e{};
  const cudaError_t rc1 = cudaMemcpyAsync(&e, d_err, sizeof(DevError), cudaMemcpyDeviceToHost, st);
  const cudaError_t rc2 = cudaStreamSynchronize(st);
  if (rc1 != cudaSuccess || rc2 != cudaSuccess) return SEREN_GPU_ERR_CUDA;
  return e.code;
}

// Launches through cudaLaunchKernel, whose return code is this launch's own.
template <typename... P, typename... A>
cudaError_t noalloc_launch(void (*kern)(P...), unsigned grid, unsigned block, cudaStream_t st,
                           A... a) {
  auto args = std::make_tuple(static_cast<P>(a)...);
  void* ptrs[sizeof...(P)];
  std::apply([&](auto&... x) {
    int k = 0;
    ((ptrs[k++] = (void*)&x), ...);
  }, args);
  return cudaLaunchKernel((const void*)kern, dim3(grid), dim3(block), ptrs, 0, st);
}

}  // namespace
}  // namespace seren

extern "C" int seren_gpu_hydro_forces_noalloc(int32_t n, const double* parray, const double* v,
                                              const double* rho, const double* omega,
                                              const double* press, const double* sound,
                                              const int32_t* pptot, const int32_t* pplist,
                                              int32_t pp_limit, int32_t kernel, int32_t precision,
                                              double alpha, double* a, void* stream) {
  using namespace seren;
  if (n < 0 || pp_limit < 1 || (kernel != 0 && kernel != 1) ||
      (precision != 0 && precision != 1) || !(alpha >= 0.0))
    return SEREN_GPU_ERR_ARG;
  if (n > NOALLOC_PMAX) return SEREN_GPU_ERR_CAPACITY;
  if (n == 0) return SEREN_GPU_OK;
  if (!parray || !v || !rho || !omega || !press || !sound || !pptot || !pplist || !a)
    return SEREN_GPU_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return SEREN_GPU_ERR_CUDA;
  double* base = nullptr;
  int rc = noalloc_setup(dev, &base);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DevError* d_err = reinterpret_cast<DevError*>(base + NA_ERR);
  double4* pm = reinterpret_cast<double4*>(base + NA_PM);
  double2* hz = reinterpret_cast<double2*>(base + NA_HZ);
  double4* vel = reinterpret_cast<double4*>(base + NA_VEL);
  double* pf = base + NA_PF;
  double* hf4 = base + NA_HF4;
  const double4* tab = reinterpret_cast<const double4*>(base + NA_TAB + kernel * NA_TABLEN);
  // the array keeps the previous call's contents: only the error block must start at zero
  if (cudaMemsetAsync(d_err, 0, sizeof(DevError), st) != cudaSuccess) return SEREN_GPU_ERR_CUDA;
  if (noalloc_launch(k_noalloc_pack, nb(n, 256), 256, st, n, parray, v, pptot, pplist, pp_limit,
                     pm, hz, vel, d_err) != cudaSuccess)
    return SEREN_GPU_ERR_CUDA;
  if ((rc = noalloc_status(st, d_err))) return rc;
  if (noalloc_launch(k_hydro_prep, nb(n, 256), 256, st, n, hz, rho, omega, press, pf, hf4) !=
      cudaSuccess)
    return SEREN_GPU_ERR_CUDA;
  const HydroTree none{};   // every row fits its list, so the kernel never walks a tree
  const int* no_act = nullptr;
  double* no_map = nullptr;
  const double4* no_rec = nullptr;   // the separate arrays, not packed records
  const cudaError_t lrc =
      precision == 0
          ? noalloc_launch(k_hydro<false, 1>, nb(n, 128), 128, st, n, no_act, pm, hz, vel, rho,
                           pf, hf4, sound, pptot, pplist, pp_limit, none, tab, alpha,
                           kernel == 1, a, no_map, d_err, no_rec)
          : noalloc_launch(k_hydro<true, HY_SUB>, nb((long)n * HY_SUB, 128), 128, st, n, no_act,
                           pm, hz, vel, rho, pf, hf4, sound, pptot, pplist, pp_limit, none, tab,
                           alpha, kernel == 1, a, no_map, d_err, no_rec);
  if (lrc != cudaSuccess) return SEREN_GPU_ERR_CUDA;
  return noalloc_status(st, d_err);
}
