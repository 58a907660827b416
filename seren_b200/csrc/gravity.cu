// gravity.cu - Barnes-Hut gravity walk with the geometric MAC, quadrupole
// cell terms and the kernel-softened grad-h near field; direct sink gravity.
//
// Two arithmetic forms share one walk:
//  * FP64: every cell and pair term is the reference expression
//    (BHtree/BHgrav_accel.F90:146-226, gravity/gravity_gradh.F90:57-86) in
//    FP64 with its association and no contraction.
//  * mixed: the walk, the MAC test (drsqd > dminsqd) and the separations stay
//    FP64, so exactly the same cells are accepted and the same pairs visited;
//    the separation is then cast to FP32 and the cell/pair term evaluated in
//    FP32 (rsqrtf, FMA), with the M4 softening kernel read at the reference's
//    table bin from an FP32 copy of its table; terms are summed in FP32 with
//    Kahan compensation and added to the FP64 result once.
#include <algorithm>

#include "ctx.cuh"

namespace seren {

namespace {

struct GravTree {
  const int4* link;
  const double4* gA;   // COM, m
  const double4* gB;   // q1..q4
  const double2* gC;   // q5, dminsqd
  int ctot;
};

// ---------------------------------------------------------------------------
// FP64 terms
__device__ __forceinline__ void cell_term64(double d0, double d1, double d2, double drsqd,
                                            const double4& a, const double4& q, double q5,
                                            double& ax, double& ay, double& az, double& pot) {
  const double invdrsqd = 1.0 / (drsqd + SMALL_NUMBER);
  const double invdrmag = sqrt(invdrsqd);
  const double mm = (a.w * invdrsqd) * invdrmag;
  double t0 = -(mm * d0), t1 = -(mm * d1), t2 = -(mm * d2);
  double dpot = a.w * invdrmag;
  const double invdr5 = (invdrsqd * invdrsqd) * invdrmag;
  const double q1 = q.x, q2 = q.y, q3 = q.z, q4 = q.w;
  const double qscalar = (((q1 * d0) * d0 + (q3 * d1) * d1) - ((q1 + q3) * d2) * d2) +
                         2.0 * ((((q2 * d0) * d1) + ((q4 * d0) * d2)) + ((q5 * d1) * d2));
  t0 = (t0 + (((q1 * d0 + q2 * d1) + q4 * d2) * invdr5)) - ((((2.5 * qscalar) * d0) * invdr5) * invdrsqd);
  t1 = (t1 + (((q2 * d0 + q3 * d1) + q5 * d2) * invdr5)) - ((((2.5 * qscalar) * d1) * invdr5) * invdrsqd);
  t2 = (t2 + (((q4 * d0 + q5 * d1) - (q1 + q3) * d2) * invdr5)) - ((((2.5 * qscalar) * d2) * invdr5) * invdrsqd);
  dpot = dpot + (0.5 * qscalar) * invdr5;
  ax = ax + t0; ay = ay + t1; az = az + t2; pot = pot + dpot;
}

// gravity/gravity_gradh.F90:11-95, dr = rpp - rp
__device__ __forceinline__ void pair_term64(double d0, double d1, double d2, double invhp, double zo_p,
                                            double mq, double hq, double zq,
                                            const double4* __restrict__ tabG, double& ax, double& ay,
                                            double& az, double& pot) {
  const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
  const double drmag = sqrt(drsqd) + SMALL_NUMBER;
  const double invdrmag = 1.0 / drmag;
  double grav, dpot;
  if (invdrmag > INVKERNRANGE * invhp) {
    int kern = (int)((HALFKERNTOT * drmag) * invhp);
    kern = min(kern, KERNTOT);
    const double4 w = tabG[kern];
    grav = (invhp * invhp) * (w.x + ((zo_p * w.y) * invhp) * invhp);
    dpot = invhp * w.z;
  } else {
    grav = invdrmag * invdrmag;
    dpot = invdrmag;
  }
  if (drmag < KERNRANGE * hq) {
    const double invhq = 1.0 / hq;
    int kern = (int)((HALFKERNTOT * drmag) * invhq);
    kern = min(kern, KERNTOT);
    const double4 w = tabG[kern];
    grav = grav + (invhq * invhq) * (w.x + ((zq * w.y) * invhq) * invhq);
    dpot = dpot + invhq * w.z;
  } else {
    grav = grav + invdrmag * invdrmag;
    dpot = dpot + invdrmag;
  }
  const double f = ((0.5 * mq) * invdrmag) * grav;
  ax = ax + f * d0; ay = ay + f * d1; az = az + f * d2;
  pot = pot + (0.5 * mq) * dpot;
}

// gravity/gravity_meanh.F90:12-69
__device__ __forceinline__ void meanh_term64(double d0, double d1, double d2, double hmean, double mq,
                                             const double4* __restrict__ tabG, double& ax,
                                             double& ay, double& az, double& pot) {
  const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
  const double drmag = sqrt(drsqd) + SMALL_NUMBER;
  const double invdrmag = 1.0 / drmag;
  double grav, dpot;
  if (drmag < KERNRANGE * hmean) {
    const double invhmean = 1.0 / hmean;
    int kern = (int)((HALFKERNTOT * drmag) * invhmean);
    kern = min(kern, KERNTOT);
    const double4 w = tabG[kern];
    grav = ((invdrmag * invhmean) * invhmean) * w.x;
    dpot = invhmean * w.z;
  } else {
    grav = invdrmag * (invdrmag * invdrmag);
    dpot = invdrmag;
  }
  const double f = mq * grav;
  ax = ax + f * d0; ay = ay + f * d1; az = az + f * d2;
  pot = pot + mq * dpot;
}

// ---------------------------------------------------------------------------
// FP32 terms (mixed form)
struct Kahan4 {
  float s[4] = {0.f, 0.f, 0.f, 0.f};
  float c[4] = {0.f, 0.f, 0.f, 0.f};
  __device__ __forceinline__ void add(int k, float x) {
    const float y = x - c[k];
    const float t = s[k] + y;
    c[k] = (t - s[k]) - y;
    s[k] = t;
  }
  __device__ __forceinline__ double get(int k) const { return (double)s[k] - (double)c[k]; }
};

__device__ __forceinline__ void count_add(unsigned long long* counts, unsigned long long ncell,
                                          unsigned long long npair) {
  // warp-aggregated interaction counters
  for (int o = 16; o > 0; o >>= 1) {
    ncell += __shfl_down_sync(0xffffffffu, ncell, o);
    npair += __shfl_down_sync(0xffffffffu, npair, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(counts + 0, ncell);
    atomicAdd(counts + 1, npair);
  }
}

// ---------------------------------------------------------------------------
// Frontier walk.  One warp walks the tree for 32 consecutive active particles
// (tree order: spatially adjacent) with the reference's per-particle decisions
// intact.  The walk state is a per-warp stack of entries (cell, mask): the
// cell, and the lanes whose walk reaches it (every ancestor was opened for
// them).  Each step pops up to 32 entries; the lanes load those cells in
// parallel, then every lane runs the reference's MAC test drsqd > dminsqd for
// its own particle against each popped cell in its mask.  That test runs first
// in FP32 on root-relative coordinates against a bracket [lo, hi] around
// dminsqd that covers the FP32 rounding; inside the bracket it is redone in
// FP64 exactly as BHgrav_accel.F90:146-155 does, so every decision equals the
// FP64 one.  Accepted cells go to a cell list with the mask of lanes that took
// them; opened leaves put their particles on a near-field list
// (BHgrav_accel.F90:128-136, :242-253); opened branch cells push their children
// with the mask of lanes that opened them.  Each cell is reached at most once
// per group, so a group processes at most ctot+1 entries.  Full lists are
// flushed by all lanes together (lane-parallel record preparation, then
// broadcast loads and a per-lane predicate).
constexpr int GW_THREADS = 128;
constexpr int GW_WARPS = GW_THREADS / 32;
constexpr int GW_STACK = 8192;   // frontier entries per warp (at most ctot+1 are ever live)
constexpr int GW_PITEMS = 384;   // near-field (particle, mask) items per warp list
constexpr unsigned FULLMASK = 0xffffffffu;

struct GravWalk {
  // two float4 per cell: (FP32 COM relative to the root centre, hi bracket),
  // (lo bracket, first particle of a leaf / first child of a branch, leaf
  // count / -children, 0) as int bits
  const float4* wN;
  const double4* gA;
  const double4* gB;
  const double2* gC;
  int ctot;
  int scap;             // stack entries per warp
  double rootx, rooty, rootz;
  int root;             // root cell of the walks
  const CloudInfo* cl;  // a forest of ncl trees (NULL: one tree)
  int ncl;
};

// gravity_gradh.F90:57-86 in FP32, dr = rpp - rp, invhq precomputed.  The M4
// softened-gravity functions w5, w4, w6 (setup/kernel.F90:80-81, :99-102) come
// from an FP32 copy of the reference's table at bin int(5000 r/h), clamped to
// KERNTOT (tab32[k] = w5, w4, w6).
// (inv = 1/r and drmag = r as the caller formed them from d for its branch test)
__device__ __forceinline__ void pair32(float d0, float d1, float d2, float inv, float drmag,
                                       float invhp, float zo_p, float mq, float invhq, float zq,
                                       const float4* __restrict__ tab32, float& ax, float& ay,
                                       float& az, float& ap) {
  const float xp = drmag * invhp;
  const float xq = drmag * invhq;
  const float4 wp = tab32[(int)fminf(5000.0f * xp, (float)KERNTOT)];
  const float4 wq = tab32[(int)fminf(5000.0f * xq, (float)KERNTOT)];
  const float ihp2 = invhp * invhp;
  const float inv2 = inv * inv;
  float grav = xp < KERNRANGE ? ihp2 * fmaf(zo_p * wp.y, ihp2, wp.x) : inv2;
  float dpot = xp < KERNRANGE ? invhp * wp.z : inv;
  const float ihq2 = invhq * invhq;
  grav += xq < KERNRANGE ? ihq2 * fmaf(zq * wq.y, ihq2, wq.x) : inv2;
  dpot += xq < KERNRANGE ? invhq * wq.z : inv;
  const float f = 0.5f * mq * inv * grav;
  ax = fmaf(f, d0, ax);
  ay = fmaf(f, d1, ay);
  az = fmaf(f, d2, az);
  ap = fmaf(0.5f * mq, dpot, ap);
}

// pair32 when r >= 2h_p and r >= 2h_q: both kernel branches are Newtonian
// (the same operations pair32 performs for such a pair)
__device__ __forceinline__ void pair32_far(float d0, float d1, float d2, float inv, float mq,
                                           float& ax, float& ay, float& az, float& ap) {
  const float inv2 = inv * inv;
  const float grav = inv2 + inv2;
  const float dpot = inv + inv;
  const float f = 0.5f * mq * inv * grav;
  ax = fmaf(f, d0, ax);
  ay = fmaf(f, d1, ay);
  az = fmaf(f, d2, az);
  ap = fmaf(0.5f * mq, dpot, ap);
}

// BHgrav_accel.F90:159-189 in FP32, dr = rp - rc, q holds q1..q4, q5z (q5,
// -(q1 + q3)), m the cell mass.  Written with the unit vector n = dr/r so that
// no power of 1/r above the second is formed: with Qn = Q.n and nQn = n.Q.n,
//   a = (1/r^2) [ n (-m - 2.5 nQn/r^2) + Qn/r^2 ],  phi = (1/r) (m + nQn/(2 r^2)),
// the reference's -m dr/r^3 + (Q.dr)/r^5 - 2.5 (dr.Q.dr) dr/r^7 and
// m/r + (dr.Q.dr)/(2 r^5).  |Q|/r^2 is of order m theta^2 for an accepted cell,
// so every FP32 intermediate stays in range however small the cell and its
// distance (1/r^7 alone overflows FP32 below r ~ 4e-6).
__device__ __forceinline__ void cell32(float d0, float d1, float d2, float m, const float4& q,
                                       const float2& q5z, float& ax, float& ay, float& az,
                                       float& ap) {
  const float drsqd = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
  const float invr = rsqrtf(drsqd);
  const float invr2 = invr * invr;
  const float n0 = d0 * invr, n1 = d1 * invr, n2 = d2 * invr;
  const float qx = fmaf(q.w, n2, fmaf(q.y, n1, q.x * n0));
  const float qy = fmaf(q5z.x, n2, fmaf(q.z, n1, q.y * n0));
  const float qz = fmaf(q5z.y, n2, fmaf(q5z.x, n1, q.w * n0));
  const float nqn = fmaf(qz, n2, fmaf(qy, n1, qx * n0)) * invr2;
  const float g = fmaf(-2.5f, nqn, -m);
  ax = fmaf(invr2, fmaf(g, n0, qx * invr2), ax);
  ay = fmaf(invr2, fmaf(g, n1, qy * invr2), ay);
  az = fmaf(invr2, fmaf(g, n2, qz * invr2), az);
  ap = fmaf(invr, fmaf(0.5f, nqn, m), ap);
}

template <bool MIXED>
struct GwTypes {
  using R = float;
  using R2 = float2;
  using R4 = float4;
  using Q5 = float2;               // q5, -(q1 + q3)
  static constexpr int CAP = 64;   // accepted-cell entries per warp list
  static constexpr int PREP = 96;  // near-field records prepared per flush pass
};
template <>
struct GwTypes<false> {
  using R = double;
  using R2 = double2;
  using R4 = double4;
  using Q5 = double;
  static constexpr int CAP = 64;
  static constexpr int PREP = 64;
};

// Per-warp shared state: interaction lists, prepared records, popped cells.
// CAPV: accepted-cell entries per list (the cell-list tile; a tuning knob of
// the mixed-precision kernel, 64 for the FP64 one).
template <bool MIXED, int CAPV>
struct GwRec {
  using T = GwTypes<MIXED>;
  typename T::R4 ca[CAPV];         // cell: mixed (r_ref - COM, m), FP64 (COM, m)
  typename T::R4 cb[CAPV];         // q1..q4
  typename T::Q5 cq5[CAPV];
  int cid[CAPV];
  unsigned cmask[CAPV];
  int qid[GW_PITEMS];
  unsigned qmask[GW_PITEMS];
  typename T::R4 pa[T::PREP];      // particle: mixed (r_q - r_ref, m), FP64 (r_q, m)
  typename T::R2 pb[T::PREP];      // mixed (1/h, zeta), FP64 (h, zeta)
  float4 fw[32];                   // popped cells: wA
  float flo[32];                   // lower MAC bracket
  unsigned ftest[32];              // lanes that test the cell (0 for one-particle leaves)
  int fcell[32];
  int fund[32];                    // popped cells the group test leaves undecided
};

__device__ __forceinline__ int warp_incl(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULLMASK, v, o);
    if (lane >= o) v += y;
  }
  return v;
}

template <bool MIXED, int CAPV>
__global__ void __launch_bounds__(GW_THREADS, MIXED ? 5 : 4)
k_grav_walk(int nact, const int* __restrict__ act, const double4* __restrict__ pm,
            const double2* __restrict__ hz, GravWalk t, const double4* __restrict__ tabG,
            const float4* __restrict__ tab32, double* __restrict__ acc,
            double* __restrict__ gpot, const double* abase, double* amap, double* __restrict__ gmap,
            int nsink, const double* __restrict__ sinks,
            int2* __restrict__ stacks, int* work, DevError* err, unsigned long long* counts) {
  using Cfg = GwTypes<MIXED>;
  constexpr int CAP = CAPV;
  __shared__ GwRec<MIXED, CAPV> srec[GW_WARPS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  GwRec<MIXED, CAPV>& R = srec[w];
  int2* const S = stacks + (size_t)(blockIdx.x * GW_WARPS + w) * t.scap;
  const unsigned lt = (1u << lane) - 1u;
  unsigned long long ncell = 0, npair = 0, nent = 0;
  unsigned ce_all = 0, ce_full = 0, pi_all = 0, pi_full = 0;   // list fill statistics

  while (true) {
    int g = 0;
    if (lane == 0) g = atomicAdd(work, 1);
    g = __shfl_sync(FULLMASK, g, 0);
    if ((long long)g * 32 >= nact) break;
    const int i = g * 32 + lane;
    // act[i] < 0 pads a cloud's last group in a forest; dead lanes take lane
    // 0's particle (always live)
    int p = i < nact ? (act ? act[i] : i) : -1;
    const bool live = p >= 0;
    const int p0 = __shfl_sync(FULLMASK, p, 0);        // every lane takes part
    p = live ? p : p0;
    // the lanes' tree (a forest: their cloud's), as locals so that t stays a
    // kernel parameter
    int root = t.root;
    double rootx = t.rootx, rooty = t.rooty, rootz = t.rootz;
    if (t.cl) {
      const CloudInfo& C = t.cl[cloud_of(t.cl, t.ncl, p)];
      root = C.cell;
      rootx = C.root[0];
      rooty = C.root[1];
      rootz = C.root[2];
    }
    const double4 P = pm[p];
    const double2 HZ = hz[p];
    // warp reference point (lane 0 is always live)
    const double rx = __shfl_sync(FULLMASK, P.x, 0);
    const double ry = __shfl_sync(FULLMASK, P.y, 0);
    const double rz = __shfl_sync(FULLMASK, P.z, 0);
    const float px32 = (float)(P.x - rootx), py32 = (float)(P.y - rooty),
                pz32 = (float)(P.z - rootz);
    const float ux = (float)(P.x - rx), uy = (float)(P.y - ry), uz = (float)(P.z - rz);
    // A separation formed in FP32 from two offsets to the reference point
    // (d = a - u) carries an error of order 2^-24 |u|, relative 2^-23 |u|/|d|;
    // the FP64 particle is used instead when some lane lies more than 64
    // smoothing lengths (the group's least) from the reference point, e.g. a
    // group that straddles a dense clump and its sparse surroundings (within
    // that bound a pair at distance h is off by less than 1e-5 relative).
    bool wide = false;
    if constexpr (MIXED) {
      float umax = live ? sqrtf(fmaf(uz, uz, fmaf(uy, uy, ux * ux))) : 0.0f;
      float hmin = live ? (float)HZ.x : 3.0e38f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        umax = fmaxf(umax, __shfl_xor_sync(FULLMASK, umax, o));
        hmin = fminf(hmin, __shfl_xor_sync(FULLMASK, hmin, o));
      }
      wide = umax > 64.0f * hmin;
    }
    // the group's bounding sphere in the walk's FP32 coordinates: centre the
    // middle of the live lanes' bounding box, radius the farthest live lane's
    // distance from it, rounded up
    float gx, gy, gz;
    {
      const float x0 = __shfl_sync(FULLMASK, px32, 0), y0 = __shfl_sync(FULLMASK, py32, 0),
                  z0 = __shfl_sync(FULLMASK, pz32, 0);
      float lox = live ? px32 : x0, loy = live ? py32 : y0, loz = live ? pz32 : z0;
      float hix = lox, hiy = loy, hiz = loz;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        lox = fminf(lox, __shfl_xor_sync(FULLMASK, lox, o));
        loy = fminf(loy, __shfl_xor_sync(FULLMASK, loy, o));
        loz = fminf(loz, __shfl_xor_sync(FULLMASK, loz, o));
        hix = fmaxf(hix, __shfl_xor_sync(FULLMASK, hix, o));
        hiy = fmaxf(hiy, __shfl_xor_sync(FULLMASK, hiy, o));
        hiz = fmaxf(hiz, __shfl_xor_sync(FULLMASK, hiz, o));
      }
      gx = 0.5f * (lox + hix);
      gy = 0.5f * (loy + hiy);
      gz = 0.5f * (loz + hiz);
    }
    float grad;
    {
      const float e0 = px32 - gx, e1 = py32 - gy, e2 = pz32 - gz;
      float r2 = live ? fmaf(e2, e2, fmaf(e1, e1, e0 * e0)) : 0.0f;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) r2 = fmaxf(r2, __shfl_xor_sync(FULLMASK, r2, o));
      grad = sqrtf(r2) * 1.00001f;
    }
    const double invhp = 1.0 / HZ.x;
    const double zo_p = HZ.y;
    const float invhp32 = (float)invhp, zo32 = (float)zo_p;
    Kahan4 kc;
    double cx = 0.0, cy = 0.0, cz = 0.0, cp = 0.0, qx = 0.0, qy = 0.0, qz = 0.0, qp = 0.0;
    int nc = 0, np = 0;

    auto flush_cells = [&]() {
      __syncwarp();
      for (int e = lane; e < nc; e += 32) {                  // lane-parallel preparation
        const int cid = R.cid[e];
        const double4 a = t.gA[cid];
        const double4 q = t.gB[cid];
        const double q5 = t.gC[cid].x;
        if constexpr (MIXED) {
          ncell += __popc(R.cmask[e]);                       // the terms this entry gives
          R.ca[e] = make_float4((float)(rx - a.x), (float)(ry - a.y), (float)(rz - a.z), (float)a.w);
          R.cb[e] = make_float4((float)q.x, (float)q.y, (float)q.z, (float)q.w);
          R.cq5[e] = make_float2((float)q5, (float)(-(q.x + q.z)));
        } else {
          R.ca[e] = a;
          R.cb[e] = q;
          R.cq5[e] = q5;
        }
      }
      __syncwarp();
      if constexpr (MIXED) {
        float sx = 0.f, sy = 0.f, sz = 0.f, sp = 0.f;
        if (!wide) {
#pragma unroll 2
          for (int e = 0; e < nc; ++e) {
            if ((R.cmask[e] >> lane) & 1u) {
              const float4 a = R.ca[e];
              cell32(ux + a.x, uy + a.y, uz + a.z, a.w, R.cb[e], R.cq5[e], sx, sy, sz, sp);
            }
          }
        } else {
          for (int e = 0; e < nc; ++e) {
            if ((R.cmask[e] >> lane) & 1u) {
              const double4 A = t.gA[R.cid[e]];
              cell32((float)(P.x - A.x), (float)(P.y - A.y), (float)(P.z - A.z), R.ca[e].w,
                     R.cb[e], R.cq5[e], sx, sy, sz, sp);
            }
          }
        }
        kc.add(0, sx); kc.add(1, sy); kc.add(2, sz); kc.add(3, sp);
      } else {
        for (int e = 0; e < nc; ++e) {
          if ((R.cmask[e] >> lane) & 1u) {
            const double4 a = R.ca[e];
            const double d0 = P.x - a.x, d1 = P.y - a.y, d2 = P.z - a.z;
            cell_term64(d0, d1, d2, (d0 * d0 + d1 * d1) + d2 * d2, a, R.cb[e], R.cq5[e], cx, cy,
                        cz, cp);
            ++ncell;
          }
        }
      }
      nc = 0;
      __syncwarp();
    };
    auto flush_pairs = [&]() {
      for (int b0 = 0; b0 < np; b0 += Cfg::PREP) {
        const int nb = min(Cfg::PREP, np - b0);
        __syncwarp();
        for (int e = lane; e < nb; e += 32) {
          const int q = R.qid[b0 + e];
          const double4 Q = pm[q];
          const double2 H = hz[q];
          if constexpr (MIXED) {
            // the pairs this item gives (each lane's own particle, one item
            // of its list, is taken off at the end of the group)
            npair += __popc(R.qmask[b0 + e]);
            R.pa[e] = make_float4((float)(Q.x - rx), (float)(Q.y - ry), (float)(Q.z - rz), (float)Q.w);
            R.pb[e] = make_float2((float)(1.0 / H.x), (float)H.y);
          } else {
            R.pa[e] = Q;
            R.pb[e] = H;
          }
        }
        __syncwarp();
        if constexpr (MIXED) {
          float sx = 0.f, sy = 0.f, sz = 0.f, sp = 0.f;
          auto item = [&](int e, float d0, float d1, float d2) {
            const bool on = ((R.qmask[b0 + e] >> lane) & 1u) && R.qid[b0 + e] != p;
            const float4 a = R.pa[e];
            const float2 b = R.pb[e];
            const float drsqd = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
            const float inv = rsqrtf(fmaxf(drsqd, 1.0e-30f));
            const float drmag = drsqd * inv;
            // pair32's own branch tests: the kernel is needed only inside 2h of either particle
            const bool soft = on && (drmag * invhp32 < KERNRANGE || drmag * b.x < KERNRANGE);
            if (__any_sync(FULLMASK, soft)) {
              if (on) pair32(d0, d1, d2, inv, drmag, invhp32, zo32, a.w, b.x, b.y, tab32, sx, sy,
                             sz, sp);
            } else if (on) {
              pair32_far(d0, d1, d2, inv, a.w, sx, sy, sz, sp);
            }
          };
          if (!wide) {
#pragma unroll 2
            for (int e = 0; e < nb; ++e) {
              const float4 a = R.pa[e];
              item(e, a.x - ux, a.y - uy, a.z - uz);
            }
          } else {
            for (int e = 0; e < nb; ++e) {
              const double4 Q = pm[R.qid[b0 + e]];
              item(e, (float)(Q.x - P.x), (float)(Q.y - P.y), (float)(Q.z - P.z));
            }
          }
          kc.add(0, sx); kc.add(1, sy); kc.add(2, sz); kc.add(3, sp);
        } else {
          for (int e = 0; e < nb; ++e) {
            if (((R.qmask[b0 + e] >> lane) & 1u) && R.qid[b0 + e] != p) {
              const double4 Q = R.pa[e];
              const double2 H = R.pb[e];
              pair_term64(Q.x - P.x, Q.y - P.y, Q.z - P.z, invhp, zo_p, Q.w, H.x, H.y, tabG, qx,
                          qy, qz, qp);
              ++npair;
            }
          }
        }
      }
      np = 0;
      __syncwarp();
    };

    const unsigned rootmask = __ballot_sync(FULLMASK, live);
    if (lane == 0) S[0] = make_int2(root, (int)rootmask);
    int sp = 1;
    long long gent = 0;
    while (sp > 0) {
      __syncwarp();
      const int k = min(32, sp);
      sp -= k;
      gent += k;
      int cc = 0, cnt = 0, base = 0;     // cnt: leaf particles, or -children of a branch
      unsigned m = 0;
      // group test of the popped cell: 1 when every lane's FP32 prefilter
      // would pass it (d2s > hi: nearest possible lane beyond the bracket),
      // 2 when none would reach the bracket (d2s < lo for the farthest
      // possible lane, or a one-particle leaf, which has no MAC test), 0 when
      // each lane tests it; margins of 1e-5 cover every FP32 rounding, so the
      // decisions are the per-lane ones
      int dec = 0;
      if (lane < k) {
        const int2 ent = S[sp + lane];
        cc = ent.x;
        m = (unsigned)ent.y;
        const float4 na = t.wN[2 * cc], nb2 = t.wN[2 * cc + 1];
        cnt = __float_as_int(nb2.z);
        base = __float_as_int(nb2.y);
        R.fw[lane] = na;
        R.flo[lane] = nb2.x;
        R.ftest[lane] = cnt == 1 ? 0u : m;
        R.fcell[lane] = cc;
        if (cnt == 1) {
          dec = 2;
        } else {
          const float e0 = gx - na.x, e1 = gy - na.y, e2 = gz - na.z;
          const float D = sqrtf(fmaf(e2, e2, fmaf(e1, e1, e0 * e0)));
          const float dn = fmaf(D, 0.99999f, -grad);      // at most the nearest lane's distance
          const float df = fmaf(D, 1.00001f, grad);       // at least the farthest lane's
          if (dn > 0.0f && (dn * dn) * 0.99999f > na.w) dec = 1;
          else if ((df * df) * 1.00001f < nb2.x) dec = 2;
        }
      }
      unsigned macc = dec == 1 ? m : 0u;
      const unsigned und = __ballot_sync(FULLMASK, lane < k && dec == 0);
      if (lane < k && dec == 0) R.fund[__popc(und & lt)] = lane;
      __syncwarp();
      // each lane's MAC test on the undecided cells, four at a time with their
      // loads issued first; a lane inside the FP32 bracket takes the exact
      // FP64 test (rare, a warp-uniform branch)
      const int ku = __popc(und);
      for (int e0 = 0; e0 < ku; e0 += 4) {
        int ie[4];
        float4 wa[4];
        float lo[4];
        unsigned mt[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          ie[u] = R.fund[min(e0 + u, ku - 1)];
          wa[u] = R.fw[ie[u]];
          lo[u] = R.flo[ie[u]];
          mt[u] = e0 + u < ku ? R.ftest[ie[u]] : 0u;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const bool mine = (mt[u] >> lane) & 1u;
          const float d0 = px32 - wa[u].x, d1 = py32 - wa[u].y, d2 = pz32 - wa[u].z;
          const float d2s = fmaf(d2, d2, fmaf(d1, d1, d0 * d0));
          const bool hi = d2s > wa[u].w;
          unsigned b = __ballot_sync(FULLMASK, mine && hi);
          const bool amb = mine && !hi && d2s >= lo[u];
          if (__any_sync(FULLMASK, amb)) {                   // exact test, :146-155
            bool a2 = false;
            if (amb) {
              const int ce = R.fcell[ie[u]];
              const double4 a = t.gA[ce];
              const double e0d = P.x - a.x, e1d = P.y - a.y, e2d = P.z - a.z;
              a2 = ((e0d * e0d + e1d * e1d) + e2d * e2d) > t.gC[ce].y;
            }
            b |= __ballot_sync(FULLMASK, a2);
          }
          if (e0 + u < ku && lane == ie[u]) macc = b;
        }
      }
      const unsigned mopn = m & ~macc;
      // accepted cells
      const unsigned bc = __ballot_sync(FULLMASK, macc != 0u);
      if (macc != 0u) {
        const int o = nc + __popc(bc & lt);
        R.cid[o] = cc;
        R.cmask[o] = macc;
        ++ce_all;
        ce_full += macc == rootmask;
      }
      nc += __popc(bc);
      // opened leaves: their particles join the near-field list
      const int npush = (cnt > 0 && mopn != 0u) ? cnt : 0;
      pi_all += npush;
      pi_full += mopn == rootmask ? npush : 0;
      const int pin = warp_incl(npush, lane);
      for (int q = 0; q < npush; ++q) {
        R.qid[np + pin - npush + q] = base + q;
        R.qmask[np + pin - npush + q] = mopn;
      }
      np += __shfl_sync(FULLMASK, pin, 31);
      // opened branch cells: children onto the stack
      const int nch = (cnt < 0 && mopn != 0u) ? -cnt : 0;
      const int cin = warp_incl(nch, lane);
      const int ctotal = __shfl_sync(FULLMASK, cin, 31);
      if (sp + ctotal > t.scap || gent > (long long)t.ctot + 1) {
        if (lane == 0) set_error(err, SEREN_GPU_ERR_WALK, MIXED ? KID_GRAV_MIXED : KID_GRAV, p, cc);
        break;
      }
      for (int q = 0; q < nch; ++q) S[sp + cin - nch + q] = make_int2(base + q, (int)mopn);
      sp += ctotal;
      if (nc > CAP - 32) flush_cells();
      if (np > GW_PITEMS - 32 * LEAFMAX) flush_pairs();
    }
    nent += gent;
    flush_cells();
    flush_pairs();
    if constexpr (MIXED) npair -= live ? 1u : 0u;           // the lane's own particle
    if (live) {
      double ax, ay, az, pot;
      if constexpr (MIXED) {
        ax = kc.get(0); ay = kc.get(1); az = kc.get(2); pot = kc.get(3);
      } else {
        ax = cx + qx; ay = cy + qy; az = cz + qz; pot = cp + qp;
      }
      double* a = acc + (size_t)p * 3;
      // the acceleration gravity adds to: acc, or a mapped host buffer
      const double* ab = abase ? abase + (size_t)p * 3 : a;
      a[0] = ab[0] + ax;
      a[1] = ab[1] + ay;
      a[2] = ab[2] + az;
      if (nsink > 0) {                                       // sinks/direct_sink_gravity.F90
        double sx = 0.0, sy = 0.0, sz = 0.0, sp2 = 0.0;
        for (int s = 0; s < nsink; ++s) {
          const double* sr = sinks + s * 5;
          meanh_term64(sr[0] - P.x, sr[1] - P.y, sr[2] - P.z, 0.5 * (HZ.x + sr[4]), sr[3], tabG,
                       sx, sy, sz, sp2);
        }
        a[0] = a[0] + sx;
        a[1] = a[1] + sy;
        a[2] = a[2] + sz;
        pot = pot + sp2;
      }
      gpot[p] = pot;
      // host buffers mapped into the device address space: the results
      // cross PCIe while the other groups still compute
      if (amap) {
        amap[(size_t)p * 3] = a[0];
        amap[(size_t)p * 3 + 1] = a[1];
        amap[(size_t)p * 3 + 2] = a[2];
      }
      if (gmap) gmap[p] = pot;
    }
  }
  count_add(counts, ncell, npair);
  count_add(counts + 9, ce_all, ce_full);
  count_add(counts + 11, pi_all, pi_full);
  if (lane == 0) atomicAdd(counts + 2, nent);
}


// sph_sim/sph_sink_forces.F90:49-110: BHgrav_accel(-s) with gravity_meanh
// near field (BHgrav_accel.F90:299-314), then the other sinks directly.
__global__ void k_sink_walk(int nsink, const double* __restrict__ sinks, const double4* __restrict__ pm,
                            const double2* __restrict__ hz, GravTree t,
                            const double4* __restrict__ tabG, double* __restrict__ out,
                            DevError* err) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsink) return;
  const double* sr = sinks + s * 5;
  const double rx = sr[0], ry = sr[1], rz = sr[2];
  const double invhp = 1.0 / sr[4];
  const double hp = 1.0 / invhp;
  double cx = 0.0, cy = 0.0, cz = 0.0, cp = 0.0, px = 0.0, py = 0.0, pz = 0.0, pp = 0.0;
  int c = 0, visits = 0;
  const int cap = t.ctot + 2;
  while (true) {
    if (++visits > cap) {
      set_error(err, SEREN_GPU_ERR_WALK, KID_SINK, s, c);
      break;
    }
    const int4 lk = t.link[c];
    if (lk.x == 1) {
      const double4 Q = pm[lk.w];
      meanh_term64(Q.x - rx, Q.y - ry, Q.z - rz, 0.5 * (hp + hz[lk.w].x), Q.w, tabG, px, py, pz, pp);
      c = lk.y;
    } else {
      const double4 a = t.gA[c];
      const double d0 = rx - a.x, d1 = ry - a.y, d2 = rz - a.z;
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      const double2 cc = t.gC[c];
      if (drsqd > cc.y) {
        cell_term64(d0, d1, d2, drsqd, a, t.gB[c], cc.x, cx, cy, cz, cp);
        c = lk.y;
      } else if (lk.x > 0) {
        for (int k = 0; k < lk.x; ++k) {
          const double4 Q = pm[lk.w + k];
          meanh_term64(Q.x - rx, Q.y - ry, Q.z - rz, 0.5 * (hp + hz[lk.w + k].x), Q.w, tabG, px, py,
                       pz, pp);
        }
        c = lk.y;
      } else if (lk.x == 0) {
        c = lk.z;
      } else {
        c = lk.y;
      }
    }
    if (c > t.ctot) break;
  }
  double ax = cx + px, ay = cy + py, az = cz + pz, pot = cp + pp;
  double sx = 0.0, sy = 0.0, sz = 0.0, sp = 0.0;
  for (int ss = 0; ss < nsink; ++ss) {
    if (ss == s) continue;
    const double* o = sinks + ss * 5;
    meanh_term64(o[0] - rx, o[1] - ry, o[2] - rz, 0.5 * (sr[4] + o[4]), o[3], tabG, sx, sy, sz, sp);
  }
  out[s * 4 + 0] = ax + sx;
  out[s * 4 + 1] = ay + sy;
  out[s * 4 + 2] = az + sz;
  out[s * 4 + 3] = pot + sp;
}

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

GravTree grav_tree(const Ctx& c) { return GravTree{c.link, c.gA, c.gB, c.gC, c.info.ctot}; }

}  // namespace

// resident blocks per SM of the walk variant (FP64; mixed with a cell-list
// tile of 64 or 96 entries)
static int grav_blocks_per_sm(int dev, bool mixed, int cap = 64) {
  static int occ[16][3] = {};
  int dummy[3] = {0, 0, 0};
  int* o = dev >= 0 && dev < 16 ? occ[dev] : dummy;
  const int which = !mixed ? 0 : (cap > 64 ? 2 : 1);
  int& r = o[which];
  if (r == 0) {
    if (which == 2)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_grav_walk<true, 96>, GW_THREADS, 0);
    else if (which == 1)
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_grav_walk<true, 64>, GW_THREADS, 0);
    else
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, k_grav_walk<false, 64>, GW_THREADS, 0);
    if (r < 1) r = 1;
  }
  return r;
}

static int sm_count(const Ctx& c) {
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c.dev);
  return nsm;
}

int grav_walk_slots(const Ctx& c) {
  return sm_count(c) *
         std::max(std::max(grav_blocks_per_sm(c.dev, true, 64), grav_blocks_per_sm(c.dev, true, 96)),
                  grav_blocks_per_sm(c.dev, false)) *
         GW_WARPS;
}

int grav_walk_stack_cap(const Ctx& c) { return std::min(GW_STACK, c.cmax + 1); }

void launch_grav(Ctx& c, int nact, int nsink, const double* d_sinks, double* amap,
                 double* gmap, const double* abase) {
  if (nact <= 0) return;
  unsigned long long* counts = reinterpret_cast<unsigned long long*>(c.d_counts);
  const GravWalk gw{c.wA, c.gA, c.gB, c.gC, c.info.ctot, c.wstack_cap,
                    c.info.root[0], c.info.root[1], c.info.root[2], 0,
                    c.ncloud > 1 ? c.d_clouds : nullptr, c.ncloud};
  const bool mixed = c.prm.precision != 0;
  // in a forest with every particle active the groups follow the clouds
  const int* gl = c.act;
  if (!c.act && c.ncloud > 1) {
    gl = c.gact;
    nact = c.ngact;
  }
  const int groups = nb(nact, 32);
  // the tuning knobs: cell-list tile (mixed) and resident blocks per SM
  const int cap = mixed && c.tune.grav_cap > 64 ? 96 : 64;
  int bps = grav_blocks_per_sm(c.dev, mixed, cap);
  if (c.tune.grav_bps > 0) bps = std::min(bps, c.tune.grav_bps);
  const int blocks = std::min(sm_count(c) * bps, nb(groups, GW_WARPS));
  cudaMemsetAsync(c.work, 0, sizeof(int), c.st);
  if (!mixed)
    k_grav_walk<false, 64><<<blocks, GW_THREADS, 0, c.st>>>(nact, gl, c.pm, c.hz, gw, c.tabG,
        c.tabG32, c.acc, c.gpot, abase, amap, gmap, nsink, d_sinks, c.wstack, c.work, c.d_err,
        counts);
  else if (cap == 96)
    k_grav_walk<true, 96><<<blocks, GW_THREADS, 0, c.st>>>(nact, gl, c.pm, c.hz, gw, c.tabG,
        c.tabG32, c.acc, c.gpot, abase, amap, gmap, nsink, d_sinks, c.wstack, c.work, c.d_err,
        counts);
  else
    k_grav_walk<true, 64><<<blocks, GW_THREADS, 0, c.st>>>(nact, gl, c.pm, c.hz, gw, c.tabG,
        c.tabG32, c.acc, c.gpot, abase, amap, gmap, nsink, d_sinks, c.wstack, c.work, c.d_err,
        counts);
  ++c.nlaunch;
}

void launch_sink_walk(Ctx& c, int nsink, const double* d_sinks, double* d_out) {
  if (nsink <= 0) return;
  k_sink_walk<<<nb(nsink, 32), 32, 0, c.st>>>(nsink, d_sinks, c.pm, c.hz, grav_tree(c), c.tabG,
                                              d_out, c.d_err); ++c.nlaunch;
}

}  // namespace seren
