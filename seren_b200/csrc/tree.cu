// tree.cu - octree build, particle reorder, stocking, hmax update and h guess.
//
// The reference (BHtree/BHgrav_build.F90:12-309) splits cells level by level
// with linked lists and numbers the children of every level serially in
// (parent, octant) order.  Its result is a pure function of the particles'
// octant paths: a cell is the set of particles sharing a path prefix, cell
// ids are breadth-first in (level, path) order, and a leaf lists its
// particles in increasing input index.  Here the same tree is made from a
// sort: each particle's octant path is computed from the same FP64 centre
// comparisons (rp > rc with rc built by repeated +/- cellsize), packed into a
// 63-bit key, and stably radix-sorted; cells are then the runs of a common
// prefix, emitted level by level in breadth-first order, and each leaf's
// particles are put back into input-index order.
#include <cstdio>
#include <cstring>

#include "ctx.cuh"

namespace seren {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// ---------------------------------------------------------------------------
// exclusive scan of int32 (block tiles of 2048, recursive on block sums)
constexpr int SCAN_T = 512;
constexpr int SCAN_I = 4;
constexpr int SCAN_TILE = SCAN_T * SCAN_I;

__global__ void k_scan_tile(const int* __restrict__ in, int* __restrict__ out, int n,
                            int* __restrict__ block_sums) {
  __shared__ int wsum[SCAN_T / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long base = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_I;
  int v[SCAN_I];
  int s = 0;
#pragma unroll
  for (int j = 0; j < SCAN_I; ++j) {
    v[j] = (base + j < n) ? in[base + j] : 0;
    s += v[j];
  }
  int x = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int ws = (lane < SCAN_T / 32) ? wsum[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(FULL, ws, o);
      if (lane >= o) ws += y;
    }
    if (lane < SCAN_T / 32) wsum[lane] = ws;
  }
  __syncthreads();
  int excl = x - s + (w > 0 ? wsum[w - 1] : 0);
#pragma unroll
  for (int j = 0; j < SCAN_I; ++j) {
    if (base + j < n) out[base + j] = excl;
    excl += v[j];
  }
  if (threadIdx.x == SCAN_T - 1) block_sums[blockIdx.x] = excl;
}

__global__ void k_scan_add(int* __restrict__ out, int n, const int* __restrict__ offs) {
  const long base = (long)blockIdx.x * SCAN_TILE;
  const int off = offs[blockIdx.x];
  for (int j = threadIdx.x; j < SCAN_TILE; j += SCAN_T) {
    const long i = base + j;
    if (i < n) out[i] += off;
  }
}

__global__ void k_copy_int(const int* __restrict__ src, int* __restrict__ dst) { *dst = *src; }

// ---------------------------------------------------------------------------
// bounding box (main/bounding_box.F90:9-43) and root cell (BHgrav_build.F90:65-67)
constexpr int BB_T = 256;

__global__ void k_bbox_partial(const double4* __restrict__ pm, int n, double* __restrict__ part) {
  __shared__ double s[6][BB_T];
  double mx[3] = {-BIG_NUMBER, -BIG_NUMBER, -BIG_NUMBER};
  double mn[3] = {BIG_NUMBER, BIG_NUMBER, BIG_NUMBER};
  for (long i = (long)blockIdx.x * BB_T + threadIdx.x; i < n; i += (long)gridDim.x * BB_T) {
    const double4 p = pm[i];
    mx[0] = fmax(mx[0], p.x); mx[1] = fmax(mx[1], p.y); mx[2] = fmax(mx[2], p.z);
    mn[0] = fmin(mn[0], p.x); mn[1] = fmin(mn[1], p.y); mn[2] = fmin(mn[2], p.z);
  }
  for (int k = 0; k < 3; ++k) { s[k][threadIdx.x] = mx[k]; s[3 + k][threadIdx.x] = mn[k]; }
  __syncthreads();
  for (int o = BB_T / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 3; ++k) {
        s[k][threadIdx.x] = fmax(s[k][threadIdx.x], s[k][threadIdx.x + o]);
        s[3 + k][threadIdx.x] = fmin(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + o]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) part[blockIdx.x * 6 + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void k_bbox_final(const double* __restrict__ part, int nblk, TreeInfo* info) {
  __shared__ double s[6][BB_T];
  double mx[3] = {-BIG_NUMBER, -BIG_NUMBER, -BIG_NUMBER};
  double mn[3] = {BIG_NUMBER, BIG_NUMBER, BIG_NUMBER};
  for (int b = threadIdx.x; b < nblk; b += BB_T)
    for (int k = 0; k < 3; ++k) {
      mx[k] = fmax(mx[k], part[b * 6 + k]);
      mn[k] = fmin(mn[k], part[b * 6 + 3 + k]);
    }
  for (int k = 0; k < 3; ++k) { s[k][threadIdx.x] = mx[k]; s[3 + k][threadIdx.x] = mn[k]; }
  __syncthreads();
  for (int o = BB_T / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 3; ++k) {
        s[k][threadIdx.x] = fmax(s[k][threadIdx.x], s[k][threadIdx.x + o]);
        s[3 + k][threadIdx.x] = fmin(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + o]);
      }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double rmax[3] = {s[0][0], s[1][0], s[2][0]};
  const double rmin[3] = {s[3][0], s[4][0], s[5][0]};
  const double ext = fmax(fmax(rmax[0] - rmin[0], rmax[1] - rmin[1]), rmax[2] - rmin[2]);
  info->rextent = ext;
  info->cellsize = 0.5 * ext;
  for (int k = 0; k < 3; ++k) info->root[k] = 0.5 * (rmin[k] + rmax[k]);
}

// the same per cloud of a forest, one block per cloud; cloud 0 also fills the
// tree summary's root box
__global__ void k_bbox_clouds(const double4* __restrict__ pm, CloudInfo* cl, TreeInfo* info) {
  __shared__ double s[6][BB_T];
  CloudInfo& C = cl[blockIdx.x];
  const int p0 = C.pstart, n = C.n;
  double mx[3] = {-BIG_NUMBER, -BIG_NUMBER, -BIG_NUMBER};
  double mn[3] = {BIG_NUMBER, BIG_NUMBER, BIG_NUMBER};
  for (int i = threadIdx.x; i < n; i += BB_T) {
    const double4 p = pm[p0 + i];
    mx[0] = fmax(mx[0], p.x); mx[1] = fmax(mx[1], p.y); mx[2] = fmax(mx[2], p.z);
    mn[0] = fmin(mn[0], p.x); mn[1] = fmin(mn[1], p.y); mn[2] = fmin(mn[2], p.z);
  }
  for (int k = 0; k < 3; ++k) { s[k][threadIdx.x] = mx[k]; s[3 + k][threadIdx.x] = mn[k]; }
  __syncthreads();
  for (int o = BB_T / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 3; ++k) {
        s[k][threadIdx.x] = fmax(s[k][threadIdx.x], s[k][threadIdx.x + o]);
        s[3 + k][threadIdx.x] = fmin(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + o]);
      }
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double rmax[3] = {s[0][0], s[1][0], s[2][0]};
  const double rmin[3] = {s[3][0], s[4][0], s[5][0]};
  const double ext = fmax(fmax(rmax[0] - rmin[0], rmax[1] - rmin[1]), rmax[2] - rmin[2]);
  C.rextent = ext;
  C.cellsize = 0.5 * ext;
  for (int k = 0; k < 3; ++k) C.root[k] = 0.5 * (rmin[k] + rmax[k]);
  C.delta = (float)(ldexp(1.0, -22) * (C.cellsize > 0.0 ? C.cellsize : 1.0));
  C.cell = blockIdx.x;
  if (blockIdx.x == 0) {
    info->rextent = C.rextent;
    info->cellsize = C.cellsize;
    for (int k = 0; k < 3; ++k) info->root[k] = C.root[k];
  }
}

// ---------------------------------------------------------------------------
// octant path keys: the comparisons and centre updates of BHgrav_build.F90:
// octant bits x=1, y=2, z=4 (:121-126), child centre rc -/+ cellsize (:212-229)
// with cellsize halved before each level (:95).
// In a forest (cl != NULL) each particle uses its own cloud's root box, and
// keep (when given) gets a copy of the keys in input order.
__global__ void k_keys(const double4* __restrict__ pm, int n, const TreeInfo* __restrict__ info,
                       const CloudInfo* __restrict__ cl, int ncl,
                       unsigned long long* __restrict__ keys,
                       unsigned long long* __restrict__ keep, int* __restrict__ idx) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = pm[i];
  double cx = info->root[0], cy = info->root[1], cz = info->root[2];
  double cs = info->cellsize;
  if (cl) {
    const CloudInfo& C = cl[cloud_of(cl, ncl, (int)i)];
    cx = C.root[0]; cy = C.root[1]; cz = C.root[2];
    cs = C.cellsize;
  }
  unsigned long long key = 0ull;
#pragma unroll 1
  for (int lev = 0; lev < KEY_LEVELS; ++lev) {
    const int d = (p.x > cx ? 1 : 0) | (p.y > cy ? 2 : 0) | (p.z > cz ? 4 : 0);
    key = (key << 3) | (unsigned long long)d;
    cs = 0.5 * cs;
    cx = (d & 1) ? __dadd_rn(cx, cs) : __dsub_rn(cx, cs);
    cy = (d & 2) ? __dadd_rn(cy, cs) : __dsub_rn(cy, cs);
    cz = (d & 4) ? __dadd_rn(cz, cs) : __dsub_rn(cz, cs);
  }
  keys[i] = key;
  if (keep) keep[i] = key;
  idx[i] = (int)i;
}

// 30-level keys of the same comparisons, for trees deeper than KEY_LEVELS:
// levels 1..21 in hi (as k_keys), levels 22..30 in lo (27 bits, level 22 in
// the most significant digit).  keys gets lo as the first sort key.
__global__ void k_keys_deep(const double4* __restrict__ pm, int n,
                            const TreeInfo* __restrict__ info, const CloudInfo* __restrict__ cl,
                            int ncl, unsigned long long* __restrict__ keys,
                            unsigned long long* __restrict__ hi, unsigned* __restrict__ lo,
                            int* __restrict__ idx) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = pm[i];
  double cx = info->root[0], cy = info->root[1], cz = info->root[2];
  double cs = info->cellsize;
  if (cl) {
    const CloudInfo& C = cl[cloud_of(cl, ncl, (int)i)];
    cx = C.root[0]; cy = C.root[1]; cz = C.root[2];
    cs = C.cellsize;
  }
  unsigned long long kh = 0ull;
  unsigned kl = 0u;
#pragma unroll 1
  for (int lev = 0; lev < DEEP_LEVELS; ++lev) {
    const int d = (p.x > cx ? 1 : 0) | (p.y > cy ? 2 : 0) | (p.z > cz ? 4 : 0);
    if (lev < KEY_LEVELS) kh = (kh << 3) | (unsigned long long)d;
    else kl = (kl << 3) | (unsigned)d;
    cs = 0.5 * cs;
    cx = (d & 1) ? __dadd_rn(cx, cs) : __dsub_rn(cx, cs);
    cy = (d & 2) ? __dadd_rn(cy, cs) : __dsub_rn(cy, cs);
    cz = (d & 4) ? __dadd_rn(cz, cs) : __dsub_rn(cz, cs);
  }
  keys[i] = (unsigned long long)kl;
  hi[i] = kh;
  lo[i] = kl;
  idx[i] = (int)i;
}

// the last sort key of a forest: the cloud of each particle, in the order so far
__global__ void k_cloud_keys(const int* __restrict__ idx, int n, const CloudInfo* __restrict__ cl,
                             int ncl, unsigned long long* __restrict__ keys) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = (unsigned long long)cloud_of(cl, ncl, idx[i]);
}

// after the stable sort on lo: the hi words in that order, the next sort key
__global__ void k_gather_hi(const unsigned long long* __restrict__ hi, const int* __restrict__ idx,
                            int n, unsigned long long* __restrict__ keys) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = hi[idx[i]];
}

// ---------------------------------------------------------------------------
// stable LSD radix sort of (64-bit key, int) pairs, 8-bit digits
constexpr int RS_T = 256;
constexpr int RS_W = RS_T / 32;
constexpr int RS_I = 16;                  // items per lane
constexpr int RS_TILE = RS_T * RS_I;      // 4096 items per block
constexpr int RS_CHUNK = 32 * RS_I;       // 512 contiguous items per warp

__global__ void k_rs_hist(const unsigned long long* __restrict__ keys, int n, int shift,
                          int* __restrict__ hist, int nblk) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const long base = (long)blockIdx.x * RS_TILE;
#pragma unroll 4
  for (int j = 0; j < RS_I; ++j) {
    const long i = base + (long)j * RS_T + threadIdx.x;
    if (i < n) atomicAdd(&cnt[(int)((keys[i] >> shift) & 255ull)], 1);
  }
  __syncthreads();
  hist[threadIdx.x * nblk + blockIdx.x] = cnt[threadIdx.x];
}

// The tile's items ranked by (digit, then the tile's order) and staged in that
// order in shared memory (the stable order of the pass), then written out:
// consecutive threads write consecutive slots of a digit's run, so the stores
// coalesce.  Shared memory: the tile's keys and values, the per-warp digit
// counts and the tile's digit starts.
constexpr size_t RS_SMEM = (size_t)RS_TILE * (sizeof(unsigned long long) + sizeof(int)) +
                           sizeof(int) * (RS_W * 256 + 256 + RS_W);
__global__ void __launch_bounds__(RS_T) k_rs_scatter(const unsigned long long* __restrict__ kin,
                                                     const int* __restrict__ vin,
                                                     unsigned long long* __restrict__ kout,
                                                     int* __restrict__ vout, int n, int shift,
                                                     const int* __restrict__ offs, int nblk) {
  extern __shared__ __align__(16) unsigned char rs_smem[];
  unsigned long long* sk = reinterpret_cast<unsigned long long*>(rs_smem);
  int* sv = reinterpret_cast<int*>(sk + RS_TILE);
  int (*wh)[256] = reinterpret_cast<int (*)[256]>(sv + RS_TILE);
  int* tstart = reinterpret_cast<int*>(wh + RS_W);
  int* wtot = tstart + 256;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int ww = 0; ww < RS_W; ++ww) wh[ww][threadIdx.x] = 0;
  __syncthreads();
  const long chunk = (long)blockIdx.x * RS_TILE + (long)w * RS_CHUNK;
  unsigned long long k[RS_I];
  int val[RS_I], rank[RS_I], dig[RS_I];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < RS_I; ++r) {
    const long i = chunk + (long)r * 32 + lane;
    const bool valid = i < n;
    k[r] = valid ? kin[i] : 0ull;
    val[r] = valid ? vin[i] : 0;
    const int d = valid ? (int)((k[r] >> shift) & 255ull) : 256;
    const unsigned peers = __match_any_sync(FULL, d);
    int before = 0;
    if (valid) before = wh[w][d];
    __syncwarp();
    const int leader = 31 - __clz(peers);
    if (valid && lane == leader) wh[w][d] = before + __popc(peers);
    __syncwarp();
    rank[r] = before + __popc(peers & lt);
    dig[r] = d;
  }
  __syncthreads();
  int run = 0;                       // this thread's digit: counts of the earlier warps
  for (int ww = 0; ww < RS_W; ++ww) {
    const int cnum = wh[ww][threadIdx.x];
    wh[ww][threadIdx.x] = run;
    run += cnum;
  }
  // the tile's digit starts: an exclusive scan of the digits' counts
  int inc = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) wtot[w] = inc;
  __syncthreads();
  int wbase = 0;
  for (int ww = 0; ww < w; ++ww) wbase += wtot[ww];
  tstart[threadIdx.x] = wbase + inc - run;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_I; ++r) {
    if (dig[r] < 256) {
      const int lp = tstart[dig[r]] + wh[w][dig[r]] + rank[r];
      sk[lp] = k[r];
      sv[lp] = val[r];
    }
  }
  __syncthreads();
  const long t0 = (long)blockIdx.x * RS_TILE;
  const int tcount = (int)min((long)RS_TILE, (long)n - t0);
  for (int t = threadIdx.x; t < tcount; t += RS_T) {
    const unsigned long long key = sk[t];
    const int d = (int)((key >> shift) & 255ull);
    const int pos = offs[d * nblk + blockIdx.x] + (t - tstart[d]);
    kout[pos] = key;
    vout[pos] = sv[t];
  }
}

// ---------------------------------------------------------------------------
// breadth-first cell emission
__global__ void k_root(int n, int cmax, int* leaf, int* nextcell, int* ifopen, int* pstart,
                       int* pcount, int* parent, int* level, int* branch, TreeInfo* info) {
  leaf[0] = 0;                 // the root is always split (BHgrav_build.F90:74)
  nextcell[0] = cmax + 1;      // :75
  ifopen[0] = -1;
  pstart[0] = 0;
  pcount[0] = n;
  parent[0] = -1;
  level[0] = 0;
  branch[0] = 0;
  info->nbranch = 1;
  info->ctot = 0;
  info->first_cell[0] = 0;
  info->last_cell[0] = 0;
}

// the roots of a forest: cell k is cloud k's root (always split, as the
// single root, BHgrav_build.F90:74-75), its particles the cloud's sorted range
__global__ void k_roots(int ncl, const CloudInfo* __restrict__ cl, int cmax, int* leaf,
                        int* nextcell, int* ifopen, int* pstart, int* pcount, int* parent,
                        int* level, int* branch, TreeInfo* info) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < ncl) {
    leaf[k] = 0;
    nextcell[k] = cmax + 1;
    ifopen[k] = -1;
    pstart[k] = cl[k].pstart;
    pcount[k] = cl[k].n;
    parent[k] = -1;
    level[k] = 0;
    branch[k] = k;
  }
  if (k == 0) {
    info->nbranch = ncl;
    info->ctot = ncl - 1;
    info->first_cell[0] = 0;
    info->last_cell[0] = ncl - 1;
  }
}

__device__ __forceinline__ int key_digit(unsigned long long key, int lev) {
  return (int)((key >> (3 * (KEY_LEVELS - 1 - lev))) & 7ull);
}

// the octant digit of level lev+1 of the particle at sorted position i: from
// the sorted 64-bit keys for the first KEY_LEVELS levels, from the input-order
// lo words (deep builds) below that
__device__ __forceinline__ int sorted_digit(const unsigned long long* __restrict__ keys,
                                            const unsigned* __restrict__ lo,
                                            const int* __restrict__ idx, int i, int lev) {
  if (lev < KEY_LEVELS) return key_digit(keys[i], lev);
  return (int)((lo[idx[i]] >> (3 * (DEEP_LEVELS - 1 - lev))) & 7u);
}

// children of every branch cell on level lev: boundaries of the octant digit
// runs inside the cell's (sorted) particle range
__global__ void k_split(const int* __restrict__ branch, const TreeInfo* __restrict__ info, int lev,
                        const int* __restrict__ pstart, const int* __restrict__ pcount,
                        const unsigned long long* __restrict__ keys,
                        const unsigned* __restrict__ lo_words, const int* __restrict__ idx,
                        int* __restrict__ nchild, int* __restrict__ cstart) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= info->nbranch) return;
  const int b = branch[j];
  const int s = pstart[b], e = s + pcount[b];
  int st[9];
  st[0] = s;
  st[8] = e;
  for (int d = 1; d < 8; ++d) {
    int lo = st[d - 1], hi = e;
    while (lo < hi) {
      const int mid = lo + ((hi - lo) >> 1);
      if (sorted_digit(keys, lo_words, idx, mid, lev) < d) lo = mid + 1;
      else hi = mid;
    }
    st[d] = lo;
  }
  int cnt = 0;
  for (int d = 0; d < 8; ++d) {
    cstart[j * 9 + d] = st[d];
    cnt += (st[d + 1] > st[d]) ? 1 : 0;
  }
  cstart[j * 9 + 8] = e;
  nchild[j] = cnt;
}

// number the children serially in (branch order, octant) order, as
// BHgrav_build.F90:149-157 does, and link them (:239-253)
__global__ void k_emit(const int* __restrict__ branch, const TreeInfo* __restrict__ info, int lev,
                       const int* __restrict__ choff, const int* __restrict__ cstart,
                       int level_first, int* leaf, int* nextcell, int* ifopen, int* pstart,
                       int* pcount, int* parent, int* level, int* nkids,
                       int* __restrict__ bflag) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= info->nbranch) return;
  const int b = branch[j];
  const int first = level_first + choff[j];
  int k = 0, prev = -1;
  for (int d = 0; d < 8; ++d) {
    const int s = cstart[j * 9 + d], e = cstart[j * 9 + d + 1];
    if (e == s) continue;
    const int c = first + k;
    ++k;
    const int cnt = e - s;
    const int lf = cnt <= LEAFMAX ? cnt : 0;
    leaf[c] = lf;
    ifopen[c] = -1;
    pstart[c] = s;
    pcount[c] = cnt;
    parent[c] = b;
    level[c] = lev + 1;
    nkids[c] = 0;
    bflag[c - level_first] = lf == 0 ? 1 : 0;
    if (prev >= 0) nextcell[prev] = c;
    prev = c;
  }
  nextcell[prev] = nextcell[b];
  ifopen[b] = first;
  nkids[b] = k;
}

__global__ void k_next_branch(const int* __restrict__ bflag, const int* __restrict__ bscan, int nnew,
                              int level_first, int* __restrict__ branch_next) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnew) return;
  if (bflag[i]) branch_next[bscan[i]] = level_first + i;
}

__global__ void k_level_done(TreeInfo* info, int lev, int level_first, int nnew,
                             const int* __restrict__ nb_next) {
  info->ctot = level_first + nnew - 1;
  info->first_cell[lev + 1] = level_first;
  info->last_cell[lev + 1] = level_first + nnew - 1;
  info->ltot = lev + 1;
  info->nbranch = *nb_next;
  info->nchild = nnew;
}

// leaf particles back to input-index order (the linked lists of the
// reference keep the order particles had in the parent cell, and the root
// list is 1..ptot), then the permutation new -> old
__global__ void k_leaf_order(const int* __restrict__ leaf, const int* __restrict__ pstart, int ctot,
                             int* __restrict__ idx) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ctot) return;
  const int n = leaf[c];
  if (n <= 1) return;
  const int s = pstart[c];
  int v[LEAFMAX];
  for (int i = 0; i < n; ++i) v[i] = idx[s + i];
  for (int i = 1; i < n; ++i) {
    const int x = v[i];
    int j = i - 1;
    while (j >= 0 && v[j] > x) { v[j + 1] = v[j]; --j; }
    v[j + 1] = x;
  }
  for (int i = 0; i < n; ++i) idx[s + i] = v[i];
}

__global__ void k_reorder(const int* __restrict__ perm, int n, const double4* __restrict__ pm,
                          const double2* __restrict__ hz, const double4* __restrict__ vel,
                          const double* __restrict__ csq, const int* __restrict__ orig,
                          double4* __restrict__ pm2, double2* __restrict__ hz2,
                          double4* __restrict__ vel2, double* __restrict__ csq2,
                          int* __restrict__ orig2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  pm2[i] = pm[p];
  hz2[i] = hz[p];
  vel2[i] = vel[p];
  csq2[i] = csq[p];
  orig2[i] = orig[p];
}

// the reorder without v and c_s^2 (still being copied in: finish_reorder)
__global__ void k_reorder_pos(const int* __restrict__ perm, int n, const double4* __restrict__ pm,
                              const double2* __restrict__ hz, const int* __restrict__ orig,
                              double4* __restrict__ pm2, double2* __restrict__ hz2,
                              int* __restrict__ orig2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  pm2[i] = pm[p];
  hz2[i] = hz[p];
  orig2[i] = orig[p];
}

__global__ void k_reorder_vc(const int* __restrict__ perm, int n, const double4* __restrict__ vel,
                             const double* __restrict__ csq, double4* __restrict__ vel2,
                             double* __restrict__ csq2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  vel2[i] = vel[p];
  csq2[i] = csq[p];
}

__global__ void k_reorder_sph(const int* __restrict__ perm, int n, const double* __restrict__ a,
                              const double* __restrict__ b, const double* __restrict__ c,
                              const double* __restrict__ d, double* __restrict__ a2,
                              double* __restrict__ b2, double* __restrict__ c2,
                              double* __restrict__ d2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  a2[i] = a[p];
  b2[i] = b[p];
  c2[i] = c[p];
  d2[i] = d[p];
}

__global__ void k_reorder_rk(const int* __restrict__ perm, int n, const double4* __restrict__ a,
                             const double4* __restrict__ b, const double4* __restrict__ c,
                             double4* __restrict__ a2, double4* __restrict__ b2,
                             double4* __restrict__ c2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm[i];
  a2[i] = a[p];
  b2[i] = b[p];
  c2[i] = c[p];
}

__global__ void k_pack_link(int ctot, const int* __restrict__ leaf, const int* __restrict__ nextcell,
                            const int* __restrict__ ifopen, const int* __restrict__ pstart,
                            int4* __restrict__ link) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ctot) return;
  link[c] = make_int4(leaf[c], nextcell[c], leaf[c] > 0 ? -1 : ifopen[c], pstart[c]);
}

__global__ void k_unpack_parray(const double* __restrict__ st, int n, double4* __restrict__ pm,
                                double2* __restrict__ hz, DevError* err) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* r = st + i * 6;
  const double x = r[0], y = r[1], z = r[2], m = r[3], h = r[4], zt = r[5];
  if (!(isfinite(x) && isfinite(y) && isfinite(z) && isfinite(m) && isfinite(h) && isfinite(zt)))
    set_error(err, SEREN_GPU_ERR_NONFINITE, KID_REORDER, (int)i, 0);
  pm[i] = make_double4(x, y, z, m);
  hz[i] = make_double2(h, zt);
}

__global__ void k_pack_parray(double* __restrict__ st, int n, const double4* __restrict__ pm,
                              const double2* __restrict__ hz) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = pm[i];
  const double2 h = hz[i];
  double* r = st + i * 6;
  r[0] = p.x; r[1] = p.y; r[2] = p.z; r[3] = p.w; r[4] = h.x; r[5] = h.y;
}

// ---------------------------------------------------------------------------
// BHgrav_stock.F90:11-358 (QUADRUPOLE, GEOMETRIC_MAC) and BHhydro_stock.F90,
// one level at a time from the deepest up; a leaf's particles are the
// contiguous range [pstart, pstart+leaf) in tree order.
// It also writes the FP32 walk copy of each cell: COM relative to the root
// centre and a bracket [lo, hi] around dminsqd wide enough to hold every FP32
// rounding of the walk's prefilter test (coordinates rounded to within delta,
// the difference, the squares and the sum); tests inside the bracket are
// redone in FP64 by the walk.
__global__ void k_stock_level(int cfirst, int clast, const int4* __restrict__ link,
                              const double4* __restrict__ pm, const double2* __restrict__ hz,
                              double thetamaxsqd, double daux, double4* __restrict__ gA,
                              double4* __restrict__ gB, double2* __restrict__ gC,
                              double4* __restrict__ hA, double* __restrict__ hmaxa,
                              double4* __restrict__ bbmina, double4* __restrict__ bbmaxa,
                              double rootx, double rooty, double rootz, double delta,
                              const int* __restrict__ nkids, float4* __restrict__ wA,
                              float4* __restrict__ hA32, float4* __restrict__ hN,
                              const CloudInfo* __restrict__ cl, int ncl) {
  const int c = cfirst + blockIdx.x * blockDim.x + threadIdx.x;
  if (c > clast) return;
  const int4 lk = link[c];
  if (cl) {                                  // a forest: the cell's own cloud's root box
    const CloudInfo& C = cl[cloud_of(cl, ncl, lk.w)];
    rootx = C.root[0]; rooty = C.root[1]; rootz = C.root[2];
    delta = ldexp(1.0, -22) * (C.cellsize > 0.0 ? C.cellsize : 1.0);
  }
  double mc = 0.0;
  double rc[3] = {0.0, 0.0, 0.0};
  double qc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  double hmax = 0.0;
  double bbmin[3] = {BIG_NUMBER, BIG_NUMBER, BIG_NUMBER};
  double bbmax[3] = {-BIG_NUMBER, -BIG_NUMBER, -BIG_NUMBER};
  double dr[3];
  if (lk.x == 1) {                                                   // :100-113
    const double4 p = pm[lk.w];
    rc[0] = p.x; rc[1] = p.y; rc[2] = p.z;
    mc = p.w;
    hmax = hz[lk.w].x;
    for (int k = 0; k < 3; ++k) { bbmin[k] = rc[k]; bbmax[k] = rc[k]; }
  } else if (lk.x > 0) {                                             // :118-183
    const int s = lk.w, npart = lk.x;
    for (int i = 0; i < npart; ++i) {
      const double4 p = pm[s + i];
      const double mp = p.w;
      mc = mc + mp;
      hmax = fmax(hmax, hz[s + i].x);
      rc[0] = rc[0] + mp * p.x;
      rc[1] = rc[1] + mp * p.y;
      rc[2] = rc[2] + mp * p.z;
      bbmax[0] = fmax(bbmax[0], p.x); bbmin[0] = fmin(bbmin[0], p.x);
      bbmax[1] = fmax(bbmax[1], p.y); bbmin[1] = fmin(bbmin[1], p.y);
      bbmax[2] = fmax(bbmax[2], p.z); bbmin[2] = fmin(bbmin[2], p.z);
    }
    for (int k = 0; k < 3; ++k) rc[k] = rc[k] / mc;
    for (int i = 0; i < npart; ++i) {
      const double4 p = pm[s + i];
      dr[0] = p.x - rc[0]; dr[1] = p.y - rc[1]; dr[2] = p.z - rc[2];
      const double mp = p.w;
      const double drsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
      qc[0] = qc[0] + mp * ((3.0 * dr[0]) * dr[0] - drsqd);
      qc[1] = qc[1] + mp * ((3.0 * dr[0]) * dr[1]);
      qc[2] = qc[2] + mp * ((3.0 * dr[1]) * dr[1] - drsqd);
      qc[3] = qc[3] + mp * ((3.0 * dr[2]) * dr[0]);
      qc[4] = qc[4] + mp * ((3.0 * dr[2]) * dr[1]);
    }
  } else {                                                           // :188-312
    const int cend = lk.y;
    int cc = lk.z;
    while (true) {
      const double4 a = gA[cc];
      mc = mc + a.w;
      rc[0] = rc[0] + a.w * a.x;
      rc[1] = rc[1] + a.w * a.y;
      rc[2] = rc[2] + a.w * a.z;
      hmax = fmax(hmaxa[cc], hmax);
      const double4 b0 = bbmina[cc], b1 = bbmaxa[cc];
      bbmax[0] = fmax(b1.x, bbmax[0]); bbmin[0] = fmin(b0.x, bbmin[0]);
      bbmax[1] = fmax(b1.y, bbmax[1]); bbmin[1] = fmin(b0.y, bbmin[1]);
      bbmax[2] = fmax(b1.z, bbmax[2]); bbmin[2] = fmin(b0.z, bbmin[2]);
      cc = link[cc].y;
      if (cc == cend) break;
    }
    if (mc > 0.0) for (int k = 0; k < 3; ++k) rc[k] = rc[k] / mc;
    cc = lk.z;
    while (true) {
      const double4 a = gA[cc];
      const double4 q = gB[cc];
      const double2 q5 = gC[cc];
      const double mcc = a.w;
      qc[0] = qc[0] + q.x; qc[1] = qc[1] + q.y; qc[2] = qc[2] + q.z; qc[3] = qc[3] + q.w;
      qc[4] = qc[4] + q5.x;
      dr[0] = a.x - rc[0]; dr[1] = a.y - rc[1]; dr[2] = a.z - rc[2];
      const double drsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
      qc[0] = qc[0] + mcc * ((3.0 * dr[0]) * dr[0] - drsqd);
      qc[1] = qc[1] + mcc * ((3.0 * dr[0]) * dr[1]);
      qc[2] = qc[2] + mcc * ((3.0 * dr[1]) * dr[1] - drsqd);
      qc[3] = qc[3] + mcc * ((3.0 * dr[2]) * dr[0]);
      qc[4] = qc[4] + mcc * ((3.0 * dr[2]) * dr[1]);
      cc = link[cc].y;
      if (cc == cend) break;
    }
  }
  // MAC quantities, :317-348
  for (int k = 0; k < 3; ++k) dr[k] = fmax(bbmax[k] - rc[k], rc[k] - bbmin[k]);
  const double diagonalsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
  const double rsize = sqrt(diagonalsqd) + KERNRANGE * hmax;
  double dminsqd = thetamaxsqd > 0.0 ? diagonalsqd / thetamaxsqd : BIG_NUMBER;
  dminsqd = fmax(dminsqd, rsize * rsize);
  if (dminsqd < daux) dminsqd = daux;
  gA[c] = make_double4(rc[0], rc[1], rc[2], mc);
  gB[c] = make_double4(qc[0], qc[1], qc[2], qc[3]);
  gC[c] = make_double2(qc[4], dminsqd);
  {
    const double marg = 2.0 * (8.0 * sqrt(dminsqd) * delta + 1.0e-6 * dminsqd + 16.0 * delta * delta);
    wA[2 * c] = make_float4((float)(rc[0] - rootx), (float)(rc[1] - rooty),
                            (float)(rc[2] - rootz), __double2float_ru(dminsqd + marg));
    wA[2 * c + 1] = make_float4(__double2float_rd(dminsqd - marg),
                                __int_as_float(lk.x > 0 ? lk.w : lk.z),
                                __int_as_float(lk.x > 0 ? lk.x : -nkids[c]), 0.0f);
  }
  hmaxa[c] = hmax;
  bbmina[c] = make_double4(bbmin[0], bbmin[1], bbmin[2], 0.0);
  bbmaxa[c] = make_double4(bbmax[0], bbmax[1], bbmax[2], 0.0);
  // BHhydro_stock.F90:69-150: bounding-box centre and half diagonal
  double4 hn;
  if (lk.x == 1) {
    hn = make_double4(rc[0], rc[1], rc[2], 0.0);
  } else {
    double hc[3], diag = 0.0;
    for (int k = 0; k < 3; ++k) {
      hc[k] = 0.5 * (bbmax[k] + bbmin[k]);
      const double hb = bbmax[k] - hc[k];
      diag = diag + hb * hb;
    }
    hn = make_double4(hc[0], hc[1], hc[2], sqrt(diag));
  }
  hA[c] = hn;
  const float4 h32 = make_float4((float)(hn.x - rootx), (float)(hn.y - rooty),
                                 (float)(hn.z - rootz), __double2float_ru(hn.w));
  hA32[c] = h32;
  hN[2 * c] = h32;
  hN[2 * c + 1] = make_float4(0.0f, __int_as_float(lk.x > 0 ? lk.w : lk.z),
                              __int_as_float(lk.x > 0 ? lk.x : -nkids[c]), 0.0f);
}

// BHhydro_update_hmax.F90:29-88
__global__ void k_hmax_level(int cfirst, int clast, const int4* __restrict__ link,
                             const double2* __restrict__ hz, double* __restrict__ hrm,
                             float* __restrict__ hrm32, float4* __restrict__ hN) {
  const int c = cfirst + blockIdx.x * blockDim.x + threadIdx.x;
  if (c > clast) return;
  const int4 lk = link[c];
  double hr = 0.0;
  if (lk.x == 1) {
    hr = KERNRANGE * hz[lk.w].x;
  } else if (lk.x > 0) {
    for (int i = 0; i < lk.x; ++i) hr = fmax(hr, KERNRANGE * hz[lk.w + i].x);
  } else {
    int cc = lk.z;
    const int cend = lk.y;
    while (true) {
      hr = fmax(hr, hrm[cc]);
      cc = link[cc].y;
      if (cc == cend) break;
    }
  }
  hrm[c] = hr;
  hrm32[c] = __double2float_ru(hr);
  reinterpret_cast<float*>(hN)[8 * (size_t)c + 4] = hrm32[c];
}

// BHhydro_hguess.F90:106-155 (GRAD_H_SPH number criterion): the h of a
// leaf's particles is half the rmax of its deepest ancestor-or-self holding
// more than int(pp_gather/2) particles, or of the root.
__global__ void k_hguess(int ctot, const int4* __restrict__ link, const int* __restrict__ pcount,
                         const int* __restrict__ parent, const int* __restrict__ level,
                         const double4* __restrict__ hA, int thresh, double2* __restrict__ hz) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > ctot) return;
  const int4 lk = link[c];
  if (lk.x <= 0) return;
  int a = c;
  while (pcount[a] <= thresh && level[a] > 0) a = parent[a];
  const double hg = INVKERNRANGE * hA[a].w;
  for (int i = 0; i < lk.x; ++i) hz[lk.w + i].x = hg;
}

inline int nb(long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------------------
int scan_scratch_alloc(ScanScratch& s, int nmax) {
  long n = nmax;
  for (int lv = 0; lv < 4; ++lv) {
    const long nblk = (n + SCAN_TILE - 1) / SCAN_TILE;
    s.level_cap[lv] = (int)nblk + 1;
    if (cudaMalloc(&s.level_buf[lv], sizeof(int) * (nblk + 1)) != cudaSuccess) return -1;
    n = nblk;
    if (nblk <= 1) break;
  }
  if (cudaMalloc(&s.total, sizeof(int)) != cudaSuccess) return -1;
  return 0;
}

static void scan_rec(Ctx& c, const int* in, int* out, int n, int lv) {
  const int nblk = nb(n, SCAN_TILE);
  int* sums = c.scan.level_buf[lv];
  k_scan_tile<<<nblk, SCAN_T, 0, c.st>>>(in, out, n, sums); ++c.nlaunch;
  if (nblk == 1) {
    k_copy_int<<<1, 1, 0, c.st>>>(sums, c.scan.total); ++c.nlaunch;
    return;
  }
  scan_rec(c, sums, sums, nblk, lv + 1);
  k_scan_add<<<nblk, SCAN_T, 0, c.st>>>(out, n, sums); ++c.nlaunch;
}

void scan_exclusive(Ctx& c, const int* in, int* out, int n) {
  if (n <= 0) {
    cudaMemsetAsync(c.scan.total, 0, sizeof(int), c.st);
    return;
  }
  scan_rec(c, in, out, n, 0);
}

__global__ void k_publish(const int* __restrict__ src, int n, volatile int* dst) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

int read_dev(Ctx& c, const void* dsrc, void* hdst, size_t bytes) {
  if (bytes % 4 != 0 || bytes > 1024) return SEREN_GPU_ERR_ARG;
  if (c.h_map == nullptr) {
    void* h = nullptr;
    void* d = nullptr;
    if (cudaHostAlloc(&h, 1024, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
      if (h) cudaFreeHost(h);
      cudaGetLastError();
      // no mapped memory: an ordinary copy
      cudaMemcpyAsync(hdst, dsrc, bytes, cudaMemcpyDeviceToHost, c.st);
      return cudaStreamSynchronize(c.st) == cudaSuccess ? SEREN_GPU_OK : SEREN_GPU_ERR_CUDA;
    }
    c.h_map = static_cast<int*>(h);
    c.d_map = static_cast<int*>(d);
  }
  k_publish<<<1, 128, 0, c.st>>>(static_cast<const int*>(dsrc), (int)(bytes / 4), c.d_map);
  ++c.nlaunch;
  if (cudaStreamSynchronize(c.st) != cudaSuccess) return SEREN_GPU_ERR_CUDA;
  std::memcpy(hdst, const_cast<const int*>(c.h_map), bytes);
  return SEREN_GPU_OK;
}

void finish_reorder(Ctx& c) {
  if (c.vel_wait) {
    cudaStreamWaitEvent(c.st, c.vel_wait, 0);
    c.vel_wait = nullptr;
  }
  if (!c.reorder_late) return;
  cudaStreamWaitEvent(c.st, c.reorder_wait, 0);
  k_reorder_vc<<<nb(c.ptot, 256), 256, 0, c.st>>>(c.idx, c.ptot, c.vel, c.csq, c.vel_alt,
                                                   c.csq_alt); ++c.nlaunch;
  std::swap(c.vel, c.vel_alt);
  std::swap(c.csq, c.csq_alt);
  c.reorder_late = false;
  c.reorder_wait = nullptr;
}

void launch_unpack_parray(Ctx& c, const double* stage, int n) {
  k_unpack_parray<<<nb(n, 256), 256, 0, c.st>>>(stage, n, c.pm, c.hz, c.d_err); ++c.nlaunch;
}

void launch_pack_parray(Ctx& c, double* stage, int n, cudaStream_t s) {
  k_pack_parray<<<nb(n, 256), 256, 0, s ? s : c.st>>>(stage, n, c.pm, c.hz); ++c.nlaunch;
}

// stable LSD sort of (keys, idx) on the key bits [0, bits), 8 at a time; an
// even number of passes leaves the sorted data in keys/idx
static void radix_sort(Ctx& c, int n, int bits) {
  static bool smem_set[16] = {};   // the scatter's shared memory is above the 48 KB default
  bool& ss = smem_set[c.dev >= 0 && c.dev < 16 ? c.dev : 0];
  if (!ss) {
    cudaFuncSetAttribute(k_rs_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS_SMEM);
    ss = true;
  }
  const int nblk = nb(n, RS_TILE);
  unsigned long long* ka = c.keys;
  unsigned long long* kb = c.keys_alt;
  int* va = c.idx;
  int* vb = c.idx_alt;
  for (int shift = 0; shift < bits; shift += 8) {
    k_rs_hist<<<nblk, RS_T, 0, c.st>>>(ka, n, shift, c.rs_hist, nblk); ++c.nlaunch;
    scan_exclusive(c, c.rs_hist, c.rs_hist, 256 * nblk);
    k_rs_scatter<<<nblk, RS_T, RS_SMEM, c.st>>>(ka, va, kb, vb, n, shift, c.rs_hist, nblk);
    ++c.nlaunch;
    std::swap(ka, kb);
    std::swap(va, vb);
  }
}

constexpr int NEED_DEEP_KEYS = -1;

// cells level by level from the sorted keys; with 21-level keys, a tree that
// needs level 22 returns NEED_DEEP_KEYS
static int build_cells(Ctx& c, bool deep, int& ctot_out) {
  const int n = c.ptot;
  const int ncl = c.ncloud;
  if (ncl > 1)
    k_roots<<<nb(ncl, 128), 128, 0, c.st>>>(ncl, c.d_clouds, c.cmax, c.leaf, c.nextcell, c.ifopen,
                                            c.pstart, c.pcount, c.parent, c.level, c.branch,
                                            c.d_info);
  else
    k_root<<<1, 1, 0, c.st>>>(n, c.cmax, c.leaf, c.nextcell, c.ifopen, c.pstart, c.pcount,
                              c.parent, c.level, c.branch, c.d_info);
  ++c.nlaunch;
  int nbranch = ncl, ctot = ncl - 1, lev = 0;
  int* br = c.branch;
  int* br_next = c.branch_next;
  while (true) {
    if (lev >= c.prm.lmax) {                // BHgrav_build.F90:289
      c.err = "Reached maximum level (tree deeper than lmax)";
      return SEREN_GPU_ERR_LMAX;
    }
    if (!deep && lev >= KEY_LEVELS) return NEED_DEEP_KEYS;
    k_split<<<nb(nbranch, 128), 128, 0, c.st>>>(br, c.d_info, lev, c.pstart, c.pcount, c.keys,
                                                c.keys_lo, c.idx, c.nchild, c.cstart); ++c.nlaunch;
    scan_exclusive(c, c.nchild, c.choff, nbranch);
    int nnew = 0;
    if (read_dev(c, c.scan.total, &nnew, sizeof(int))) return SEREN_GPU_ERR_CUDA;
    const int level_first = ctot + 1;
    if ((long)ctot + nnew > (long)c.cmax) {
      c.err = "cell count exceeds cmax = 2*pmax";
      return SEREN_GPU_ERR_CAPACITY;
    }
    k_emit<<<nb(nbranch, 128), 128, 0, c.st>>>(br, c.d_info, lev, c.choff, c.cstart, level_first,
                                               c.leaf, c.nextcell, c.ifopen, c.pstart, c.pcount,
                                               c.parent, c.level, c.nkids, c.bflag); ++c.nlaunch;
    scan_exclusive(c, c.bflag, c.bscan, nnew);
    k_next_branch<<<nb(nnew, 256), 256, 0, c.st>>>(c.bflag, c.bscan, nnew, level_first, br_next); ++c.nlaunch;
    k_level_done<<<1, 1, 0, c.st>>>(c.d_info, lev, level_first, nnew, c.scan.total); ++c.nlaunch;
    int nbn = 0;
    if (read_dev(c, c.scan.total, &nbn, sizeof(int))) return SEREN_GPU_ERR_CUDA;
    ctot += nnew;
    ++lev;
    std::swap(br, br_next);
    nbranch = nbn;
    if (nbranch == 0) break;
  }
  ctot_out = ctot;
  return SEREN_GPU_OK;
}

// a forest: a last stable pass on the cloud of each particle makes the order
// cloud-major again, then the octant words (kept in input order in keys_hi)
// are gathered into that order for the cell split
static void sort_by_cloud(Ctx& c, int n) {
  k_cloud_keys<<<nb(n, 256), 256, 0, c.st>>>(c.idx, n, c.d_clouds, c.ncloud, c.keys); ++c.nlaunch;
  radix_sort(c, n, c.ncloud <= 65536 ? 16 : 32);      // an even number of passes
  k_gather_hi<<<nb(n, 256), 256, 0, c.st>>>(c.keys_hi, c.idx, n, c.keys); ++c.nlaunch;
}

int build_tree(Ctx& c) {
  const int n = c.ptot;
  const bool forest = c.ncloud > 1;
  const CloudInfo* cl = forest ? c.d_clouds : nullptr;
  if (forest) {
    k_bbox_clouds<<<c.ncloud, BB_T, 0, c.st>>>(c.pm, c.d_clouds, c.d_info); ++c.nlaunch;
  } else {
    const int bblk = std::min(nb(n, BB_T), 1184);
    k_bbox_partial<<<bblk, BB_T, 0, c.st>>>(c.pm, n, c.bbox_part); ++c.nlaunch;
    k_bbox_final<<<1, BB_T, 0, c.st>>>(c.bbox_part, bblk, c.d_info); ++c.nlaunch;
  }
  k_keys<<<nb(n, 256), 256, 0, c.st>>>(c.pm, n, c.d_info, cl, c.ncloud, c.keys,
                                        forest ? c.keys_hi : nullptr, c.idx); ++c.nlaunch;
  radix_sort(c, n, 64);
  if (forest) sort_by_cloud(c, n);
  int ctot = 0;
  int rc = build_cells(c, false, ctot);
  if (rc == NEED_DEEP_KEYS) {
    // sort on (levels 1..21, levels 22..30): stable passes on the low word,
    // then on the high word in that order
    k_keys_deep<<<nb(n, 256), 256, 0, c.st>>>(c.pm, n, c.d_info, cl, c.ncloud, c.keys, c.keys_hi,
                                               c.keys_lo, c.idx); ++c.nlaunch;
    radix_sort(c, n, 32);
    k_gather_hi<<<nb(n, 256), 256, 0, c.st>>>(c.keys_hi, c.idx, n, c.keys); ++c.nlaunch;
    radix_sort(c, n, 64);
    if (forest) sort_by_cloud(c, n);
    rc = build_cells(c, true, ctot);
  }
  if (rc) return rc;
  k_leaf_order<<<nb(ctot + 1, 256), 256, 0, c.st>>>(c.leaf, c.pstart, ctot, c.idx); ++c.nlaunch;
  if (c.reorder_wait) {                     // velocities and c_s^2 still being copied in
    k_reorder_pos<<<nb(n, 256), 256, 0, c.st>>>(c.idx, n, c.pm, c.hz, c.orig, c.pm_alt, c.hz_alt,
                                                 c.orig_alt); ++c.nlaunch;
    c.reorder_late = true;
  } else {
    k_reorder<<<nb(n, 256), 256, 0, c.st>>>(c.idx, n, c.pm, c.hz, c.vel, c.csq, c.orig, c.pm_alt,
                                             c.hz_alt, c.vel_alt, c.csq_alt, c.orig_alt); ++c.nlaunch;
    std::swap(c.vel, c.vel_alt);
    std::swap(c.csq, c.csq_alt);
  }
  std::swap(c.pm, c.pm_alt);
  std::swap(c.hz, c.hz_alt);
  std::swap(c.orig, c.orig_alt);
  // rho, omega, div v, drho/dt of the last evaluation follow the particles
  // (main/reorder_array.F90): particles left out of an active subset keep theirs
  k_reorder_sph<<<nb(n, 256), 256, 0, c.st>>>(c.idx, n, c.rho, c.omega, c.div_v, c.drhodt,
                                               c.rho_alt, c.omega_alt, c.div_v_alt,
                                               c.drhodt_alt); ++c.nlaunch;
  std::swap(c.rho, c.rho_alt);
  std::swap(c.omega, c.omega_alt);
  std::swap(c.div_v, c.div_v_alt);
  std::swap(c.drhodt, c.drhodt_alt);
  if (c.r_old) {                            // Runge-Kutta state follows the particles
    k_reorder_rk<<<nb(n, 256), 256, 0, c.st>>>(c.idx, n, c.r_old, c.v_old, c.v_half, c.r_old_alt,
                                                c.v_old_alt, c.v_half_alt); ++c.nlaunch;
    std::swap(c.r_old, c.r_old_alt);
    std::swap(c.v_old, c.v_old_alt);
    std::swap(c.v_half, c.v_half_alt);
  }
  if (c.blk.on) reorder_block(c);           // block-timestep state, a and gpot too
  k_pack_link<<<nb(ctot + 1, 256), 256, 0, c.st>>>(ctot, c.leaf, c.nextcell, c.ifopen, c.pstart,
                                                   c.link); ++c.nlaunch;
  static_assert(sizeof(TreeInfo) % 4 == 0 && sizeof(TreeInfo) <= 1024, "TreeInfo through read_dev");
  if (read_dev(c, c.d_info, &c.info, sizeof(TreeInfo))) return SEREN_GPU_ERR_CUDA;
  c.have_tree = true;
  return SEREN_GPU_OK;
}

// the largest per-axis distance of a particle from the root cell centre, as
// the bit pattern of a non-negative double (ordered as an integer)
__global__ void k_max_offset(const double4* __restrict__ pm, int n, double rx, double ry,
                             double rz, unsigned long long* out) {
  double m = 0.0;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double4 p = pm[i];
    m = fmax(m, fmax(fabs(p.x - rx), fmax(fabs(p.y - ry), fabs(p.z - rz))));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

int restock(Ctx& c, bool& rebuilt) {
  rebuilt = false;
  if (c.ncloud > 1) {                      // a forest is built at every evaluation
    rebuilt = true;
    const int rc = build_tree(c);
    if (rc) return rc;
    launch_stock(c);
    return SEREN_GPU_OK;
  }
  // the FP32 node records bound the rounding of a coordinate relative to the
  // root centre by 2^-22 cellsize, which holds while every particle is within
  // two root half widths of the centre; past that (or on non-finite
  // positions) the tree is built again instead
  unsigned long long* out = reinterpret_cast<unsigned long long*>(c.bbox_part);
  cudaMemsetAsync(out, 0, sizeof(unsigned long long), c.st);
  k_max_offset<<<std::min(nb(c.ptot, 256), 1184), 256, 0, c.st>>>(
      c.pm, c.ptot, c.info.root[0], c.info.root[1], c.info.root[2], out); ++c.nlaunch;
  unsigned long long bits = 0;
  if (read_dev(c, out, &bits, sizeof(bits))) return SEREN_GPU_ERR_CUDA;
  double maxoff = 0.0;
  std::memcpy(&maxoff, &bits, sizeof(double));
  if (!(maxoff <= 2.0 * c.info.cellsize)) {
    rebuilt = true;
    const int rc = build_tree(c);
    if (rc) return rc;
  }
  launch_stock(c);
  return SEREN_GPU_OK;
}

void launch_stock(Ctx& c) {
  const double daux = 10.0 * pow(1.7976931348623157e308, -0.2);
  // bound on the rounding of a coordinate relative to the root centre when
  // cast to FP32: every position lies within cellsize (the root half width)
  // of the centre on each axis, so half an ulp is below 2^-23 * cellsize
  const double delta = ldexp(1.0, -22) * (c.info.cellsize > 0.0 ? c.info.cellsize : 1.0);
  for (int l = c.info.ltot; l >= 0; --l) {
    const int f = c.info.first_cell[l], la = c.info.last_cell[l];
    const int cnt = la - f + 1;
    if (cnt <= 0) continue;
    k_stock_level<<<nb(cnt, 128), 128, 0, c.st>>>(f, la, c.link, c.pm, c.hz, c.prm.thetamaxsqd, daux,
                                                 c.gA, c.gB, c.gC, c.hA, c.hmax, c.bbmin, c.bbmax,
                                                 c.info.root[0], c.info.root[1], c.info.root[2],
                                                 delta, c.nkids, c.wA, c.hA32, c.hN,
                                                 c.ncloud > 1 ? c.d_clouds : nullptr, c.ncloud);
    ++c.nlaunch;
  }
}

void launch_update_hmax(Ctx& c) {
  for (int l = c.info.ltot; l >= 0; --l) {
    const int f = c.info.first_cell[l], la = c.info.last_cell[l];
    const int cnt = la - f + 1;
    if (cnt <= 0) continue;
    k_hmax_level<<<nb(cnt, 128), 128, 0, c.st>>>(f, la, c.link, c.hz, c.hrm, c.hrm32, c.hN); ++c.nlaunch;
  }
}

void launch_hguess(Ctx& c) {
  const int thresh = (int)(0.5 * (double)c.prm.pp_gather);
  k_hguess<<<nb(c.info.ctot + 1, 256), 256, 0, c.st>>>(c.info.ctot, c.link, c.pcount, c.parent,
                                                       c.level, c.hA, thresh, c.hz); ++c.nlaunch;
}

}  // namespace seren
