// common.cuh - constants, device layouts and helpers of the force path.
//
// Device data are structure-of-arrays in tree order (particles renumbered by
// the depth-first leaf order of the octree, as BH_reorder_particles does), so
// the particles of a leaf are the contiguous range [pstart, pstart+leaf).
// Cells use the reference's breadth-first numbering (BHgrav_build.F90:149-157).
//
// This translation unit family is compiled with -fmad=false: every FP64
// expression that mirrors a Fortran statement is evaluated with the same
// association and no contraction, so integer decisions taken from floats
// (octants, MAC tests, kernel bins, neighbour tests) agree with the FP64
// reference arithmetic.  Kernels that want FMA (the mixed-precision pair
// arithmetic) call fmaf()/fma() explicitly.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace seren {

// headers/macros.h (NDIM = 3, M4 kernel, PR = DP)
constexpr int KERNTOT = 10000;
constexpr double HALFKERNTOT = 5000.0;
constexpr double KERNRANGE = 2.0;
constexpr double KERNRANGESQD = 4.0;
constexpr double INVKERNRANGE = 0.5;
constexpr double INVPI = 0.318309886;
constexpr double ONETHIRD = 0.333333333;   // INVNDIM
constexpr double NDIMPR = 3.0;
constexpr double NDIMPLUS1 = 4.0;
constexpr double SMALL_NUMBER = 1.0e-20;
constexpr double BIG_NUMBER = 9.9e20;
constexpr double HMULT = 1.1;
constexpr double H_CON = 0.02;
constexpr int GRADH_ITERATION_MAX = 20;
constexpr int LEAFMAX = 8;
constexpr int LISTSIZE = 10000;
constexpr int GLISTSIZE = 10000;

// key layout: 21 octree levels of 3 bits in one 64-bit word, level-1 octant
// in the most significant digit.  A tree deeper than that is built again from
// 30-level keys (DEEP_LEVELS, the reference's LMAX, headers/macros.h:139):
// levels 1..21 in the 64-bit word, levels 22..30 in a 27-bit second word.
constexpr int KEY_LEVELS = 21;
constexpr int DEEP_LEVELS = 30;
constexpr int LO_LEVELS = DEEP_LEVELS - KEY_LEVELS;
// cap on h growths in the grad-h candidate search (the reference loops forever
// when fewer than pp_gather particles exist)
constexpr int HGROW_CAP = 2000;

// device error record: the first error wins
struct DevError {
  int code;      // SEREN_GPU_ERR_*
  int where;     // kernel id
  int index;     // particle or cell
  int aux;
};

enum KernelId : int {
  KID_BBOX = 1, KID_KEYS, KID_SORT, KID_SPLIT, KID_EMIT, KID_REORDER, KID_STOCK, KID_HGUESS,
  KID_GRADH, KID_HMAX, KID_NEIB, KID_HYDRO, KID_GRAV, KID_GRAV_MIXED, KID_SINK, KID_THERMAL,
  KID_SINK_SEARCH
};

__device__ __forceinline__ void set_error(DevError* e, int code, int where, int index, int aux) {
  if (atomicCAS(&e->code, 0, code) == 0) {
    e->where = where;
    e->index = index;
    e->aux = aux;
  }
}

// Tree summary kept on the device (and mirrored on the host after a build).
struct TreeInfo {
  int ctot;          // last cell id
  int ltot;          // deepest level
  int nbranch;       // branch cells on the level being split
  int nchild;        // children made on that level
  double rextent;    // maxval(rmax - rmin) of the bounding box (bounding_box.F90:348)
  double root[3];    // root cell centre
  double cellsize;   // 0.5*maxval(rmax - rmin) (BHgrav_build.F90:66)
  int first_cell[32];
  int last_cell[32];
};

// One of several independent clouds sharing a context (seren_gpu_set_clouds).
// The particles stay cloud-major in every order (upload order, tree order),
// cloud k holding [pstart, pstart + n); its tree has root cell `cell` (the
// roots are cells 0..ncloud-1) and its own root box, so each cloud's tree,
// walks and sums are those of a context holding that cloud alone.
struct CloudInfo {
  double root[3];    // root cell centre (BHgrav_build.F90:65-67)
  double cellsize;   // root half width
  double rextent;    // largest bounding-box extent (bounding_box.F90)
  float delta;       // bound on the FP32 rounding of a root-relative coordinate
  int pstart;
  int n;
  int cell;
};

// the cloud of particle p (cloud-major order): the last k with pstart <= p
__host__ __device__ __forceinline__ int cloud_of(const CloudInfo* cl, int ncl, int p) {
  int lo = 0, hi = ncl - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cl[mid].pstart <= p) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Kernel table rows (setup/kernel.F90), packed by use:// Kernel table rows (setup/kernel.F90), packed by use:
//   tabA[i] = (w0, wh, w4, wg): grad-h density, omega, div v, zeta
//   tabG[i] = (w5, w4, w6, w1): gravity softening, potential, hydro gradient
struct KernelTables {
  const double4* A;
  const double4* G;
};

template <typename T>
__host__ __device__ __forceinline__ T cdiv(T a, T b) { return (a + b - 1) / b; }

}  // namespace seren
