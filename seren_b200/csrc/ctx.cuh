// ctx.cuh - the device context behind one seren_gpu_ctx, and the launchers
// each .cu file provides to the C ABI layer.
#pragma once

#include <string>
#include <vector>

#include "../../include/seren_gpu.h"
#include "common.cuh"

namespace seren {

// Scratch for the multi-level exclusive scan of int32 arrays.
struct ScanScratch {
  int* level_buf[4] = {nullptr, nullptr, nullptr, nullptr};  // block sums per level
  int level_cap[4] = {0, 0, 0, 0};
  int* total = nullptr;  // device int: total of the last scan
};

// Block timesteps of the device-resident step loop (blockstep.cu): the
// scalars of the reference's time_module on the host, the per-particle level
// state in tree order on the device (permuted at every build, as
// reorder_particle_arrays does).
// Tuning knobs of the kernels (seren_gpu_autotune, seren_gpu_set_tuning).
// The FP64 path's results do not depend on them; the mixed path's change in
// the FP32 rounding of its partial sums only (hydro_sub, grav_cap).
struct Tuning {
  int hydro_sub = 4;   // threads per particle of the mixed hydro kernel: 2, 4 or 8
  int grav_cap = 64;   // cell-list tile of the mixed gravity walk: 64 or 96 entries
  int grav_bps = 0;    // resident blocks per SM of the gravity walk (0: as many as fit)
  int gradh_bps = 0;   // of the grad-h pass kernel
  int neib_bps = 0;    // of the neighbour-row kernel
};

struct BlockState {
  bool on = false;
  int nlevels = 1;
  int level_mode = 1;        // 0 free, 1 RESTRICTED_TIMESTEP_LEVELS, 2 FIXED_TIMESTEP_LEVELS
  int check_neib = 1;        // CHECK_NEIB_TIMESTEP: 0, 1 or 2
  double dt_fixed = 1.0, courant = 0.2, accel = 0.5;
  long long n = 0, nresync = 0, nsteps = 0;
  int level_max = 0, level_step = 0, nactive = 0;
  double timestep = 0.0, dt_max = 0.0, time = 0.0;
  int* nlevel = nullptr;
  long long* nlast = nullptr;
  int* nminneib = nullptr;
  int* accdo = nullptr;
  double* laststep = nullptr;
  int* nlevel_alt = nullptr;
  long long* nlast_alt = nullptr;
  int* nminneib_alt = nullptr;
  int* accdo_alt = nullptr;
  double* laststep_alt = nullptr;
  double* acc_alt = nullptr;             // a and gpot follow the particles in block mode
  double* gpot_alt = nullptr;
  double* dt = nullptr;                  // per-particle timestep_size
  unsigned long long* red = nullptr;     // [4] reduction words
};

struct Ctx {
  seren_gpu_params prm{};
  int64_t pmax = 0;
  int cmax = 0;          // 2*pmax, the reference's cmax_grav
  int ptot = 0;
  int dev = 0;
  cudaStream_t st = nullptr;
  std::string err;

  // particles in tree order
  double4* pm = nullptr;     // x, y, z, m
  double2* hz = nullptr;     // h, zeta
  double4* vel = nullptr;    // vx, vy, vz, 0
  double* csq = nullptr;     // isothermal c_s^2 = Pconst*T
  int* orig = nullptr;       // id of each slot in the first upload's order
  double4* pm_alt = nullptr;
  double2* hz_alt = nullptr;
  double4* vel_alt = nullptr;
  double* csq_alt = nullptr;
  int* orig_alt = nullptr;
  double* rho = nullptr;
  double* omega = nullptr;
  double* div_v = nullptr;
  double* drhodt = nullptr;
  // reorder targets of rho, omega, div_v, drhodt: a tree build permutes them
  // with the particles, as main/reorder_array.F90 does the host's arrays
  double* rho_alt = nullptr;
  double* omega_alt = nullptr;
  double* div_v_alt = nullptr;
  double* drhodt_alt = nullptr;
  double* press = nullptr;
  double* sound = nullptr;
  double* acc = nullptr;     // [ptot][3]
  // second-order Runge-Kutta state (seren_gpu_rk2_step), made on first use and
  // reordered with the particles: positions and velocities at the start of
  // the step and the velocities at its half
  double4* r_old = nullptr;
  double4* v_old = nullptr;
  double4* v_half = nullptr;
  double4* r_old_alt = nullptr;
  double4* v_old_alt = nullptr;
  double4* v_half_alt = nullptr;
  double* gpot = nullptr;
  double* pf = nullptr;      // hydro: press/rho/rho/omega per particle
  double* hf4 = nullptr;     // hydro: (1/h)**(NDIM+1) per particle
  int* pptot = nullptr;
  int* pplist = nullptr;     // [ptot][pp_limit]
  int* act = nullptr;        // active list (0-based), when given
  double* stage = nullptr;   // [pmax][6] device staging of host-layout arrays
  int* istage = nullptr;     // [pmax*pp_limit] device staging of id arrays
  double* h_pin = nullptr;   // pinned host staging, [pmax][6] doubles
  // mapped page-locked host words the device writes small results into
  // (read_dev): no copy-engine transfer, so they never queue behind bulk copies
  int* h_map = nullptr;
  int* d_map = nullptr;
  int* hi_pin = nullptr;     // pinned host staging, ids

  // build scratch
  unsigned long long* keys = nullptr;
  unsigned long long* keys_alt = nullptr;
  unsigned long long* keys_hi = nullptr;   // deep builds: levels 1..21 in input order
  unsigned* keys_lo = nullptr;             // deep builds: levels 22..30 in input order
  int* idx = nullptr;
  int* idx_alt = nullptr;
  int* rs_hist = nullptr;     // [256][nblk]
  double* bbox_part = nullptr;
  int* branch = nullptr;      // branch cells of the level being split
  int* branch_next = nullptr;
  int* nchild = nullptr;      // children per branch cell
  int* choff = nullptr;       // exclusive scan of nchild
  int* cstart = nullptr;      // [nbranch][9] child range boundaries
  int* bflag = nullptr;       // 1 for a branch child on the new level
  int* bscan = nullptr;
  ScanScratch scan;

  // tree, breadth-first cell ids 0..ctot
  int* leaf = nullptr;
  int* nextcell = nullptr;
  int* ifopen = nullptr;
  int* pstart = nullptr;
  int* pcount = nullptr;
  int* parent = nullptr;
  int* level = nullptr;
  int* nkids = nullptr;       // number of children (0 for leaves); they are ifopen..ifopen+n-1
  int4* link = nullptr;       // {leaf, nextcell, ifopen, pstart}, packed for walks
  double4* gA = nullptr;      // gravity: COM x, y, z, m
  double4* gB = nullptr;      // gravity: q1..q4 (xx, xy, yy, zx)
  double2* gC = nullptr;      // gravity: q5 (zy), dminsqd
  // gravity walk node, two float4 per cell (one 32-byte sector): FP32 COM -
  // root centre and the upper MAC bracket; the lower bracket, then (as int
  // bits) the first particle of a leaf or first child of a branch, and the
  // leaf's particle count or minus the branch's number of children
  float4* wA = nullptr;
  // hydro walk node, two float4 per cell: hA32; hrm32, then (as int bits)
  // the first particle of a leaf or first child of a branch, and the leaf's
  // particle count or minus the branch's number of children
  float4* hN = nullptr;
  double4* hA = nullptr;      // hydro: bbox centre x, y, z, rmax
  double* hrm = nullptr;      // hydro: hrangemax
  float4* hA32 = nullptr;     // hydro walk: FP32 centre - root centre, rmax rounded up
  float* hrm32 = nullptr;     // hydro walk: hrangemax rounded up
  double* hmax = nullptr;     // stock: max h in the cell (at stock time)
  double4* bbmin = nullptr;
  double4* bbmax = nullptr;
  TreeInfo* d_info = nullptr;
  TreeInfo info{};            // host mirror after a build
  DevError* d_err = nullptr;
  int* d_counts = nullptr;    // [16] int64 interaction counters (as 2 ints each)
  int* work = nullptr;        // work counter of the persistent kernels
  double* sinks = nullptr;    // [1024][5] sinks of the device-resident step (x, y, z, m, h)
  int nsink = 0;
  double* sink_out = nullptr; // [1024][4] sink accelerations and potentials of the last walk
  // sinks that seren_gpu_rk2_step moves (seren_gpu_set_sink_motion): host
  // copies of their state, [nsink][5] x y z m h, [nsink][3] v and a, radius,
  // potential, and the Runge-Kutta start and half-step values
  bool sink_move = false;
  bool sink_a_valid = false;
  std::vector<double> sink_rmh, sink_v, sink_a, sink_pot, sink_radius, sink_rold, sink_vold,
      sink_vhalf;
  int* leaves = nullptr;      // [pmax][256] opened leaves of each particle's grad-h walk
  int* nleaf = nullptr;       // their number (-1: overflow)
  int* npot = nullptr;        // [pmax] particles in those leaves (pp_pot)
  int* redo = nullptr;        // [pmax] particles whose grad-h is redone alone; count in work[1]
  int* wide = nullptr;        // [pmax] particles whose grad-h walks cover most of the tree; count in work[2]
  void* wst = nullptr;        // state of a batch of those particles (sph.cu)
  double* wacc = nullptr;     // their walk accumulators, 4 per particle
  double* wpart = nullptr;        // their partial sums per walk slice (made on first use)
  double* wpart_brute = nullptr;  // and per particle tile of the passes
  size_t wpart_brute_cap = 0;
  bool gsets = false;             // the last grad-h recorded the gather neighbours (launch_neib)
  int* wcover = nullptr;          // the cells their walks are spread over (made on first use)
  int wcover_cap = 0;
  double4* hrec = nullptr;        // hydro: 96-byte neighbour records, 3 per particle (first use)
  int2* wstack = nullptr;     // walk stacks, wstack_cap (cell, lane mask) entries per warp slot
  int wstack_cap = 0;
  int wstack_slots = 0;

  // kernel tables
  double4* tabA = nullptr;
  double4* tabG = nullptr;
  float4* tabG32 = nullptr;   // FP32 w5, w4, w6 of tabG (mixed gravity)

  // sink accretion and search (seren_gpu_accrete, seren_gpu_sink_search), made
  // on first use: sink records and results, ACC_STRIDE doubles per sink for up
  // to 1024 sinks, and 4 * pmax + 16 ints of scratch (sinks.cu)
  double* acc_sinks = nullptr;
  double* acc_out = nullptr;
  int* acc_ws = nullptr;

  BlockState blk;
  Tuning tune;

  // independent clouds (seren_gpu_set_clouds): ncloud > 1 makes every tree
  // build a forest of ncloud trees and the group kernels take gact, the
  // particles cloud by cloud with each cloud padded (-1) to a multiple of 32,
  // so that no group of 32 spans two clouds
  int ncloud = 1;
  std::vector<CloudInfo> clouds;       // host copy (after a build: roots and extents)
  CloudInfo* d_clouds = nullptr;
  int* gact = nullptr;
  int ngact = 0;

  // build schedule of the device-resident force steps (main/tree_update.F90:
  // build every nbuildstep evaluations, restock in between)
  int nbuildstep = 1;
  int since_build = 0;

  bool have_tree = false;
  bool have_sph = false;
  bool have_v = false;
  bool have_csq = false;

  // seren_gpu_force_step_io: a copy stream, its events and a staging buffer
  // of 6*pmax doubles, made on first use; build_tree waits for reorder_wait
  // (when set) before it reorders the particles
  cudaStream_t st_io = nullptr;
  cudaEvent_t ev_io[3] = {};
  double* stage_io = nullptr;
  cudaEvent_t reorder_wait = nullptr;
  bool reorder_late = false;    // v and c_s^2 still to reorder (finish_reorder)
  cudaEvent_t vel_wait = nullptr;   // velocities still being copied in (finish_reorder waits)

  // timing of the last force step
  cudaEvent_t ev[10] = {};
  double stage_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int nlaunch = 0;          // kernels launched since the counter was reset
  int step_launches = 0;    // kernels of the last seren_gpu_force_step
};

// tree.cu
int build_tree(Ctx& c);               // bbox, keys, sort, cells, leaf order, reorder
void finish_reorder(Ctx& c);          // the deferred v, c_s^2 reorder (reorder_wait set)
// the stock of the last build's cells at the current positions (no build, no
// reorder), as tree_update does between builds; rebuilt = true when the
// particles left the range the node records allow and the tree was built
int restock(Ctx& c, bool& rebuilt);
// copy `bytes` (a multiple of 4, at most 1 KiB) of device memory to the host
// through the mapped words, after the work queued on c.st; 0 or an error code
int read_dev(Ctx& c, const void* dsrc, void* hdst, size_t bytes);
void launch_unpack_parray(Ctx& c, const double* stage, int n);
void launch_pack_parray(Ctx& c, double* stage, int n, cudaStream_t s = nullptr);
void launch_stock(Ctx& c);            // BHgrav_stock + BHhydro_stock
void launch_update_hmax(Ctx& c);      // BHhydro_update_hmax
void launch_hguess(Ctx& c);           // BHhydro_hguess
void scan_exclusive(Ctx& c, const int* in, int* out, int n);   // total -> c.scan.total
int scan_scratch_alloc(ScanScratch& s, int nmax);

// blockstep.cu
void reorder_block(Ctx& c);           // the block state follows a build's permutation
int block_active(Ctx& c, int& nact);  // c.act = the accdo particles (tree order)
int block_start(Ctx& c);              // state after a first force step of every particle
int block_after_forces(Ctx& c);       // sph_timesteps, neighbour checks, advance, reduction
void block_free(Ctx& c);
int rk_alloc(Ctx& c);                 // r_old, v_old, v_half (and their reorder targets)

// sph.cu
void launch_gradh(Ctx& c, int nact);
void launch_hgather(Ctx& c, int nact);  // h_gather (standard SPH)
// sorted = false: right after grad-h with every particle active, the rows
// hold the reference's neighbours and counts in a fixed order of their own
// (the device's own hydro forces do not depend on it beyond rounding); true:
// in the reference's order, for lists the caller reads
void launch_neib(Ctx& c, int nact, bool sorted = true);
void launch_hydro(Ctx& c, int nact, double* amap = nullptr);   // amap: mapped host a (optional)
void launch_thermal(Ctx& c);
int hydro_walk_slots(const Ctx& c);     // resident warps of the grad-h / neighbour grids
int wide_scratch_alloc(Ctx& c);         // c.wst, c.wacc; 0 or -1
// check_neighbour_timesteps: every active particle's level reaches the
// nminneib of its neighbours (its list, or the same test on the fly)
void launch_neib_levels(Ctx& c, int nact, const int* nlevel, int* nminneib);

// gravity.cu
// amap/gmap (optional): host buffers mapped into the device address space
// that receive a and gpot of each particle as soon as its group is done;
// abase (optional): where the acceleration gravity adds to is read (else acc)
void launch_grav(Ctx& c, int nact, int nsink, const double* d_sinks, double* amap = nullptr,
                 double* gmap = nullptr, const double* abase = nullptr);
void launch_sink_walk(Ctx& c, int nsink, const double* d_sinks, double* d_out /*[nsink][4]*/);
int grav_walk_slots(const Ctx& c);      // resident warps of the gravity walk grid
int grav_walk_stack_cap(const Ctx& c);  // stack entries per warp

// sinks.cu
constexpr int ACC_STRIDE = 16;
// the options of sinks/sink_search.F90 (setup/default_parameters.F90:120-129)
struct SinkSearchArgs {
  double rhosink;
  double sinkrad;
  int hmult_sinkrad;
  int rho_search;
  int potmin_search;
  int hill_sphere_search;
  int div_v_search;
  int div_a_search;
  int timescale_search;
};
// sink_search + create_sink on the device-resident particles with the sinks
// in c.acc_sinks: psink = the particle made a sink (-1: none; psink_id its id),
// out = {m, x, y, z, vx, vy, vz, ax, ay, az, Lx, Ly, Lz, radius}, nremoved
// particles removed (psink and its neighbours); c.ptot is the kept count
int launch_sink_search(Ctx& c, int nsink, const SinkSearchArgs& sa, int& psink, int& psink_id,
                       std::vector<double>& out, int& nremoved);
// accrete_particles + remove_from_list on the device-resident particles with
// the sinks in c.acc_sinks: ndead particles accreted (0: nothing changed); when
// ndead > 0, out holds ACC_STRIDE doubles per sink and c.ptot is the kept count
int launch_accrete(Ctx& c, int nsink, int energy, std::vector<double>& out, int& ndead);

// tables.cpp
void make_kernel_tables(int kernel, std::vector<double>& w0, std::vector<double>& w1,
                        std::vector<double>& w4, std::vector<double>& w5, std::vector<double>& w6,
                        std::vector<double>& wh, std::vector<double>& wg);

}  // namespace seren
