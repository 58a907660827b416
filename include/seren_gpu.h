/*
 * seren_gpu.h - C ABI of the B200 force hot path of the SEREN grad-h SPH code.
 *
 * One call replaces one OpenMP particle loop of the Fortran reference.  All
 * arrays are HOST arrays laid out like the Fortran module arrays they replace:
 * column-major Fortran parray(1:6,1:ptot) is C row-major parray[ptot][6] with
 * columns x, y, z, m, h, zeta (headers/macros.h:44-55, NDIM=3 block);
 * v(1:3,p) and a(1:3,p) are [ptot][3]; pplist(1:pp_limit,p) is
 * [ptot][pp_limit].  Particle ids that cross the boundary (perm_out, pplist,
 * acclist) use the base given in seren_gpu_params.index_base (1 for Fortran).
 *
 * Every function returns SEREN_GPU_OK (0) or one of the SEREN_GPU_ERR_* codes
 * below; seren_gpu_last_error() gives a one-line reason.  No device code ever
 * traps: walk caps and capacity limits set an error flag that the host reads.
 * A context is not thread-safe; call it from one host thread (the Fortran
 * master thread, outside !$OMP regions).  Each call synchronises its stream
 * before returning.
 */
#ifndef SEREN_GPU_H
#define SEREN_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SEREN_GPU_OK 0
#define SEREN_GPU_ERR_ARG 1        /* bad argument or unsupported option         */
#define SEREN_GPU_ERR_CAPACITY 2   /* ptot > pmax, or cell count > 2*pmax          */
#define SEREN_GPU_ERR_LMAX 3       /* tree deeper than the supported level count   */
#define SEREN_GPU_ERR_NONFINITE 4  /* NaN/Inf in positions, masses or h            */
#define SEREN_GPU_ERR_WALK 5       /* a tree walk hit its iteration cap            */
#define SEREN_GPU_ERR_NEGATIVE_H 6 /* grad-h produced h < 0 (all_sph_gradh.F90:486) */
#define SEREN_GPU_ERR_CUDA 7       /* CUDA runtime error                           */
#define SEREN_GPU_ERR_STATE 8      /* call made before the state it needs exists   */

typedef struct seren_gpu_ctx seren_gpu_ctx;

/* Runtime options of the hot path.  Values come from params.dat and the
 * compile-time macros of the reference (setup/default_parameters.F90:104-117,
 * setup/initialize_seren_variables_1.F90:30-39, headers/macros.h:138-139). */
typedef struct {
  int32_t ndim;        /* must be 3                                              */
  int32_t kernel;      /* 0 = M4 (KERNEL=M4), 1 = M4 Thomas-Couchman (M4TC)      */
  int32_t visc;        /* 0 = MON97 artificial viscosity                         */
  int32_t precision;   /* 0 = FP64 throughout, 1 = mixed FP32 pair arithmetic    */
  int32_t pp_gather;   /* target neighbour number (57 for h_fac = 1.2)           */
  int32_t pp_limit;    /* neighbour-list width, 2*pp_gather                      */
  int32_t leafmax;     /* must be 8 (LEAFMAX)                                    */
  int32_t lmax;        /* maximum tree level, <= 30 (LMAX)                       */
  int32_t index_base;  /* 1: Fortran ids (1..ptot); 0: C ids (0..ptot-1)         */
  int32_t redo_cap;    /* 0: default; n > 0: a grad-h redo walk that needs more than n
                          frontier cells or leaves moves to the whole-GPU path (results
                          unchanged; small n exercises that path in tests). The CPU
                          oracle ignores it.                                        */
  double h_fac;        /* h = h_fac*(m/rho)^(1/3)                                */
  double thetamaxsqd;  /* geometric MAC opening angle squared                    */
  double alpha;        /* artificial viscosity alpha (beta is always 2*alpha)    */
  double alpha_min;    /* unused by MON97 without time-dependent viscosity       */
} seren_gpu_params;

/* Context: device mirrors of the particle arrays, the gravity/hydro tree and
 * scratch, sized for pmax particles.  Replaces allocate_memory.F90:43-221 for
 * the arrays of the hot path. */
int seren_gpu_create(seren_gpu_ctx** ctx, int64_t pmax, const seren_gpu_params* prm);
void seren_gpu_destroy(seren_gpu_ctx* ctx);
int seren_gpu_last_error(seren_gpu_ctx* ctx, char* buf, int32_t len);

/* tree_update (main/tree_update.F90:27-60): when do_build != 0,
 * BHgrav_build (BHtree/BHgrav_build.F90:12-309) and, when do_reorder != 0,
 * BH_reorder_particles (BHtree/BH_reorder_particles.F90:57-123) with the
 * device mirrors permuted; then BHgrav_stock (BHtree/BHgrav_stock.F90:11-358),
 * copy_BHgrav_to_BHhydro and BHhydro_stock.  parray is uploaded first and,
 * after a reorder, written back in tree order; perm_out[new] = old id
 * (the reference's dummylist) when not NULL.  The stock uses the h in parray,
 * i.e. the h from before this step's grad-h solve, as the reference does. */
int seren_gpu_tree_update(seren_gpu_ctx* ctx, int32_t ptot, double* parray,
                          int32_t do_build, int32_t do_reorder, int32_t* perm_out);

/* sph_update, GRAD_H_SPH branch (sph_sim/sph_update.F90:57-100):
 * [BHhydro_hguess when first_call] -> all_sph_gradh for the active particles
 * -> BHhydro_update_hmax -> get_neib.  v is uploaded; parray columns h and
 * zeta, rho, omega, div_v and drhodt are written back for the active
 * particles (with every particle active, whole parray rows are written, their
 * x, y, z, m being the ones uploaded by the last tree_update).  pptot/pplist
 * may be NULL (then the lists stay on the device for seren_gpu_hydro_forces).
 * acclist == NULL means every particle is active. */
int seren_gpu_sph_update(seren_gpu_ctx* ctx, int32_t ptot, const int32_t* acclist,
                         int32_t nacc, double* parray, const double* v, double* rho,
                         double* omega, double* div_v, double* drhodt, int32_t* pptot,
                         int32_t* pplist, int32_t first_call);

/* get_neib alone (sph/get_neib.F90:10-140) after BHhydro_update_hmax, at the
 * smoothing lengths h[ptot] given (NULL: the ones on the device). */
int seren_gpu_get_neib(seren_gpu_ctx* ctx, int32_t ptot, const int32_t* acclist,
                       int32_t nacc, const double* h, int32_t* pptot, int32_t* pplist);

/* h_gather (sph/h_gather.F90:14-203), the standard-SPH smoothing length loop
 * of sph_sim/sph_update.F90:111-119, then BHhydro_update_hmax (:121-124):
 * for each active particle (acclist, NULL: all) of the last tree_update,
 * h = INVKERNRANGE*sqrt(d2) with d2 the pp_gather-th smallest squared
 * distance to another particle, the value the reference's search and
 * insertion sort select whatever the guess (MINIMUM_H is not applied).  The
 * new h is written to column 4 of the active rows of parray (tree order) and
 * kept on the device for a following seren_gpu_get_neib.  Fewer than
 * pp_gather other particles (the reference loops forever) give
 * SEREN_GPU_ERR_WALK. */
int seren_gpu_h_gather(seren_gpu_ctx* ctx, int32_t ptot, const int32_t* acclist, int32_t nacc,
                       double* parray);

/* sph_hydro_forces (sph_sim/sph_hydro_forces.F90:41-85) with hydro_gradh
 * (sph/hydro_gradh.F90:9-339, MON97): a[p] is OVERWRITTEN with the hydro
 * acceleration of each active particle (inactive rows are left as they are). */
int seren_gpu_hydro_forces(seren_gpu_ctx* ctx, const int32_t* acclist, int32_t nacc,
                           const double* press, const double* sound, double* a);

/* sph_grav_forces (sph_sim/sph_grav_forces.F90:94-157): BHgrav_accel with
 * gravity_gradh (BHtree/BHgrav_accel.F90:21-348, gravity/gravity_gradh.F90)
 * ADDED to a, gpot OVERWRITTEN with the (positive) potential; then, when
 * nsink > 0, direct_sink_gravity (sinks/direct_sink_gravity.F90:10-64) with
 * sink_rmh[s] = {x, y, z, m, h} added to a and gpot. */
int seren_gpu_grav_forces(seren_gpu_ctx* ctx, const int32_t* acclist, int32_t nacc,
                          double* a, double* gpot, int32_t nsink, const double* sink_rmh);

/* sph_sink_forces (sph_sim/sph_sink_forces.F90:49-110): for each sink, the
 * tree walk BHgrav_accel(-s) with gravity_meanh plus the sink-sink direct sum.
 * sink_a[s][3] and sink_gpot[s] are overwritten. */
int seren_gpu_sink_forces(seren_gpu_ctx* ctx, int32_t nsink, const double* sink_rmh,
                          double* sink_a, double* sink_gpot);

/* Device-resident force step, the path the Fortran caller reaches with
 * positions kept on the device between steps: seren_gpu_upload() copies
 * parray, v and csq = Pconst*T (isothermal c_s^2) once; seren_gpu_force_step()
 * runs tree build + reorder + stock, [h guess], grad-h, hmax update,
 * neighbour lists, isothermal thermal (sph/thermal.F90:52-59), hydro and
 * gravity without touching the host; seren_gpu_drift() moves r += v*dt;
 * seren_gpu_download() copies results back in tree order (any pointer may be
 * NULL).  The uploaded particles are all gas particles (the reference's
 * pgasstart..pgasend range): the device-resident calls that loop over
 * particles (accretion, sink search) take every uploaded particle as gas, so
 * a caller with boundary or intercloud particles uploads only its gas range. */
int seren_gpu_upload(seren_gpu_ctx* ctx, int32_t ptot, const double* parray,
                     const double* v, const double* csq);
int seren_gpu_force_step(seren_gpu_ctx* ctx, int32_t first_call);
int seren_gpu_drift(seren_gpu_ctx* ctx, double dt);
/* Per-particle timesteps on the state of the last force evaluation
 * (timestep/timestep_size.F90:52-120 with HYDRO and MON97 viscosity,
 * beta = 2*alpha, no internal energy):
 *   dt_p = min(accel_mult*sqrt(h/(|a| + 1e-20)),
 *              courant_mult*h/(c + h|div v| + 0.6*(alpha*c + beta*h|div v|))).
 * *dt_min receives the least of them (the global step of
 * sph_sim/sph_timesteps.F90:58-66); dt (may be NULL) every dt_p, in tree
 * order.  Not a reference entry point: it replaces the loop that calls
 * timestep_size for every particle. */
int seren_gpu_timestep(seren_gpu_ctx* ctx, double courant_mult, double accel_mult,
                       double* dt_min, double* dt);
/* One step of the reference's second-order Runge-Kutta scheme
 * (advance/advance_runge_kutta.F90:40-72) for all particles on one timestep
 * level, kept on the device: r_half = r + v*dt/2, v_half = v + a*dt/2; the
 * forces at the half step; r' = r + v_half*dt, v' = v + a_half*dt; the forces
 * at the end, so the state is at t + dt with its accelerations, ready for
 * seren_gpu_timestep.  Two force evaluations, each as seren_gpu_force_step
 * (tree rebuilt; the step's state follows the particle reorder).  Needs
 * seren_gpu_upload and one seren_gpu_force_step first.  Not a reference
 * entry point: it replaces sph_advance's per-particle loop for one level. */
int seren_gpu_rk2_step(seren_gpu_ctx* ctx, double dt);
/* Many independent clouds in one context (no counterpart in the reference,
 * which evolves one cloud per run).  After seren_gpu_upload of the clouds'
 * particles one cloud after another (counts[k] particles each, summing to
 * ptot), every tree build makes a forest of ncloud trees at once: one sort of
 * all particles (octant keys from each cloud's own root box, then a stable
 * pass on the cloud) and one level-by-level split of all clouds' cells, the
 * roots being cells 0..ncloud-1; the walks, passes, hydro and gravity then
 * run as single launches over every cloud, each group of 32 particles inside
 * one cloud (each cloud's particles padded to a multiple of 32) and walking
 * its own cloud's tree from its own root box.  Every cloud's results equal
 * those of a context holding that cloud alone, bit for bit.  Particles stay
 * cloud-major in tree order: cloud k is rows [pstart_k, pstart_k + counts[k])
 * of seren_gpu_download with pstart_k the sum of the counts before it, and
 * perm maps them to upload indices.  ncloud = 1 returns to one cloud; a new
 * upload does too.  Active lists, sinks and block timesteps are refused while
 * ncloud > 1.  The device-resident force steps build the forest every
 * evaluation. */
int seren_gpu_set_clouds(seren_gpu_ctx* ctx, int32_t ncloud, const int32_t* counts);

/* Kernel tuning (no counterpart in the reference).  The knobs: threads per
 * particle of the mixed-precision hydro kernel (2, 4 or 8), the cell-list tile
 * of the mixed-precision gravity walk (64 or 96 entries), and the resident
 * blocks per SM of the gravity walk, the grad-h pass and the neighbour-row
 * kernels (0: as many as fit).  The defaults (4, 64, 0, 0, 0) suit the 4M-
 * particle core.  seren_gpu_autotune, after seren_gpu_upload and a first
 * seren_gpu_force_step, times `trials` force steps on the current state for
 * each of four configurations, keeps for every stage its fastest, applies
 * the result to the context and records it for the process under (device,
 * precision, ceil(log2 ptot)); with trials <= 0 it applies the recorded
 * choice instead (SEREN_GPU_ERR_STATE when there is none).  The FP64 path's
 * results do not depend on the knobs; the mixed path's change within FP32
 * rounding (the order of its partial sums).  ms_per_step (out) is the force
 * step the chosen knobs give. */
typedef struct {
  int32_t hydro_sub;
  int32_t grav_cap;
  int32_t grav_bps;
  int32_t gradh_bps;
  int32_t neib_bps;
  int32_t reserved;
  double ms_per_step;
} seren_gpu_tuning;
int seren_gpu_autotune(seren_gpu_ctx* ctx, int32_t trials, seren_gpu_tuning* out);
int seren_gpu_set_tuning(seren_gpu_ctx* ctx, const seren_gpu_tuning* tuning);

/* Block timesteps (nlevels > 1) of the reference's main loop for the
 * second-order Runge-Kutta scheme, on the device-resident particles
 * (sph_sim/sph_integrate.F90:27-136).  seren_gpu_block_start, after
 * seren_gpu_upload and a first seren_gpu_force_step (the setup evaluation of
 * every particle), takes that state as the start of every particle's step
 * (initialize_sph_variables_2.F90:72-73, :157; n = nresync = 0).  Each
 * seren_gpu_block_step is one call of sph_integrate: tree_update on the
 * build schedule (seren_gpu_set_build_step), sph_update, thermal, hydro and
 * gravity for the accdo particles only, sph_timesteps
 * (sph_sim/sph_timesteps.F90:11-341: resynchronisation at n == nresync,
 * levels int(INVLOGETWO*log(dt_max/dt)) + 1, one level up at a time when
 * synchronised, integer times rescaled when level_max changes),
 * check_neighbour_timesteps (timestep/check_neighbour_timesteps.F90:11-85),
 * advance_runge_kutta for every particle (advance/advance_runge_kutta.F90:
 * 9-111) and, with check_neib = 2, reduce_timesteps
 * (timestep/reduce_timesteps.F90, reduce_particle_timestep.F90).  The
 * per-particle level state stays on the device in tree order and follows
 * every build, with a and gpot.  Timesteps are timestep_size.F90's (as
 * seren_gpu_timestep).  Moving sinks, accretion and sink search are refused
 * while block timesteps are on; a new upload turns them off. */
typedef struct {
  int32_t nlevels;      /* timestep levels, 1..24 (setup/default_parameters.F90:66)       */
  int32_t level_mode;   /* 0 free, 1 RESTRICTED_TIMESTEP_LEVELS (the reference's default:
                           dt_min = dt_fixed/2^k), 2 FIXED_TIMESTEP_LEVELS                 */
  int32_t check_neib;   /* CHECK_NEIB_TIMESTEP: 0 none, 1 CHECK_NEIGHBOUR_TIMESTEPS (the
                           default), 2 with IMMEDIATE_TIMESTEP_REDUCTION                   */
  int32_t reserved;     /* 0 */
  double dt_fixed;      /* setup/default_parameters.F90:67                                 */
  double courant_mult;  /* timestep_size.F90 multipliers                                   */
  double accel_mult;
} seren_gpu_block_params;
/* The time_module scalars after a step (sph_timesteps.F90 state). */
typedef struct {
  int64_t n;            /* integer time after the step                                  */
  int64_t nresync;      /* integer time of the next resynchronisation                    */
  int64_t nsteps;
  int32_t level_max;
  int32_t level_step;
  int32_t nactive;      /* particles whose forces this step evaluated                    */
  int32_t reserved;
  double timestep;      /* length of one integer step                                    */
  double dt_max;
  double time;
} seren_gpu_block_state;
int seren_gpu_block_start(seren_gpu_ctx* ctx, const seren_gpu_block_params* prm);
int seren_gpu_block_step(seren_gpu_ctx* ctx, seren_gpu_block_state* out);
/* Per-particle block state in tree order (any pointer may be NULL): level,
 * integer time of the start of the current step, least neighbour level, accdo. */
int seren_gpu_block_levels(seren_gpu_ctx* ctx, int32_t* nlevel, int64_t* nlast,
                           int32_t* nminneib, int32_t* accdo);

/* Sinks that seren_gpu_rk2_step moves with the gas (sinks/advance_sink_RK.F90:
 * 22-51, same step; their accelerations are sph_sink_forces.F90:49-110 on each
 * step's trees): velocities [nsink][3] and radii for the sinks last given to
 * seren_gpu_set_sinks (which stops their motion until this is called again). */
int seren_gpu_set_sink_motion(seren_gpu_ctx* ctx, int32_t nsink, const double* sink_v,
                              const double* sink_radius);
/* The sinks' current state (any pointer may be NULL): x, y, z, m, h
 * [nsink][5], v [nsink][3], acceleration [nsink][3] and potential. */
int seren_gpu_get_sinks(seren_gpu_ctx* ctx, int32_t nsink, double* sink_rmh, double* sink_v,
                        double* sink_a, double* sink_gpot);
/* The least sink timestep (sinks/sink_timestep.F90:28-52: sink_mult times
 * sqrt(radius/|a|) and radius/|v|, and the sink-sink crossing times), which
 * sph_sim/sph_timesteps.F90:69-74 folds into the global minimum. */
int seren_gpu_sink_timestep(seren_gpu_ctx* ctx, double sink_mult, double* dt_min);
/* Sink accretion on the device-resident particles, replacing
 * sinks/accrete_particles.F90:16-365 with main/remove_from_list.F90:10-96
 * (called by sinks/sink_update.F90:24 after the step's advance).  Each particle
 * inside the radius of an accreting sink (accrete[s] != 0; NULL: every sink)
 * goes to the nearest one; with energy_accrete it must also be bound to it
 * (kinetic energy of the reduced mass below m_p times the pair potential of
 * gravity/gravity_gradh.F90, called as the reference calls it).  An accreting
 * sink takes the mass of its particles, moves to their common centre of mass,
 * velocity and mass-weighted acceleration, and sink_angmom[s] (when given,
 * [nsink][3], added to) takes the angular momentum about the new centre of
 * mass.  The accreted particles leave the device arrays, the others keep their
 * order; naccreted[s] (when given) counts them per sink, *ptot_out (when
 * given) is the new particle count.  Needs seren_gpu_set_sinks,
 * seren_gpu_set_sink_motion and a force step; afterwards the next force step
 * builds a new tree (calls that reuse the tree fail until then). */
int seren_gpu_accrete(seren_gpu_ctx* ctx, int32_t nsink, const int32_t* accrete,
                      int32_t energy_accrete, double* sink_angmom, int32_t* naccreted,
                      int32_t* ptot_out);

/* Options of the sink search (setup/default_parameters.F90:120-129; the
 * logical ones 0 or 1).  sinkrad is the new sink's radius, in units of the
 * particle's h when hmult_sinkrad (the reference's SINK_RADIUS = HMULT). */
typedef struct {
  double rhosink;
  double sinkrad;
  int32_t hmult_sinkrad;
  int32_t rho_search;
  int32_t potmin_search;
  int32_t hill_sphere_search;
  int32_t div_v_search;
  int32_t div_a_search;
  int32_t timescale_search;
  int32_t reserved;        /* 0 */
} seren_gpu_sink_search_params;

/* Sink search and creation on the device-resident particles, replacing
 * sinks/sink_search.F90:25-433 with sinks/create_sink.F90:11-268 (called by
 * sinks/sink_update.F90:16-20 every nsearchstep steps).  Candidates: rho >=
 * rhosink (rho_search), a minimum of the potential over the gather
 * neighbours (potmin_search), not within 2 radii of a sink, the Hill test
 * (hill_sphere_search; it reads accelerations that only the reference's
 * DEBUG_FORCES builds fill, and so rejects nothing, as there), div v and div
 * a of the neighbours within max(sinkrad, 2h) not positive, and the timescale
 * test (timescale_search).  When a candidate passes, the densest candidate
 * of the last test loop becomes a sink (as the reference picks it) with the
 * particles within the sink radius of it: mass, centre of mass, velocity,
 * acceleration, h = radius/2, and its angular momentum in sink_angmom[3]
 * (when given).  Those particles leave the device arrays (the rest keep
 * their order); the new sink is appended to the sinks (seren_gpu_get_sinks)
 * and moves with seren_gpu_rk2_step.  *created is 1 or 0, *psink_id the id
 * (index_base) of the particle it was made from, *nremoved the particles
 * removed, *ptot_out the particles left (each may be NULL).  Needs a force
 * step on the current positions (the walk uses its tree); with sinks, their
 * motion set.  Afterwards the next force step builds a new tree. */
int seren_gpu_sink_search(seren_gpu_ctx* ctx, const seren_gpu_sink_search_params* prm,
                          int32_t* created, int32_t* psink_id, double* sink_angmom,
                          int32_t* nremoved, int32_t* ptot_out);
/* Sinks for the device-resident step: from the next seren_gpu_force_step on,
 * its gravity adds direct_sink_gravity (sinks/direct_sink_gravity.F90:10-64)
 * for sink_rmh[s] = {x, y, z, m, h}, as seren_gpu_grav_forces does with
 * nsink > 0 (at most 1024 sinks; nsink = 0 removes them). */
int seren_gpu_set_sinks(seren_gpu_ctx* ctx, int32_t nsink, const double* sink_rmh);
/* Build schedule of the device-resident force steps (seren_gpu_force_step and
 * the evaluations inside seren_gpu_rk2_step), as main/tree_update.F90:26-88
 * with the reference's nbuildstep (default there 8; here 1, a build every
 * evaluation): the tree is built on the next evaluation and then every
 * nbuildstep evaluations; in between the same cells are restocked at the new
 * positions (BHgrav_stock, BHhydro_stock) and the particles keep their
 * order.  A build also happens after an upload, on a first call, after
 * accretion or sink creation, and when a particle has moved beyond twice
 * the root cell's half width from its centre (the bound of the walks' FP32
 * node records).  seren_gpu_force_step_io always builds. */
int seren_gpu_set_build_step(seren_gpu_ctx* ctx, int32_t nbuildstep);
int seren_gpu_download(seren_gpu_ctx* ctx, double* parray, double* v, double* rho,
                       double* omega, double* a, double* gpot, int32_t* perm_total);

/* One force evaluation from host buffers to host buffers: the work of
 * seren_gpu_upload(ptot, parray, v, csq), seren_gpu_force_step(first_call)
 * and seren_gpu_download(parray_out, v_out, rho, omega, a, gpot, perm_total)
 * in one call, plus csq_out (c_s^2 in tree order).  The copies overlap the
 * force step on a second stream: v and c_s^2 come in during the tree build,
 * and each result goes out once the stage that makes it has run (v, c_s^2,
 * perm after the tree build; parray with the new h, rho, omega after grad-h;
 * a and gpot after gravity).  Outputs are in tree order; any output may be
 * NULL and may alias its input.  Pinned host buffers give overlapped copies.
 * Not a reference entry point: it fuses the calls a caller of
 * seren_gpu_tree_update / sph_update / hydro_forces / grav_forces makes
 * each step when it keeps no state on the device. */
int seren_gpu_force_step_io(seren_gpu_ctx* ctx, int32_t ptot, const double* parray,
                            const double* v, const double* csq, int32_t first_call,
                            double* parray_out, double* v_out, double* csq_out, double* rho,
                            double* omega, double* a, double* gpot, int32_t* perm_total);

/* Tree inspection (BHgrav_node / BHhydro_node of headers/modules.F90:907-959
 * in the reference's breadth-first cell numbering).  Counts first: pass NULL
 * arrays to get ctot and ltot.  plist rows hold particle ids (index_base) and
 * -1 past the leaf count; ifopen is -1 for leaves. */
int seren_gpu_tree_export(seren_gpu_ctx* ctx, int32_t* ctot, int32_t* ltot,
                          int32_t* leaf, int32_t* nextcell, int32_t* ifopen,
                          int32_t* plist /*[ctot+1][8]*/, int32_t* first_cell,
                          int32_t* last_cell, double* grav_r /*[ctot+1][3]*/,
                          double* grav_m, double* grav_q /*[ctot+1][5]*/,
                          double* dminsqd, double* hydro_r /*[ctot+1][3]*/,
                          double* rmax, double* hrangemax);

/* Per-stage device time of the last seren_gpu_force_step (ms: tree build +
 * stock, grad-h, hmax update + neighbour lists, thermal + hydro, gravity,
 * total), the number of kernels it launched, and the work counters of the
 * last force evaluation (16 slots): gravity [0] cell terms, [1] pair terms,
 * [2] walk entries (cell, lane mask), [8] grad-h particles whose walks
 * needed a block each (k_gradh_wide), [9] cell-list
 * entries, [10] of them taken by all 32 lanes, [11] near-field list items,
 * [12] of them for all 32 lanes; grad-h [3] walks, [4] walk entries (with
 * the neighbour-list kernel), [5] passes, [6] candidates, [13] warp
 * iterations over candidates; neighbour lists [7] candidates, [14] warp
 * iterations; [15] particles handed to a single-particle path (grad-h
 * re-walks and overflows, neighbour-row overflows). */
int seren_gpu_last_step_stats(seren_gpu_ctx* ctx, double* stage_ms /*[8]*/,
                              int32_t* nlaunch, int64_t* counts /*[16]*/);

/* The CUDA stream every kernel of this context runs on (cudaStream_t), so a
 * caller can order its own work and CUDA events against the library's. */
int seren_gpu_get_stream(seren_gpu_ctx* ctx, void** stream);

/* Measured FMA throughput of this GPU's FP32 (precision 1) or FP64
 * (precision 0) pipe in TFLOP/s (2 flops per FMA), from a kernel of
 * independent FMA chains over every SM; the roofline denominator of the
 * pair-interaction kernels, which do not use tensor cores. */
int seren_gpu_fma_peak(seren_gpu_ctx* ctx, int32_t precision, double* tflops);

/* Hydro accelerations without a context and without allocating device memory.
 * No counterpart in the reference: it serves callers that cannot call
 * cudaMalloc, such as an application whose device memory belongs to its own
 * pool allocator (a framework's caching allocator, a Fortran/OpenACC runtime
 * that reserves the GPU up front) or that runs under a fixed memory budget.
 * Such a caller cannot create a context, but it holds the particle state and
 * the neighbour lists in device buffers of its own; this call runs the hydro
 * kernel of seren_gpu_hydro_forces (grad-h pressure force and MON97
 * viscosity, every particle active) on them.
 *
 * All pointers are DEVICE pointers, laid out like the host arrays above:
 * parray[n][6], v[n][3], rho/omega/press/sound[n], pptot[n],
 * pplist[n][pp_limit] with 0-based ids, output a[n][3] (overwritten).
 * kernel and precision mean what they mean in seren_gpu_params.  stream is a
 * cudaStream_t (NULL for the default stream); the call is synchronous: it
 * waits for that stream before it returns, twice (after the list check and
 * at the end).  An error that the caller's own earlier work left pending is
 * neither reported by this call nor cleared.
 *
 * Limits: n <= SEREN_GPU_NOALLOC_PMAX (SEREN_GPU_ERR_CAPACITY beyond); every
 * row must hold its whole neighbour list, 0 <= pptot <= pp_limit
 * (SEREN_GPU_ERR_CAPACITY otherwise: the context entry point walks the tree
 * for such rows, and there is no tree here); listed ids in 0..n-1
 * (SEREN_GPU_ERR_ARG).  No message is kept: the return code is the report.
 *
 * Scratch: one fixed device array of 3.6 MiB (the kernel-layout copies of
 * the particles, per-particle factors, kernel tables and an error block),
 * held by every GPU that loads the library until the process exits.  The
 * first call on a device looks up the array's address and uploads the kernel
 * tables; make that first call before any stream capture.  That set-up is
 * kept per device ordinal for the life of the process, so the library must not
 * outlive a cudaDeviceReset of a device it has run on.  Every call on a
 * device shares the array and leaves its contents behind, so calls that
 * overlap on the GPU (other streams, other host threads) race: serialise
 * them. */
#define SEREN_GPU_NOALLOC_PMAX 32768
int seren_gpu_hydro_forces_noalloc(int32_t n, const double* parray, const double* v,
                                   const double* rho, const double* omega, const double* press,
                                   const double* sound, const int32_t* pptot,
                                   const int32_t* pplist, int32_t pp_limit, int32_t kernel,
                                   int32_t precision, double alpha, double* a, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SEREN_GPU_H */
