/*
 * sphgpu.h — C ABI of the B200 (sm_100a) SPH per-step particle hot path.
 *
 * This is the drop-in boundary for the reference's per-step module surface
 * (Guo-astro/sph-code-simulation):
 *
 *   Module::initialize / Module::calculation        include/module.hpp:10-14
 *   BHTree::initialize / resize / make / set_kernel
 *          / neighbor_search / tree_force           include/bhtree.hpp:76-81
 *   PreInteraction::calculation (ssph)              src/pre_interaction.cpp:39-169
 *   disph::PreInteraction::calculation              src/disph/d_pre_interaction.cpp:21-162
 *   gsph::PreInteraction::calculation               src/gsph/g_pre_interaction.cpp:27-144
 *   FluidForce::calculation (ssph)                  src/fluid_force.cpp:26-86
 *   disph::FluidForce::calculation                  src/disph/d_fluid_force.cpp:26-86
 *   gsph::FluidForce::calculation                   src/gsph/g_fluid_force.cpp:44-171
 *   GravityForce::calculation                       src/gravity_force.cpp:52-89
 *   TimeStep::calculation                           src/timestep.cpp:18-38
 *   Solver::predict / correct / integrate           src/solver.cpp:966-1113
 *   Solver::compute_total_energies                  src/solver.cpp:1149-1175
 *
 * Conventions
 *   - Every entry point returns int: 0 = ok, >0 = recoverable (already
 *     handled internally, e.g. a neighbour-list capacity that was grown and
 *     the walk re-run), <0 = fatal.  The message of the last error is
 *     available from sphgpu_last_error().  The C++ wrapper in
 *     sph-code-simulation_b200/host/sphgpu.hpp turns fatal codes into
 *     sph::SPHException, the way THROW_ERROR does (include/exception.hpp:9-14).
 *   - One CUDA stream per context.  A context is not thread-safe.
 *   - All device memory is owned by the context.  Host arrays passed in are
 *     plain pointers in the caller's particle order (the reference's
 *     std::vector<SPHParticle> index order); the device keeps particles in
 *     octree (Morton) order and un-permutes on download.
 *   - There is no CPU fallback: without a usable sm_100 device every compute
 *     entry point fails with SPHGPU_ERR_CUDA.
 */
#ifndef SPHGPU_H
#define SPHGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enums: same order as sph::SPHType / KernelType / RiemannSolverType
 *      (include/parameters.hpp:8-31) ---- */
enum sphgpu_sph_type { SPHGPU_SSPH = 0, SPHGPU_DISPH = 1, SPHGPU_GSPH = 2, SPHGPU_GDISPH = 3, SPHGPU_SRGSPH = 4 };
enum sphgpu_kernel   { SPHGPU_CUBIC_SPLINE = 0, SPHGPU_WENDLAND = 1, SPHGPU_GAUSSIAN = 2 };
enum sphgpu_riemann  { SPHGPU_RIEMANN_HLL = 0, SPHGPU_RIEMANN_ITERATIVE = 1 };
enum sphgpu_precision { SPHGPU_FP64 = 0, SPHGPU_MIXED = 1 };
enum sphgpu_guess    { SPHGPU_GUESS_NONE = 0, SPHGPU_GUESS_MLP = 1 };

/* return codes */
enum sphgpu_status {
    SPHGPU_OK = 0,
    SPHGPU_RETRIED = 1,            /* capacity grown and the pass re-run */
    SPHGPU_ERR_ARG = -1,           /* bad argument */
    SPHGPU_ERR_CUDA = -2,          /* CUDA runtime error / no device */
    SPHGPU_ERR_NEIGHBOR_OVERFLOW = -3, /* > neighbor_number*1000 neighbours (src/bhtree.cpp:129-135) */
    SPHGPU_ERR_NODE_POOL = -4,     /* more nodes than 5*N+1 (src/bhtree.cpp:222-224) */
    SPHGPU_ERR_STATE = -5,         /* call out of order (e.g. force before tree) */
    SPHGPU_ERR_NO_MLP = -6,        /* riemann_guess = MLP without weights */
    SPHGPU_ERR_SR_RECOVERY = -7    /* srgsph: the Lorentz-factor solve of the primitive
                                      recovery did not converge (the reference throws
                                      std::runtime_error, src/srgsph/sr_primitive_recovery.cpp:75) */
};

/* Subset of sph::SPHParameters (include/parameters.hpp:33-91) that the hot
 * path reads.  Key names follow the JSON keys of Solver::read_parameterfile
 * (src/solver.cpp:311-438); sphgpu_default_params() fills the same defaults. */
typedef struct sphgpu_params {
    int32_t sph_type;              /* SPHType: ssph / disph / gsph          */
    int32_t kernel;                /* "kernel": cubic_spline / wendland     */
    int32_t neighbor_number;       /* "neighborNumber" (50)                 */
    int32_t iterative_sml;         /* "iterativeSmoothingLength" (1)        */
    double  gamma;                 /* "gamma" (5/3)                         */
    double  cfl_sound;             /* "cflSound" (0.3)                      */
    double  cfl_force;             /* "cflForce" (0.125)                    */
    double  av_alpha;              /* "avAlpha" (1.0)                       */
    int32_t use_balsara_switch;    /* "useBalsaraSwitch" (1)                */
    int32_t use_time_dependent_av; /* "useTimeDependentAV" (0)              */
    double  alpha_max;             /* "alphaMax" (2.0)                      */
    double  alpha_min;             /* "alphaMin" (0.1)                      */
    double  epsilon_av;            /* "epsilonAV" (0.2)                     */
    int32_t use_ac;                /* "useArtificialConductivity" (0)       */
    int32_t max_tree_level;        /* "maxTreeLevel" (20)                   */
    double  alpha_ac;              /* "alphaAC" (1.0)                       */
    int32_t leaf_particle_num;     /* "leafParticleNumber" (1)              */
    int32_t periodic;              /* "periodic" (0)                        */
    double  range_min[3];          /* "rangeMin"                            */
    double  range_max[3];          /* "rangeMax"                            */
    int32_t use_gravity;           /* "useGravity" (0)                      */
    int32_t gsph_2nd_order;        /* "use2ndOrderGSPH" (1)                 */
    double  g_constant;            /* "G" (1.0)                             */
    double  theta;                 /* "theta" (0.5)                         */
    int32_t riemann_solver;        /* "riemannSolver": hll / iterative      */
    int32_t precision;             /* sphgpu_precision: FP64 drop-in / mixed */
    int32_t riemann_guess;         /* sphgpu_guess: none / learned MLP      */
    int32_t mlp_max_newton;        /* learned form: Newton iterations before
                                      falling back to the plain solver (4)  */
    /* SRGSPH (SPHParameters::srgsph, include/parameters.hpp:89-96; keys of
     * src/solver.cpp:430-438) */
    int32_t sr_2nd_order;          /* "use2ndOrderSRGSPH" (1)               */
    int32_t tree_root_origin;      /* non-periodic root cube: 1 = the bounding
                                      box of the particles and the origin, as
                                      BHTree::make computes it when OpenMP runs
                                      more than one thread (its per-thread
                                      min / max slots other than thread 0's
                                      start at 0.0: include/openmp.hpp:16-27,
                                      src/bhtree.cpp:68-91); 0 = the particles'
                                      own bounding box (one thread).  (1)   */
    double  sr_c_speed;            /* "cSpeed" (1.0)                        */
    double  sr_c_shock;            /* "cShock" (3.0)                        */
    double  sr_c_cd;               /* "cContactDiscontinuity" (1.0)         */
    double  sr_eta;                /* "etaSmoothingLength" (1.0)            */
    double  sr_c_smooth;           /* "cSmoothGradient" (2.0)               */
    /* Mixed form only (no counterpart in the reference): per-particle bound
     * on the FP32 rounding error of the FluidForce and GravityForce sums,
     * relative to the acceleration.  After GravityForce, particles whose
     * error estimate (8 x 2^-24 x the sum of the absolute values of their
     * FP32 force and gravity terms) exceeds it are re-evaluated in FP64
     * (FluidForce and GravityForce on the same lists and tree).  It bounds
     * the rounding of the force and gravity terms, not that of the FP32
     * PreInteraction outputs (density, pressure) they read.  0 = off.  (0) */
    double  mixed_acc_tol;
    /* Relative change of p at which the plain iterative Riemann solver stops
     * (src/gsph/g_fluid_force.cpp:262 stops at 1e-6; a smaller value runs
     * the same Newton iteration further, for like-for-like comparisons with
     * the learned start, which always refines to 1e-10).  (1e-6)          */
    double  riemann_tol;
    /* No counterpart in the reference (an implementation choice with the
     * same results): the gather walk builds lists of radius (1 + gather_skin)
     * times the gather radius and later steps reuse them, moved to each new
     * tree's particle order, while every particle's gather sphere stays
     * inside its list's sphere (displacements are tracked); the consumers
     * take exactly the reference's list members from them.  The skin
     * widens (2x, up to 5 x gather_skin) after two builds in a row that
     * served fewer than two steps, when the motion measured at the failed
     * check shows the wider lists would serve two; lists that serve eight
     * steps or more narrow it again.  Two builds in a row that are never
     * reused and do not widen it pause the skin for 32 steps of exact
     * walks.  0 = a fresh exact walk every step.  (0.02)                  */
    double  gather_skin;
} sphgpu_params;

/* Per-particle fields, in the order of sph::SPHParticle where it has them
 * (include/particle.hpp:8-43), then the GSPH named arrays
 * (src/solver.cpp:707-719), then the SRGSPH particle fields
 * (include/particle.hpp:31-38: S, e, N, nu, gamma_lor, enthalpy, dS, de; held
 * on the device only by SRGSPH contexts). Used by upload/download. */
enum sphgpu_field {
    SPHGPU_F_POS_X = 0, SPHGPU_F_POS_Y, SPHGPU_F_POS_Z,
    SPHGPU_F_VEL_X, SPHGPU_F_VEL_Y, SPHGPU_F_VEL_Z,
    SPHGPU_F_VELP_X, SPHGPU_F_VELP_Y, SPHGPU_F_VELP_Z,
    SPHGPU_F_ACC_X, SPHGPU_F_ACC_Y, SPHGPU_F_ACC_Z,
    SPHGPU_F_MASS, SPHGPU_F_DENS, SPHGPU_F_PRES, SPHGPU_F_ENE, SPHGPU_F_ENE_P,
    SPHGPU_F_DENE, SPHGPU_F_SML, SPHGPU_F_SOUND, SPHGPU_F_BALSARA,
    SPHGPU_F_ALPHA, SPHGPU_F_GRADH, SPHGPU_F_PHI, SPHGPU_F_NEIGHBOR,
    SPHGPU_F_GRAD_D_X, SPHGPU_F_GRAD_D_Y, SPHGPU_F_GRAD_D_Z,
    SPHGPU_F_GRAD_P_X, SPHGPU_F_GRAD_P_Y, SPHGPU_F_GRAD_P_Z,
    SPHGPU_F_GRAD_V0_X, SPHGPU_F_GRAD_V0_Y, SPHGPU_F_GRAD_V0_Z,
    SPHGPU_F_GRAD_V1_X, SPHGPU_F_GRAD_V1_Y, SPHGPU_F_GRAD_V1_Z,
    SPHGPU_F_GRAD_V2_X, SPHGPU_F_GRAD_V2_Y, SPHGPU_F_GRAD_V2_Z,
    SPHGPU_F_SR_S_X, SPHGPU_F_SR_S_Y, SPHGPU_F_SR_S_Z, SPHGPU_F_SR_E,
    SPHGPU_F_SR_N, SPHGPU_F_SR_NU, SPHGPU_F_SR_GAMMA_LOR, SPHGPU_F_SR_ENTHALPY,
    SPHGPU_F_SR_DS_X, SPHGPU_F_SR_DS_Y, SPHGPU_F_SR_DS_Z, SPHGPU_F_SR_DE,
    SPHGPU_NFIELDS
};

/* Device-side counters (no reference counterpart except the Newton
 * non-convergence log line, src/pre_interaction.cpp:277-280). */
typedef struct sphgpu_counters {
    int64_t newton_nonconverged;   /* smoothing-length Newton fallbacks      */
    int64_t riemann_solves;        /* iterative/learned Riemann solves       */
    int64_t riemann_iterations;    /* Newton iterations summed over solves   */
    int64_t riemann_fallbacks;     /* learned guess -> plain solver fallbacks */
    int64_t gather_capacity;       /* current per-particle list capacity     */
    int64_t max_gather;            /* largest gather list of the last search */
    int64_t max_pair;              /* largest symmetric list                 */
    int64_t node_count;            /* octree nodes of the last tree_make     */
    int64_t retries;               /* neighbour walks re-run after growing   */
    int64_t walk_group_warps;      /* warps walked as one group of 32        */
    int64_t walk_split_warps;      /* warps walked as several sub-groups     */
    int64_t walk_fallbacks;        /* group walks redone per lane (overflow) */
    int64_t mlp_guesses;           /* pairs whose start came from the network */
    int64_t force_list_builds;     /* FluidForce calls that took the pair lists
                                      built from the gather lists (no walk) */
    /* work done since the last reset, the units of the FLOP roofline */
    int64_t pre_candidates;        /* gather-list entries tested, summed over
                                      the Newton sweeps and the final pass  */
    int64_t pre_newton_pairs;      /* pairs inside h in the Newton sweeps    */
    int64_t pre_pairs;             /* pairs inside h in the final pass       */
    int64_t pre_list_entries;      /* gather-list entries read by the final pass
                                      (each list once)                       */
    int64_t force_candidates;      /* pair-list entries tested by FluidForce */
    int64_t force_pairs;           /* pairs inside max(h_i, h_j)             */
    int64_t gravity_nodes;         /* tree nodes met (opening tests)         */
    int64_t gravity_monopoles;     /* nodes taken as monopoles               */
    int64_t gravity_leaf_pairs;    /* softened particle pairs                */
    int64_t mixed_rechecks;        /* mixed form: particles whose FluidForce and
                                      GravityForce were re-evaluated in FP64
                                      (mixed_acc_tol)                       */
    int64_t skin_builds;           /* gather walks that built skin lists      */
    int64_t skin_reuses;           /* steps that reused them (no walk)        */
} sphgpu_counters;

/* Stage timers (ms, summed since the last reset; CUDA events on the
 * context stream, recorded only when timing is enabled). */
enum sphgpu_stage {
    SPHGPU_T_TIMESTEP = 0, SPHGPU_T_PREDICT, SPHGPU_T_TREE, SPHGPU_T_GATHER_WALK,
    SPHGPU_T_PRE, SPHGPU_T_SET_KERNEL, SPHGPU_T_PAIR_WALK, SPHGPU_T_FORCE,
    SPHGPU_T_GRAVITY, SPHGPU_T_CORRECT,
    SPHGPU_T_RECHECK,   /* mixed form: FP64 re-evaluation (mixed_acc_tol) */
    SPHGPU_NSTAGES
};

typedef struct sphgpu_ctx sphgpu_ctx;

/* ---------------- parameters / lifetime ---------------- */
void        sphgpu_default_params(sphgpu_params* p);
int         sphgpu_create(const sphgpu_params* p, sphgpu_ctx** out);
/* Simulation(param) + BHTree::initialize (src/simulation.cpp:13-33,
   src/bhtree.cpp:13-41). */
int         sphgpu_destroy(sphgpu_ctx* ctx);
const char* sphgpu_last_error(const sphgpu_ctx* ctx);
int         sphgpu_device_ok(void);  /* 1 if an sm_100 device is usable */

/* ---------------- state transfer ---------------- */
/* Largest particle count a context holds: octree nodes (up to 5 n + 2, the
   reference's pool of BHTree::resize, src/bhtree.cpp:43-51) are int32 indices. */
#define SPHGPU_MAX_PARTICLES 429496729
/* fields[k] may be NULL (field zero-filled).  Arrays are length n, in the
   caller's particle order; the caller's index is the particle id.  Device
   buffers are reused when n is unchanged; time, dt and h_per_v_sig persist
   across uploads, and the next PreInteraction runs initial_smoothing unless
   sphgpu_set_initial_smoothing(ctx, 0) is called. */
int sphgpu_upload(sphgpu_ctx* ctx, int64_t n, const double* const* fields);
/* fields[k] may be NULL (field skipped). */
int sphgpu_download(sphgpu_ctx* ctx, double* const* fields);
int64_t sphgpu_particle_num(const sphgpu_ctx* ctx);
int sphgpu_get_time(const sphgpu_ctx* ctx, double* time, double* dt);
int sphgpu_set_dt(sphgpu_ctx* ctx, double dt);
int sphgpu_get_h_per_v_sig(const sphgpu_ctx* ctx, double* h_per_v_sig);

/* ---------------- modules ---------------- */
/* BHTree::make (src/bhtree.cpp:59-115): bbox, Morton keys replaying the
   pos > center comparisons, radix sort, bottom-up node build, mass and
   centre of mass.  Permutes the device particle arrays into tree order. */
int sphgpu_tree_make(sphgpu_ctx* ctx);
/* BHTree::set_kernel (src/bhtree.cpp:117-120,249-275). */
int sphgpu_tree_set_kernel(sphgpu_ctx* ctx);
/* Batched BHTree::neighbor_search (src/bhtree.cpp:122-144,277-316) for every
   particle with radius sml (is_ij=0) or max(sml, node kernel_size)
   (is_ij=1).  Writes a host CSR in caller order: offsets[n+1], ids[].
   Pass ids=NULL to get the offsets (sizes) only.  Lists are in tree-walk
   order (not distance-sorted). */
int sphgpu_neighbor_search(sphgpu_ctx* ctx, int is_ij, int64_t* offsets,
                           int32_t* ids, int64_t ids_capacity);
/* The pairs FluidForce sums over for the current state, as a CSR in caller
   order like sphgpu_neighbor_search: every j with r_ij < max(h_i, h_j).
   After PreInteraction they are built from the gather lists (own entries in
   gather-list order, then the pairs only j's kernel reaches, by index);
   otherwise, or when those are incomplete, the symmetric walk's lists.  No
   reference counterpart (the reference searches inside FluidForce::calculation,
   src/fluid_force.cpp:45-60); parity checks use it. */
int sphgpu_force_pairs(sphgpu_ctx* ctx, int64_t* offsets, int32_t* ids, int64_t ids_capacity);
/* Same, with the O(N^2) exhaustive predicate of exhaustive_search
   (src/exhaustive_search.cpp:11-42). Debug/parity only. */
int sphgpu_exhaustive_search(sphgpu_ctx* ctx, int is_ij, int64_t* offsets,
                             int32_t* ids, int64_t ids_capacity);
/* PreInteraction::calculation for params.sph_type, including
   initial_smoothing on the first call and set_kernel at the end. */
int sphgpu_pre_interaction(sphgpu_ctx* ctx);
/* FluidForce::calculation for params.sph_type (overwrites acc and dene). */
int sphgpu_fluid_force(sphgpu_ctx* ctx);
/* GravityForce::calculation (adds to acc, sets phi). No-op without gravity. */
int sphgpu_gravity_force(sphgpu_ctx* ctx);
/* GravityForce::calculation under -DEXHAUSTIVE_SEARCH: direct summation
   (src/gravity_force.cpp:70-84). Debug/parity only. */
int sphgpu_gravity_direct(sphgpu_ctx* ctx);
/* TimeStep::calculation: sets and returns dt. */
int sphgpu_timestep(sphgpu_ctx* ctx, double* dt);
/* Solver::predict / Solver::correct with the context dt. */
int sphgpu_predict(sphgpu_ctx* ctx);
int sphgpu_correct(sphgpu_ctx* ctx);
/* Tail of Solver::initialize (src/solver.cpp:941-964): alpha = avAlpha,
   balsara = 1, sound = sqrt(gamma (gamma-1) u), tree make, pre, force,
   gravity. */
int sphgpu_initialize(sphgpu_ctx* ctx);
/* Solver::integrate (src/solver.cpp:966-978) followed by
   Simulation::update_time. */
int sphgpu_integrate(sphgpu_ctx* ctx);
/* One sphgpu_integrate on host buffers, for a host that keeps the particle
   state (the reference's Solver::integrate with every module on the GPU and
   SPHParticle as the record): in_fields replace the device state as
   sphgpu_upload does, except that the simulation time and the
   initial-smoothing flag carry on (the particle count must be the uploaded
   one); the step runs; out_fields receive the state as sphgpu_download
   writes it.  Fields that are final early in the step (positions and mass
   after the tree build, the PreInteraction outputs after it) are copied to
   the host while the rest of the step runs, on a second stream, and the
   alpha, Balsara, grad-h, density and pressure inputs (first read by
   PreInteraction) are copied up while the step's first modules run; the
   call returns when every copy
   is done.  Either table may hold NULL entries. */
int sphgpu_integrate_host(sphgpu_ctx* ctx, const double* const* in_fields, double* const* out_fields);
/* Solver::compute_total_energies (src/solver.cpp:1149-1175), plus total
   momentum (mom[3]); FP64 device reductions. mom may be NULL. */
int sphgpu_energies(sphgpu_ctx* ctx, double* kinetic, double* thermal,
                    double* potential, double* mom);

/* ---- Lane-Emden relaxation ---------------------------------------------
 * One step of Solver's relaxation loop (src/solver.cpp:779-829): tree, pre,
 * force, gravity (when on); minus LaneEmdenRelaxation's analytic equilibrium
 * acceleration (src/relaxation/lane_emden_relaxation.cpp:35-138) interpolated
 * in the caller's table (LaneEmdenData, src/relaxation/lane_emden_data.cpp:
 * 66-113; the reference reads it from data/lane_emden/n1.5_3d.dat); TimeStep's
 * dt x 0.1 -> *dt_relax; v = 0, x += a dt^2 / 2.  `first` != 0 sets the sound
 * speeds first, as the set-up before the loop does.  The simulation time is
 * not advanced (the reference accumulates dt_relax separately). */
typedef struct sphgpu_lane_emden {
    double alpha_scaling;          /* r = alpha * xi                         */
    double K;                      /* polytropic constant                    */
    double xi_1;                   /* first zero of theta                    */
    const double* xi;              /* npts ascending abscissae (host)        */
    const double* theta;
    const double* dtheta;          /* dtheta / dxi                           */
    int64_t npts;
} sphgpu_lane_emden;
int sphgpu_relax_step(sphgpu_ctx* ctx, const sphgpu_lane_emden* le, int first, double* dt_relax);

/* ---- Snapshots in the reference's CSV v1 format ------------------------
 * CSVWriter (src/writers/csv_writer.cpp:18-170) with the header of
 * OutputManager::build_metadata (src/output_manager.cpp:254-299): code units,
 * doubles as "%.*e" with `precision` digits (the reference's default 16),
 * rows ordered by caller index with id = that index.  The reference's own
 * plotting scripts and load_for_resume (src/output_manager.cpp:150-233) read
 * these files. */
typedef struct sphgpu_csv_meta {
    int step;                      /* header "Step"                          */
    double time;                   /* "Time (code)" and "Time (physical)"    */
    int sph_type;                  /* enum sphgpu_sph_type; others: Unknown  */
    int kernel;                    /* enum sphgpu_kernel; others: Unknown    */
    double gamma, g_constant;
    int neighbor_number;
    int use_gravity, use_balsara, use_time_dependent_av;
    double kinetic, thermal, potential;  /* "Total" is their sum          */
    int precision;                 /* decimal digits after the point (1..30) */
    const char* timestamp;         /* NULL or "": the current UTC time       */
} sphgpu_csv_meta;
/* The context's state (downloaded in caller order), its time, parameters
   and device energies, written to `path`. */
int sphgpu_write_csv(sphgpu_ctx* ctx, const char* path, int step, int precision);
/* OutputManager::load_for_resume (src/output_manager.cpp:150-233) for a CSV
   snapshot: its particles, in file order, become the context's state (as
   sphgpu_upload) and its "Time (code)" the simulation time; *step (may be
   NULL) receives its "Step". */
int sphgpu_read_csv(sphgpu_ctx* ctx, const char* path, int* step);
/* Host-only writer: n rows from host arrays indexed like sphgpu_download's
   (NULL arrays print 0; ids NULL = 0..n-1).  Needs no device. */
int sphgpu_csv_write_host(const char* path, int64_t n, const double* const* fields,
                          const int64_t* ids, const sphgpu_csv_meta* meta);
/* Reader (CSVWriter::read_metadata / read_particles, src/writers/csv_writer.cpp:
   172-369): *n = the file's row count; with fields != NULL fills up to cap rows
   (ERR_ARG when the file holds more); meta and ids may be NULL. */
int sphgpu_csv_read_host(const char* path, int64_t* n, int64_t cap, double* const* fields,
                         int64_t* ids, sphgpu_csv_meta* meta);

/* Neighbour-walk implementation: 0 (default) = warp-level group walk with
   exact fallback for pairs on the search radius; 1 = per-lane walk that
   replays the reference's recursion test by test.  Both give the same sets;
   mode 1 exists for cross-checking. */
int sphgpu_set_walk_mode(sphgpu_ctx* ctx, int mode);
/* PreInteraction::m_first (src/pre_interaction.cpp:41-44): whether the next
   PreInteraction call runs initial_smoothing first.  Set after upload; turn
   it off to continue from a state whose density is already an SPH density
   (e.g. a snapshot or another implementation's output). */
int sphgpu_set_initial_smoothing(sphgpu_ctx* ctx, int on);
/* Octree node table in depth-first preorder (children in index order), for
   tree parity: ints[3k..] = level, is_leaf, particle count;
   dbl[9k..] = center x,y,z, edge, mass, centre of mass x,y,z, kernel_size.
   Returns the node count (call with NULL buffers to size), <0 on error. */
int64_t sphgpu_tree_nodes(sphgpu_ctx* ctx, int32_t* ints, double* dbl, int64_t capacity);

/* ---------------- diagnostics ---------------- */
int sphgpu_get_counters(sphgpu_ctx* ctx, sphgpu_counters* out);
int sphgpu_reset_counters(sphgpu_ctx* ctx);
int sphgpu_enable_timing(sphgpu_ctx* ctx, int on);
int sphgpu_get_stage_times(sphgpu_ctx* ctx, double* ms /* [SPHGPU_NSTAGES] */,
                           int64_t* launches /* [SPHGPU_NSTAGES] or NULL */);
/* Wait for the context's stream.  Also reports (SPHGPU_ERR_STATE) a bound
   hit since the last wait by a device pass that runs without a host wait of
   its own: the bottom-up mass and kernel_size passes and the gravity walks,
   which bound their loops by the tree depth and node count instead of
   looping on a corrupt tree.  sphgpu_integrate, sphgpu_initialize and the
   next tree_make / neighbour walk report it the same way. */
int sphgpu_synchronize(sphgpu_ctx* ctx);
/* Test hook: set PASS_GUARD bits (1 mass, 2 set_kernel, 4 gravity, 8 mixed
   gravity) on the device as those passes do when they hit their bound, so a
   test can check that the next synchronising call reports it without
   corrupting a tree.  No counterpart in the reference. */
int sphgpu_test_flag_pass_guard(sphgpu_ctx* ctx, int bits);
/* CUDA-event timer on the context stream: elapsed device time between the
   two calls (the stop call waits for the stream). */
int sphgpu_timer_start(sphgpu_ctx* ctx);
int sphgpu_timer_stop(sphgpu_ctx* ctx, double* ms);
/* Kernels this context launched since timing was last enabled. */
int64_t sphgpu_launch_count(const sphgpu_ctx* ctx);

/* ---------------- allocation-free entry point ---------------- */
/* No counterpart in the reference.  TimeStep::calculation for callers that
   cannot allocate device memory when they need dt (e.g. a host solver whose
   device memory is entirely owned by its own pool, or code that must not
   incur the synchronisation of cudaMalloc/cudaFree).  Inputs and the result
   are caller-owned DEVICE memory: acc_xyz = 3n doubles (x, y, z per
   particle), sml = n doubles, dt_out = 1 double; stream = cudaStream_t
   (NULL = default stream).  Nothing is allocated: the reduction scratch is a
   fixed file-scope device array of SPHGPU_NOALLOC_MAX_BLOCKS doubles that
   every GPU loading the library keeps until exit.  n above
   SPHGPU_NOALLOC_MAX_PARTICLES is rejected with SPHGPU_ERR_ARG.  The first
   call on a device looks up the array's device address (make it before any
   stream capture).  All calls share the array: calls that overlap on the GPU
   race.  The looked-up address is cached per device for the life of the
   process: do not call this entry point again after cudaDeviceReset on that
   device (the cached address would then be stale). */
#define SPHGPU_NOALLOC_TILE 1024
#define SPHGPU_NOALLOC_MAX_BLOCKS 4096
#define SPHGPU_NOALLOC_MAX_PARTICLES (SPHGPU_NOALLOC_TILE * SPHGPU_NOALLOC_MAX_BLOCKS)
int sphgpu_timestep_noalloc(const double* acc_xyz, const double* sml, int64_t n,
                            double h_per_v_sig, double cfl_sound, double cfl_force,
                            double* dt_out, void* stream);

/* ---------------- learned Riemann guess (no reference counterpart) ------ */
/* The MLP maps (log rho_R/rho_L, log p_R/p_L, (u_R-u_L)/c_L, c_R/c_L, gamma)
   to log(p_star / p_L) through 3 hidden layers of 64 SiLU units. Weights are BF16
   on the device, FP32 master copies in the trainer. */
enum { SPHGPU_MLP_IN = 5, SPHGPU_MLP_HIDDEN = 64, SPHGPU_MLP_LAYERS = 3 };
/* Number of FP32 parameters (weights + biases) of the MLP. */
int64_t sphgpu_mlp_param_count(void);
/* Load / read FP32 master parameters (length sphgpu_mlp_param_count()):
   W0[64][5], b0[64], W1[64][64], b1[64], W2[64][64], b2[64], w3[64], b3. */
int sphgpu_mlp_set_params(sphgpu_ctx* ctx, const float* params);
int sphgpu_mlp_get_params(sphgpu_ctx* ctx, float* params);
/* Deterministic Glorot-uniform initialisation from a seed. */
int sphgpu_mlp_init(sphgpu_ctx* ctx, uint64_t seed);
/* Riemann states are rows of 7 doubles: u_L, rho_L, p_L, u_R, rho_R, p_R,
   gamma (left = neighbour j side, right = particle i side, as the GSPH force
   poses them, src/gsph/g_fluid_force.cpp:140).  Network output
   y = log(p_star / p_L) per state (host arrays). */
int sphgpu_mlp_predict(sphgpu_ctx* ctx, const double* states, int64_t n, float* y);
/* Adam training on labelled states (mean squared error in y) with the
   project's tensor-core forward/backward kernels; loss_history[epochs].
   epochs = 0: write the full-data gradient of the current parameters to
   grad_out[param_count] and its loss to loss_history[0]. */
int sphgpu_mlp_train(sphgpu_ctx* ctx, const double* states, const double* pstar, int64_t n, int epochs,
                     int batch, float lr, uint64_t seed, float* loss_history, float* grad_out);
/* Riemann problems in bulk on the device: mode 0 = the reference's iterative
   solver (src/gsph/g_fluid_force.cpp:209-304), 1 = learned guess + Newton
   (fallback to mode 0), 2 = converged to 1e-13 (training labels), 3 = plain
   start converged to 1e-10.  Outputs may be NULL except pstar. */
int sphgpu_riemann_batch(sphgpu_ctx* ctx, const double* states, int64_t n, int mode, double* pstar,
                         double* vstar, int32_t* iters, int32_t* fallbacks);
/* Harvest pair states from the plain solver's own runs: subsequent
   FluidForce calls append sampled pairs (records of 8 doubles: the 7 state
   values then p_star); harvest_end copies them out and stops. */
int sphgpu_harvest_begin(sphgpu_ctx* ctx, int64_t capacity, uint32_t sample_mod);
int sphgpu_harvest_end(sphgpu_ctx* ctx, double* out, int64_t capacity, int64_t* count);

/* ---------------- workload generators (inputs, not the hot path) ------- */
/* Deterministic initial conditions in the field order above; call with
   fields == NULL to get the particle count.  Evrard sphere:
   Solver::make_evrard (src/sample/evrard.cpp:13-87). */
int64_t sphgpu_sample_evrard(int N, double G, double gamma, double* const* fields);
/* 3-D periodic shear layer after Solver::make_khi (src/sample/khi.cpp:12-73). */
int64_t sphgpu_sample_shear_layer(double dx, double lz, double gamma, double* const* fields);
/* 3-D shock tube along x in [-0.5, 0.5] x [0, ly]^2. */
int64_t sphgpu_sample_shock_tube(double dx, double ly, double p_left, double p_right, double gamma,
                                 double* const* fields);
/* Special-relativistic Sod tube after Solver::make_sr_sod
   (src/sample/sr_sod.cpp:15-199) in 3-D; ly / (2 dx) a whole number. */
int64_t sphgpu_sample_sr_shock_tube(double dx, double ly, double gamma, double c_speed, double* const* fields);

#ifdef __cplusplus
}
#endif
#endif /* SPHGPU_H */
