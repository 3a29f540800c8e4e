/*
 * pd_b200.h -- C ABI of the B200-native Peridigm hot path.
 *
 * The library replaces, behind plain C entry points, the per-bond force and
 * damage path of Peridigm: the "Elastic" (LPS) material, the "Critical
 * Stretch" damage model, the "Short Range Force" contact model, the
 * velocity-Verlet explicit integrator and the quasi-static Newton/CG solve.
 * All compute runs in hand-written sm_100a CUDA kernels; there is no CPU path.
 *
 * Conventions
 *  - Every function returns an int status (PD_OK == 0). No exception crosses
 *    the ABI; pd_last_error() gives a one-line message for the last failure.
 *  - Point arrays are in the caller's order and interleaved xyz (3*i+k), as
 *    Peridigm's Epetra vectors are. Host pointers are copied in/out; the
 *    *_device variants take device pointers on the context's device.
 *  - Bond families: Peridigm's flattened neighbor list [n_0, j.., n_1, j..]
 *    (src/core/Peridigm_NeighborhoodData.hpp:56-140) or a search done here.
 *    Bond-ordered data (bond damage) follows that list's order.
 *  - Force outputs are force densities, as Material::computeForce produces
 *    (multiply by volume for forces, src/core/Peridigm.cpp:1881-1884).
 *  - The context owns its device memory. One context per host thread at a
 *    time; contexts are independent.
 *  - Every entry point that takes a context makes the context's device the
 *    calling thread's current CUDA device (cudaSetDevice) and leaves it so; a
 *    caller that drives other devices from the same thread sets its own
 *    device again after the call.
 */
#ifndef PD_B200_H
#define PD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PD_OK 0
#define PD_ERR_ARG 1         /* bad argument (Teuchos TEST_FOR_EXCEPT in the reference) */
#define PD_ERR_CUDA 2        /* CUDA runtime error */
#define PD_ERR_NONFINITE 3   /* NaN/Inf in a force (Peridigm.cpp:1551-1566 terminate) */
#define PD_ERR_TIMEOUT 4     /* a bounded device wait ran out */
#define PD_ERR_STATE 5       /* call out of order (e.g. force before bonds) */
#define PD_ERR_UNSUPPORTED 6 /* input outside what this build handles */
#define PD_ERR_NOMEM 7       /* device allocation failed */
#define PD_ERR_NOT_CONVERGED 8 /* solver stopped before its tolerance */

/* ---- enums ------------------------------------------------------------- */
/* Bond-kernel arithmetic. PD_FP64: every per-bond quantity in FP64, the
 * reference's formulas in the reference's operation order. PD_SPLIT_FP32:
 * per-bond math in FP32 with bond vectors and displacement differences formed
 * in FP64 and rounded once; stretch as (2X.du+du.du)/(|Y|+|X|); FP64 kept for
 * displacement/velocity state, weighted volume and reductions. */
#define PD_FP64 0
#define PD_SPLIT_FP32 1
/* PD_FP64_SLICED: every per-bond quantity in FP64 as PD_FP64, on the split
 * path's data layout: the sliced bond stream at 4 lanes per point with X
 * streamed in FP64 (24 B per bond), one gathered record per neighbor, one
 * division per bond and the owner constants folded (3/m, the c1 and alpha
 * terms), so rounding differs from PD_FP64 in the last bits. LPS elastic with
 * the "One" influence function; other materials and influence functions
 * return PD_ERR_UNSUPPORTED. */
#define PD_FP64_SLICED 2

/* Influence functions (src/core/Peridigm_InfluenceFunction.hpp:69-87). */
#define PD_INFLUENCE_ONE 0
#define PD_INFLUENCE_PARABOLIC_DECAY 1
#define PD_INFLUENCE_GAUSSIAN 2

/* Output fields for pd_get_field (names of Peridigm fields). */
#define PD_FIELD_DISPLACEMENT 0     /* "Displacement"       [3n] double */
#define PD_FIELD_VELOCITY 1         /* "Velocity"           [3n] double */
#define PD_FIELD_ACCELERATION 2     /* "Acceleration"       [3n] double */
#define PD_FIELD_FORCE_DENSITY 3    /* "Force_Density" (internal + contact) [3n] double */
#define PD_FIELD_CONTACT_FORCE 4    /* "Contact_Force_Density" [3n] double */
#define PD_FIELD_DILATATION 5       /* "Dilatation"         [n] double */
#define PD_FIELD_WEIGHTED_VOLUME 6  /* "Weighted_Volume"    [n] double */
#define PD_FIELD_DAMAGE 7           /* "Damage"             [n] double */
#define PD_FIELD_BOND_DAMAGE 8      /* "Bond_Damage"        [nb] double, neighbor-list order */
#define PD_FIELD_COORDINATES 9      /* "Coordinates" x+u    [3n] double */
#define PD_FIELD_NUM_NEIGHBORS 10   /* "Number_Of_Neighbors" [n] double */
#define PD_FIELD_FORCE 11           /* "Force" = Force_Density x Volume (Compute_Force) [3n] double */
#define PD_FIELD_VOLUME 12          /* "Volume"             [n] double */
#define PD_FIELD_MODEL_COORDINATES 13 /* "Model_Coordinates" x [3n] double */

typedef struct pd_ctx pd_ctx;

typedef struct {
  int device;     /* CUDA device ordinal */
  int precision;  /* PD_FP64, PD_SPLIT_FP32 or PD_FP64_SLICED */
  int influence;  /* PD_INFLUENCE_* */
  int threads_per_point; /* lanes cooperating on one point's bond family: 0 = auto, else 4/8/16/32 */
} pd_config;

/* Rectangular_Plane bond filter (src/io/pdneigh/BondFilter.h:59-93 FinitePlane;
 * parameters as parsed in src/io/discretization/Peridigm_Discretization.cpp:158-175). */
typedef struct {
  double normal[3];
  double lower_left[3];
  double bottom_unit[3];
  double bottom_length;
  double side_length;
} pd_plane_filter;

/* Run statistics of pd_verlet_run / pd_qs_solve. */
typedef struct {
  int64_t steps;          /* explicit steps taken */
  int64_t bonds;          /* directed bonds in the family */
  int64_t broken_bonds;   /* bonds with damage 1 at the end */
  int64_t contact_pairs;  /* directed pairs in the last contact list */
  double device_ms;       /* device time of the step loop (CUDA events) */
  int64_t newton_iterations;
  int64_t cg_iterations;
  double final_residual;  /* relative FP64 residual of the last linear solve */
  int64_t preconditioner_fallbacks; /* learned-preconditioner solves finished by block Jacobi */
  int64_t coarse_builds;  /* coarse operators built by pd_qs_load_step (two-level and learned) */
} pd_stats;

/* ---- lifecycle ---------------------------------------------------------- */
/* Replaces the construction done by PeridigmNS::Peridigm (src/core/Peridigm.cpp:105-792). */
int pd_create(const pd_config* cfg, pd_ctx** out);
int pd_destroy(pd_ctx* ctx);
/* Message of the last failure on ctx (never NULL). */
const char* pd_last_error(const pd_ctx* ctx);
/* Library version string. */
const char* pd_version(void);

/* ---- discretization ----------------------------------------------------- */
/* Points: model coordinates x[3n], cell volumes vol[n] and an optional block
 * id per point (NULL = all block 0). Mirrors the "Model_Coordinates"/"Volume"
 * fields a discretization hands Peridigm (Peridigm.cpp:811-930). */
int pd_set_points(pd_ctx* ctx, int64_t n, const double* x, const double* vol, const int32_t* block);
/* Per-block horizon (Blocks/"Horizon", one constant per block). */
int pd_set_block_horizons(pd_ctx* ctx, int32_t n_blocks, const double* horizon);

/* Bond family by search on the device: j in H(i) iff j != i, FP64
 * dx*dx+dy*dy+dz*dz <= h_i*h_i and no plane filter cuts the bond.
 * Replaces NeighborhoodList::buildNeighborhoodList (src/io/pdneigh/NeighborhoodList.cxx:621-761)
 * with ZoltanSearchTree::FindPointsWithinRadius (src/io/Peridigm_ZoltanSearchTree.cpp:214-247)
 * and FinitePlaneFilter (src/io/pdneigh/BondFilter.cxx:123-150). */
int pd_build_bonds(pd_ctx* ctx, const pd_plane_filter* filters, int32_t n_filters);
/* Bond family from a Peridigm neighbor list of length len (accepted verbatim).
 * Families may be one-sided (j in H(i) without i in H(j), as blocks of different
 * horizons give): each bond's force then acts as the reference's scatter of
 * i's family adds it (elastic.cxx:121-130); pd_get_bonds, pd_num_bonds and the
 * per-bond fields keep the list as given. */
int pd_set_bonds(pd_ctx* ctx, const int32_t* neighborhood_list, int64_t len);
int pd_num_bonds(const pd_ctx* ctx, int64_t* nb);
/* Neighbor list in Peridigm format; *len receives the length (cap may be 0 to query). */
int pd_get_bonds(pd_ctx* ctx, int32_t* neighborhood_list, int64_t cap, int64_t* len);

/* ---- material / damage -------------------------------------------------- */
/* "Elastic" material (PeridigmNS::ElasticMaterial ctor, src/materials/Peridigm_ElasticMaterial.cpp:59-118):
 * bulk modulus, shear modulus, density of one block. */
int pd_material_lps(pd_ctx* ctx, int32_t block, double bulk_modulus, double shear_modulus, double density);
/* Per-point moduli (an extension for heterogeneous bodies; the owner's values
 * take the place of the block constants at src/materials/elastic.cxx:99,119). */
int pd_material_lps_field(pd_ctx* ctx, const double* bulk_modulus, const double* shear_modulus);
/* Elastic bond-based material of a block ("Elastic Bond Based",
 * PeridigmNS::ElasticBondBasedMaterial, src/materials/Peridigm_ElasticBondBasedMaterial.cpp:52-95;
 * force MATERIAL_EVALUATION::computeInternalForceElasticBondBased,
 * src/materials/elastic_bond_based.cxx:55-124): pair force
 * 0.5 (1 - d) s c per bond and end, c = 18K/(pi delta^4) in 3D, or
 * 12K/(pi height delta^3) with plane != 0 ("Plane Strain" / "Plane Stress",
 * height > 0). One bond pass per evaluation (no dilatation, no influence
 * function). All blocks of a context use one material model; the
 * quasi-static entry points support the LPS model only. */
#define PD_MATERIAL_LPS 0
#define PD_MATERIAL_BOND_BASED 1
int pd_material_bond_based(pd_ctx* ctx, int32_t block, double K, double rho, int32_t plane, double height);
/* Linear LPS material of a block ("Linear LPS Partial Volume" with partial
 * volumes and improved quadrature off, PeridigmNS::LinearLPSPVMaterial,
 * src/materials/Peridigm_LinearLPSPVMaterial.cpp:62-394): the LPS model
 * linearised about the reference configuration,
 * theta = 3/m sum omega (1-d) zeta.(u_j - u_i) V_j and per bond
 * (1-d) ((9K - 15mu) omega theta/(3m) zeta + 15mu omega/(m |zeta|^2) zeta zeta^T (u_j - u_i)).
 * FP64 contexts evaluate it in the class's operation order; split-FP32
 * contexts at 4 lanes per point (the default) evaluate it from the sliced bond
 * stream, with X in FP32 and the owner terms (9K - 15mu) theta/(3m) and 15mu/m
 * of the LPS state record. The quasi-static and implicit solves support the
 * LPS model only. */
#define PD_MATERIAL_LINEAR_LPS 2
int pd_material_linear_lps(pd_ctx* ctx, int32_t block, double K, double mu, double rho);
/* "Critical Stretch" damage (CriticalStretchDamageModel ctor, src/damage/Peridigm_CriticalStretchDamageModel.cpp:52-77)
 * for one block; s_c < 0 disables damage on that block. */
int pd_damage_critical_stretch(pd_ctx* ctx, int32_t block, double critical_stretch);
/* Per-point critical stretch of the bond's owner (extension). */
int pd_damage_critical_stretch_field(pd_ctx* ctx, const double* critical_stretch);

/* ElasticMaterial::initialize -> computeWeightedVolume
 * (Peridigm_ElasticMaterial.cpp:124-139, material_utilities.cxx:161-188,501-520).
 * m_out may be NULL. */
int pd_weighted_volume(pd_ctx* ctx, double* m_out);

/* ModelEvaluator::evalModel for one configuration (src/core/Peridigm_ModelEvaluator.cpp:57-131):
 * CriticalStretchDamageModel::computeDamage (Peridigm_CriticalStretchDamageModel.cpp:108-184),
 * then ElasticMaterial::computeForce (Peridigm_ElasticMaterial.cpp:141-172:
 * computeDilatation + computeInternalForceLinearElastic). y = current
 * coordinates [3n] (host). Damage is trial damage (NP1) on top of the
 * committed state (N); pd_update_state commits it. force_density_out [3n]
 * may be NULL. On the split path the coordinates go up in point chunks
 * beside the dilatation pass and the force density comes down in chunks
 * beside the force pass (page-locked host buffers let the copies run
 * asynchronously; pageable ones work but serialise them). */
int pd_compute_force(pd_ctx* ctx, const double* y, double* force_density_out);
/* Same with device pointers. */
int pd_compute_force_device(pd_ctx* ctx, const double* y_dev, double* force_density_dev);
/* DamageModel::computeDamage alone (Peridigm_DamageModel.hpp:107-112). */
int pd_compute_damage(pd_ctx* ctx, const double* y);
/* DataManager::updateState (Peridigm_DataManager.hpp:159): commit NP1 damage. */
int pd_update_state(pd_ctx* ctx);
/* Bond damage in neighbor-list order (doubles 0/1), in and out. */
int pd_set_bond_damage(pd_ctx* ctx, const double* bond_damage);

/* ---- contact -------------------------------------------------------------- */
/* "Short Range Force" contact: ShortRangeForceContactModel
 * (src/contact/Peridigm_ShortRangeForceContactModel.cpp:50-87) with the
 * ContactManager's "Search Radius" / "Search Frequency"
 * (src/core/Peridigm_ContactManager.cpp:79-84). The horizon of the spring
 * coefficient is each point's block horizon (Peridigm_ContactManager.cpp:241-249).
 * contact_radius <= 0 disables contact. Once set, pd_verlet_run searches at
 * setup and every search_frequency steps and adds the contact force. */
int pd_contact_short_range(pd_ctx* ctx, double search_radius, int32_t search_frequency, double contact_radius,
                           double spring_constant, double friction_coefficient);
/* ContactManager::contactSearch + ShortRangeForceContactModel::computeForce
 * (Peridigm_ContactManager.cpp:696-748, Peridigm_ShortRangeForceContactModel.cpp:98-261)
 * on host coordinates y[3n] and velocities v[3n]; fc_out[3n] receives the
 * contact force density. */
int pd_contact_force(pd_ctx* ctx, const double* y, const double* v, double* fc_out);

/* ---- explicit integration ----------------------------------------------- */
/* ComputeCriticalTimeStep (src/core/Peridigm_CriticalTimeStep.cpp:52-130), min over points. */
int pd_critical_time_step(pd_ctx* ctx, double* dt_out);
/* The same critical time step, computed with no device allocation. No
 * counterpart in the reference: it exists for callers that cannot allocate
 * device memory around the call. pd_critical_time_step allocates and frees a
 * small device buffer on each call; a host whose pool allocator has reserved
 * the device's memory sees that allocation fail, and the free synchronises the
 * whole device, stalling the host's other streams inside its time loop. Here
 * the block minima live in a static 512 KiB device array (65,536 doubles) in
 * the library, so:
 *  - the context must already be set up (bonds, material, and one
 *    pd_weighted_volume or evaluation done), else PD_ERR_STATE;
 *  - at most 65,536 blocks of 256 threads: 1,048,576 points at the default 16
 *    lanes per point; larger contexts get PD_ERR_ARG (use pd_critical_time_step);
 *  - nothing needs to start at zero: each call writes every partial it reads;
 *  - the array is shared by all contexts on a device, so calls that overlap on
 *    one device (from two threads) race and must be serialised by the caller;
 *  - the first call on each device resolves the array's address and may load
 *    the library's module there: make it before any stream capture begins;
 *  - the resolved address is kept for the life of the process: no
 *    cudaDeviceReset of that device may come between calls (a reset unloads
 *    the module the address belongs to).
 * The result is copied to the host double *dt_out after a stream synchronise. */
int pd_critical_time_step_static(pd_ctx* ctx, double* dt_out);
/* Initial displacement / velocity (DirichletBC "Initial Displacement"/"Initial Velocity",
 * src/core/Peridigm_BoundaryCondition.cpp:157-187). NULL leaves the field unchanged. */
int pd_set_state(pd_ctx* ctx, const double* u, const double* v);
/* Prescribed displacement u_c(t) = a*t + b on coordinate c of the listed points
 * (DirichletIncrementBC, Peridigm_BoundaryCondition.cpp:202-241: each step sets
 * v_c = (u_c(t) - u_c(t_prev)) / (t - t_prev)). */
int pd_add_prescribed_displacement(pd_ctx* ctx, int64_t n_points, const int64_t* points, int32_t coordinate,
                                   double a, double b);
/* Prescribed displacement u_c = f(x, y, z, t) on coordinate c of the listed
 * points, f given as the reference's "Value" string: the body its run-time
 * compiler runs with variables x, y, z (the point's model coordinates), t and
 * value, "value = " prepended when the string does not mention value
 * (Peridigm_BoundaryCondition.cpp:68-84, 217-220), e.g. "0.001*y*t/1.0e-8" or
 * "if (t <= 1) { value = -y*1.0e-6*t; } else { value = -y*1.0e-6; }".
 * Language: numbers, + - * / % ^ (power), comparisons, && || !, if/else,
 * assignments to new variables, and sin cos tan asin acos atan sinh cosh
 * tanh exp log log10 sqrt abs fabs floor ceil pow atan2 fmod min max. Each
 * explicit step evaluates f at the step's two times on the device (FP64) and
 * sets v_c = (f(t) - f(t_prev)) / (t - t_prev) as DirichletIncrementBC does
 * (:222-241); a zero increment takes f(t_prev) from the displacement field
 * (:137-142). PD_ERR_ARG with the message in pd_last_error on a syntax error
 * or an unknown name; PD_ERR_NONFINITE when a value is not finite. The
 * quasi-static solve evaluates them at each load step's two times (the same
 * increment rule); the implicit solve refuses contexts with such functions
 * (PD_ERR_UNSUPPORTED). */
int pd_add_prescribed_displacement_function(pd_ctx* ctx, int64_t n_points, const int64_t* points,
                                            int32_t coordinate, const char* function);
/* Evaluates such a function once on the host (no context, no device): for
 * checking a "Value" string. PD_ERR_ARG when it does not compile. */
int pd_expr_eval(const char* function, double x, double y, double z, double t, double* value);
int pd_clear_boundary_conditions(pd_ctx* ctx);
/* Velocity-Verlet loop of Peridigm::executeExplicit (src/core/Peridigm.cpp:1290-1593):
 * initial evaluation at t0, then nsteps steps of size dt. State stays on the
 * device; read it with pd_get_field. stats may be NULL. */
int pd_verlet_run(pd_ctx* ctx, double dt, double t0, int64_t nsteps, pd_stats* stats);
/* Stepping form of pd_verlet_run for hosts that act between steps, e.g. the
 * halo exchange of a domain decomposition (no counterpart in the reference,
 * whose step loop exchanges ghosts through Epetra imports inside
 * executeExplicit, Peridigm.cpp:1497-1546). pd_verlet_begin does the initial
 * evaluation at t0 and the first half of step 1; pd_verlet_step(k) completes k
 * steps and starts the next; pd_verlet_finish completes the last one and fills
 * stats (device_ms spans begin to finish, host time between calls included).
 * begin + step(n - 1) + finish gives the same state as pd_verlet_run(n). */
int pd_verlet_begin(pd_ctx* ctx, double dt, double t0);
int pd_verlet_step(pd_ctx* ctx, int64_t nsteps);
int pd_verlet_finish(pd_ctx* ctx, pd_stats* stats);
/* Ghost-state exchange between pd_verlet_begin and pd_verlet_finish (device
 * pointers on the context's device, ordered on its stream; both return after
 * the copy). pack: out[6k..6k+5] = (u, y) of point idx[k], the displacement
 * and current coordinates the next step's evaluation reads. unpack: makes
 * points idx[k] hold in[6k..6k+5] exactly as the packing context held them.
 * Indices outside [0, n) are skipped and reported as PD_ERR_ARG. */
int pd_pack_state_device(pd_ctx* ctx, int64_t n_idx, const int32_t* idx, double* out);
int pd_unpack_state_device(pd_ctx* ctx, int64_t n_idx, const int32_t* idx, const double* in);
/* Reads a field (PD_FIELD_*) into host memory in the caller's order. */
int pd_get_field(pd_ctx* ctx, int32_t field, double* out);

/* ---- compute classes ------------------------------------------------------ */
/* Block_Data (src/compute/Peridigm_Compute_Block_Data.cpp:121-210): the
 * minimum, maximum or sum (PD_CALC_*) of a per-point field (PD_FIELD_*,
 * scalar or vector) over the points of one block, into out[3] (scalars in
 * out[0]). As in the reference the maximum starts from DBL_MIN. Sums run in
 * a fixed order (bit-reproducible). */
#define PD_CALC_MINIMUM 0
#define PD_CALC_MAXIMUM 1
#define PD_CALC_SUM 2
int pd_block_data(pd_ctx* ctx, int32_t field, int32_t block, int32_t calculation, double* out);
/* Kinetic_Energy (src/compute/Peridigm_Compute_Kinetic_Energy.cpp:79-150):
 * global sum of 0.5 V rho |v|^2; per_point[n] (may be NULL) the local values. */
int pd_kinetic_energy(pd_ctx* ctx, double* global, double* per_point);
/* Linear_Momentum (src/compute/Peridigm_Compute_Linear_Momentum.cpp:110-150):
 * global sum of rho V v into global[3]; per_point[3n] (may be NULL). */
int pd_linear_momentum(pd_ctx* ctx, double* global, double* per_point);

/* ---- quasi-static ---------------------------------------------------------- */
#define PD_PRECOND_NONE 0         /* plain CG (the reference's default, usePreconditioner=false, Peridigm.cpp:2740) */
#define PD_PRECOND_BLOCK_JACOBI 1 /* inverse 3x3 diagonal blocks ("Block 3x3", Peridigm.cpp:1603-1646) */
#define PD_PRECOND_MPNN 2         /* learned message-passing correction on top of PD_PRECOND_TWO_LEVEL, or of block
                                   * Jacobi alone after pd_mpnn_coarse(ctx, -1) (no reference counterpart) */
#define PD_PRECOND_TWO_LEVEL 3    /* block Jacobi + exact Galerkin coarse correction on aggregate cells (no reference
                                   * counterpart): z = P_bj r + P0 (P0^T K P0)^-1 P0^T r, P0 = piecewise-constant
                                   * translations of the non-empty cells of a grid of side >= 2 * max horizon */

typedef struct {
  double newton_tolerance;      /* on ||r||_2 + 20 ||r||_inf (Peridigm.cpp:4316): > 0 absolute ("Absolute
                                 * Tolerance"), < 0 relative to the value at the load step's start with
                                 * only the prescribed increments applied (before any predictor) */
  double cg_relative_tolerance; /* ||r_cg|| / ||r_cg,0|| of each linear solve (Belos "Relative Tolerance", :2556) */
  int32_t max_newton_iterations;/* "Maximum Solver Iterations" */
  int32_t max_cg_iterations;
  int32_t preconditioner;       /* PD_PRECOND_* */
  int32_t use_predictor;        /* start the free dofs from the previous step's increment (Peridigm.cpp:2764-2769) */
  double coarse_cell;           /* PD_PRECOND_TWO_LEVEL: aggregate cell side; the side used is max(coarse_cell,
                                 * 2 * max horizon), grown 1.25x at a time until the coarse space has at most
                                 * 6144 dofs (0: the default) */
} pd_qs_options;

/* One quasi-static load step t_prev -> t_cur of Peridigm::executeQuasiStatic
 * (src/core/Peridigm.cpp:2651-3043): prescribed-displacement increments on
 * their dofs, then Newton on r = V (f_int + f_ext) (computeQuasiStaticResidual,
 * :4176-4317) with CG on the matrix-free tangent -dr/du. Updates the
 * displacement (u += du) and velocity (v = du / (t_cur - t_prev)). Bond damage
 * is held fixed. stats (may be NULL) accumulates steps, Newton and CG
 * iterations and device time. */
int pd_qs_load_step(pd_ctx* ctx, double t_prev, double t_cur, const pd_qs_options* options, pd_stats* stats);

/* ---- implicit dynamics ------------------------------------------------------ */
typedef struct {
  double beta;                  /* Newmark "Beta" (Peridigm.cpp:3647, default 0.25) */
  double gamma;                 /* Newmark "Gamma" (:3648, default 0.50) */
  double absolute_tolerance;    /* on ||R||_2, R = beta dt^2 (rho a - f) with the prescribed rows zeroed
                                 * ("Absolute Tolerance", :3644, default 1e-6) */
  double cg_relative_tolerance; /* of each linear solve (Belos "Convergence Tolerance" 1e-10, :3668) */
  int32_t max_newton_iterations;/* "Maximum Solver Iterations" (:3645, default 10); as in the reference the
                                 * Newton loop runs while the iteration count is <= this (:3815) */
  int32_t max_cg_iterations;
  int32_t preconditioner;       /* PD_PRECOND_NONE (the reference: plain CG) or PD_PRECOND_BLOCK_JACOBI on the
                                 * 3x3 blocks of rho I + beta dt^2 K */
} pd_implicit_options;

/* nsteps implicit Newmark-beta steps of dt from t0, Peridigm::executeImplicit
 * (src/core/Peridigm.cpp:3620-4016): per step the predictor u2 = u + dt v +
 * dt^2 (1/2 - beta) a, v2 = v + dt (1 - gamma) a, then Newton on
 * R = beta dt^2 (rho a - f) with the operator rho I + beta dt^2 K
 * (computeImplicitJacobian :4319-4338, K = -d(V f)/du applied matrix-free)
 * and CG; after each correction a = (u - u2)/(beta dt^2), v = v2 + dt gamma a.
 * Prescribed dofs start at u = a t0 + b with velocity a and follow the
 * predictor; their rows are left out of the solve. Bond damage is held fixed;
 * LPS material only; the solve is FP64 whatever the context's precision.
 * Updates displacement, velocity, acceleration and force density. stats (may
 * be NULL) accumulates steps, Newton and CG iterations and device time. */
int pd_implicit_run(pd_ctx* ctx, double dt, double t0, int64_t nsteps, const pd_implicit_options* options,
                    pd_stats* stats);

/* Material::computeJacobian (src/materials/Peridigm_Material.hpp:174-180,
 * FULL_MATRIX) in matrix-free form: kw = K w with K = -d(V f)/du at
 * displacement u (V-weighted, Scale(-1): Peridigm_ElasticMaterial.cpp:366-370,
 * Peridigm.cpp:2800); rows and columns of prescribed dofs are identity
 * (applyKinematicBC_InsertZerosAndSetDiagonal, Peridigm.cpp:2799). Host arrays [3n]. */
int pd_jacobian_apply(pd_ctx* ctx, const double* u, const double* w, double* kw);
/* BLOCK_DIAGONAL Jacobian (SerialMatrix::addBlockDiagonalValues,
 * src/core/Peridigm_SerialMatrix.cpp:110-170): the 3x3 diagonal blocks of K
 * at displacement u, row-major, 9 per point. */
int pd_jacobian_block_diagonal(pd_ctx* ctx, const double* u, double* blocks);

/* ---- learned preconditioner (no counterpart in the reference) -------------
 * A learned middle level added to the two-level preconditioner:
 *   z = P_bj r + P0 Ac^-1 P0^T r + Q S G^T G S Q^T r
 * Q: piecewise-constant prolongation from patches (the non-empty cells of a
 * grid of side `patch`, about two lattice spacings); S: per-patch scales from
 * the block-Jacobi blocks; G: a linear message-passing network on the patch
 * graph (3 layers, hidden 64, BF16 weights, FP32 activations and
 * accumulation). M is symmetric positive definite, so PD_PRECOND_MPNN solves
 * run preconditioned CG, with the flexible (Polak-Ribiere) beta
 * z_new.(r_new - r_old) / (z_old.r_old): the standard beta for a fixed SPD M,
 * and tolerant of the FP32 rounding of the network's product. A stall, or a
 * true FP64 residual above the tolerance, falls back to 3x3 block Jacobi
 * from the current iterate (the FP64 residual decides). */
int pd_mpnn_init(pd_ctx* ctx, uint64_t seed, double patch);
/* While every > 0, block-Jacobi and two-level CG solves of pd_qs_load_step
 * store training pairs (r_k, x* - x_k) from every every-th iterate
 * (K (x* - x_k) = r_k). */
int pd_mpnn_collect(pd_ctx* ctx, int32_t every);
int pd_mpnn_num_pairs(pd_ctx* ctx, int64_t* count);
/* Adam on the stored pairs, loss L = 1 - (r.z)^2 / ((z.K z)(e.r)) (the
 * energy-norm error left by one optimally scaled preconditioned step) with K
 * the tangent at the context's current displacement, rescaled to each pair's
 * modulus. */
int pd_mpnn_train(pd_ctx* ctx, int32_t epochs, double learning_rate, int32_t batch, double* loss);
int pd_mpnn_num_params(int64_t* count);
int pd_mpnn_get_weights(pd_ctx* ctx, float* weights);
int pd_mpnn_set_weights(pd_ctx* ctx, const float* weights);
/* Loss and parameter gradient for one pair (a = P_bj r, r = K e, e; 9n
 * floats) with the tangent at the current displacement, for gradient checks.
 * With the coarse level on, z includes P0 Ac^-1 P0^T r of the current
 * displacement. */
int pd_mpnn_loss_grad(pd_ctx* ctx, const float* pair, double* loss, float* grad);
/* The middle level alone, z = Q S G^T G S Q^T r (host arrays [3n], prescribed
 * dofs of z left zero), with S from the block-Jacobi blocks at the current
 * displacement: the product each PD_PRECOND_MPNN CG iteration adds, for
 * parity checks of the inference kernels. It runs as one cooperative launch
 * whose phases meet at grid barriers with bounded waits; PD_ERR_TIMEOUT if
 * one ran out (here, or at the end of a PD_PRECOND_MPNN CG solve). */
int pd_mpnn_apply(pd_ctx* ctx, const double* r, double* z);
/* Coarse level under the network (training, loss and PD_PRECOND_MPNN solves):
 * cell >= 0 puts the network on top of the two-level preconditioner with
 * aggregate cells of side max(cell, 2 * max horizon) (the default after
 * pd_mpnn_init, cell 0); cell < 0 puts it on block Jacobi alone. */
int pd_mpnn_coarse(pd_ctx* ctx, double cell);
/* Coarse dofs per aggregate of the two-level preconditioner (no counterpart
 * in the reference): 3 (the default) = translations; 6 = translations and the
 * three rotations about the aggregate's center, orthonormalised per aggregate
 * (Gram-matrix Cholesky; near-dependent modes dropped), the Galerkin matrix
 * assembled from 162 matrix-free tangent products per build (aggregates
 * colored by cell coordinates mod 3). At most 6144 coarse dofs either way:
 * with 6 modes the cells grow to hold at most 1024 aggregates. Applies to
 * every coarse level of the context (two-level, and the learned
 * preconditioner's base). */
int pd_qs_coarse_modes(pd_ctx* ctx, int32_t modes);
/* The coarse space of PD_PRECOND_TWO_LEVEL at displacement u (host [3n]):
 * n_coarse receives 3 (6 with pd_qs_coarse_modes(ctx, 6)) x the number of
 * aggregates; aggregate[n] the aggregate of each point, A the assembled
 * P0^T K P0 and A_inv its inverse (row-major n_coarse^2, coarse dof 3I + c =
 * component c of aggregate I; with 6 modes, 6I + k = orthonormal mode k). Call first with
 * aggregate, A and A_inv NULL to get n_coarse; on the second call *n_coarse
 * must hold at least that. */
int pd_qs_coarse_operator(pd_ctx* ctx, const double* u, double cell, int64_t* n_coarse, int32_t* aggregate,
                          double* A, double* A_inv);

/* ---- instrumentation ----------------------------------------------------- */
/* Named stopwatches around the hot calls are the reference's Timer
 * (src/core/Peridigm_Timer.hpp:77-86); here CUDA events bracket every launch
 * of the two bond passes while enabled. ms_out[0]/[1] receive the summed
 * device time of the dilatation (+damage) pass and of the force (+Verlet)
 * pass since the last reset; launches_out the number of evaluations. */
int pd_set_kernel_timing(pd_ctx* ctx, int enable);
int pd_get_kernel_timing(pd_ctx* ctx, double* ms_out, int64_t* launches_out);

#ifdef __cplusplus
}
#endif
#endif /* PD_B200_H */
