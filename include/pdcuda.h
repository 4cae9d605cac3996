/*
 * pdcuda.h -- C ABI of libpdcuda, the B200 (sm_100a) explicit-dynamics engine behind
 * Peridynamics.jl's Body / material! / velocity_bc! / VelocityVerlet / Job / submit surface.
 *
 * The library replaces the per-chunk calls that the reference's threads data handler makes
 * on one BodyChunk (src/core/threads_body_data_handler.jl, src/discretization/body_chunk.jl)
 * with one device-resident body. Every entry point below names the reference function it
 * replaces (file:line inside Peridynamics.jl).
 *
 * Conventions
 *  - Plain C types only. Arrays are host pointers, valid for the duration of the call; the
 *    library copies them into device memory it owns. Point vectors use the reference's
 *    3 x N column-major layout (x, y, z of point 0, then point 1, ...). Point tensors are
 *    9 x N column-major 3x3 matrices. Indices are 0-based.
 *  - Every function returns a pd_status. PD_OK is 0. On error, pd_last_error() returns a
 *    message for the calling thread.
 *  - Calls on one handle must be serialised by the caller (one host thread per handle).
 *    Handles are independent.
 */
#ifndef PDCUDA_H
#define PDCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t pd_status;
#define PD_OK 0
#define PD_ERR_ARG 1      /* invalid argument (reference: ArgumentError) */
#define PD_ERR_CUDA 2     /* CUDA runtime error */
#define PD_ERR_NAN 3      /* NaN in the internal force density (reference: NaNError) */
#define PD_ERR_TIMEOUT 4  /* a bounded device wait gave up */
#define PD_ERR_OOM 5      /* device allocation failed */
#define PD_ERR_UNSUPPORTED 6
#define PD_ERR_NOCONV 7   /* Newton iterations exhausted (reference: ErrorException "did not converge") */

/* material families (src/physics/bond_based.jl, ordinary_state_based.jl, correspondence.jl) */
#define PD_MAT_BB 0
#define PD_MAT_OSB 1
#define PD_MAT_CMAT 2

/* correspondence constitutive models (src/physics/constitutive_models.jl) */
#define PD_CM_SVK 0
#define PD_CM_NEOHOOKE 1
#define PD_CM_NEOHOOKE_PENALTY 2

/* CMat zero-energy mode stabilisation (src/discretization/zem_stabilization.jl) */
#define PD_ZEM_SILLING 0  /* ZEMSilling(Cs), zem_stabilization.jl:16-21 */
#define PD_ZEM_WAN 1      /* ZEMWan(), zem_stabilization.jl:30-42 (stiffness C : K^-1 per point) */

/* influence functions (src/discretization/kernels.jl:10-52) */
#define PD_KERNEL_CONST_ONE 0
#define PD_KERNEL_LINEAR 1
#define PD_KERNEL_CUBIC_BSPLINE 2

/* arithmetic of the bond loops */
#define PD_PREC_FP64 0        /* FP64 everywhere; positions kept incrementally as the reference does */
#define PD_PREC_FP32_KAHAN 1  /* FP32 bond math on xi + (u_j - u_i), compensated sums, FP64 integration */

/* storage fields (src/time_solvers/velocity_verlet.jl:342-352, bond_system.jl:408-412,
 * correspondence.jl:173-181) */
#define PD_FIELD_POSITION 0       /* double[3n] */
#define PD_FIELD_DISPLACEMENT 1   /* double[3n] */
#define PD_FIELD_VELOCITY 2       /* double[3n] */
#define PD_FIELD_VELOCITY_HALF 3  /* double[3n] */
#define PD_FIELD_ACCELERATION 4   /* double[3n] */
#define PD_FIELD_B_INT 5          /* double[3n] */
#define PD_FIELD_B_EXT 6          /* double[3n] */
#define PD_FIELD_DAMAGE 7         /* double[n] */
#define PD_FIELD_N_ACTIVE_BONDS 8 /* int64[n] */
#define PD_FIELD_BOND_ACTIVE 9    /* uint8[n_bonds] */
#define PD_FIELD_DEFGRAD 10       /* double[9n] (CMaterial) */
#define PD_FIELD_CAUCHY_STRESS 11 /* double[9n] (CMaterial) */
#define PD_FIELD_N_NEIGHBORS 12   /* int64[n]: bonds per point (BondSystem.n_neighbors, bond_system.jl:48) */

/* boundary-condition targets (velocity_bc! writes velocity_half, forcedensity_bc! b_ext:
 * src/physics/boundary_conditions.jl:422-435, 559-575) */
#define PD_BC_VELOCITY_HALF 0
#define PD_BC_B_EXT 1
/* boundary-condition value kinds */
#define PD_BC_KIND_TIME 0        /* f(t): one value per step, tabulated by the host */
#define PD_BC_KIND_POINT_TIME 1  /* f(p, t): one value per point of the set per step */
#define PD_BC_KIND_DATA 2        /* DataBC: one constant value per point of the set */

/* StandardPointParameters (src/core/parameters.jl:107-125); CPointParameters
 * (src/physics/correspondence.jl:148-161) without the Hooke tensor. */
typedef struct {
    double delta, rho, E, nu, G, K, lambda, mu, Gc, epsilon_c, bc;
} pd_point_params;

/* One body chunk with its bond system (src/discretization/bond_system.jl:44-65). */
typedef struct {
    int64_t n_points;
    const double *position;        /* [3n] reference positions */
    const double *volume;          /* [n] */
    int64_t n_bonds;
    const int64_t *bond_offsets;   /* [n+1]: bonds of point i are [off[i], off[i+1]) */
    const int32_t *neighbors;      /* [n_bonds], 0-based */
    const double *bond_length;     /* [n_bonds] or NULL (then |X_j - X_i|) */
    const uint8_t *fail_permit;    /* [n_bonds] or NULL (then all 1) */
    const uint16_t *param_id;      /* [n] or NULL (then all 0) */
    int32_t n_params;
    const pd_point_params *params; /* [n_params] */
    int32_t material;              /* PD_MAT_* */
    int32_t kernel;                /* PD_KERNEL_* (OSB, CMat) */
    int32_t cmodel;                /* PD_CM_* (CMat) */
    int32_t precision;             /* PD_PREC_* */
    int32_t multi_params;          /* 1: ParameterHandler semantics of the reference
                                      (bond-averaged parameters, bond_based.jl:163-180,
                                      ordinary_state_based.jl:151-174) */
    double zem_cs;                 /* ZEMSilling Cs (zem_stabilization.jl:16-21), default 0.5 */
    double maxdmg;                 /* CMaterial maxdmg (correspondence.jl:123-128), default 0.85 */
    int32_t device;                /* CUDA device ordinal */
    int32_t zem;                   /* PD_ZEM_* (CMat); 0 (ZEMSilling with zem_cs) when zeroed */
} pd_body_desc;

/* One boundary condition on one point set and one dimension. */
typedef struct {
    int32_t field;        /* PD_BC_VELOCITY_HALF / PD_BC_B_EXT */
    int32_t dim;          /* 0, 1, 2 */
    int32_t kind;         /* PD_BC_KIND_* */
    int32_t n_points;
    const int32_t *points;/* [n_points] */
    const double *data;   /* PD_BC_KIND_DATA: [n_points] values, else NULL */
} pd_bc_desc;

typedef struct pd_handle pd_handle;

/* Message of the last failed call on this thread (empty if none). */
const char *pd_last_error(void);

/* Library version, e.g. "0.1.0". */
const char *pd_version(void);

/* Neighbour search: replaces find_bonds / find_bonds! / filter_bonds! and the
 * duplicate-point check (src/discretization/bond_system.jl:96-165). Runs on the device.
 * Bond i->j exists for j != i with |X_j - X_i|^2 <= delta_i^2; bonds of a point are ordered
 * by ascending j. fail_permit of a bond is fp_point[i] & fp_point[j]. n_filters filter-mode
 * pre-cracks (precrack!(...; update_dmg=false), predefined_cracks.jl:106-112) are given as
 * point masks filter_a/filter_b of n_filters x n bytes. Call first with capacity 0 to get
 * *n_bonds, then with arrays of that capacity. */
pd_status pd_find_bonds(int64_t n, const double *position, const double *delta,
                        const uint8_t *fp_point, int32_t n_filters, const uint8_t *filter_a,
                        const uint8_t *filter_b, int64_t capacity, int64_t *bond_offsets,
                        int32_t *neighbors, double *bond_length, uint8_t *fail_permit,
                        int64_t *n_bonds, int32_t device);

/* Creates the device body: replaces BodyChunk construction with its storage
 * (src/discretization/body_chunk.jl:41-52, src/core/storages.jl) for one chunk holding all
 * points. All fields start as the reference initialises them (zeros, all bonds active,
 * n_active_bonds = n_neighbors). */
pd_status pd_create(const pd_body_desc *desc, pd_handle **out);

/* pd_create with the bonds found on the device by the neighbour search of pd_find_bonds
 * (desc->bond_offsets, neighbors, bond_length and fail_permit are ignored): the horizon of a
 * point is the delta of its parameter set, fp_point (n bytes, may be NULL = all 1) is the
 * failure permission per point (failure_permit!, fracture.jl:38-42) and the n_filters
 * filter-mode pre-cracks are point masks as in pd_find_bonds. search_position (3n, may be
 * NULL = desc->position) are the coordinates the search runs on: several independent bodies
 * are kept apart there while the body stores their own coordinates. */
pd_status pd_create_search(const pd_body_desc *desc, const double *search_position,
                           const uint8_t *fp_point, int32_t n_filters, const uint8_t *filter_a,
                           const uint8_t *filter_b, pd_handle **out);

/* Frees all device memory of the handle. */
pd_status pd_destroy(pd_handle *h);

/* Overwrites point fields (any pointer may be NULL = keep): replaces the initial-condition
 * and pre-crack setup of a chunk (apply_initial_conditions!, initial_conditions.jl:86-94;
 * break_bonds! + calc_damage!, bond_system.jl:249-267, 338-343). bond_active is one byte
 * per bond; n_active_bonds is recomputed from it. position NULL keeps the current one. */
pd_status pd_set_state(pd_handle *h, const double *position, const double *displacement,
                       const double *velocity, const double *velocity_half,
                       const double *acceleration, const double *b_ext,
                       const uint8_t *bond_active);

/* Damage-mode pre-crack: replaces break_bonds! + calc_damage! of apply_precracks!
 * (bond_system.jl:249-267, predefined_cracks.jl:31-60). Bonds joining a point of set a
 * with a point of set b become inactive. set_a / set_b: n bytes, nonzero = member. */
pd_status pd_break_bonds(pd_handle *h, const uint8_t *set_a, const uint8_t *set_b);

/* Initial damage of synthetic workloads (no counterpart in the reference, which has no API
 * for random initial damage): each unordered pair {i, j} is broken with probability
 * `fraction`, decided by a hash of (min(i,j), max(i,j), seed), so both directions agree. */
pd_status pd_break_random_pairs(pd_handle *h, double fraction, uint64_t seed);

/* Bonds that may fail and whose current stretch (l - L) / L, evaluated in FP64, lies within
 * tol of the owner's critical stretch: the decisions of calc_failure! (bond_system.jl:309-327)
 * that a different summation order can flip. Reported beside broken-bond comparisons. */
pd_status pd_count_near_critical(pd_handle *h, double tol, int64_t *count);

/* pd_break_random_pairs hashing point_ids[i] (n int64, host) instead of the row numbers: a
 * partition passes the body's point numbers of its rows and breaks the same pairs as the
 * undivided body. */
pd_status pd_break_random_pairs_ids(pd_handle *h, double fraction, uint64_t seed,
                                    const int64_t *point_ids);

/* Copies one storage field to host memory of `bytes` bytes (export_results,
 * threads_body_data_handler.jl:197-212). */
pd_status pd_get_field(pd_handle *h, int32_t field, void *out, size_t bytes);

/* Installs the boundary conditions of the chunk (ConditionHandler,
 * src/discretization/condition_handler.jl:1-36). Replaces any previous set. */
pd_status pd_set_bcs(pd_handle *h, int32_t n_bcs, const pd_bc_desc *bcs);

/* Values of the time-dependent boundary conditions for steps first_step ..
 * first_step + n_steps - 1: the host evaluates each f(t) (apply_bc!,
 * boundary_conditions.jl:37-51, 91-108) at t = step * dt. `values` holds, step after step,
 * one value per PD_BC_KIND_TIME condition and n_points values per PD_BC_KIND_POINT_TIME
 * condition, in the order of pd_set_bcs. NaN / Inf values leave the field unchanged. */
pd_status pd_set_bc_values(pd_handle *h, int64_t first_step, int64_t n_steps,
                           const double *values, int64_t n_values);

/* CFL time step: replaces calc_stable_timestep / calc_timestep_point
 * (velocity_verlet.jl:132-163, bond_system.jl:269-277). dt_per_param (may be NULL) receives
 * the minimum per parameter set times the safety factor (one body per set in an ensemble). */
pd_status pd_stable_timestep(pd_handle *h, double safety_factor, double *dt,
                             double *dt_per_param);

/* Integration step per parameter set (ensemble of bodies with their own CFL steps).
 * pd_run_vv with dt <= 0 uses these. */
pd_status pd_set_param_timesteps(pd_handle *h, const double *dt_per_param);

/* One force evaluation at the current positions: replaces calc_force_density!(chunk, t, dt)
 * (bond_system.jl:279-297) with calc_failure!, calc_damage! and force_density_point! for
 * every point, followed by check_for_nans (nans.jl:10-18). Used by initialize!
 * (core/data_handler.jl:1-4) and the Newton-Krylov matrix-free products. */
pd_status pd_force(pd_handle *h, double t, double dt);

/* n_steps Velocity Verlet steps first_step .. first_step + n_steps - 1 at t = step * dt:
 * replaces solve! / verlet_timestep! (velocity_verlet.jl:165-237: update_vel_half!,
 * apply_boundary_conditions!, update_disp_and_pos!, calc_force_density!,
 * update_acc_and_vel!). On NaN in the force density it stops with PD_ERR_NAN and leaves the
 * state as the reference does when it throws NaNError; pd_nan_step reports the step. */
pd_status pd_run_vv(pd_handle *h, int64_t first_step, int64_t n_steps, double dt);

/* Step at which the last PD_ERR_NAN was raised (NaNError.step). */
pd_status pd_nan_step(pd_handle *h, int64_t *step);

/* pd_run_vv with CUDA events on the handle's stream around every kernel (no graph):
 * elapsed milliseconds of the whole run, of the first force kernel (BB: the force kernel;
 * OSB / CMat: phase A), of the second force kernel (OSB / CMat phase B) and of the
 * integration kernels, summed over the steps. Same effect on the state as pd_run_vv. When
 * ms_phase_a, ms_phase_b and ms_integrate are all NULL, the steps are issued as pd_run_vv
 * issues them (CUDA-graph blocks when pd_set_graph is on) and only ms_total is measured,
 * between two events on the handle's stream. */
pd_status pd_run_vv_timed(pd_handle *h, int64_t first_step, int64_t n_steps, double dt,
                          double *ms_total, double *ms_phase_a, double *ms_phase_b,
                          double *ms_integrate);

/* Groups of bodies advanced together. No counterpart in the reference, which runs a study's
 * jobs one after the other (Study / submit!, src/core/study.jl:193-283); here the size classes
 * of an ensemble, each body with its own mapping (pd_autotune / pd_set_mapping), advance in one
 * CUDA graph: the launches of every body on its own stream, forked from and joined into the
 * stream of handles[0]. The bodies share one device and have distinct streams; the group keeps
 * the handle pointers (destroy the group first). */
typedef struct pd_group pd_group;
pd_status pd_group_create(pd_handle *const *handles, int32_t n, pd_group **out);
/* pd_run_vv for every body of the group (same steps, dt as pd_run_vv: <= 0 takes each
 * parameter set's step from pd_set_param_timesteps), in CUDA graphs of steps_per_graph steps
 * (0: eager launches); ms_total (may be NULL): device time of the run on handles[0]'s stream.
 * Returns after the steps completed; PD_ERR_NAN etc. as pd_run_vv, the first failing body's. */
pd_status pd_group_run_vv(pd_group *g, int64_t first_step, int64_t n_steps, double dt,
                          int32_t steps_per_graph, double *ms_total);
pd_status pd_group_destroy(pd_group *g);

/* Chooses the point-to-lane mapping (points per thread / warp) and block size of the force
 * kernels by timing each candidate on this body. Leaves the state unchanged. */
pd_status pd_autotune(pd_handle *h, int32_t *group_out, int32_t *block_out);

/* Forces a mapping: group lanes per point in {1, 2, 4, 8, 16, 32}, or 0 for the FP64
 * serial-order mapping (one lane per point summing in the reference's order: bit-identical
 * to a serial CPU evaluation); block size 64, 128 or 256. */
pd_status pd_set_mapping(pd_handle *h, int32_t group, int32_t block);

/* How the FP32 force kernels read the bond stream: 0 = direct loads; 1, 2, 3 = chunks of
 * the sliced bond arrays staged in shared memory by TMA bulk copies (4 rows x 3 stages,
 * 4 rows x 4 stages, 8 rows x 3 stages per warp; one lane per point, BB or OSB); 4 = direct
 * loads two rows at a time, all their neighbour gathers in flight together (BB, OSB; results
 * identical to 0); 5 = BB, OSB and CMat with the x and y components of every bond vector and
 * 3x3 row in packed FP32 pairs, the bond states selecting instead of branching, and the next
 * row pair's bond stream loaded (as streaming loads) while the current pair is computed (one
 * lane per point and one parameter set; phase B needs symmetric bond states and, for CMat,
 * ZEMSilling; BB and OSB need no surface correction; where they do not apply the phase runs
 * as 4, CMat as 0; same FP32 form, roundings differ in the order of a few operations).
 * pd_autotune times all that apply. */
pd_status pd_set_pipeline(pd_handle *h, int32_t pipe);

/* The current mapping (group 0 = serial order), block size and bond-stream variant. */
pd_status pd_get_mapping(pd_handle *h, int32_t *group, int32_t *block, int32_t *pipe);

/* Enables CUDA-graph capture of blocks of `steps_per_graph` steps (0 disables). */
pd_status pd_set_graph(pd_handle *h, int32_t steps_per_graph);

/* Sizes: points, bonds, and 1 if the fast symmetric-pair bond mode is active. */
pd_status pd_info(pd_handle *h, int64_t *n_points, int64_t *n_bonds, int32_t *symmetric);

/* Number of kernel launches issued by the handle since creation. */
pd_status pd_launch_count(pd_handle *h, int64_t *count);

/* The cudaStream_t of the handle, as an opaque pointer. */
pd_status pd_stream(pd_handle *h, void **stream);

/* ---------------------------------------------------------------------------------------
 * Partitioned bodies: one partition per GPU with halo exchange between the stages of a
 * step (the reference's MPI data handler, src/core/mpi_body_data_handler.jl: chop_body_mpi
 * :102-109, exchange_loc_to_halo! :239-318, calc_force_density! :400-409; decomposition
 * PointDecomposition / distribute_equally, src/discretization/decomposition.jl:32-63).
 * --------------------------------------------------------------------------------------- */

/* A partition of a body: desc holds its rows (owned points and halo points, in the body's
 * point order) and owned[i] != 0 marks the owned rows. The search gives every owned row all
 * its bonds and every halo row only its bonds to owned rows; halo rows take no part in the
 * stable time step and leave the killed-point decision of CMaterial to their owner. Other
 * arguments as pd_create_search. */
pd_status pd_create_partition(const pd_body_desc *desc, const double *search_position,
                              const uint8_t *fp_point, int32_t n_filters, const uint8_t *filter_a,
                              const uint8_t *filter_b, const uint8_t *owned, pd_handle **out);

/* Issues all further work of the handle on `stream` (a cudaStream_t of the same device; NULL
 * returns to the handle's own stream), so that a communication library's transfers on that
 * stream order with the kernels. Waits for the work issued so far. */
pd_status pd_set_stream(pd_handle *h, void *stream);

/* Velocity Verlet in stages (verlet_timestep!, velocity_verlet.jl:181-237, with the force
 * density split at its halo exchanges): pd_vv_begin(first_step, n_steps, dt) opens a run
 * (boundary values from pd_set_bc_values as for pd_run_vv); for kstep = 0 .. n_steps - 1 the
 * caller issues stage 0 (half kick, conditions, drift), stage 1 (the first force kernel; BB:
 * the whole force) and stage 2 (the second force kernel of OSB / CMat; nothing for BB);
 * pd_vv_end issues the closing half kick, waits and reports PD_ERR_NAN as pd_run_vv. The
 * sequence has the effect of pd_run_vv(first_step, n_steps, dt). Asynchronous except
 * pd_vv_begin / pd_vv_end. */
pd_status pd_vv_begin(pd_handle *h, int64_t first_step, int64_t n_steps, double dt);
/* pd_force split like the stages: phase 1 issues the first force kernel, phase 2 the second
 * one, then waits and reports PD_ERR_NAN (initialize! of a partition, with the kind-1
 * exchange between the phases). */
pd_status pd_force_phase(pd_handle *h, int32_t phase, double t, double dt);
pd_status pd_vv_stage(pd_handle *h, int32_t stage, int64_t kstep);
pd_status pd_vv_end(pd_handle *h);

/* Halo data (exchange_loc_to_halo!): kind 0 = the point state the force kernels gather from
 * neighbours, exchanged after stage 0; kind 1 = the per-point state of the first force kernel
 * that the second one gathers (OSB, CMat; nothing for BB), exchanged after stage 1; kind 2 =
 * the surface-correction multiplication factors, exchanged once between pd_esc_init(h, 1)
 * and pd_esc_init(h, 2) (exchange_loc_to_halo!(get_mfactor, ...), :82, :92). Every row
 * is pd_halo_row_bytes bytes. pd_halo_pack gathers rows d_rows[0 .. n_rows) (int32, device)
 * into d_buf (device); pd_halo_unpack writes d_buf into rows d_rows[0 .. n_rows) and finishes
 * them (FP32: the split displacement; CMat with directed bond states: the bonds of killed
 * rows). Both are asynchronous on the handle's stream; a row index outside the body is
 * reported by the next pd_vv_end. */
pd_status pd_halo_row_bytes(pd_handle *h, int32_t kind, int64_t *bytes);
pd_status pd_halo_pack(pd_handle *h, int32_t kind, const int32_t *d_rows, int64_t n_rows,
                       void *d_buf);
pd_status pd_halo_unpack(pd_handle *h, int32_t kind, const int32_t *d_rows, int64_t n_rows,
                         const void *d_buf);

/* ---------------------------------------------------------------------------------------
 * EnergySurfaceCorrection (src/discretization/bond_system_corrections.jl) of BBMaterial and
 * OSBMaterial: BBMaterial{EnergySurfaceCorrection}() / OSBMaterial{EnergySurfaceCorrection}().
 * --------------------------------------------------------------------------------------- */

/* initialize! of the correction (:78-94), after the pre-cracks: what = 0 computes the
 * multiplication factors of every point from the current bond states (calc_mfactor!, :96-124)
 * and the factor of every bond from them (calc_scfactor!, :156-204); from then on every force
 * evaluation multiplies each bond by its factor (BB: bond_based.jl:156, 175; OSB: weighted
 * volume, dilatation and force, ordinary_state_based.jl:143-198). what = 1 computes only the
 * multiplication factors and what = 2 only the bond factors (a partition exchanges the halo
 * rows' multiplication factors between the two). FP32 OSB uses the one-row bond stream (pipe
 * 0) with the correction. PD_ERR_UNSUPPORTED for CMaterial. */
pd_status pd_esc_init(pd_handle *h, int32_t what);

/* The multiplication factors (3n doubles, {x, y, z} per point, may be NULL) and the bond
 * factors (n_bonds doubles in CSR order, may be NULL), host arrays. */
pd_status pd_esc_get(pd_handle *h, double *mfactor, double *scfactor);

/* ---------------------------------------------------------------------------------------
 * Dynamic relaxation (src/time_solvers/dynamic_relaxation.jl): adaptive-damping explicit
 * steps towards a static state on the same force kernels as Velocity Verlet.
 * --------------------------------------------------------------------------------------- */

/* init_density_matrix! (dynamic_relaxation.jl:109-164): the fictitious density
 * Lambda_i = damping_factor / 4 dt^2 n_i 5 pi delta^2 bc of every point, v_half_old and
 * b_int_old cleared. dt is the relaxation step (DynamicRelaxation stepsize). */
pd_status pd_dr_init(pd_handle *h, double dt, double damping_factor);

/* relaxation_timestep! (:191-211, 269-370) for steps first_step .. first_step + n_steps - 1:
 * conditions and drift, force density, damping coefficient (steps > 1), velocity update.
 * Boundary values come from pd_set_bc_values as for pd_run_vv. PD_ERR_NAN as pd_run_vv. With
 * the serial mapping (pd_set_mapping group 0) the damping sums follow the reference's order. */
pd_status pd_run_dr(pd_handle *h, int64_t first_step, int64_t n_steps);

/* pd_run_dr with CUDA events around every phase: elapsed milliseconds of the whole run, of the
 * conditions and drift kernels, of the force kernels and of the damping and velocity-update
 * kernels, summed over the steps. Same effect on the state as pd_run_dr. */
pd_status pd_run_dr_timed(pd_handle *h, int64_t first_step, int64_t n_steps, double *ms_total,
                          double *ms_drift, double *ms_force, double *ms_relax);

/* Lambda of every point (n doubles, host). */
pd_status pd_dr_density_matrix(pd_handle *h, double *out);

/* ---------------------------------------------------------------------------------------
 * Quasi-static Jacobian-free Newton-Krylov solve (src/time_solvers/newton_krylov.jl).
 * Needs a PD_PREC_FP64 handle without fracture (validate_chunk_for_newton_krylov!,
 * newton_krylov.jl:219-253). Position-dependent conditions f(p) are evaluated by the host at
 * the reference positions and uploaded once; every load increment scales them by
 * beta = n / n_steps on the device (apply_incr_boundary_conditions!,
 * boundary_conditions.jl:148-163, 229-236).
 * --------------------------------------------------------------------------------------- */

/* Frechet step of the Jacobian-vector product */
#define PD_NK_CENTRAL 0  /* eps = s cbrt(eps_mach)(|u|+1)/|v|, Jv = (F(u+eps v) - F(u-eps v))/(2 eps)
                            (compute_perturbation / jacobian_vector_product!, newton_krylov.jl:504-567) */
#define PD_NK_FORWARD 1  /* eps = s sqrt(eps_mach)|u|/|v| (|u| = 0: 1), Jv = (F(u+eps v) - F(u))/eps */

/* preconditioner of the Krylov solve (right preconditioning, flexible GMRES) */
#define PD_PC_NONE 0          /* plain restarted GMRES, as the reference (newton_krylov.jl:448-450) */
#define PD_PC_BLOCK_JACOBI 1  /* z_i = P_i v_i, P_i = inverse of the 3x3 diagonal block J_ii (BB) */
#define PD_PC_BLOCK_POLY 2    /* z = P (2v - K0 P v), K0 the small-strain bond stiffness (BB) */
#define PD_PC_LEARNED_POLY 3  /* z = B (2v - K0 B v), B_i = P_i (I + D_i), D from pd_nk_set_corrections */
#define PD_PC_LEARNED 4       /* z_i = B_i v_i */

typedef struct pd_nk_condition {
  int32_t field;           /* 0: displacement (constrains the dof), 1: b_ext */
  int32_t dim;             /* 0, 1, 2 */
  int64_t n_points;
  const int32_t *points;   /* 0-based point indices */
  const double *values;    /* f(p) at the reference position of every point (full load) */
} pd_nk_condition;

typedef struct pd_nk_params {
  int32_t maxiter;              /* Newton iterations per increment (NewtonKrylov maxiter) */
  double tol;                   /* Newton tolerance on ||r||, r = (b_int + b_ext) V */
  int32_t tol_relative;         /* 0: ||r|| < tol (reference); 1: ||r|| <= tol ||r_first|| */
  double perturbation_scale;    /* s */
  int32_t frechet;              /* PD_NK_* */
  int32_t gmres_maxiter;        /* Arnoldi steps per linear solve */
  double gmres_reltol, gmres_abstol;
  int32_t gmres_restart;        /* Krylov basis size between restarts */
  int32_t precond;              /* PD_PC_* */
} pd_nk_params;

typedef struct pd_nk_stats {
  int32_t newton_iters;     /* residual evaluations of the increment */
  int32_t converged;
  int64_t gmres_iters;      /* Arnoldi steps (Jacobian-vector products inside the bases) */
  int64_t matvecs;          /* all Jacobian-vector products, restart residuals included */
  int64_t force_evals;      /* force-density evaluations of the increment */
  int64_t precond_applies;
  double residual_first;    /* ||r|| at the first Newton iteration of the increment */
  double residual;          /* ||r|| at the last Newton iteration */
} pd_nk_stats;

/* Conditions of the solve (pos_single_dim_bcs of the body, condition_handler.jl:5-36):
 * replaces earlier ones. Displacement conditions define the constrained dofs. */
pd_status pd_nk_set_conditions(pd_handle *h, int32_t n, const pd_nk_condition *conds);

/* One load increment, newton_krylov_step! (newton_krylov.jl:298-332): apply the conditions at
 * beta, then Newton iterations of force, residual and a (F)GMRES solve of J du = -r.
 * `step` is the increment number used in NaN reports. PD_ERR_NOCONV when maxiter Newton
 * iterations did not reach the tolerance (stats are filled either way). */
pd_status pd_nk_step(pd_handle *h, int64_t step, double beta, const pd_nk_params *p,
                     pd_nk_stats *stats);

/* Learned corrections D (9 floats per point, 3x3 column-major) of PD_PC_LEARNED*; NULL
 * clears them. Host pointer. No counterpart in the reference. */
pd_status pd_nk_set_corrections(pd_handle *h, const float *D);

/* Operators at the current state, for tests: op 0 out = J v (the Frechet product of p),
 * 1 out = K0 v, 2 out = M v (the preconditioner p->precond), 3 out = residual r (v unused).
 * Host vectors of 3n doubles. */
pd_status pd_nk_apply(pd_handle *h, int32_t op, const pd_nk_params *p, const double *v,
                      double *out);

/* Record the unit residual direction of every (re)start of the Krylov solves, FP32, up to
 * `capacity` vectors (0 stops and frees); pd_nk_recorded returns how many are held. The
 * recorded vectors are the training data of the learned preconditioner. */
pd_status pd_nk_record(pd_handle *h, int64_t capacity);
pd_status pd_nk_recorded(pd_handle *h, int64_t *n);
/* Recorded direction k as 3n floats (host). */
pd_status pd_nk_recorded_vector(pd_handle *h, int64_t k, float *out);

/* ---------------------------------------------------------------------------------------
 * Learned block preconditioner of the Newton-Krylov solve. No counterpart in the reference
 * (its Newton systems are solved by plain GMRES): a two-layer message-passing network over
 * the bond graph (16 point features, hidden width 64, BF16 tensor-core layers with FP32
 * accumulation) predicts per-point corrections D_i of the block-Jacobi blocks,
 * B_i = P_i (I + D_i), used by PD_PC_LEARNED(_POLY). Bond-based bodies; the body's
 * conditions (pd_nk_set_conditions) must be set before pd_mpnn_infer / pd_mpnn_loss_grad.
 * --------------------------------------------------------------------------------------- */
typedef struct pd_mpnn pd_mpnn;
#define PD_MPNN_N_PARAMS 18185  /* W0[64x16] b0[64] W1[64x128] b1 W2[64x128] b2 Wo[9x64] bo[9] */

pd_status pd_mpnn_create(int32_t device, pd_mpnn **out);
pd_status pd_mpnn_destroy(pd_mpnn *net);
/* FP32 parameter vector (row-major weights, layout above); setting resets the optimiser. */
pd_status pd_mpnn_set_params(pd_mpnn *net, const float *theta);
pd_status pd_mpnn_get_params(pd_mpnn *net, float *theta);
/* Runs the network on the body and installs its corrections D (as pd_nk_set_corrections).
 * Optional host outputs: features [n x 16], D [n x 9]. */
pd_status pd_mpnn_infer(pd_mpnn *net, pd_handle *h, float *features, float *D);
/* Training loss L = sum_s w_s ||(I - alpha_s K0 B)^2 r_s||^2 / S over recorded residual
 * directions (rec_ids into pd_nk_record's store; alpha = w = 1) and host samples
 * [n_host x 3n] (FP32; alpha = host_alpha, w = host_weight); the gradient is added to the
 * network's accumulator (copied to grad [PD_MPNN_N_PARAMS] when not NULL). */
pd_status pd_mpnn_loss_grad(pd_mpnn *net, pd_handle *h, int32_t n_rec, const int64_t *rec_ids,
                            int32_t n_host, const float *host_samples, double host_alpha,
                            double host_weight, double *loss, float *grad);
/* Spectral training loss L = -mean_rec rho(r) + weight mean_host max(rho(q) - tau, 0)^2 with
 * rho(v) = v . K0 B v: recorded residual directions (the slow end) are pulled up, host samples
 * (top eigenvectors of K0 B) are held below tau. Gradient handling as pd_mpnn_loss_grad. */
pd_status pd_mpnn_spectral_grad(pd_mpnn *net, pd_handle *h, int32_t n_rec, const int64_t *rec_ids,
                                int32_t n_host, const float *host_samples, double tau,
                                double weight, double *loss, float *grad);
pd_status pd_mpnn_zero_grad(pd_mpnn *net);
/* One Adam step (beta 0.9 / 0.999) with the accumulated gradient, which is then cleared. */
pd_status pd_mpnn_adam(pd_mpnn *net, float lr);

/* Ordinary state-based force evaluation that allocates no device memory. No counterpart in
 * the reference: it exists for callers that must not let the library allocate GPU memory --
 * a host that owns every device buffer through its own pool, a time loop that must not stall
 * on the allocator, or memory carved out of a fixed arena (the reference itself asserts that
 * its force loop allocates nothing, test/perf/perf.jl).
 * Every array is a device pointer owned by the caller, in the reference's CSR bond order
 * (every bond list sorted by neighbour, one parameter set): ref_position, position [3n],
 * volume [n], bond_offsets [n+1], neighbors, bond_length, fail_permit [n_bonds];
 * bond_active [n_bonds] is updated by the failure test; b_int [3n] and n_active [n] are
 * written. Bond states need not agree in the two directions of a pair: the term of
 * neighbour j on point i uses j's own bond j -> i (its state and length), found by a binary
 * search of j's sorted list, as the reference's scatter does; a neighbour without a bond to
 * i adds nothing. Kernels run on `stream` (NULL: the default stream); the call does not
 * wait. A CUDA error left pending by earlier work of the calling thread is reported
 * (PD_ERR_CUDA) before anything is launched and stays pending.
 * Limit: n <= 262144 points. The per-point coefficients live in a static device array of
 * that size (8 MiB, held by every GPU that loads the library until the process exits);
 * larger bodies are rejected with PD_ERR_ARG. All calls share that array: calls whose
 * kernels may overlap on the GPU (other streams, other host threads) race. Every entry a
 * call reads is written earlier in the same call, so nothing has to start at zero. The
 * first call in each CUDA context (normally a device's primary context) looks up the
 * array's device address with that context current and keeps it for the context; make that
 * first call before any stream capture. A context destroyed and created again at the same
 * handle (cudaDeviceReset) is not told apart from the old one. Errors: pd_static_last_error(). */
pd_status pd_osb_force_static(int64_t n, const double *ref_position, const double *position,
                              const double *volume, const int64_t *bond_offsets,
                              const int32_t *neighbors, const double *bond_length,
                              const uint8_t *fail_permit, uint8_t *bond_active,
                              const pd_point_params *params, int32_t kernel, double *b_int,
                              int64_t *n_active, void *stream);

/* Message of the last failed pd_osb_force_static call on this thread. */
const char *pd_static_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* PDCUDA_H */
