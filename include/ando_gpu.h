/*
 * ando_gpu.h -- C ABI of the B200 (sm_100a) implementation of AndoSim's
 * implicit cloth/shell step.
 *
 * Plain C types only: no C++, no CUDA and no torch types cross this boundary.
 * Every entry point returns an ando_status (0 = ANDO_OK); nothing throws.
 *
 * The reference binds its C++ core to Python with pybind11
 * (src/py/bindings.cpp:27-633). The pybind11 module shipped here
 * (andosim_b200/csrc/bindings.cpp, module name `ando_barrier_core`) keeps that
 * Python surface and calls the entry points below; any other host (ctypes,
 * cffi, a C++ add-on) can bind them directly. Each declaration names the
 * reference interface it replaces.
 */
#ifndef ANDO_GPU_H
#define ANDO_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ANDO_ABI_VERSION 1

#if defined(__GNUC__)
#define ANDO_API __attribute__((visibility("default")))
#else
#define ANDO_API
#endif

typedef enum {
  ANDO_OK = 0,
  ANDO_ERR_INVALID = 1,      /* bad argument (null pointer, size, index out of range) */
  ANDO_ERR_CUDA = 2,         /* a CUDA runtime call failed; see ando_last_error() */
  ANDO_ERR_STATE = 3,        /* call out of order (e.g. step before mesh/state upload) */
  ANDO_ERR_TIMEOUT = 4,      /* a device-side bounded wait gave up (grid barrier) */
  ANDO_ERR_NO_DEVICE = 5,    /* no CUDA device / wrong architecture */
  ANDO_ERR_CAPACITY = 6      /* a caller-supplied buffer is too small */
} ando_status;

/* Step semantics. REFERENCE reproduces the reference step exactly, including
 * its documented quirks (elastic gradient on the rest mesh, repelling pins,
 * literal BVH broad phase, frozen contact gaps, sampled CCD). CORRECTED runs
 * the step the reference intends: elastic gradient at the current positions,
 * attracting pins, contact gaps re-evaluated per Newton iteration, conservative
 * time of impact, the block-scaled PCG, each step restarting from the last
 * step's end (ando_state_set_start) with v = (x - x_start) / dt. */
typedef enum { ANDO_SEMANTICS_REFERENCE = 0, ANDO_SEMANTICS_CORRECTED = 1 } ando_semantics;

/* Preconditioner of the PCG inner solve. */
typedef enum { ANDO_PRECOND_BLOCK_JACOBI = 0, ANDO_PRECOND_LEARNED = 1 } ando_precond;

/* ContactType (collision.h:70-75). */
typedef enum {
  ANDO_CONTACT_POINT_TRIANGLE = 0,
  ANDO_CONTACT_EDGE_EDGE = 1,
  ANDO_CONTACT_WALL = 2,
  ANDO_CONTACT_RIGID_POINT_TRIANGLE = 3
} ando_contact_type;

/* Material (types.h:51-57). */
typedef struct {
  double youngs_modulus, poisson_ratio, density, thickness, bending_stiffness;
} ando_material;

/* SimParams (types.h:60-100), every field, plus the GPU-only knobs at the end. */
typedef struct {
  double dt, beta_max;
  int32_t min_newton_steps, max_newton_steps, friction_min_newton_steps;
  double pcg_tol;
  int32_t pcg_max_iters;
  double contact_gap_max, wall_gap;
  int32_t enable_ccd;
  double contact_normal_epsilon, barrier_tolerance;
  int32_t enable_friction;
  double friction_mu, friction_epsilon, friction_tangent_threshold;
  double velocity_damping, contact_restitution;
  int32_t enable_strain_limiting;
  double strain_limit, strain_tau, strain_epsilon, strain_svd_epsilon;
  double hessian_epsilon, min_gap;
  int32_t semantics; /* ando_semantics */
  int32_t precond;   /* ando_precond */
  /* Learned preconditioner: Newton iterations between evaluations of the
   * network (<= 1: every iteration). In between, S is rebuilt from the
   * current scaled system with the last coefficients (still SPD). */
  int32_t precond_refresh;
  /* CORRECTED membrane Hessian in the Newton system: ANDO_MEMBRANE_FIXED_ROTATION
   * (0, the constant 2k (G G^T) (x) I3) or ANDO_MEMBRANE_PROJECTED (1, the exact
   * as-rigid-as-possible Hessian projected to positive semidefinite per face,
   * rebuilt every Newton iteration: face rotations, such as a clamped sheet
   * swinging down, are not resisted). */
  int32_t membrane_hessian;
} ando_params;

typedef enum { ANDO_MEMBRANE_FIXED_ROTATION = 0, ANDO_MEMBRANE_PROJECTED = 1 } ando_membrane_hessian;

/* PinConstraint (constraints.h:12-17). */
typedef struct { int32_t vertex; int32_t active; double target[3]; } ando_pin;

/* WallConstraint (constraints.h:22-28); normal already normalised by add_wall. */
typedef struct { double normal[3]; double offset; double gap; int32_t active; int32_t pad_; } ando_wall;

/* RigidBody (rigid_body.h), copied in and out by value around a step exactly
 * as bindings.cpp:476-491 does. Mesh arrays are read-only; the dynamic fields
 * are updated in place by ando_step. */
typedef struct {
  int32_t num_vertices, num_triangles;
  const double* local_vertices;  /* (num_vertices, 3), body frame */
  const int32_t* triangles;      /* (num_triangles, 3) */
  double mass;
  double inertia_body_inv[9];    /* row-major */
  double position[3];
  double rotation[9];            /* row-major */
  double linear_velocity[3];
  double angular_velocity[3];
} ando_rigid;

/* ContactPair (collision.h:78-103). */
typedef struct {
  int32_t type, idx0, idx1, idx2, idx3, rigid_body_index, vertex_count, pad_;
  double gap;
  double normal[3], witness_p[3], witness_q[3], barycentric[3];
  double weights[4];
} ando_contact;

/* Per-step counters (no reference counterpart: the reference only logs to stderr). */
typedef struct {
  int32_t newton_iters;        /* Newton iterations that solved a system */
  int32_t pcg_iters;           /* PCG iterations summed over the step */
  int32_t pcg_max_per_newton;
  int32_t pcg_not_converged;
  int32_t line_search_fail;    /* inner steps whose line search returned alpha < 1e-6 */
  int32_t contacts;            /* contacts detected at the start of the step */
  int32_t strain_active;       /* strain-limit constraints active at the last gradient */
  int32_t status;              /* ando_status of the step */
  int32_t precond_fallbacks;   /* learned-preconditioner solves redone with block-Jacobi */
  int32_t graph_launched;      /* 1 when the whole step ran as one CUDA graph launch */
  double beta;
  double last_alpha;
  double device_ms;            /* device time of the step (CUDA events) */
  int32_t substeps;            /* CORRECTED: sub-steps taken for a fast drive or fast motion (1 = none) */
  int32_t pad_;
} ando_step_stats;

typedef struct ando_ctx_s* ando_ctx;

/* Phases of a step timed by the profiler (no reference counterpart; the
 * reference only times whole steps from Python, demo_framework.py:144-170). */
typedef enum {
  ANDO_PHASE_SETUP = 0,        /* prediction, contact detection, per-step contact constants */
  ANDO_PHASE_STRAIN = 1,       /* per-face strain-limit SVD and barrier terms */
  ANDO_PHASE_GRADIENT = 2,     /* per-vertex Newton gradient and diagonal terms */
  ANDO_PHASE_ASSEMBLE = 3,     /* BSR Hessian assembly + block-Jacobi inverse */
  ANDO_PHASE_PCG = 4,          /* persistent PCG solve */
  ANDO_PHASE_LINE_SEARCH = 5,  /* feasibility masks and position update */
  ANDO_PHASE_FINISH = 6,       /* velocity update, restitution, rigid coupling, gravity */
  ANDO_PHASE_PRECOND = 7,      /* learned preconditioner: features, network, S */
  ANDO_PHASE_COUNT = 8
} ando_phase;

typedef struct {
  int64_t launches;                        /* this library's kernel launches since the last reset */
  int64_t phase_launches[ANDO_PHASE_COUNT];
  double phase_ms[ANDO_PHASE_COUNT];       /* summed CUDA-event time of each phase (profiling on) */
  int64_t pcg_iterations;                  /* PCG iterations inside the profiled PCG launches */
  int64_t newton_iterations;               /* Newton iterations that assembled and solved */
  int64_t pcg_learned_iterations;          /* of pcg_iterations: iterations with the learned preconditioner */
  int64_t pcg_extra_block_iterations;      /* sum over PCG iterations of the contact blocks outside the mesh pattern */
} ando_profile;

/* Library identity. */
ANDO_API int32_t ando_abi_version(void);
ANDO_API const char* ando_status_string(int32_t status);
/* Message of the last CUDA/argument error on this thread (never NULL). */
ANDO_API const char* ando_last_error(void);

/* Create / destroy a device context holding one scene (mesh topology, rest
 * data and simulation state) on `device`. No reference counterpart: the
 * reference keeps everything in host objects. */
ANDO_API int32_t ando_ctx_create(int32_t device, ando_ctx* out);
ANDO_API void ando_ctx_destroy(ando_ctx ctx);

/* Upload mesh topology, rest data and the current mesh vertices.
 * Replaces Mesh::initialize / Mesh::compute_rest_state (mesh.h:137-142,
 * mesh.cpp:8-75): the caller passes the rest areas and Dm_inv it computed
 * (row-major 2x2 per face); the device builds the block-sparse pattern,
 * scatter maps and the constant elastic Hessian blocks from them. */
ANDO_API int32_t ando_mesh_upload(ando_ctx ctx, const double* vertices, int32_t num_vertices,
                         const int32_t* triangles, int32_t num_triangles,
                         const double* rest_areas, const double* dm_inv,
                         const ando_material* material);

/* Replace only the mesh vertices (Mesh::set_positions, mesh.cpp:121-123, and
 * the `vertices` property setter, bindings.cpp:185-191). */
ANDO_API int32_t ando_mesh_set_vertices(ando_ctx ctx, const double* vertices, int32_t num_vertices);

/* Upload the simulation state (State::initialize, state.cpp:6-16; any of the
 * pointers may be NULL to keep the device copy). */
ANDO_API int32_t ando_state_upload(ando_ctx ctx, const double* positions, const double* velocities,
                          const double* positions_prev, const double* masses, int32_t num_vertices);

/* CORRECTED semantics: the positions the next step starts from. A step
 * starts where the previous one ended, or at the positions of the last
 * ando_state_upload; State.apply_gravity's position update is not a start
 * (it is an explicit, collision-unchecked move whose velocity change the
 * implicit predictor x_hat = x + dt v already carries). No reference
 * counterpart: the reference starts from the moved positions. */
ANDO_API int32_t ando_state_set_start(ando_ctx ctx, const double* positions, int32_t num_vertices);
ANDO_API int32_t ando_state_get_start(ando_ctx ctx, double* positions, int32_t num_vertices);

/* Download positions and/or velocities (State.get_positions/get_velocities,
 * bindings.cpp:248-267). Either pointer may be NULL. */
ANDO_API int32_t ando_state_download(ando_ctx ctx, double* positions, double* velocities, int32_t num_vertices);

/* v += g*dt; x += v*dt for every vertex (State.apply_gravity, bindings.cpp:284-300). */
ANDO_API int32_t ando_apply_gravity(ando_ctx ctx, const double gravity[3], double dt);

/* One implicit step (Integrator::step, integrator.h:33-35, integrator.cpp:70-150).
 * `rigids` may be NULL when num_rigids == 0; their dynamic fields are updated.
 * `stats` may be NULL. */
ANDO_API int32_t ando_step(ando_ctx ctx, const ando_params* params,
                  const ando_pin* pins, int32_t num_pins,
                  const ando_wall* walls, int32_t num_walls,
                  ando_rigid* rigids, int32_t num_rigids,
                  ando_step_stats* stats);

/* Contact detection at the current state (Integrator::compute_contacts,
 * integrator.h:44-46, integrator.cpp:238-244). Writes up to `capacity`
 * contacts and the total count to *num_out; returns ANDO_ERR_CAPACITY when
 * the total exceeds `capacity`. */
ANDO_API int32_t ando_compute_contacts(ando_ctx ctx, const ando_rigid* rigids, int32_t num_rigids,
                              ando_contact* out, int32_t capacity, int32_t* num_out);

/* The contact set the CORRECTED step uses at the current positions: every
 * vertex-triangle and edge-edge pair of the mesh closer than gap_max (LBVH
 * broad phase, FP64 narrow phase, unsigned distances), then vertices against
 * rigid triangles. Integrator.compute_contacts(..., semantics="corrected")
 * and CollisionValidator read it; the reference's own query
 * (integrator.cpp:238-244) finds no self contact (its BVH drops every leaf of
 * 2-4 primitives, collision.cpp:65-159). Same output conventions as
 * ando_compute_contacts. */
ANDO_API int32_t ando_compute_contacts_corrected(ando_ctx ctx, double gap_max, const ando_rigid* rigids, int32_t num_rigids,
                                                 ando_contact* out, int32_t capacity, int32_t* num_out);

/* CollisionMetrics (collision_validator.h) reduced on the device over the
 * context's current contact list (the last ando_compute_contacts*, or the
 * last Newton iteration of a step) and its velocities: counts, extremes and
 * sums; the averages and flags follow from them (avg_gap = sum_gap /
 * num_total_contacts, has_major_penetration = num_major_penetrations > 0, and
 * so on). Gaps are compared in single precision like the reference's Real.
 * With no contacts every field is zero. */
typedef struct {
  int32_t num_total_contacts, num_point_triangle, num_edge_edge, num_wall;
  int32_t num_penetrations;        /* gap < 0 */
  int32_t num_major_penetrations;  /* penetration > 1 mm */
  int32_t num_tunneling;           /* penetration > 0.1 gap_max */
  int32_t num_ccd_contacts;        /* ccd_enabled and gap < 0.5 gap_max */
  int32_t num_relative_velocities; /* point-triangle, edge-edge and wall contacts */
  double min_gap, max_gap, sum_gap, max_penetration, sum_penetration;
  double max_relative_velocity, sum_relative_velocity;
} ando_metrics;

/* Replaces CollisionMetrics::compute_from_contacts and
 * CollisionValidator::compute_metrics / compute_relative_velocities
 * (collision_validator.cpp:7-111,133-157,179-221) for a contact list that is
 * still on the device: no contact or state download. */
ANDO_API int32_t ando_collision_metrics(ando_ctx ctx, double gap_max, int32_t ccd_enabled, ando_metrics* out);

/* Moments of the device state: 1/2 sum m |v|^2, sum m v, sum x cross m v and
 * max |v|. Replaces EnergyTracker::compute_kinetic_energy /
 * compute_linear_momentum / compute_angular_momentum / compute_max_velocity
 * (energy_tracker.cpp:7-42) and AdaptiveTimestep::compute_max_velocity
 * (adaptive_timestep.cpp:132-149) without a state download. */
typedef struct {
  double kinetic_energy, linear_momentum[3], angular_momentum[3], max_speed;
} ando_moments;
ANDO_API int32_t ando_state_moments(ando_ctx ctx, ando_moments* out);

/* Discrete intersection count at the current positions: mesh edges whose
 * segment passes through a triangle they share no vertex with (exact FP64
 * test over an LBVH of the triangles). No reference counterpart: the
 * reference's CollisionValidator only reads a contact list and cannot see a
 * crossing that no contact reports; this is the direct check that a
 * trajectory stays intersection-free. */
ANDO_API int32_t ando_edge_triangle_crossings(ando_ctx ctx, int64_t* crossings);

/* Block-sparse (3x3 BSR) system of the most recent Newton iteration, for
 * inspection and for the preconditioner-training dump. Pass NULL pointers to
 * query sizes. rowptr: num_vertices+1; cols: nnzb; vals: 9*nnzb (row-major
 * blocks); rhs: 3*num_vertices. Extra contact blocks are not included. */
ANDO_API int32_t ando_last_system(ando_ctx ctx, int32_t* num_vertices, int32_t* nnzb,
                         int32_t* rowptr, int32_t* cols, float* vals, float* rhs, float* solution);

/* Evaluate, without stepping, the system the first Newton iteration of a step
 * would solve at the current state: prediction x_hat = x + dt*v, contact
 * detection, Newton gradient (Integrator::compute_gradient,
 * integrator.cpp:246-396) and Hessian (assemble_system_matrix, :398-544).
 * Read the results with ando_last_gradient / ando_last_system. This is the
 * solver's system dump for preconditioner training and for parity checks. */
ANDO_API int32_t ando_eval_system(ando_ctx ctx, const ando_params* params,
                                  const ando_pin* pins, int32_t num_pins,
                                  const ando_wall* walls, int32_t num_walls,
                                  const ando_rigid* rigids, int32_t num_rigids);

/* The per-step contact blocks between vertices that share no mesh face
 * (vertex-triangle and edge-edge barrier terms), which live outside the
 * static pattern of ando_last_system: block k sits at (rows[k], cols[k]).
 * Pass NULL pointers to query the count. */
ANDO_API int32_t ando_last_contact_blocks(ando_ctx ctx, int32_t* count, int32_t* rows, int32_t* cols, float* vals);

/* Broad-phase candidate pairs at the current positions from the device LBVH
 * (replaces Collision::build_*_bvh / broad_phase_*, collision.cpp:65-276, with
 * the query the reference intends; its own BVH drops every leaf holding 2..4
 * primitives). kind 0: (vertex, triangle) pairs, the vertex not a corner of
 * the triangle; kind 1: (edge, edge) pairs with e1 < e2 and no shared vertex,
 * edges numbered in Mesh::compute_edges' first-seen order. Boxes are FP32 with
 * the reference's inclusive overlap test and +-1e-4 point box, each inflated
 * by `pad`. Pairs (2 ints each) come sorted by (first, second); with too small
 * a `capacity` the call returns ANDO_ERR_CAPACITY and the total in *count. */
ANDO_API int32_t ando_broad_phase(ando_ctx ctx, int32_t kind, double pad, int32_t* pairs, int32_t capacity, int32_t* count);

/* Start (enable != 0) or stop per-phase CUDA-event timing; resets the counters.
 * Kernel launches are counted whether or not timing is on. */
ANDO_API int32_t ando_profile_enable(ando_ctx ctx, int32_t enable);
ANDO_API int32_t ando_profile_read(ando_ctx ctx, ando_profile* out);

/* Many scenes in one call: item i runs ando_step(ctx, params, pins, walls,
 * rigids, stats) and stores its status. The contexts (all distinct) step
 * concurrently from up to `threads` host threads (0: one per item, at most
 * 16), each on its own CUDA stream, so small scenes share the GPU. Every
 * scene's result is the one its own ando_step call gives. Returns ANDO_OK
 * when every item did, else the first failing item's status. Replaces the
 * caller's loop over scenes (the reference steps one scene per call,
 * integrator.h:33-35). */
typedef struct {
  ando_ctx ctx;
  const ando_params* params;
  const ando_pin* pins; int32_t num_pins;
  const ando_wall* walls; int32_t num_walls;
  ando_rigid* rigids; int32_t num_rigids;
  ando_step_stats* stats;                 /* may be null */
  int32_t status;                         /* out */
} ando_batch_item;
ANDO_API int32_t ando_step_batch(ando_batch_item* items, int32_t count, int32_t threads);

/* Launch shape of the scaled PCG (CORRECTED semantics) for the current mesh,
 * per preconditioner (learned = 0: block Jacobi, 1: learned). The candidates
 * (threads per CTA, CTAs, column slots loaded ahead) all give the same result
 * bits. By default (index -1) the first solve of a mesh times every candidate
 * and keeps the fastest; index >= 0 fixes candidate `index`. No reference
 * counterpart (the reference solves on the CPU). */
ANDO_API int32_t ando_ctx_select_pcg_shape(ando_ctx ctx, int32_t learned, int32_t index);
/* Number of candidates for the current mesh and the shape in use
 * (shape[0..2] = threads per CTA, CTAs, slots ahead; zeros before the first
 * solve of the mesh). `tune_ms` (may be null): device time spent timing. */
ANDO_API int32_t ando_ctx_pcg_shape(ando_ctx ctx, int32_t learned, int32_t* count, int32_t* shape, double* tune_ms);

/* Capacity, in candidate pairs, of the context's broad-phase candidate
 * buffers (contact and time-of-impact passes). They grow on demand (a larger
 * buffer and the pass redone, with the same result), so this only sets where
 * they start: a caller short of device memory can start small. A mesh upload
 * resets them to their default size (about 4 per vertex + 8 per edge). No
 * reference counterpart. */
ANDO_API int32_t ando_ctx_set_pair_capacity(ando_ctx ctx, int32_t pairs);

/* Nodes above the refit's cut (more than 1,024 leaves) that one CTA finishes
 * in shared memory, 0..4096 (-1: 4096, the default). A hierarchy with more
 * top nodes is refit through global acquire/release arrival counters instead;
 * both give the same boxes. Lowering it exercises that path on small meshes.
 * No reference counterpart. */
ANDO_API int32_t ando_ctx_set_refit_top_capacity(ando_ctx ctx, int32_t nodes);

/* Threads per block of the CORRECTED block-scaled assembly (candidates 128,
 * 256, 512; one thread per vertex or block slot, so every candidate gives the
 * same bits). Index -1 (default): the first assembly of a mesh times every
 * candidate and keeps the fastest; 0..2 fixes one. ando_ctx_assembly_tpb
 * returns the number of candidates and the block size in use (0 before the
 * first assembly of the mesh). No reference counterpart. */
ANDO_API int32_t ando_ctx_select_assembly_tpb(ando_ctx ctx, int32_t index);
ANDO_API int32_t ando_ctx_assembly_tpb(ando_ctx ctx, int32_t* count, int32_t* tpb);

/* CORRECTED steps assemble the block-scaled system the PCG solves and, by
 * default, not the unscaled block values: ando_last_system then has no values
 * to return for a CORRECTED step and fails with ANDO_ERR_STATE. keep != 0 makes
 * every CORRECTED Newton iteration also write them (36 bytes per block), so
 * ando_last_system returns the last system solved. ando_eval_system always
 * writes them. No reference counterpart. */
ANDO_API int32_t ando_ctx_keep_system(ando_ctx ctx, int32_t keep);

/* The CUDA stream (cudaStream_t) every kernel of this context runs on, for
 * callers that time or order work around the library's. */
ANDO_API int32_t ando_ctx_stream(ando_ctx ctx, void** stream);

/* Newton gradient (FP64, 3*num_vertices) of the most recent Newton iteration. */
ANDO_API int32_t ando_last_gradient(ando_ctx ctx, double* gradient, int32_t num_vertices);

/* Largest system ando_pcg_solve_noalloc accepts (3 * num_rows must fit int32). */
#define ANDO_NOALLOC_MAX_ROWS 715827882

/* Block-Jacobi PCG on a caller-owned 3x3-block BSR system that allocates no
 * device memory. No reference counterpart: the reference's PCGSolver::solve
 * (pcg_solver.cpp:8-146) allocates its vectors on every call. It is for
 * callers that cannot allocate at solve time: a host that hands out all device
 * memory from its own fixed arena, or one that cannot take the device-wide
 * synchronisation of cudaFree between frames. The iteration is the one
 * ando_step runs (x0 = 0, stop when |r|_inf < tol * |b|_inf, FP64 dots).
 *
 * Device pointers: rowptr (num_rows+1), cols (sorted per row), vals (9 floats
 * per block, row-major), rhs (3*num_rows), x (3*num_rows, overwritten) and
 * work (>= 24*num_rows floats, any contents; smaller work buffers are rejected
 * with ANDO_ERR_CAPACITY, as are num_rows > ANDO_NOALLOC_MAX_ROWS). `stream` is a
 * cudaStream_t of `device` (NULL = legacy default stream). Reduction partials
 * and grid-barrier words live in a 16 KiB static device array per device
 * (partials for up to 640 CTAs; the grid is capped there); the call zeroes its
 * control words itself, so nothing has to start at zero.
 *
 * The first call on a device looks up that array's device address and the
 * kernel's grid size (which may load the module): make it before any stream
 * capture. Calls on one device share the scratch, so overlapping calls (other
 * streams or threads without ordering) race; serialise them. With all three
 * outputs NULL the call is asynchronous on `stream` and reports launch errors
 * only: a grid-barrier timeout, a not-SPD stop or reaching max_iters is not
 * reported, and the next call clears the status words. A caller that needs the
 * PCG status passes at least one output; the call then synchronises `stream`
 * and reports iterations, the PCG status (0 converged, 1 max iterations, 2 not
 * SPD, 3 barrier timeout) and the final relative residual. */
ANDO_API int32_t ando_pcg_solve_noalloc(int32_t device, void* stream, int32_t num_rows, const int32_t* rowptr,
                                        const int32_t* cols, const float* vals, const float* rhs, float* x, float* work,
                                        int64_t work_floats, double tol, int32_t max_iters, int32_t* iterations,
                                        int32_t* pcg_status, double* rel_residual);

/* ---------------------------------------------------------------------------
 * Learned preconditioner (no reference counterpart: the reference's only
 * preconditioner is block Jacobi, pcg_solver.cpp:77-114).
 *
 * In CORRECTED semantics the PCG runs on the block-scaled system
 * A^ = L^-1 A L^-T (A_ii = L_i L_i^T). With params.precond =
 * ANDO_PRECOND_LEARNED a mesh-graph message-passing network (3 layers, 64
 * wide, BF16 weights, FP32 accumulation) turns per-vertex and per-edge
 * features of A^ into a symmetric positive definite block-sparse S ~ A^-1 on
 * the mesh pattern:
 *   S = sum_i delta_i E_ii + sum_{edges i<j} W_e W_e^T,  W_e = [a_e I ; b_e A^_ij^T],
 * delta_i > 0. A solve whose S loses definiteness, stalls or reaches the
 * iteration cap is redone with block Jacobi (ando_step_stats.precond_fallbacks).
 * Weights are a flat float vector of ando_precond_num_params() entries. */
ANDO_API int32_t ando_precond_num_params(void);
/* Deterministic initial weights for `seed` (starts near S = 0.25 (2 I - A^)). */
ANDO_API int32_t ando_precond_init_weights(uint64_t seed, float* out, int32_t n);
/* Load weights into a context (rounded to BF16 for inference). */
ANDO_API int32_t ando_ctx_set_precond_weights(ando_ctx ctx, const float* weights, int32_t n);
/* Evaluate S for the context's current scaled system (after ando_eval_system
 * or a CORRECTED step) without solving; read it with ando_last_precond. */
ANDO_API int32_t ando_precond_eval(ando_ctx ctx);
/* S of the last learned evaluation: 9 floats per static pattern slot. */
ANDO_API int32_t ando_last_precond(ando_ctx ctx, float* S);
/* The scaled system of the last CORRECTED Newton iteration: A^ on the static
 * pattern (9 * nnzb), A^ of the contact blocks of ando_last_contact_blocks
 * (9 * count), b^ = L^-1 b (3 V), L packed lower-triangular per vertex
 * (6 V, FP32) and L^-1 (6 V, FP64). Any pointer may be NULL. */
ANDO_API int32_t ando_last_scaled_system(ando_ctx ctx, float* valh, float* xvalh, float* bhat, float* Lf, double* Linv);

/* Training of the preconditioner on the device (forward and backward
 * kernels of this library, Adam). A trainer holds weights, optimiser state
 * and a set of scaled Newton systems, each with probe vectors dumped by the
 * solver itself: the residuals of a block-Jacobi solve after 2^k - 1
 * iterations. The loss of a system is the mean over its probes r of the
 * relative energy error of one preconditioned step, 1 + (y^T A^ y - 2 r^T y)
 * / (r^T A^-1 r) with y = S r. */
typedef struct ando_trainer_s* ando_trainer;
ANDO_API int32_t ando_trainer_create(int32_t device, const float* weights, int32_t n, ando_trainer* out);
ANDO_API void ando_trainer_destroy(ando_trainer t);
/* Add the context's current scaled system (ando_eval_system in CORRECTED
 * semantics), solving it with block Jacobi to `tol` (at most `max_iters`
 * iterations) to record up to `max_probes` probes. */
ANDO_API int32_t ando_trainer_add_system(ando_trainer t, ando_ctx ctx, int32_t max_probes, double tol, int32_t max_iters);
ANDO_API int32_t ando_trainer_num_systems(ando_trainer t);
/* Probes of system `idx` (3 V floats each) and their energy norms. */
ANDO_API int32_t ando_trainer_probes(ando_trainer t, int32_t idx, float* probes, double* norms, int32_t* num);
/* Loss of system `idx` at the current weights; with `grad` (num_params
 * floats) also its gradient w.r.t. the FP32 master weights. */
ANDO_API int32_t ando_trainer_loss(ando_trainer t, int32_t idx, double* loss, float* grad);
/* One Adam step (beta 0.9 / 0.999) on the next system in turn. */
ANDO_API int32_t ando_trainer_step(ando_trainer t, float lr, double* loss);
ANDO_API int32_t ando_trainer_get_weights(ando_trainer t, float* weights, int32_t n);
ANDO_API int32_t ando_trainer_set_weights(ando_trainer t, const float* weights, int32_t n);

#ifdef __cplusplus
}
#endif

#endif /* ANDO_GPU_H */
