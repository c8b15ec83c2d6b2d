/*
 * chysx_cloth.h — C ABI of the B200-native implicit cloth step.
 *
 * Drop-in boundary for ChysX's ClothSimulator hot path
 * (caixiao-0725/Ai-Phyiscs, src/cloth/cloth_simulator.h and the pybind11
 * facade src/bindings.cpp:25-600).  Plain pointers and sizes only; device
 * buffers are passed as uintptr_t (a cudaMalloc'd address), CUDA streams as
 * uintptr_t (a cudaStream_t, 0 = legacy default stream), exactly as the
 * reference's Python layer passes Warp pointers.
 *
 * Every function returns a status code (CHYSX_OK on success).  On failure
 * chysx_last_error() returns a thread-local message.  The status codes map
 * onto the exception types the reference raises:
 *   CHYSX_ERR_INVALID_ARGUMENT -> std::invalid_argument (Python ValueError)
 *   CHYSX_ERR_OUT_OF_RANGE     -> std::out_of_range     (Python IndexError)
 *   CHYSX_ERR_RUNTIME          -> std::runtime_error    (Python RuntimeError)
 *   CHYSX_ERR_CUDA             -> CUDA failure          (Python RuntimeError)
 */
#ifndef CHYSX_CLOTH_H_
#define CHYSX_CLOTH_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CHYSX_OK = 0,
    CHYSX_ERR_INVALID_ARGUMENT = 1,
    CHYSX_ERR_OUT_OF_RANGE = 2,
    CHYSX_ERR_RUNTIME = 3,
    CHYSX_ERR_CUDA = 4
};

/* Outcome of the last PCG solve (chysx_cloth_last_stats). */
enum {
    CHYSX_SOLVE_CONVERGED = 0, /* ||r||/||b|| <= rel_tol, or fixed count done */
    CHYSX_SOLVE_MAX_ITER = 1,  /* rel_tol > 0 and max_iter reached first */
    CHYSX_SOLVE_NONFINITE = 2, /* NaN/Inf met; caller's pos/vel left untouched */
    CHYSX_SOLVE_KERNEL_ERROR = 3 /* solver grid barrier timed out; pos/vel untouched */
};

/* Initial guess of the PCG solve. */
enum {
    CHYSX_WARM_ZERO = 0,     /* zero guess (plain PCG) */
    CHYSX_WARM_PREVIOUS = 1, /* previous step's dx (reference behaviour,
                                src/cloth/cloth_simulator.cu:1219-1228) */
    CHYSX_WARM_LEARNED = 2,  /* per-vertex network guess, energy-scaled,
                                zero-guess fallback */
    CHYSX_WARM_PREVIOUS_SCALED = 3 /* previous dx, energy-scaled, zero-guess
                                      fallback */
};
/* Energy scaling: a guess x0 starts the solve as c x0 with
 * c = x0.b / x0.A x0, the factor that minimises 1/2 x.A x - b.x along x0, so
 * the start is never worse than the zero guess in the A-norm; c <= 0 (or a
 * non-finite partial) falls back to the zero guess.  CHYSX_WARM_PREVIOUS
 * keeps the reference's unscaled start. */

/* POD material, field-for-field src/cloth/cloth_material.h:20-43. */
typedef struct chysx_cloth_material {
    float lame_mu;
    float lame_lambda;
    float bending;
    float density;
    float damping;
    float gx;
    float gy;
    float gz;
} chysx_cloth_material;

typedef struct chysx_cloth chysx_cloth; /* opaque simulator handle */

/* Thread-local message of the last failing call on this thread. */
const char* chysx_last_error(void);

/* ClothSimulator() / ~ClothSimulator(): src/cloth/cloth_simulator.h:67-75. */
int chysx_cloth_create(chysx_cloth** out);
int chysx_cloth_destroy(chysx_cloth* h);

/* ClothSimulator::set_material (copy): src/cloth/cloth_simulator.h:81. */
int chysx_cloth_set_material(chysx_cloth* h, const chysx_cloth_material* m);
int chysx_cloth_get_material(const chysx_cloth* h, chysx_cloth_material* out);

/* ClothSimulator::set_external_buffers: src/cloth/cloth_simulator.h:95-99,
 * src/cloth/cloth_simulator.cu:248-258.  Borrowed float3 (12-byte AoS)
 * device arrays; inv_mass / force may be 0.  Never copied or freed. */
int chysx_cloth_set_external_buffers(chysx_cloth* h, uintptr_t pos, uintptr_t vel,
                                     int particle_count, uintptr_t inv_mass,
                                     uintptr_t force);

/* ClothSimulator::set_mesh: src/cloth/cloth_simulator.cu:315-377.  Host
 * int32 triangle triples; builds the sorted unique edge list. */
int chysx_cloth_set_mesh(chysx_cloth* h, const int32_t* tris, int n_triangles);
int chysx_cloth_num_edges(const chysx_cloth* h, int* out);
int chysx_cloth_get_edges(const chysx_cloth* h, int32_t* out /* 2*num_edges */);

/* ClothSimulator::set_pins / clear_pins / update_pin_targets:
 * src/cloth/cloth_simulator.cu:277-313 (host index + float3 target arrays). */
int chysx_cloth_set_pins(chysx_cloth* h, const int32_t* idx, const float* targets, int n,
                         float stiffness);
int chysx_cloth_clear_pins(chysx_cloth* h);
int chysx_cloth_num_pins(const chysx_cloth* h, int* out);
int chysx_cloth_update_pin_targets(chysx_cloth* h, const float* targets, int n,
                                   uintptr_t stream);

/* ClothSimulator::build_springs_from_current_positions:
 * src/cloth/cloth_simulator.cu:379-398.  k_per_edge (host, num_edges
 * floats, may be NULL) overrides the scalar stiffness per edge. */
int chysx_cloth_build_springs(chysx_cloth* h, float stiffness, const float* k_per_edge,
                              uintptr_t stream);
int chysx_cloth_num_springs(const chysx_cloth* h, int* out);

/* ClothSimulator::build_fem_stretch_from_current_positions:
 * src/cloth/cloth_simulator.cu:400-421.  k_per_tri (host, may be NULL)
 * overrides the scalar per-area stiffness per triangle. */
int chysx_cloth_build_fem_stretch(chysx_cloth* h, float stiffness, const float* k_per_tri,
                                  uintptr_t stream);

/* ClothSimulator::build_fem_shear_from_current_positions:
 * src/cloth/cloth_simulator.cu:423-449.  The stretch element with its rest
 * frame turned by pi/4 (triangle_stretch_constraint.cu:87-109), assembled
 * beside the stretch set; k_per_tri (host, may be NULL) overrides the scalar
 * per-area stiffness per triangle. */
int chysx_cloth_build_fem_shear(chysx_cloth* h, float stiffness, const float* k_per_tri,
                                uintptr_t stream);

/* ClothSimulator::build_bending_from_current_positions:
 * src/cloth/cloth_simulator.cu:451-514.  One discrete-bending dihedral per
 * interior edge of the (consistently oriented) mesh, rest angles from the
 * current positions, stiffness k for all (constraint/cloth/
 * bending_constraint.h).  Its Hessian blocks are not symmetric, so a step
 * with bending stores full 3x3 off-diagonal blocks and runs the streamed or
 * graph-loop PCG kernel. */
int chysx_cloth_build_bending(chysx_cloth* h, float stiffness, uintptr_t stream);
int chysx_cloth_num_dihedrals(const chysx_cloth* h, int* out);

/* Static-shape contact, ClothSimulator::add_static_plane / add_static_box /
 * clear_static_shapes / set_static_contact_{thickness,stiffness,friction,
 * friction_epsilon} (src/cloth/cloth_simulator.h:383-452; shapes as
 * collision::PlaneShape / BoxShape, src/collision/static_contact.h:73-105).
 * Each particle's deepest penetration below `thickness` adds the penalty
 * gradient, the lagged IPC friction force, the diagonal block
 * k n n^T + alpha (I - n n^T) and the Coulomb-cone projection of its residual
 * (static_contact.cu:111-381); active while stiffness > 0 and a shape exists.
 * A plane is n (3 floats, unit, pointing to the free side) and d with
 * n.x + d = 0 on the surface; a box is center, half extents and its three
 * unit axes (3 floats each). */
int chysx_cloth_add_static_plane(chysx_cloth* h, const float* n, float d);
int chysx_cloth_add_static_box(chysx_cloth* h, const float* center, const float* half_ext, const float* ex,
                               const float* ey, const float* ez);
int chysx_cloth_clear_static_shapes(chysx_cloth* h);
int chysx_cloth_static_shape_counts(const chysx_cloth* h, int* planes, int* boxes);
int chysx_cloth_set_static_contact_thickness(chysx_cloth* h, float thickness);
int chysx_cloth_set_static_contact_stiffness(chysx_cloth* h, float stiffness);
int chysx_cloth_set_static_contact_friction(chysx_cloth* h, float mu);
int chysx_cloth_set_static_contact_friction_epsilon(chysx_cloth* h, float eps_u);
int chysx_cloth_get_static_contact(const chysx_cloth* h, float* thickness, float* stiffness, float* mu,
                                   float* eps_u);

/* Contact operator, collision::ContactSpMVOp (src/collision/contact_spmv.h:
 * 58-96): a contact list filled on the device by the caller's detector
 * every step (the reference's SelfCollisionDetector output,
 * src/collision/self_collision.h:22-57) that the step folds into its system
 * as the penalty Hessian sum_c w_ci w_cj (k n n^T + alpha (I - n n^T)):
 * gradient and diagonal blocks into the assembly (self_collision_constraint.
 * cu:45-95, contact_spmv.cu:84-165), the off-diagonal blocks into every
 * solver SpMV (contact_spmv.cu:171-236; cloth_simulator.cu:941-962,
 * 1160-1165, 1243-1248).  The pointers are borrowed device addresses read
 * when each step runs, so the list and *count may change between steps
 * without any call here.  alpha = mu k depth f1(|u_t|) when friction_mu > 0
 * and slips are given.  A contact whose stiffness is not finite and
 * positive is skipped; one with a weighted particle index outside the
 * particle range is dropped and counted (contact_stats).  Needs the
 * single-instance layout; a step with a contact operator uses the streamed
 * or graph-loop PCG kernel. */
typedef struct chysx_contact_op {
    uintptr_t pairs;       /* int32 x 4 per contact, 16-byte aligned */
    uintptr_t weights;     /* float x 8 per contact: w0..w3, nx, ny, nz, depth; 16-byte aligned */
    uintptr_t count;       /* int32: contacts written this step (clamped to max_contacts) */
    int max_contacts;
    float stiffness;       /* uniform k */
    uintptr_t stiffnesses; /* optional float per contact, overrides stiffness */
    uintptr_t slips;       /* optional float x 4 per contact: u_t xyz, |u_t|; 16-byte aligned */
    float friction_mu;
    float friction_epsilon;
    /* 0: the warm-start residual r = b - (A + C) x0 (default);
     * 1: the reference's r = b - A x0 without the off-diagonal contact part
     *    (src/solver/pcg_solver.cu:512-513 passes alpha = -1, which
     *    contact_spmv.cu:193-196 skips) */
    int residual_mode;
} chysx_contact_op;
int chysx_cloth_set_contact_op(chysx_cloth* h, const chysx_contact_op* op);
int chysx_cloth_clear_contact_op(chysx_cloth* h);
/* Contacts live in the last step, contacts dropped for an out-of-range
 * index, and row slots written (synchronises). */
int chysx_cloth_contact_stats(chysx_cloth* h, int* live, int* dropped, int* slots);

/* ClothSimulator::redistribute_mass_area_weighted:
 * src/cloth/cloth_simulator.cu:516-575.  Writes the caller's inv_mass. */
int chysx_cloth_redistribute_mass(chysx_cloth* h, float surface_density, uintptr_t inv_mass,
                                  int particle_count, uintptr_t stream);

/* ClothSimulator::set_pcg_iterations / pcg_iterations:
 * src/cloth/cloth_simulator.h:597-600. */
int chysx_cloth_set_pcg_iterations(chysx_cloth* h, int max_iter);
int chysx_cloth_pcg_iterations(const chysx_cloth* h, int* out);

/* Solver controls the reference lacks (no counterpart; defaults reproduce
 * the reference: max_iter 50, rel_tol 0 = fixed iteration count, warm start
 * from the previous dx).  rel_tol > 0 stops when ||r||/||b|| <= rel_tol
 * with FP64 norms. */
int chysx_cloth_set_solver(chysx_cloth* h, int max_iter, double rel_tol, int warm_start);

/* Behaviour switches (no counterpart in the reference).  springs_in_step:
 * assemble springs into step() (the reference skips them,
 * src/cloth/cloth_simulator.cu:921; default 1).  apply_external_force: use
 * the force buffer in the predictor (the reference passes nullptr,
 * src/cloth/cloth_simulator.cu:892-894; default 0).  fem_det_eps: rest-shape
 * degeneracy threshold (src/constraint/cloth/triangle_stretch_constraint.cu:
 * 39,88-91; default 1e-6). */
int chysx_cloth_set_options(chysx_cloth* h, int springs_in_step, int apply_external_force,
                            float fem_det_eps);

/* ClothSimulator::step: src/cloth/cloth_simulator.cu:814-1261.  Enqueues the
 * whole step (assembly, PCG, update) on `stream` as one CUDA graph launch and
 * returns without synchronising. */
int chysx_cloth_step(chysx_cloth* h, float dt, uintptr_t stream);

/* Iterations, relative residual ||r||/||b|| and CHYSX_SOLVE_* status of the
 * last step (synchronises the last step's stream).  Replaces
 * PCGSolver::last_residual (src/solver/pcg_solver.cu:897-923). */
int chysx_cloth_last_stats(chysx_cloth* h, int* iterations, double* rel_residual, int* status);

/* The rel_residual above is the solver's recurrence residual.  With on != 0
 * every later step also recomputes r = b - (A + C) dx from the stored system
 * and the returned dx (FP64 accumulation) in a graph branch beside the
 * update: PCGParams::compute_true_residual (src/solver/pcg_solver.h:78) and
 * its pass (src/solver/pcg_solver.cu:595-641).  Off by default. */
int chysx_cloth_set_true_residual(chysx_cloth* h, int on);
/* ||b - (A + C) dx|| / ||b|| of the last step per instance (relres: n
 * entries, n = chysx_cloth_num_instances, or NULL) and the largest (worst,
 * or NULL); synchronises.  Replaces PCGSolver::host_last_true_relative_residual
 * (src/solver/pcg_solver.h:191).  CHYSX_ERR_RUNTIME unless the last step ran
 * with the pass on. */
int chysx_cloth_true_residual(chysx_cloth* h, int n, double* relres, double* worst);

/* Double-buffered step, the Newton bridge's stepping (SolverChysX, reference
 * README.md:113-130, which copies state_in to state_out and then steps
 * state_out in place): reads x_n, v_n from pos_in / vel_in and writes
 * x_{n+1}, v_{n+1} to pos_out / vel_out in the same kernels, with no copy
 * pass; the inputs become the external buffers.  pos_out == pos_in together
 * with vel_out == vel_in is an in-place step; otherwise the outputs must not
 * overlap the inputs.  A failed solve (status NONFINITE) copies the inputs to
 * the outputs.  Float3 AoS device buffers of num_particles entries. */
int chysx_cloth_step_into(chysx_cloth* h, float dt, uintptr_t pos_in, uintptr_t vel_in, uintptr_t pos_out,
                          uintptr_t vel_out, uintptr_t stream);

/* ClothSimulator::num_particles / num_off_diag_blocks (used by the
 * reference's debug dump, src/bindings.cpp:551-596). */
int chysx_cloth_num_particles(const chysx_cloth* h, int* out);
int chysx_cloth_num_off_diag_blocks(const chysx_cloth* h, int* out);

/* debug_dump_last_solve in the reference's layout (src/bindings.cpp:551-596,
 * src/cloth/cloth_simulator.cu:1272-1348): diag (N*9 row-major), row_offsets
 * (N+1), col_indices (nnz), values (nnz*9), rhs (N*3), dx (N*3); host
 * buffers, synchronises the device. */
int chysx_cloth_debug_dump(chysx_cloth* h, float* diag, int32_t* row_offsets,
                           int32_t* col_indices, float* values, float* rhs, float* dx);
/* The two-level preconditioner's coarse level of the last step (test
 * support, no counterpart in the reference): info[6] = {in use, coarse
 * blocks, CTAs per block, fields per block, unknowns m, 0};
 * with ac / ainv non-null (host, m * m floats each, cap >= m * m) the coarse
 * matrix A_c dense and the inverse the solver used (of A_c + shift
 * diag(A_c), shift 0 on the register-resident kernel, 1e-5 on the streamed
 * one; for the batched level the inverse is block-diagonal by instance),
 * unknown
 * index block * 3 * fields + 3 * field + component.  Synchronises. */
int chysx_cloth_debug_coarse(chysx_cloth* h, int32_t* info, float* ac, float* ainv, int cap);
/* The coarse blocks' first internal rows of the last graph build (test
 * support, no counterpart in the reference): *count = blocks + 1 (0 without
 * a coarse level); with row0 non-null (cap >= *count entries) the rows, the
 * last one the internal row count rounded up to whole 32-row slices. */
int chysx_cloth_debug_coarse_rows(chysx_cloth* h, int32_t* row0, int cap, int32_t* count);

/* Learned warm start (no counterpart in the reference).  A per-vertex
 * network (20 1-ring features -> 3 x 64 GELU -> dv, BF16 on tensor cores)
 * predicts each step's velocity change; the PCG starts from dx0 = dt (v + dv)
 * and still runs to the same tolerance, falling back to the zero guess per
 * instance when ||b - A dx0|| > ||b||.  set_network takes the flat FP32
 * parameter vector (chysx_mlp_num_params() floats: input mean/std, output
 * mean/std, then W1 [20][64], b1, W2 [64][64], b2, W3, b3, W4 [64][3], b4)
 * and enables set_solver(..., CHYSX_WARM_LEARNED). */
int chysx_cloth_set_network(chysx_cloth* h, const float* params, int n_params);
/* Every following step also writes its raw features (particle_count x 20
 * floats, caller order) to this device buffer (0 = off): the training-data
 * tap.  The target of a step is v_{n+1} - v_n (undamped).  With a network
 * loaded and the learned warm start on, `predictions` (may be 0) receives
 * the predicted dv (particle_count x 3). */
int chysx_cloth_set_feature_output(chysx_cloth* h, uintptr_t features, uintptr_t predictions);
/* Number of instances whose last solve kept the warm-start guess (the rest
 * fell back to the zero guess); synchronises. */
int chysx_cloth_guess_kept(chysx_cloth* h, int* kept);
int chysx_mlp_num_params(void);
int chysx_mlp_num_features(void);
/* Device workspace needed by the training / prediction calls for `rows`. */
uint64_t chysx_mlp_workspace_bytes(int rows);
/* Loss (mean squared error of standardised dv) and its gradient in the flat
 * parameter layout, for `rows` feature / target rows (device pointers;
 * synchronises `stream` to return the loss). */
int chysx_mlp_gradients(uintptr_t params, uintptr_t features, uintptr_t targets, int rows, uintptr_t grad,
                        double* loss, uintptr_t workspace, uint64_t workspace_bytes, uintptr_t stream);
/* Predicted dv (rows x 3) for feature rows. */
int chysx_mlp_predict(uintptr_t params, uintptr_t features, int rows, uintptr_t dv, uintptr_t workspace,
                      uint64_t workspace_bytes, uintptr_t stream);
/* One Adam step (lr, step count >= 1) on the FP32 master parameters, using
 * the gradient of the minibatch; m1 / m2 are the moment buffers. */
int chysx_mlp_train_step(uintptr_t params, uintptr_t grad, uintptr_t m1, uintptr_t m2, uintptr_t features,
                         uintptr_t targets, int rows, float lr, int adam_step, uintptr_t workspace,
                         uint64_t workspace_bytes, double* loss, uintptr_t stream);

/* Largest `rows` accepted by chysx_mlp_gradients_noalloc; the library's
 * value is also returned by chysx_mlp_noalloc_max_rows(), for callers that
 * bind the C ABI without this header. */
#define CHYSX_MLP_NOALLOC_MAX_ROWS 4096
int chysx_mlp_noalloc_max_rows(void);
/* chysx_mlp_gradients without a workspace argument (no counterpart in the
 * reference, which has no training entry point at all).  Same kernels, same
 * results; the workspace is a fixed static device array inside this library
 * (5,308,672 bytes per device, enough for CHYSX_MLP_NOALLOC_MAX_ROWS rows),
 * so the call allocates no device memory and, on success, no host memory.
 * It is for callers that cannot allocate: a host program that drives the
 * training through this C ABI (ctypes, cgo, JNI) without a device allocator
 * of its own, and a caller that keeps cudaMalloc / cudaFree out of its loop
 * because they can synchronise the device while the solver runs.
 *   - rows > CHYSX_MLP_NOALLOC_MAX_ROWS (or rows <= 0, a null pointer, or
 *     targets = 0) returns CHYSX_ERR_INVALID_ARGUMENT and launches nothing;
 *     use chysx_mlp_gradients with a caller workspace for larger batches.
 *   - The first call on each device is its set-up: with that device current
 *     it looks up the device address of the scratch array (which may load
 *     the library's device code).  Make that first call before any stream
 *     capture on the device.
 *   - Nothing in the scratch has to start at zero: every byte the kernels
 *     read was written earlier in the same call.  The first 46 entries of
 *     `grad` (the normalisation slots) are zeroed by the call itself.
 *   - All calls on one device share the one scratch array: two calls that
 *     overlap in time (different streams, or host threads without ordering)
 *     race on it and corrupt each other's results.  Issue them on one stream
 *     or order them with events.
 *   - loss != NULL synchronises `stream`, as chysx_mlp_gradients does. */
int chysx_mlp_gradients_noalloc(uintptr_t params, uintptr_t features, uintptr_t targets, int rows,
                                uintptr_t grad, double* loss, uintptr_t stream);

/* Batched solve (no counterpart in the reference): the particles of the
 * external buffers form n_instances independent cloths, instance b owning
 * particles [offsets[b], offsets[b+1]) (offsets[0] = 0, offsets[n] = the
 * particle count; no triangle may connect two instances).  All instances are
 * assembled into one concatenated block system and solved by one persistent
 * PCG kernel with a separate convergence test per instance; last_stats then
 * reports the slowest / worst instance.  n_instances = 0 restores the single
 * system. */
int chysx_cloth_set_instances(chysx_cloth* h, const int32_t* offsets, int n_instances);
int chysx_cloth_num_instances(const chysx_cloth* h, int* out);
/* Per-instance iterations, relative residual and status of the last step
 * (arrays of n = num_instances entries; synchronises). */
int chysx_cloth_instance_stats(chysx_cloth* h, int n, int* iterations, double* rel_residual,
                               int* status);

/* Solver kernel selection (no counterpart in the reference, whose PCG is a
 * fixed chain of 8 launches per iteration, src/solver/pcg_solver.cu:542-592):
 * solver_path 0 = one persistent cooperative kernel per solve, with rows held
 * in registers when the system fits (default), 1 = CUDA-graph WHILE loop of
 * two kernels per iteration, 2 = the streamed persistent kernel forced.
 * block (0, 128, 256, 512) and grid (0 = automatic) size the streamed
 * persistent kernel; block 0 lets the planner choose (64-thread CTAs, a
 * build of its own, for batches that get the coarse level, whose blocks are
 * the instances' CTA segments; else 256). */
int chysx_cloth_set_tuning(chysx_cloth* h, int solver_path, int block, int grid);
/* Synchronisation of the persistent PCG kernels (no counterpart in the
 * reference): 0 = one grid-wide counter barrier per reduction (default),
 * 1 = polled per-instance reduction slots, in which each instance waits only
 * for the CTAs holding its rows and the reduction read is the wait itself.
 * Both sum the same partials in the same order: identical iterates. */
int chysx_cloth_set_sync_mode(chysx_cloth* h, int mode);

/* Autotuner (no counterpart in the reference).  Times, on the current state,
 * every solver configuration that applies to the current system: the
 * planner's persistent kernel (register-resident rows when they fit, else
 * streamed), the streamed kernel at 128 / 256 / 512 threads per CTA (4 / 8 /
 * 16 32-row slices per CTA; one thread per row), both synchronisation modes,
 * and the graph-loop path; each `repetitions` times (best kept).  All run the
 * same PCG recurrence.  The caller's positions / velocities and the previous-step guess are
 * restored after every trial, so the simulation does not advance; the
 * fastest configuration stays selected.  Synchronises `stream`. */
int chysx_cloth_autotune(chysx_cloth* h, float dt, int repetitions, uintptr_t stream);
/* The autotuner's table: per candidate 8 ints (path, block, sync, kernel used
 * as in solver_info, its grid, its block, iterations, solve status) and the
 * solve time in ms; *count = the number of candidates. */
int chysx_cloth_autotune_results(const chysx_cloth* h, int capacity, int* count, int32_t* config,
                                 float* solve_ms);
int chysx_cloth_sync_mode(const chysx_cloth* h, int* mode);
/* Row order (no counterpart in the reference, whose rows are the particles):
 * mode 0 = the caller's particle order (default); mode 1 = spatially
 * compact blocks: at the next topology build the particles of each instance
 * are ordered by recursive coordinate bisection of their positions (split
 * sizes multiples of 512 rows, then of 32), so every 32-row slice and every
 * block of rows one CTA holds is a patch of the cloth.  The order is kept
 * until the mesh, the instances or the particle count change.  Results do
 * not depend on it beyond summation order; the CTA-local preconditioner
 * gains from it.  row_of_particles reports the internal row of each of the
 * n particles. */
int chysx_cloth_set_row_order(chysx_cloth* h, int mode);
int chysx_cloth_row_of_particles(const chysx_cloth* h, int n, int32_t* rows);

/* Preconditioner (no counterpart in the reference, whose PCG preconditions
 * with the 3x3 diagonal blocks, src/solver/pcg_solver.cu:29-51): kind 0 =
 * block-Jacobi (default; the reference's iterates); kind 1 = CTA-local
 * Chebyshev: z = p(D^-1 A_cc) D^-1 r, A_cc the diagonal block of the rows one
 * CTA of the register-resident kernel holds (couplings to other CTAs left
 * out), p the Chebyshev polynomial of odd `degree` on
 * [lambda_max / ratio, lambda_max], lambda_max estimated per CTA and solve by
 * power iteration with a 10% margin.  A fixed polynomial, so the outer
 * iteration stays plain PCG with the same stopping test (||r|| / ||b||);
 * odd degrees keep p positive on the whole spectrum.  Kind 2 = kind 1 plus
 * a coarse level: z += R A_c^-1 R^T r, A_c = R^T A R assembled on the device
 * each step, R the coarse space: on blocks of 2 consecutive CTAs (1024 rows
 * of a spatially ordered 256 x 256 grid) the translation and the three
 * linear fields along the principal axes of the block's positions, where the
 * plan has at least 8 CTAs, else the translation of every CTA's block;
 * A_c^-1 is formed densely each step by an FP64 Gauss-Jordan kernel (at
 * most 2048 unknowns).  It applies to single-instance systems of at most
 * 160 CTAs and acts as kind 1 elsewhere.  Kinds 1 and 2 apply where the
 * register-resident kernel runs with synchronisation mode 0.  On systems too
 * large for that kernel (the streamed kernel), kinds 1 and 2 give
 * block-Jacobi plus the coarse level on blocks of about 5120 rows, A_c
 * shifted by 1e-5 diag(A_c) (single instance, synchronisation mode 0); on
 * batches of instances there (zero-guess solves, synchronisation mode 0),
 * block-Jacobi plus coarse blocks inside the instances (an instance's rows in
 * one CTA, or runs of such segments, at most 12 per instance; translation and
 * linear fields; A_c block-diagonal by instance, each instance's dense
 * inverse formed on its own, same shift).
 * in_use reports what the last graph build uses (0 block-Jacobi, 1 local,
 * 2 two-level with translations, 3 two-level with translations and linear
 * fields). */
int chysx_cloth_set_preconditioner(chysx_cloth* h, int kind, int degree, float ratio);
int chysx_cloth_preconditioner(const chysx_cloth* h, int* kind, int* degree, float* ratio, int* in_use);
/* Kernel used at the last graph build: path 0 register-resident persistent,
 * 1 graph loop, 2 streamed persistent; with its grid and block size. */
int chysx_cloth_solver_info(const chysx_cloth* h, int* path, int* grid, int* block);

/* Measurement hooks (no counterpart in the reference): when enabled, the
 * step graph records CUDA events around assembly, the PCG solve and the
 * finalize kernel on the step's stream; last_timing synchronises on the
 * last event and returns the three durations of the last step. */
int chysx_cloth_enable_timing(chysx_cloth* h, int on);
int chysx_cloth_last_timing(chysx_cloth* h, float* assemble_ms, float* solve_ms, float* finalize_ms);

/* Host-only introspection of the off-diagonal block pattern the step
 * assembles for a mesh (no counterpart in the reference; the equivalent there
 * is BlockCSR3::build_topology, src/sparse/block_csr.cu:91-147, fed by
 * src/cloth/cloth_simulator.cu:698-793).  Triangle pairs plus spring edges,
 * sorted unique columns per row; row_offsets has n+1 entries, col_indices
 * up to max_nnz.  Also reports the sliced-ELL entry count and widest slice.
 * Needs no GPU. */
int chysx_topology_pattern(int n, const int32_t* tris, int n_tris, const int32_t* edges, int n_edges,
                           int32_t* row_offsets, int32_t* col_indices, int max_nnz, int* nnz_out,
                           int* ell_entries_out, int* max_width_out);

#ifdef __cplusplus
}
#endif

#endif /* CHYSX_CLOTH_H_ */
