/* vortex_b200: B200-native (sm_100a, FP64) nodal-DG right-hand side and
 * explicit RK4 / forward-Euler stepper for the 2D compressible Euler equations
 * on affine triangles, as a drop-in for Vortex-Transport's CPU element loop.
 *
 * C ABI only: plain pointers and sizes, no C++ or torch types. Every entry point
 * returns VT_OK (0) or a status code; nothing in the library calls exit().
 * A context owns its device memory and one CUDA stream; calls on one context
 * are serialised by a per-context lock and may come from any host thread.
 *
 * Host array layouts follow the reference's nested vectors, flattened
 * element-major:
 *   U   K x Np x 4       (rho, rho u, rho v, rho E)   Element.H:30
 *   F   K x Np x 2 x 4   (x flux, y flux)              Element.H:31
 * Np = (p+1)(p+2)/2 nodes per element, K = 2 nx ny elements.
 */
#ifndef VORTEX_B200_H
#define VORTEX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define VT_OK 0
/* The reference's non-physical-state exits (Numericalflux.cpp:42-54, 75-79,
 * 111-115) become these codes instead of exit(EXIT_FAILURE). */
#define VT_ERR_NONPHYSICAL_LEFT 1  /* pL <= 0 or rhoL <= 0 */
#define VT_ERR_NONPHYSICAL_RIGHT 2 /* pR <= 0 or rhoR <= 0 */
#define VT_ERR_NONPHYSICAL_C2 3    /* Roe-averaged c^2 <= 0 */
#define VT_ERR_INVALID (-1)        /* bad argument or input file */
#define VT_ERR_UNSUPPORTED (-2)    /* p, integration order or method out of range */
#define VT_ERR_CUDA (-3)           /* CUDA runtime error (message in vt_last_message) */
#define VT_ERR_NO_MEMORY (-4)

/* ---- input file --------------------------------------------------------- */
/* Mirrors `struct parameters` (Parameters.H:5-19), same fields and types. */
typedef struct vt_params {
  int p;
  float domain_x;
  float domain_y;
  int num_element_in_x;
  int num_element_in_y;
  float perturb_grid;
  int integration_order;
  float simulation_time;
  int number_time_steps;
  double time_step;
  int write_every_steps;
  int U_initialization_type;
  int stepping_method;
} vt_params;

/* Replaces read_input_files (Parameters.cpp:12-64): same `key=value` keys and
 * std::stoi/stof/stod conversions (so perturb_grid=0.2 reads as 0, as in the
 * reference); a missing or malformed key returns VT_ERR_INVALID instead of
 * throwing. */
int vt_read_input_file(const char* path, vt_params* out);
int vt_parse_input(const char* text, vt_params* out);

/* Message for the last non-OK status returned on the calling thread. */
const char* vt_last_message(void);

/* ---- initial condition -------------------------------------------------- */
/* The isentropic-vortex constants that Element::initialize_hydrodinamics
 * hard-codes (Element.cpp:134-143), as parameters. */
typedef struct vt_vortex {
  double rho_infty, rc, epsilon, gamma, M_infty, p_infty, U_infty, V_infty, x0, y0;
} vt_vortex;

/* The reference's literals: rho=1, rc=1, eps=0.3, gamma=1.4, M=0.5, p=20/7,
 * U=V=1/sqrt(2), centre (0,0). */
void vt_default_vortex(vt_vortex* out);

/* ---- host precompute (main.cpp:99-147) ---------------------------------- */
typedef struct vt_problem vt_problem;

typedef struct vt_problem_info {
  int K, p, Np, nfq, nqa, nx, ny;
} vt_problem_info;

/* Builds the mesh (Meshgeneration.cpp:16-186), quadrature
 * (Quadraturerule.cpp), reference operators (Preevolve.cpp:15-144),
 * per-element geometry (Element.cpp:54-116), face tables (Evolve.cpp:76-132)
 * and the initial state (Element.cpp:119-333). perturb_grid is used as the
 * float in `prm` (callers wanting the reference's std::stoi quirk go through
 * vt_read_input_file). ic == NULL uses the reference's vortex. */
vt_problem* vt_problem_create(const vt_params* prm, const vt_vortex* ic, int* status);
void vt_problem_destroy(vt_problem* prob);
int vt_problem_get_info(const vt_problem* prob, vt_problem_info* out);

/* Copies one named array (doubles, or int32 for "conn"/"type") into dst of
 * `bytes` bytes. Names: vertices, conn, type, nodes_ref, nodes_phys, line_quad,
 * area_quad, minv_ref, stiff_ref, phi_plus, phi_minus, jac, jinv, detj,
 * detjinv, normals, sides, U0, F0. */
int vt_problem_get_array(const vt_problem* prob, const char* name, void* dst, size_t bytes);

/* The exactly translated vortex at time t at the problem's nodes (K x Np x 4):
 * the initial condition's formula (Element.cpp:134-179) with the centre moved
 * by (U_infty, V_infty) t and taken as each node's nearest periodic image (the
 * reference's formula does not wrap). */
int vt_problem_exact_state(const vt_problem* prob, double t, double* U);

/* Nodal flux of a state, the formula the reference applies after every stage
 * (Timestepping.cpp:141-158). U: K x Np x 4 -> F: K x Np x 2 x 4. */
int vt_flux_from_state(int K, int p, const double* U, double* F);

/* ---- drop-in boundary: the device solver -------------------------------- */
/* Everything the reference's Element / Evolve_element objects hold that the
 * element loop reads (Element.H:19-45, Evolve.H:19-33), as flat host arrays.
 * The stepper never needs the per-element physical matrices: the elements are
 * affine, so the reference-space operators plus each element's inverse
 * Jacobian and determinant carry the same information. */
typedef struct vt_mesh_desc {
  int32_t p;                     /* Lagrange order, 0..3 */
  int32_t n_elements;            /* K */
  int32_t n_line_points;         /* nfq = gau_integ_line.size(), 1..10 */
  const int32_t* element_type;   /* K: Element::type */
  const int32_t* neighbours;     /* K x 3: right, left, vertical element */
  const double* det_jacobian;    /* K: Element::determinant_jacobian */
  const double* inv_jacobian;    /* K x 4: Element::inverse_jacobian [00,01,10,11] */
  const double* normals;         /* K x 3 x 2: outward unit normal per side */
  const double* side_lengths;    /* K x 3: Element::sides_lenght */
  const double* inv_mass_ref;    /* Np x Np: inverse_mass_matrix_reference_space */
  const double* stiffness_ref;   /* 2 x Np x Np: sitffness_matrix_reference_space */
  const double* line_quadrature; /* nfq x 2: (sigma, weight), gauss_line_integral */
  const double* phi_plus;        /* 3 x Np x nfq: plus_phi_in_quadrature_points_side_1..3 */
  const double* phi_minus;       /* 3 x Np x nfq: minus_phi_in_quadrature_points_side_1..3 */
} vt_mesh_desc;

/* Fills a descriptor whose pointers refer to arrays owned by `prob`. */
int vt_problem_mesh_desc(const vt_problem* prob, vt_mesh_desc* out);

typedef struct vt_ctx vt_ctx;

/* First failing check of the last step call, in the reference's serial order
 * (element, then face point, then side, Evolve.cpp:215-221). code 0 = none. */
typedef struct vt_error_info {
  int code;
  int element;
  int point;
  int side;
  int64_t step;  /* 0-based step within the failing call */
  int stage;     /* 0..3 for RK4, 0 for forward Euler */
} vt_error_info;

/* Uploads operators and geometry to `device` and allocates the state. Replaces
 * the per-step work of rk4 / forward_euler (Timestepping.H:8-9). */
vt_ctx* vt_create(const vt_mesh_desc* desc, int device, int* status);
void vt_destroy(vt_ctx* ctx);
/* The whole set-up on the device for the reference's own mesh: the periodic
 * structured triangulation with its perturbation (Meshgeneration.cpp:16-186),
 * the per-element geometry (Element.cpp:54-93) and the initial condition
 * (nodal or projected, Element.cpp:119-333, vortex `ic` or the reference's when
 * NULL) are generated per element on the GPU; only the reference-space tables
 * are built on the host. The mesh perturbation uses CUDA's sin/cos/pow, so
 * perturbed vertices agree with vt_problem_create's (glibc) to rounding; the
 * connectivity is identical. num_element_in_y must be at least 2: with one
 * row the reference's vertical neighbour index is negative (VT_ERR_INVALID,
 * as vt_create and vt_batch_create return for such a mesh). */
vt_ctx* vt_create_structured(const vt_params* prm, const vt_vortex* ic, int device, int* status);

/* State transfer with host arrays in the reference layout (U: K x Np x 4). */
int vt_upload_state(vt_ctx* ctx, const double* U);
/* F (K x Np x 2 x 4) may be NULL; when given it is the nodal flux of U, as the
 * reference stores it after each step. */
int vt_download_state(vt_ctx* ctx, double* U, double* F);
/* Same, with U a device pointer (K x Np x 4, reference layout) on ctx's device. */
int vt_upload_state_device(vt_ctx* ctx, const double* dU);
int vt_download_state_device(vt_ctx* ctx, double* dU);

/* nsteps classical RK4 steps (Timestepping.cpp:85-306) / forward-Euler steps
 * (Timestepping.cpp:39-82) of size dt. Blocks until done and returns VT_OK or
 * the first non-physical-state code (details via vt_last_error). */
int vt_step_rk4(vt_ctx* ctx, double dt, int nsteps);
int vt_step_euler(vt_ctx* ctx, double dt, int nsteps);

/* Same as vt_step_rk4 but only enqueues the work on the context's stream and
 * returns; vt_synchronize() waits and reports the status. */
int vt_step_rk4_async(vt_ctx* ctx, double dt, int nsteps);
int vt_synchronize(vt_ctx* ctx);

/* One right-hand-side evaluation of the current state, DG_time_derivative_U of
 * evolve_elem (Timestepping.cpp:18-36); Udot is a host K x Np x 4 array. */
int vt_rhs(vt_ctx* ctx, double* Udot);

int vt_last_error(const vt_ctx* ctx, vt_error_info* out);

/* Simulation time, advanced by dt per step as Element::time is
 * (Timestepping.cpp:80, :304). */
double vt_get_time(const vt_ctx* ctx);
int vt_set_time(vt_ctx* ctx, double t);

/* Conservation totals sum_e detJ_e sum_i W_i U_e,i (W_i = integral of the
 * i-th basis function), computed on the device. out[4]. */
int vt_totals(vt_ctx* ctx, double* out);

/* The L2 difference between the current state and U_ref (K x Np x 4, host or
 * device memory), in the form of the reference's post-processing script
 * (plottools/l2stateerror.py:65-98): squared nodal differences interpolated
 * with the basis at the area-rule points area_quad (nq x 3: xi, eta, weight),
 * integrated with det J, then sqrt(integral / 25) per component; out[4].
 * Computed on the device. */
int vt_l2_error(vt_ctx* ctx, int nq, const double* area_quad, const double* U_ref, int device_pointers,
                double* out);

/* Sets the state to the L2 projection of the vortex `ic` at time t on the
 * device (U_initialization_type=1, Element.cpp:180-326): vertices is the
 * problem's K x 3 x 2 host array (vt_problem_get_array "vertices"), area_quad
 * the nq x 3 area rule (xi, eta, weight). */
int vt_project_vortex(vt_ctx* ctx, const double* vertices, const vt_vortex* ic, double t, int nq,
                      const double* area_quad);

/* Full-precision dump and restart, replacing the reference's 6-decimal
 * per-element text dumps (Element::write_data, Element.cpp:336-425) where a
 * run must resume exactly. A state file is "VTSTATE" + NUL, int32 version (1),
 * p, K, Np, float64 time, then K x Np x 4 float64 in the reference's U layout.
 * vt_save_state writes the context's state and time; vt_load_state restores
 * them (the file must match the context's p and K). The file functions below
 * need no GPU. */
int vt_save_state(vt_ctx* ctx, const char* path);
int vt_load_state(vt_ctx* ctx, const char* path);
int vt_write_state_file(const char* path, int p, int n_elements, double time, const double* U);
int vt_state_file_info(const char* path, int* p, int* n_elements, double* time);
int vt_read_state_file(const char* path, double* U);

/* The context's cudaStream_t, for callers that interleave their own work. */
void* vt_stream(vt_ctx* ctx);

/* Warp mapping of the context's stage kernel: 0 one thread per element and
 * conserved component, 1 (the default) one thread per element, component pair
 * and half of the nodes. Both compute the same arithmetic (results agree to
 * rounding); the choice only changes the speed. No reference counterpart. */
int vt_set_stage_mapping(vt_ctx* ctx, int mapping);
int vt_get_stage_mapping(const vt_ctx* ctx);

/* Test hook of the stage kernels' bounded waits (no reference counterpart:
 * the reference has no asynchronous copies). Every wait of a stage kernel on
 * its tile's bulk copies gives up after a fixed number of polls, records
 * "a bulk-copy wait gave up" and stops the block, so a lost copy cannot hang
 * the GPU. tries > 0 sets that bound for the context's later steps;
 * issue_no_copies != 0 makes the kernels issue no state copies at all, so
 * every wait gives up (with no copy in flight) and vt_step_rk4 returns
 * VT_ERR_CUDA with the state unchanged. vt_test_bulk_wait(ctx, 0, 0) restores
 * the defaults; the context then steps as before. */
int vt_test_bulk_wait(vt_ctx* ctx, unsigned tries, int issue_no_copies);

/* Device time of each kernel kind of one RK4 step, measured with CUDA events
 * around individual launches (no graph): ms[0..3] = stages 0..3, averaged over
 * `reps` steps of size dt. Advances the state by `reps` steps. */
int vt_profile_rk4_stages(vt_ctx* ctx, double dt, int reps, float* ms);

/* ---- batched ensemble --------------------------------------------------- */
/* Many independent problems (meshes of any size, p = 0..3) advanced together:
 * the reference runs one problem per process (main.cpp:81-197), so this is
 * `n` calls of rk4 (Timestepping.cpp:85-306) sharing each kernel launch.
 * Instances with the same p and reference tables form a group stored as one
 * ragged element array; one stage launch per group advances all its
 * instances, and one CUDA graph holds a whole RK4 step. Each instance keeps
 * its own time step, and its elements see exactly the arithmetic of a
 * vt_ctx built from the same descriptor. */
typedef struct vt_batch vt_batch;

vt_batch* vt_batch_create(const vt_mesh_desc* descs, int n, int device, int* status);
void vt_batch_destroy(vt_batch* batch);
int vt_batch_size(const vt_batch* batch);
int vt_batch_groups(const vt_batch* batch);
int vt_batch_group_info(const vt_batch* batch, int group, int* p, int* n_instances, int64_t* n_elements);
/* Per-instance state transfer, host arrays in the reference layout. */
int vt_batch_upload_state(vt_batch* batch, int instance, const double* U);
int vt_batch_download_state(vt_batch* batch, int instance, double* U, double* F);
/* The same with U a device array (K_i x Np_i x 4) on the batch's device. */
int vt_batch_upload_state_device(vt_batch* batch, int instance, const double* dU);
int vt_batch_download_state_device(vt_batch* batch, int instance, double* dU);
/* Per-instance time steps, dt[n]. */
int vt_batch_set_dt(vt_batch* batch, const double* dt);
/* nsteps RK4 steps of every instance; blocks until done. A non-physical state
 * returns its code; vt_batch_last_error names the instance. */
int vt_batch_step_rk4(vt_batch* batch, int nsteps);
int vt_batch_last_error(const vt_batch* batch, int* instance, vt_error_info* out);
/* Times each group's RK4 step for both warp mappings of the stage kernel
 * (0: one thread per element and component; 1: one thread per element,
 * component pair and half of the nodes) and 1..max resident blocks per SM
 * (`trials` repetitions each), keeps the fastest and reports it per group in
 * blocks_per_sm[groups] and mapping[groups] (either may be NULL); the state is
 * left unchanged. No reference counterpart (the reference has one CPU loop). */
int vt_batch_autotune(vt_batch* batch, int trials, int* blocks_per_sm, int* mapping);
/* Apply a stored tuning (as reported by vt_batch_autotune). */
int vt_batch_set_blocks_per_sm(vt_batch* batch, const int* blocks_per_sm);
int vt_batch_set_mapping(vt_batch* batch, const int* mapping);
/* Device time of one RK4 step of each group on its own (group order of
 * vt_batch_group_info), averaged over `reps` steps after one warm-up step; the
 * groups' states are restored afterwards. No reference counterpart: it
 * reports how fast each order p runs inside a batch. */
int vt_batch_time_groups(vt_batch* batch, int reps, float* ms_per_step);

/* ---- discrete adjoint ---------------------------------------------------- */
/* No counterpart in the reference (which has no derivatives). The exact
 * transpose of the linearised RK4 step of vt_step_rk4: per stage the
 * transposed volume operator and nodal-flux Jacobian, the transposed Roe-flux
 * Jacobian at every face point (Roe averages, the c2^2 speed and the entropy
 * fix differentiated, Numericalflux.cpp:99-156), the transposed lift and mass
 * inverse, and the reversed RK4 combine. States are (K x Np x 4) arrays in the
 * reference layout, host memory unless `device_pointers` is non-zero (then
 * device memory on the context's device). Needs a mesh whose side s faces its
 * neighbour's side s (the reference mesh does); VT_ERR_UNSUPPORTED otherwise. */

/* Schedule of the checkpointing of an nsteps-step run with `nsnapshots`
 * stored states (U_0 included). With nsnapshots >= 4 nsteps every step's start
 * and three stage states are kept and nothing is recomputed (all_stages = 1);
 * otherwise step starts are checkpointed on the binomial schedule and each
 * step is rerun once, keeping its stage states, before its reverse. */
typedef struct vt_checkpoint_info {
  int64_t advance_steps;         /* plain RK4 steps, forward sweep included */
  int64_t forward_sweep_steps;   /* of which in the forward sweep */
  int64_t stage_steps;           /* steps run keeping stage states (= nsteps) */
  int64_t adjoint_steps;         /* = nsteps */
  int64_t optimal_advance_steps; /* Griewank's bound r n - C(S + r, S + 1) */
  int32_t slots_used;            /* state buffers actually used */
  int32_t all_stages;            /* 1: every stage state kept, no recomputation */
} vt_checkpoint_info;

/* Plans the reversal on the host only (no device needed). */
int vt_checkpoint_plan(int nsteps, int nsnapshots, vt_checkpoint_info* out);

/* Forward sweep: nsteps RK4 steps of size dt from the current state, keeping
 * at most `nsnapshots` states in device memory (nsnapshots >= nsteps keeps
 * every step's start; >= 4 nsteps also every stage state, so the reverse
 * sweep recomputes nothing). Besides the snapshots the context holds eleven
 * working state vectors, and a checkpointed sweep two more, onto which the
 * reverse sweep renames slots so that its recomputation can run ahead of its
 * reverse steps. On return the context holds U(T) exactly as vt_step_rk4
 * would leave it and the time has advanced; a non-physical state returns its
 * code. */
int vt_adjoint_forward(vt_ctx* ctx, double dt, int nsteps, int nsnapshots);
/* Reverse sweep of the last vt_adjoint_forward: given dJ/dU(T) returns
 * dJ/dU(0), recomputing the steps between checkpoints. Leaves the state and
 * the time alone, and may be called again with another dJ/dU(T). */
int vt_adjoint_backward(vt_ctx* ctx, const double* dJdU_T, double* dJdU_0, int device_pointers);
/* Both sweeps in one call, host arrays (K x Np x 4), for a cotangent dJ/dU(T)
 * known before the run (a linear functional of U(T)); a loss that depends on
 * U(T) needs the two calls above, with U(T) read in between. The one-call
 * adjoint entry of the drop-in interface. */
int vt_adjoint_rk4(vt_ctx* ctx, double dt, int nsteps, int nsnapshots, const double* dJdU_T, double* dJdU_0);
/* Schedule of the last vt_adjoint_forward. */
int vt_adjoint_info(const vt_ctx* ctx, vt_checkpoint_info* out);

/* Directional derivative of the right-hand side at U along V, dR = R'(U) V
 * (forward mode on dual numbers), and the transpose product G = R'(U)^T W
 * through the adjoint kernels. The context's state is not touched. */
int vt_rhs_jvp(vt_ctx* ctx, const double* U, const double* V, double* dR, int device_pointers);
int vt_rhs_vjp(vt_ctx* ctx, const double* U, const double* W, double* G, int device_pointers);
/* Tangent-linear model: advances the state nsteps RK4 steps as vt_step_rk4
 * does and carries a perturbation along: dU_T = (dU(T)/dU(0)) dU_0. */
int vt_tangent_rk4(vt_ctx* ctx, double dt, int nsteps, const double* dU_0, double* dU_T, int device_pointers);

/* Host-side pointwise pieces, for checks: the Roe flux in the algebra of the
 * stage kernels (Numericalflux.cpp:13-157; returns 0 or the non-physical code
 * 1/2/3), its Jacobian-vector product, and its transpose product (which adds
 * to buL and buR). */
int vt_roe_flux(const double* uL, const double* uR, double nx, double ny, double* flux);
int vt_roe_flux_jvp(const double* uL, const double* uR, double nx, double ny, const double* duL,
                    const double* duR, double* dflux);
void vt_roe_flux_vjp(const double* uL, const double* uR, double nx, double ny, const double* bflux, double* buL,
                     double* buR);

/* Adjoint of a batched run: vt_adjoint_forward / vt_adjoint_backward over each
 * group's ragged element array (one launch per stage for all instances of a
 * group, each instance with its own time step from vt_batch_set_dt). dJdU_T
 * and dJdU_0 are host arrays holding every instance's K_i x Np_i x 4 block, in
 * instance order. */
int vt_batch_adjoint_forward(vt_batch* batch, int nsteps, int nsnapshots);
int vt_batch_adjoint_backward(vt_batch* batch, const double* dJdU_T, double* dJdU_0);
/* The same with dJdU_T / dJdU_0 in device memory. */
int vt_batch_adjoint_backward_device(vt_batch* batch, const double* dJdU_T, double* dJdU_0);
int vt_batch_adjoint_info(const vt_batch* batch, int group, vt_checkpoint_info* out);

/* ---- stepping without device allocation --------------------------------- */
/* No counterpart in the reference. For callers that cannot call cudaMalloc:
 * code running while a host framework's pool or arena owns all device memory,
 * real-time loops where a cudaMalloc or cudaFree would synchronise the device,
 * and plugins that may only use buffers their host passes in. All scratch
 * (packed geometry, the state in the kernel's layout, the RK accumulator and
 * stage buffers, error words) lives in one fixed device array of
 * VT_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads the
 * library holds until the process exits. */
#define VT_NOALLOC_SCRATCH_BYTES (16u << 20)

/* vt_mesh_desc with the per-element arrays in DEVICE memory (same layouts);
 * the reference-space tables stay in host memory. */
typedef struct vt_device_mesh {
  int32_t p;
  int32_t n_elements;
  int32_t n_line_points;
  const int32_t* element_type;   /* device, K */
  const int32_t* neighbours;     /* device, K x 3: right, left, vertical */
  const double* det_jacobian;    /* device, K */
  const double* inv_jacobian;    /* device, K x 4 */
  const double* normals;         /* device, K x 3 x 2 */
  const double* side_lengths;    /* device, K x 3 */
  const double* inv_mass_ref;    /* host, Np x Np */
  const double* stiffness_ref;   /* host, 2 x Np x Np */
  const double* line_quadrature; /* host, nfq x 2 */
  const double* phi_plus;        /* host, 3 x Np x nfq */
  const double* phi_minus;       /* host, 3 x Np x nfq */
} vt_device_mesh;

/* Bytes of the fixed scratch a problem of this size needs (0 if p is out of
 * range); problems needing more than VT_NOALLOC_SCRATCH_BYTES are rejected. At
 * p = 3 that is about 11,700 elements. */
size_t vt_noalloc_scratch_bytes(int p, int n_elements);

/* nsteps RK4 steps from dU_in to dU_out (device, K x Np x 4, the reference
 * layout; they may be the same buffer) on `stream` (a cudaStream_t, NULL for
 * the default stream), the same kernels as vt_step_rk4, with no cudaMalloc,
 * cudaFree or allocating library call. Blocks until done. Returns VT_OK, a
 * non-physical-state code with `err` filled in, VT_ERR_INVALID for a problem
 * larger than the scratch, a bad neighbour index or a misaligned array (dU_in
 * and dU_out 16-byte aligned, the mesh's doubles 8 and ints 4; checked before
 * any device work), or VT_ERR_CUDA.
 * Every call looks up the scratch array's device address on the current device
 * (cudaGetSymbolAddress: a lookup, not an allocation), so the address is never
 * stale, not even after cudaDeviceReset; the first call on a device also reads
 * its SM count and may load the library's kernels, so make that first call
 * before any stream capture. Every call shares the one array and leaves its
 * contents behind (each call clears the words that must start at zero); calls
 * whose work overlaps on the GPU race on it. */
int vt_step_rk4_noalloc(const vt_device_mesh* mesh, const double* dU_in, double* dU_out, double dt,
                        int nsteps, void* stream, vt_error_info* err);

#ifdef __cplusplus
}
#endif

#endif /* VORTEX_B200_H */
