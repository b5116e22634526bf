/*
 * fem_b200.h — C ABI of the B200 (sm_100a) matrix-free FEM solver path.
 *
 * Drop-in boundary for jax_fem_cfd's solver hot path. The reference has no
 * FFI; its boundary is a set of Python callables (cited per entry point below,
 * paths relative to the jax_fem_cfd project root). Each entry point here is the
 * native implementation a binding (XLA FFI handler, ctypes, torch op) calls in
 * place of the cited reference function.
 *
 * Conventions
 *  - All array arguments are DEVICE pointers owned by the caller, FP64 unless
 *    stated. Vector fields are stacked component-major [u; v; (w)] of length
 *    ndim*nn, exactly as in the reference.
 *  - Every call is asynchronous on the given stream and returns an int status:
 *    FEM_OK or a negative FEM_E_* code for argument / CUDA errors detected at
 *    launch. Solver outcomes (iterations, convergence flags) are written to
 *    device memory (int32), like the reference's device-array iteration counts.
 *  - Connectivity is implicit: meshes are the structured lattices of
 *    setup/regular_mesh.py and kernels compute nconn on the fly.
 *  - A context owns its mesh-resident data and solver workspace (allocated at
 *    create / setup time, never on the solve path). One context is driven by
 *    one stream at a time.
 */
#ifndef FEM_B200_H
#define FEM_B200_H

#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FEM_OK 0
#define FEM_E_ARG (-1)
#define FEM_E_CUDA (-2)
#define FEM_E_OOM (-3)
#define FEM_E_STATE (-4)

/* element families */
#define FEM_KIND_Q1_2D 0 /* quad4  */
#define FEM_KIND_Q2_2D 1 /* quad9  */
#define FEM_KIND_HEX8 2  /* hex8   */
/* shape-function families for fem_shape_functions */
#define FEM_SHAPE_QUAD4 0
#define FEM_SHAPE_QUAD9 1
#define FEM_SHAPE_HEX8 2
#define FEM_SHAPE_LIN2 3
#define FEM_SHAPE_LIN3 4

/* pressure preconditioners (solvers/standard.py:219-247) */
#define FEM_PREC_NONE 0
#define FEM_PREC_JACOBI 1
#define FEM_PREC_APPROX_INV 2
#define FEM_PREC_APPROX_INV_PT 3 /* solvers/passive_transport.py:141-150 variant */
#define FEM_PREC_MG 4

/* solver status bits written to the device status word */
#define FEM_STATUS_BARRIER_TIMEOUT 1
#define FEM_STATUS_NONFINITE 2
#define FEM_STATUS_MAXITER 4
#define FEM_STATUS_BREAKDOWN 8
#define FEM_STATUS_WATCHDOG 32 /* a solve exceeded its 10 s device-side wall budget */

typedef struct fem_mesh_desc {
  int kind;     /* FEM_KIND_* */
  int periodic; /* 2D only */
  int nex, ney, nez;
  double lx, ly, lz;
} fem_mesh_desc;

typedef struct fem_ctx fem_ctx;

/* ---------------------------------------------------------------- mesh ---- */

/* Node/element counts of a mesh (host only). */
int fem_mesh_counts(const fem_mesh_desc* mesh, int* nn, int* ne, int* nen);

/* Node coordinates (nn x dim) and connectivity (ne x nen, int64).
 * Replaces setup/regular_mesh.py:6 create_mesh_2d, :46 create_mesh_3d,
 * :108 create_mesh_2d_quad9, :150 create_periodic_mesh_2d,
 * :183 create_periodic_mesh_2d_quad9. */
int fem_mesh_generate(const fem_mesh_desc* mesh, double* node_coords, int64_t* nconn, cudaStream_t stream);

/* Gauss-point data wq (q), N (q x I), Nderiv (q x dim x I) of one element
 * with nodal coordinates coords (I x dim). Replaces core/shape_functions.py:11
 * lin2, :27 quad4, :47 hex8, :89 lin3, :108 quad9 *_shape_functions. */
int fem_shape_functions(int family, const double* coords, double* wq, double* N, double* Nderiv,
                        cudaStream_t stream);

/* ------------------------------------------------------------- context ---- */

/* Create a context for a mesh: evaluates shape functions on element 0 and the
 * shared element matrices Me, Le, Ge, the lumped mass M (ndim*nn) and diag(L)
 * (core/element_calc.py:9 lumped_mass_matrix, :27 laplacian_element_calc,
 * :34 gradient_element_calc, :99 laplacian_diag; solvers/standard.py:211-214),
 * all on the device. */
int fem_ctx_create(const fem_mesh_desc* mesh, int device, fem_ctx** out);
void fem_ctx_destroy(fem_ctx* ctx);

/* nn, ne, nen, ndim, nq of the context mesh (host). */
int fem_ctx_dims(const fem_ctx* ctx, int* nn, int* ne, int* nen, int* ndim, int* nq);

/* Copy the element data out (device pointers, any may be NULL):
 * wq (nq), N (nq*nen), Nderiv (nq*ndim*nen), Me, Le (nen*nen), Ge (ndim*nen*nen),
 * M_lumped (ndim*nn), L_diag (nn). */
int fem_ctx_element_data(const fem_ctx* ctx, double* wq, double* N, double* Nderiv, double* Me, double* Le,
                         double* Ge, double* M_lumped, double* L_diag, cudaStream_t stream);

/* Boundary sets. dmask: uint8 (ndim*nn), 1 on gamma_d entries
 * (setup/simulation.py:169-173). pmask: uint8 (nn), 1 on gamma_p nodes (outlet
 * nodes, or node 0 when there is no outlet: setup/simulation.py:178-181).
 * set_zeroP selects pinned (1) or mean-zero (0) pressure (StandardSolverConfig). */
int fem_ctx_set_bc(fem_ctx* ctx, const uint8_t* dmask, const uint8_t* pmask, int set_zeroP, cudaStream_t stream);

/* Multigrid hierarchy (core/multigrid.py:9-88): nlev levels obtained by halving
 * nex, ney; level_pmasks is the concatenation over levels of the uint8 gamma_p
 * masks of each level mesh (NULL: node 0 of every level). coarse_tol is the
 * coarsest-level CG tolerance (the reference passes solver_tol).
 * hex8 meshes (an extension: the reference refuses 3D multigrid,
 * setup/simulation.py:75-76) get the 3D form of the scheme: every axis halved
 * per level (nex, ney, nez divisible by 2^(nlev-1)), trilinear prolongation
 * and R = P^T, a degree-3 Chebyshev smoother on D^-1 A with its interval from
 * a power-iteration estimate of lambda_max, and the coarsest level (at most
 * 4096 nodes) solved exactly by its inverse, formed on the device here;
 * coarse_tol is then unused. Pinned pressure only. */
int fem_ctx_setup_multigrid(fem_ctx* ctx, int nlev, const uint8_t* level_pmasks, double coarse_tol,
                            cudaStream_t stream);

/* Level metadata of the hierarchy: nn and full lattice extents per level. */
int fem_ctx_level_info(const fem_ctx* ctx, int level, int* nn, int* nnx_full, int* nny_full, int* nex, int* ney);

/* ---------------------------------------------------- element products ---- */

/* y_c = sum_e P_e^T (alpha*A + beta*B_e (B_e^T if transB) + gamma*C_e) P_e x_c
 * for c < ncomp (x_c = x + c*nn). A: shared nen x nen, B/C: per element
 * (ne x nen x nen); any may be NULL. Covers core/element_mult.py:11
 * consistent_mass_mult, :38 laplacian_element_mult, :79 visc_conv_mult,
 * :106 stabilized_visc_conv_mult, :159 scalar_visc_conv_mult,
 * :174 scalar_stabilized_visc_conv_mult, :190 scalar_consistent_mass_SUPG_mult. */
int fem_ebe_apply(fem_ctx* ctx, int ncomp, const double* x, double* y, double alpha, const double* A, double beta,
                  const double* B, int transB, double gamma, const double* C, cudaStream_t stream);

/* y = [G_1 P; ...; G_ndim P] (core/element_mult.py:51 gradient_element_mult). */
int fem_grad_apply(fem_ctx* ctx, const double* P, const double* Ge, double* y, cudaStream_t stream);

/* y = sum_i G_i^T u_i (core/element_mult.py:133 divergence_element_mult). */
int fem_div_apply(fem_ctx* ctx, const double* U, const double* Ge, double* y, cudaStream_t stream);

/* Quadrature arguments: wq (q), N (q x I), Nderiv (q x dim x I) of the element
 * (the reference evaluates them on element 0); NULL selects the context's own. */

/* Ce (ne x nen x nen) from U (core/element_calc.py:165 conservative_convec_elem_calc). */
int fem_convection_build(fem_ctx* ctx, const double* U, double beta, const double* wq, const double* N,
                         const double* Nderiv, double* Ce, cudaStream_t stream);

/* Ctau_tilde (ne x nen x nen) (core/element_calc.py:188 Ctau_tilde_elem_calc). */
int fem_ctau_tilde_build(fem_ctx* ctx, const double* U, const double* wq, const double* N, const double* Nderiv,
                         double* Ct, cudaStream_t stream);

/* Vector-Jacobian product of the convection operator in its velocity:
 * y = d/dU <a, Ce(U) b>, y (ndim*nn), for a, b of ncomp components (ncomp*nn,
 * Ce acting on each) with the divergence weight beta (Ce of
 * core/element_calc.py:165 conservative_convec_elem_calc). Ce is linear in U,
 * so y does not depend on U. Deterministic (per-node sums in a fixed order).
 * No reference counterpart: the reference gets it from jax.grad. */
int fem_conv_vjp(fem_ctx* ctx, int ncomp, const double* a, const double* b, double beta, double* y,
                 cudaStream_t stream);

/* The velocity-dependent element matrices of the passive-scalar step
 * (solvers/passive_transport.py:80-88 feeding :14-62): the lhs operator is
 * K_A + E_k and the rhs operator K_B + B_k with the shared K_A = Me/dt + (D/2) Le,
 * K_B = Me/dt - (D/2) Le and
 *   SUPG:  E_k = Mtau/dt + (Ce(U) + Ctau)/2,  B_k = Mtau/dt - (Ce(U_n) + Ctau)/2
 *   plain: E_k = Ce(U)/2,                     B_k = -Ce(U_n)/2
 * Ek, Bk: ne * nen * nen each, element-major; transpose != 0 writes each
 * element's block transposed (what the adjoint's transposed solve applies). */
int fem_transport_elements(fem_ctx* ctx, const double* U_n, const double* U, double dt, double D, int supg,
                           int transpose, double* Ek, double* Bk, cudaStream_t stream);

/* Velocity side of the adjoint of the passive-scalar step (2D): for
 * s = <lam, B(U_n) phi_n - E(U_n, U) phi>, with E, B the step's lhs and rhs
 * operators without their shared parts (solvers/passive_transport.py:14-97;
 * SUPG with supg != 0: Ce(U), Ctau = tau Ct(U_n), Mtau = tau Ce(U_n)^T and tau
 * of core/element_calc.py:165-229), gUn = ds/dU_n and gU = ds/dU (2*nn each).
 * lam is the adjoint solve's solution with its Dirichlet rows zeroed. No
 * reference counterpart: the reference gets it from jax.grad. */
int fem_transport_vjp(fem_ctx* ctx, const double* U_n, const double* U, const double* lam, const double* phi_n,
                      const double* phi, double dt, double D, int supg, double* gU_n, double* gU,
                      cudaStream_t stream);

/* Per-element SUPG tau (core/element_calc.py:202 calculate_tau). */
int fem_supg_tau(fem_ctx* ctx, const double* U, const double* Ce, const double* Ct, double D, double dt, double r,
                 const double* N, double* tau, cudaStream_t stream);

/* Shared element matrices from quadrature data (nq points, nen nodes, dim):
 * Me = sum_q w N(x)N (core/element_calc.py:13), Le = sum_q w dN^T dN (:27-32),
 * Ge[i] = sum_q w N (x) dN_i (:34-40). Any output may be NULL except scratch
 * use: Le_off (nen x nen) receives Le with a zero diagonal (core/multigrid.py:66). */
int fem_element_matrices(int nq, int nen, int dim, const double* wq, const double* N, const double* Nderiv,
                         double* Me, double* Le, double* Le_off, double* Ge, cudaStream_t stream);

/* Assembled diagonals on the context mesh: M = assemble(rowsum(Me)) tiled
 * ndim times (core/element_calc.py:9-25) and L_diag = assemble(diag(Le))
 * (:99-109). Me / Le may be NULL (skip that output). */
int fem_assemble_diag(fem_ctx* ctx, const double* Me, const double* Le, int ndim, double* M, double* L_diag,
                      cudaStream_t stream);

/* ------------------------------------------------------------ multigrid ---- */

/* Lattice-bilinear prolongation of xH on the (nnH_x, nnH_y) lattice to the
 * (nnh_x, nnh_y) lattice; extents include the periodic duplicate row/column
 * (core/multigrid.py:90 interpolation_operator). */
int fem_lattice_interpolate(int nnH_x, int nnH_y, int nnh_x, int nnh_y, int periodic, const double* xH, double* xh,
                            cudaStream_t stream);
/* Restriction R = I^T (core/multigrid.py:142 restriction_operator). */
int fem_lattice_restrict(int nnh_x, int nnh_y, int nnH_x, int nnH_y, int periodic, const double* xh, double* xH,
                         cudaStream_t stream);
/* z = one V-cycle applied to r (core/multigrid.py:231 v_cycle). */
int fem_mg_vcycle(fem_ctx* ctx, const double* r, double* z, cudaStream_t stream);

/* -------------------------------------------------------------- solvers ---- */

/* Pressure Poisson solve by (P)CG on the context Laplacian, one persistent
 * launch (solvers/standard.py:85 solve_pressure with utils/
 * jax_iterative_solvers.py:214 cg). Pinned rows (set_zeroP) or mean-zero
 * handling follow the context's boundary setup. center_rhs subtracts mean(b)
 * first; post applies the final pin/mean fix of solve_pressure. x holds x0 on
 * entry and the solution on exit. iters/status: device int32.
 * On hex8 with FEM_PREC_MG the solve is the same CG (stop rule, iteration
 * count) preconditioned by the hex8 V-cycle, run as one CUDA graph whose loop
 * condition is evaluated on the device; pinned pressure only, and the stream
 * must not be capturing (FEM_E_STATE). */
int fem_pressure_solve(fem_ctx* ctx, const double* b, double* x, double tol, double atol, int maxiter, int precond,
                       int center_rhs, int post, int* iters, int* status, cudaStream_t stream);

/* General EBE-operator BiCGSTAB (utils/jax_iterative_solvers.py:685 bicgstab)
 * on A = alpha*Ash + beta*B_e + gamma*C_e with identity rows where mask != 0
 * (solvers/standard.py:20-28 lhs_operator). ncomp components share the element
 * matrices; mask (uint8, ncomp*nn) may be NULL. maxiter <= 0 selects the
 * reference default 10*size. x holds x0 on entry, the solution on exit;
 * iters is the reference's iteration count (negative on breakdown). */
int fem_bicgstab_solve(fem_ctx* ctx, int ncomp, double alpha, const double* Ash, double beta, const double* B,
                       double gamma, const double* C, const uint8_t* mask, const double* b, double* x, double tol,
                       double atol, int maxiter, int* iters, int* status, cudaStream_t stream);

/* Precision of fem_step4's solves: FEM_PRECISION_FP64 (default, the
 * reference's FP64 solvers) or FEM_PRECISION_MIXED. Mixed: the multigrid
 * pressure solve is fem_pressure_solve_mixed's scheme (FP64 refinement,
 * `inner` FP32 multigrid-PCG iterations per cycle, at most max_cycles cycles;
 * iters[1] receives the cycle count), and on 2D meshes the momentum solve is
 * FP64 refinement around 3 FP32 BiCGSTAB iterations per cycle with FP32 Gauss
 * factors of the convection (iters[0] receives the cycle count). Each mixed
 * solve is one CUDA graph with a device-side loop, so a mixed step cannot be
 * captured (FEM_E_STATE on a capturing stream). Needs the multigrid pressure
 * preconditioner. No reference counterpart: the reference solves in FP64 only. */
#define FEM_PRECISION_FP64 0
#define FEM_PRECISION_MIXED 1
int fem_ctx_set_precision(fem_ctx* ctx, int precision, int inner, int max_cycles);

/* One 4-step projection time step (solvers/standard.py:148 four_step_timestep
 * as called by setup_solver.timestep_loaded :264): Ce(U_n), momentum
 * BiCGSTAB, U*, pressure PCG, projection, Dirichlet values. U_d_full is the
 * ndim*nn vector holding U_d on gamma_d entries; F_p (nn) and F (ndim*nn) may
 * be NULL for zero. iters: device int32[2] = {U_iters, P_iters}. */
int fem_step4(fem_ctx* ctx, const double* U_n, const double* P_n, double dt, double rho, double mu,
              const double* U_d_full, const double* F_p, const double* F, double tol, int precond, double* U_out,
              double* P_out, int* iters, int* status, cudaStream_t stream);

/* Passive-scalar step after the NS step (solvers/passive_transport.py:64
 * timestep, phi part :80-95): builds Ce(U_n, 1), Ce(U, 1) and, with supg,
 * Ctau_tilde/tau, then BiCGSTAB for phi. phi_mask (uint8 nn) / phi_d_full may
 * be NULL. iters: device int32 (phi iterations). */
int fem_transport_phi(fem_ctx* ctx, const double* U_n, const double* U, const double* phi_n, double dt, double D,
                      int supg, const uint8_t* phi_mask, const double* phi_d_full, double tol, double* phi_out,
                      int* iters, int* status, cudaStream_t stream);

/* F_p = int_Gamma_d q (u_d . n) over the boundary edges/faces listed in bconn
 * (nb x I, int32, I = 2 lin2, 3 lin3, 4 quad4 faces) with outward normals nvec
 * (nb x dim) and Dirichlet values at their nodes U_b (ndim*nn, full vector)
 * (core/element_calc.py:111 u_dot_n_boundary_integral_1d, :137 _2d). quad4
 * faces belong to the axis-aligned hex8 lattice: their in-plane axes are the
 * two other than the normal's largest component. The assembly runs
 * node-parallel: a node -> face-entry table is built on the device on every
 * call, and each node sums its entries in face order. The result is bitwise
 * that of a serial scatter in face order (the reference's segment_sum order).
 * A face that names a node outside [0, nn) is skipped (nothing of it is read
 * or written); fem_boundary_flux_skipped reports how many were. */
int fem_boundary_flux(fem_ctx* ctx, const int32_t* bconn, const double* nvec, int nb, int nodes_per_face,
                      const double* U_full, double* F_p, cudaStream_t stream);

/* Number of faces the last fem_boundary_flux / fem_boundary_flux_noalloc call
 * on ctx skipped because they named a node outside [0, nn); 0 for valid input.
 * Waits for `stream` (the stream of that call). No reference counterpart: the
 * reference's segment_sum drops out-of-range segment ids without a report. */
int fem_boundary_flux_skipped(fem_ctx* ctx, int* count, cudaStream_t stream);

/* Same result as fem_boundary_flux, but the call never allocates or frees
 * device memory. No counterpart in the reference: the reference has one
 * boundary integral and leaves device memory to XLA.
 *
 * fem_boundary_flux keeps its scratch in the context: nb * nodes_per_face
 * doubles and as many ints per face entry, plus 2 nn + 1 ints for the node
 * table. When a larger boundary arrives, it grows that scratch with a stream
 * synchronize, cudaFree and cudaMalloc, and cudaFree synchronizes the whole
 * device. Some callers cannot do that: a host framework whose handlers must
 * take every device byte from the framework's own allocator, or a
 * time-stepping loop that must not stall the device when its set of boundary
 * faces changes. This entry point is for them. Its scratch is one fixed
 * structure inside this library (the face values plus the tables of the
 * node-parallel assembly, whose node table is a hash table of
 * 2 * FEM_NOALLOC_FACE_VALUES slots rather than nn entries; 2.9 MB), one copy
 * per device, held by every GPU that loads the library until the process
 * exits. The work is the same node-parallel gather as fem_boundary_flux's, and
 * the flux is bitwise the same.
 *  - nb * nodes_per_face must be <= FEM_NOALLOC_FACE_VALUES (for example 32768
 *    lin2 edges or 16384 quad4 faces). Larger requests return FEM_E_ARG with
 *    the limit in fem_last_error(), and nothing is launched.
 *  - The calling thread's current device must be ctx's device (else
 *    FEM_E_STATE). The first call on each device looks up that device's copy
 *    of the structure (cudaGetSymbolAddress, which may load the library's
 *    device code). Make that first call before any stream capture begins.
 *  - Nothing has to start at zero: each call clears the tables it counts in
 *    and writes every other scratch value it reads, on `stream`, before
 *    reading it.
 *  - All calls on one device share the one structure, and it keeps the last
 *    call's contents. Two calls that can overlap on the GPU (different streams
 *    with no event between them, or different host threads) race on it and
 *    may return wrong fluxes: order them on one stream. */
#define FEM_NOALLOC_FACE_VALUES 65536
int fem_boundary_flux_noalloc(fem_ctx* ctx, const int32_t* bconn, const double* nvec, int nb,
                              int nodes_per_face, const double* U_full, double* F_p, cudaStream_t stream);

/* out[idx[k]] = vals[k] for k < n (idx int64; vals NULL writes `value`),
 * the functional x.at[idx].set(v) of the reference. */
int fem_scatter(const int64_t* idx, const double* vals, double value, int n, double* out, cudaStream_t stream);
/* mask[idx[k]] = 1 for k < n (mask uint8, cleared to len first). */
int fem_make_mask(const int64_t* idx, int n, int len, uint8_t* mask, cudaStream_t stream);

/* Deterministic dot product and axpby helpers used by host-driven generic
 * solver loops: out[0] = x . y (device), y = a*x + b*y. */
int fem_dot(fem_ctx* ctx, const double* x, const double* y, int n, double* out, cudaStream_t stream);
int fem_axpby(fem_ctx* ctx, double a, const double* x, double b, double* y, int n, cudaStream_t stream);

/* Stage timing of fem_step4 / fem_transport_phi. When enabled, the context
 * records a CUDA event on the call's stream before each stage (Ce build,
 * momentum rhs, momentum BiCGSTAB, U*, PPE rhs, pressure PCG, projection) and
 * after the last. fem_ctx_stage_times synchronizes on the last event and writes
 * up to max_n stage durations in ms; it returns the number written (or < 0). */
int fem_ctx_enable_timing(fem_ctx* ctx, int enable);
int fem_ctx_stage_times(fem_ctx* ctx, float* ms, int max_n);

/* Barrier trace of the persistent solver kernels (diagnostics): when set,
 * CTA 0 appends the %globaltimer value (ns) at every grid-barrier exit to
 * buf[1..cap-1] and keeps the count in buf[0] (the caller zeroes buf[0]).
 * cap = 0 disables tracing. */
int fem_ctx_set_trace(fem_ctx* ctx, unsigned long long* buf, int cap);

/* Cap on the CTAs of this context's persistent cooperative launches (the PCG,
 * V-cycle and BiCGSTAB solver kernels); ctas = 0 restores the co-resident
 * capacity found at create, and ctas above it is clamped to it. *capacity
 * (optional) receives that capacity (SMs x resident solver CTAs per SM). A
 * request loop that runs several contexts at once on separate streams gives
 * each a share of the capacity, so every cooperative grid in flight fits on
 * the device at the same time. Results depend on the cap (the reduction
 * partials are per CTA) and are reproducible for a given cap. No reference
 * counterpart: the reference runs one problem at a time. */
int fem_ctx_set_max_ctas(fem_ctx* ctx, int ctas, int* capacity);

/* nsteps (even, >= 2) consecutive fem_step4 calls captured into one CUDA
 * graph: step k reads (U0,P0) and writes (U1,P1) for even k and the reverse
 * for odd k, so after a launch the result is back in (U0,P0). Every argument
 * has fem_step4's meaning and is fixed in the graph (pointers and scalars): a
 * new dt or mu needs a new graph. iters / status receive each step's values
 * (the last step's remain). Nothing runs at capture; fem_graph_launch replays
 * the steps on any stream, fem_graph_destroy frees the graph. The context must
 * not have stage timing enabled (FEM_E_STATE). A graph and direct calls on the
 * same context must not overlap, as for two direct calls. No reference
 * counterpart: it replaces the host launches of a chunk of time steps. */
typedef struct fem_graph fem_graph;
int fem_step4_graph(fem_ctx* ctx, double* U0, double* P0, double* U1, double* P1, double dt, double rho, double mu,
                    const double* Ud, const double* Fp, const double* F, double tol, int precond, int nsteps,
                    int* iters, int* status, fem_graph** out);
int fem_graph_launch(fem_graph* graph, cudaStream_t stream);
int fem_graph_destroy(fem_graph* graph);

/* Mixed-precision pressure-Poisson solve of the context's pinned Q1 2D or hex8 problem
 * (the system of fem_pressure_solve with FEM_PREC_MG: gamma_p rows zeroed).
 * FP64 iterative refinement, x += d after each cycle, until
 * ||b - A x|| <= tol ||b|| or max_cycles cycles. The inner solve is `inner`
 * iterations of a multigrid-preconditioned CG on FP32 vectors from d = 0; its
 * coarsest level is solved in FP64. x (FP64, device) holds the initial guess on
 * entry and is zeroed on gamma_p at the end. *cycles and *relres (host) receive
 * the cycle count and the final relative FP64 residual; the call waits for the
 * stream once per cycle to read the residual norm. It needs the context's
 * multigrid hierarchy (fem_ctx_setup_multigrid) with a coarsest level of at most
 * 128 nodes (FEM_E_STATE otherwise), and allocates its FP32 work vectors on the
 * first call. On hex8 the inner solve uses the hex8 V-cycle (Chebyshev
 * smoother, FP32 vectors, FP64 sums and FP64 coarsest solve) and the whole
 * refinement loop is one CUDA graph with a device-side loop condition; the
 * call then waits for the stream once, at the end. No reference counterpart:
 * the reference solves in FP64 only. */
int fem_pressure_solve_mixed(fem_ctx* ctx, const double* b, double* x, double tol, int inner, int max_cycles,
                             int* cycles, double* relres, cudaStream_t stream);

/* Self-test of failure detection (diagnostics, about 2 s on the GPU): one
 * CTA waits at the solvers' grid barrier for a party that never arrives, so
 * the wait ends only by the barrier's time limit, which sets the timeout bit
 * of the context's error word and returns, as in a solver. *status (device
 * int) receives FEM_STATUS_BARRIER_TIMEOUT; the context stays usable, since
 * every solve clears the error word first. No reference counterpart (the
 * reference has no device-side waits). */
int fem_selftest_barrier_timeout(fem_ctx* ctx, int* status, cudaStream_t stream);

/* Number of this library's kernel launches issued so far in this process. */
long long fem_launch_count(void);

/* Last CUDA error string recorded by the library (host, static storage). */
const char* fem_last_error(void);

/* Packed steps (serving): k contexts of one mesh size advanced together, one
 * persistent cooperative launch per call. Member m is the context ctxs[m]
 * (Q1 2D, multigrid hierarchy, pinned pressure, on-the-fly convection, FP64
 * precision) with its ping-pong fields (U[0], P[0]) = (U0[m], P0[m]) and
 * (U[1], P[1]) = (U1[m], P1[m]) and its Dirichlet values Ud[m]; every member's
 * cooperative CTA count (its max-CTA cap, fem_ctx_set_max_ctas) must be the
 * same and fit on the device (FEM_E_STATE otherwise); the members active in
 * one call must fit together. stat: device int32 [k * 5], per member the momentum and
 * pressure iterations of its last step, their statuses, and at [5m + 4] the
 * OR of every status since the caller last zeroed it. tol and precond have
 * fem_step4's meaning. Each member's step is fem_step4's on the same CTA count
 * (solvers/standard.py:148-165, rho = 1), bit for bit. No reference
 * counterpart: the reference runs one problem at a time. */
typedef struct fem_pack fem_pack;
int fem_pack_create(fem_ctx* const* ctxs, int k, double* const* U0, double* const* P0, double* const* U1,
                    double* const* P1, const double* const* Ud, int* stat, double tol, int precond,
                    fem_pack** out);
/* steps[m] steps of member m (0: idle this call) from buffer cur[m] (0 or 1)
 * with its dt[m] and viscosity mu[m] (host arrays of k values, read before
 * the call returns); the result of member m is in buffer cur[m] ^ (steps[m] & 1).
 * Only the members with steps[m] > 0 are launched, so the launch holds
 * (active members) x ctas CTAs.
 * Calls on one pack run in stream order; a member's buffers may be written by
 * the caller between calls on the same stream. */
int fem_pack_step(fem_pack* pack, const double* dt, const double* mu, const int* steps, const int* cur,
                  cudaStream_t stream);
/* Members and CTAs per member of a pack; the device's capacity for one packed
 * launch (SMs x resident CTAs per SM of the packed kernel). */
int fem_pack_info(const fem_pack* pack, int* k, int* ctas, int* capacity);
int fem_pack_destroy(fem_pack* pack);

#ifdef __cplusplus
}
#endif
#endif /* FEM_B200_H */
