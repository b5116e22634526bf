// Kernel argument structs and host launcher declarations of libfemb200.
#pragma once
#include <stdint.h>
#include "fem_solvers.cuh"
#include "fem_conv.cuh"
#include "fem_conv3.cuh"

#define FEM_THREADS 512
#define FEM_OP_THREADS 256
// whole dynamic smem of k_cg / k_vcycle: reduction scratch + tile staging + stencil tables
#define FEM_DYN_SMEM_MAX ((128 + FEM_TILE_SMEM + FEM_TAB_SMEM + FEM_BLK_SMEM) * 8)
// coarse multigrid levels: at most FEM_MG_TEAM CTAs, levels of at most
// FEM_MG_TEAM_NN nodes (both can be overridden by the environment variables of
// the same names)
#define FEM_MG_TEAM 16
#define FEM_MG_TEAM_NN 4096

struct BiArgs {
  FemSync sync;
  FemGrid g;
  MatCombo op;
  const uint8_t* mask;  // ncomp*nn identity rows, or null
  const double* b;
  double* x;
  double *r, *rhat, *p0, *p1, *q0, *q1, *t;
  double tol, atol;
  int maxiter;
  int* iters;
  int* status;
  // convection applied from Gauss-point factors (fem_conv.cuh) instead of op.B:
  // op.B is then unused and the operator is op.alpha op.A + cv_coef Ce
  const double* cvf;
  double cv_coef;
  FemQuadTab qt;
};

struct StepArgs {
  FemGrid g;
  int ndim;
  double dt, rho, mu, theta;
  const double *Me, *Le, *Ge, *M;  // shared element matrices and lumped mass
  const double* Ce;
  const double* vcv;                // if set: (mu Le + rho Ce) U_n, precomputed (Ce is then unused)
  const uint8_t* dmask;             // ndim*nn
  const uint8_t* pmask;             // nn (pinned pressure)
  int pinned;
  // hex8: assembled stencil tables (FEM_TAB_MAX doubles apart) of Me, Ge_x, Ge_y,
  // Ge_z and their transposes, used by the step bodies instead of per-node
  // element gathers; null: gathers
  const double* tab3 = nullptr;
};

// One request of a packed step launch (k_pack.cu): the device pointers and
// solver arguments of its context, built once per pack. The 4-step step of
// fem_step4 (Q1, pinned multigrid pressure, on-the-fly convection, FP64).
struct PackMember {
  StepArgs S;  // dt and mu come from the launch's PackStep
  BiArgs B;    // momentum solve: x = Uhat, b = rhsU; its shared matrix is built in smem
  CgArgs C;    // pressure solve: b = rhsP; x is the step's output pressure
  double* U[2];
  double* P[2];
  const double* Ud;
  double *cvf, *vcv, *rhsU, *Uhat, *gPn, *Ustar, *rhsP;
  double *cr, *cp, *cq;
  int* stat;  // [0..1] iterations, [2..3] statuses of the last step (momentum, pressure), [4] OR of all statuses
};
#define FEM_PACK_MAX 64
struct PackStep {
  double dt, mu;
  int steps;  // steps of this launch (0: the member is idle)
  int cur;    // buffer (0 or 1) holding the member's current U, P
};
struct PackParams {
  PackStep m[FEM_PACK_MAX];  // per member
  int idx[FEM_PACK_MAX];     // member of each grid row (blockIdx.y): only the active ones are launched
};

// ----------------------------------------------------------------------------
// Host launchers (one translation unit per kernel family; fem_capi.cu drives them)
// ----------------------------------------------------------------------------
int fem_after_launch(const char* what);  // records launch count / error; 0 or FEM_E_CUDA
int fem_cuda_error(const char* where, cudaError_t e);  // records e for fem_last_error; FEM_E_CUDA
char* fem_err_buf();  // the calling thread's fem_last_error buffer (256 bytes)

int fem_launch_mesh_generate(const FemGrid& g, double dx, double dy, double dz, double* coords, int64_t* nconn,
                             cudaStream_t s);
int fem_launch_shape_functions(int family, const double* coords, double* wq, double* N, double* dN, cudaStream_t s);
int fem_launch_element_matrices(int nq, int nen, int dim, const double* wq, const double* N, const double* dN,
                                double* Me, double* Le, double* Leoff, double* Ge, cudaStream_t s);
int fem_launch_assemble_diag(const FemGrid& g, int ndim, const double* Me, const double* Le, double* M, double* Ldiag,
                             cudaStream_t s);
int fem_launch_stencil_build(const FemGrid& g, const double* A, int transpose, int skip_diag, double* out,
                             cudaStream_t s);
int fem_launch_invdiag(int n, const double* D, const uint8_t* pin, double* invD, double* winvD, cudaStream_t s);
int fem_launch_level_sums(const FemGrid& g, const FemLattice& lat, const double* diag, double* out, cudaStream_t s);

int fem_launch_ebe(int ncomp, const FemGrid& g, const MatCombo& m, const double* x, double* y, cudaStream_t s);
// y = alpha A x per component for one shared element matrix A, as its assembled
// stencil (tab: FEM_TAB_MAX doubles of scratch, used by the 3D kind)
int fem_launch_shared_apply(int ncomp, const FemGrid& g, const double* A, double* tab, double alpha, const double* x,
                            double* y, int sms, cudaStream_t s);
int fem_launch_grad(int ndim, const FemGrid& g, const double* Ge, const double* P, double* y, cudaStream_t s);
int fem_launch_div(int ndim, const FemGrid& g, const double* Ge, const double* U, double* y, cudaStream_t s);
int fem_launch_convection(const FemGrid& g, const FemQuad& Q, const double* U, double beta, int mode, double* out,
                          cudaStream_t s);
int fem_launch_supg_tau(const FemGrid& g, const FemQuad& Q, const double* U, const double* Ce, const double* Ct,
                        double D, double dt, double r, double* tau, cudaStream_t s);
int fem_launch_scale_elem(int ne, int nen, const double* tau, const double* X, int trans, double* out, cudaStream_t s);
// out = s_m Mt + s_c (C + Ct); transpose_nen = nen writes each element block transposed, 0 as is
int fem_launch_elem_combine(size_t n, double s_m, const double* Mt, double s_c, const double* C, const double* Ct,
                            double* out, int transpose_nen, cudaStream_t s);
int fem_launch_lincomb(int n, double a, const double* X, double b, const double* Y, double* out, cudaStream_t s);
int fem_launch_interp(const FemLattice& H, const FemLattice& h, const double* xH, double* xh, cudaStream_t s);
int fem_launch_restrict(const FemLattice& h, const FemLattice& H, const double* xh, double* xH, cudaStream_t s);
// Boundary flux (core/element_calc.py:111-163) assembled per node in face
// order through a node -> entry CSR in cnt (nn ints), off (nn + 1) and list
// (nb * npf); faces naming a node outside [0, nn) are skipped and counted in
// *skipped.
int fem_launch_boundary_csr(const double* coords, int dim, const int32_t* bconn, const double* nvec, int nb, int npf,
                            const double* U, int nn, double* Fe, int* cnt, int* off, int* list, int* skipped,
                            double* Fp, cudaStream_t s);
// The same result with tables of a fixed size: the CSR is indexed by the slots
// of a hash table of `cap` node ids (a power of two >= 2 nb npf) instead of by
// node, so nothing depends on nn.
struct FemBoundaryHash {
  int cap;
  double* Fe;    // nb * npf
  int* keys;     // cap
  int* cnt;      // cap
  int* off;      // cap + 1
  int* slot;     // nb * npf
  int* list;     // nb * npf
  int* skipped;  // 1
};
int fem_launch_boundary_hash(const double* coords, int dim, const int32_t* bconn, const double* nvec, int nb, int npf,
                             const double* U, int nn, const FemBoundaryHash& H, double* Fp, cudaStream_t s);
int fem_launch_dot(const double* x, const double* y, int n, double* part, double* out, cudaStream_t s);
int fem_launch_axpby(double a, const double* x, double b, double* y, int n, cudaStream_t s);
int fem_launch_scatter(const int64_t* idx, const double* vals, double value, int n, double* out, cudaStream_t s);
int fem_launch_make_mask(const int64_t* idx, int n, int len, uint8_t* mask, cudaStream_t s);

int fem_launch_conv_factors(const FemGrid& g, const FemQuadTab& qt, const double* U, double bd, double* fq,
                            cudaStream_t s);
int fem_launch_conv_apply(int ncomp, const FemGrid& g, const FemQuadTab& qt, const double* fq, double cc,
                          double alpha, const double* Ash, const double* x, double* y, int grid, cudaStream_t s);
// y = d/dU <a, Ce(U) b> over ncomp components of a and b (ge: ne * dim * nen scratch)
int fem_launch_conv_vjp(const FemGrid& g, const FemQuadTab& qt, int ncomp, const double* a, const double* b,
                        double beta, double* ge, double* y, cudaStream_t s);
// velocity side of the passive-scalar step's adjoint (2D): yn = ds/dU_n, yu = ds/dU
// (ge*: ne * 2 * nen scratch each)
int fem_launch_transport_vjp(const FemGrid& g, const FemQuadTab& qt, const double* Un, const double* U,
                             const double* lam, const double* phin, const double* phi, double dt, double D, int supg,
                             double* gen, double* geu, double* yn, double* yu, cudaStream_t s);
// hex8: the Gauss-point factors (32 per element, element-major) and
// y = alpha Ash x + cc Ce x per component (3 components) from them
int fem_launch_conv_factors3(const FemGrid& g, const FemQuadTab& qt, const double* U, double bd, double* fq,
                             cudaStream_t s);
int fem_launch_conv_apply3(const FemGrid& g, const FemQuadTab& qt, const double* fq, double cc, double alpha,
                           const double* Ash, const double* x, double* y, int grid, int* err, cudaStream_t s);

// hex8, 3 components: y = (alpha A + beta B_e) x, element-centric (B per element, not transposed, no C)
int fem_launch_ebe3e(const FemGrid& g, const MatCombo& m, const double* x, double* y, int grid, cudaStream_t s);

int fem_launch_selftest_barrier(const FemSync& sync, int* status, cudaStream_t s);
// mixed-precision pinned Poisson solve (k_mixed.cu); work: 6 sum(nn_l) + 3 nn_0
// floats, dwork: grid + 8 doubles
struct MxGraphCache {
  cudaGraphExec_t exec = nullptr;  // captured inner solve of a context
  int inner = 0;
};
int fem_mixed_poisson(const CgArgs& A, int grid, float* work, double* dwork, const double* b, double* x, double tol,
                      int inner, int max_cycles, int* cycles, double* relres, cudaStream_t s, MxGraphCache* gc,
                      cudaStream_t cap);

// mixed-precision momentum solve of the 2D on-the-fly step (k_mixmom.cu)
struct MixMom;
int mixmom_create(MixMom** out, const FemGrid& g, int ncomp, int nq, int sms);
void mixmom_destroy(MixMom* M);
int mixmom_solve(MixMom* M, const FemQuadTab& qt, const double* fq64, const double* Kd, double cc,
                 const uint8_t* mask, const double* b, double* x, double tol, int inner, int max_cycles,
                 int* cycles, int* status, int sms, cudaStream_t s, cudaStream_t cs);

int fem_coop_occupancy_cg(int* occ);
int fem_coop_occupancy_bi(int* occ);
int fem_launch_cg(const CgArgs& A, int grid, double* cr, double* cp, double* cq, cudaStream_t s);
int fem_launch_vcycle(const CgArgs& A, int grid, double* cr, double* cp, double* cq, double* z, cudaStream_t s);
int fem_launch_bicgstab(int ncomp, const BiArgs& A, int grid, cudaStream_t s);
// packed step (k_pack.cu): k members of `ctas` CTAs each, one cooperative launch
int fem_launch_step_pack(int kind, const PackMember* members, const PackParams& P, int k, int ctas, int blk,
                         cudaStream_t s);
int fem_pack_occupancy(int* per_sm);

int fem_launch_mom_rhs(const StepArgs& S, const double* Un, const double* Pn, const double* Ud, const double* F,
                       double* rhs, double* x0, double* gPn, cudaStream_t s);
int fem_launch_ustar(int n, double c, const double* Uh, const double* gPn, const double* M, double* Us,
                     cudaStream_t s);
int fem_launch_p_rhs(const StepArgs& S, const double* Us, const double* Fp, const double* Pn, double* rhs, double* x0,
                     cudaStream_t s);
int fem_launch_ufinal(const StepArgs& S, const double* Us, const double* P, const double* Ud, double* U,
                      cudaStream_t s);
int fem_launch_phi_rhs(const FemGrid& g, const double* Me, const double* Le, double dt, double D, const double* Mt,
                       const double* Cn, const double* Ct, const double* phin, const uint8_t* mask,
                       const double* phid, double* rhs, double* x0, cudaStream_t s);

static inline int fem_nblocks(long long n, int threads, int cap = 148 * 16) {
  long long b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}
