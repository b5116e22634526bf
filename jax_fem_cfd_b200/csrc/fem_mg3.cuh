// Hierarchy and solve state of the hex8 geometric multigrid (k_mg3.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fem_solvers.cuh"

#define MG3_DEGREE 3              // Chebyshev smoother degree
#define MG3_CHEB_LO 0.2           // smoothing interval [lo, hi] x lambda_max(D^-1 A)
#define MG3_CHEB_HI 1.1
#define MG3_POWER_ITERS 40        // power iterations per level for lambda_max
#define MG3_COARSE_MAX 4096       // largest coarsest level (nodes): its dense inverse is n^2 doubles
#define MG3_GRAPHS 4              // cached solve graphs per hierarchy

#define MG3_MODE_PCG 0
#define MG3_MODE_MIXED 1

#define MG3_CTL_PCG0 0
#define MG3_CTL_PCG 1
#define MG3_CTL_IN0 2
#define MG3_CTL_IN 3
#define MG3_CTL_MX0 4
#define MG3_CTL_MX 5

// One lattice level: node extents, the assembled 1D rows of every axis
// ([axis][class][offset + 1], class 0 first node, 1 inside, 2 last node) and
// the z-run length of a sweep work item.
struct Mg3Geo {
  int nx, ny, nz, zs;
  double k[3][3][3];
  double m[3][3][3];
};

// One 2D lattice level (quad4 / quad9, periodic or not): the grid, its full
// lattice (transfers) and the assembled stencil table of its Laplacian
// (fem_stencil.cuh).
struct Mg2Geo {
  FemGrid g;
  FemLattice lat;
  const double* tab;
};

// Level vectors of storage type T: rhs r, residual t, iterates xa / xb,
// Chebyshev direction d; invD = 1/diag(A), 0 on gamma_p.
template <class T, class G = Mg3Geo>
struct Mg3Lev {
  G geo;
  const T* invD;
  T *r, *t, *xa, *xb, *d;
};

// Device-side scalars of a solve. Inputs (set per call): tol, atol, maxiter,
// max_cycles. The rest is written by the solve.
struct Mg3Scal {
  double tol, atol;
  int maxiter, max_cycles;
  double gamma, beta, gamma_i, beta_i;
  double rr, rr0, bb, atol2, relres;
  double zbar;       // mean of the inner preconditioned residual (mean-zero problems)
  int k, cycles, status, out_iters, out_status, pad;
  unsigned long long t0;
};

struct Mg3GraphKey {
  int mode, inner, maxiter, pad;
};
struct Mg3GraphCache {
  Mg3GraphKey key{};
  cudaGraphExec_t exec = nullptr;
};

struct Mg3 {
  int nlev = 0, sms = 148, cap = 148 * 8;
  int d2 = 0;   // 2D lattice levels (geo2, m64, m32) instead of hex8 ones (geo, l64, l32)
  int mz = 0;   // mean-zero (periodic) pressure: no gamma_p, solutions centred
  Mg3Geo geo[FEM_MAX_LEVELS];
  Mg2Geo geo2[FEM_MAX_LEVELS];
  size_t off[FEM_MAX_LEVELS] = {};
  int nn[FEM_MAX_LEVELS] = {};
  size_t total = 0;
  double lam[FEM_MAX_LEVELS] = {};
  double ca[FEM_MAX_LEVELS][MG3_DEGREE] = {}, cb[FEM_MAX_LEVELS][MG3_DEGREE] = {};
  uint8_t* pin = nullptr;          // gamma_p masks of all levels (concatenated)
  double* invD64 = nullptr;
  float* invD32 = nullptr;
  double* work64 = nullptr;        // 5 vectors per level (r, t, xa, xb, d)
  float* work32 = nullptr;
  double* v64 = nullptr;           // level-0 PCG vectors p_old, p_new, Ap (+1)
  float* v32 = nullptr;            // p_old, p_new, Ap, d of the FP32 inner solve
  double *x64 = nullptr, *b64 = nullptr;  // solve input / iterate
  double* Ainv = nullptr;          // coarsest level inverse (n x n)
  double* parts = nullptr;         // 6 partial-sum slots: p.Ap, r.r, b.b, r.z, sum z, sum r
  Mg3Scal* sc = nullptr;
  double* gj = nullptr;            // setup scratch
  cudaStream_t s2 = nullptr;       // capture stream of the loop bodies
  Mg3Lev<double> l64[FEM_MAX_LEVELS];
  Mg3Lev<float> l32[FEM_MAX_LEVELS];
  Mg3Lev<double, Mg2Geo> m64[FEM_MAX_LEVELS];
  Mg3Lev<float, Mg2Geo> m32[FEM_MAX_LEVELS];
  Mg3GraphCache graphs[MG3_GRAPHS];
};

int mg3_setup(Mg3** out, int nex, int ney, int nez, double lx, double ly, double lz, int nlev,
              const uint8_t* level_pins, int sms, cudaStream_t s);
// 2D hierarchy for the mixed-precision solve over the levels of a context's
// 2D multigrid: grids, stencil tables, diagonals and gamma_p masks per level
// (pins unused when mean_zero).
int mg2_setup(Mg3** out, int nlev, const FemGrid* grids, const double* const* tabs, const double* const* diags,
              const uint8_t* const* pins, int mean_zero, int sms, cudaStream_t s);
void mg3_destroy(Mg3* M);
int mg3_vcycle64(Mg3* M, const double* r, double* z, cudaStream_t s);
int mg3_pcg(Mg3* M, const double* b, double* x, double tol, double atol, int maxiter,
            int* iters, int* status, cudaStream_t s, cudaStream_t cs);
int mg3_mixed(Mg3* M, const double* b, double* x, double tol, int inner, int max_cycles,
              int* cycles, int* status, cudaStream_t s, cudaStream_t cs);
int mg3_last_relres(Mg3* M, double* relres, cudaStream_t s);
