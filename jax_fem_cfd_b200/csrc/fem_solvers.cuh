// Device-resident Krylov solvers: one persistent cooperative launch runs the
// whole CG / BiCGSTAB loop. Phases are separated by bounded grid barriers
// (GridTeam::sync); reductions are two-pass and deterministic; the coarse
// multigrid levels run inside CTA 0 with __syncthreads only (BlockTeam).
//
// Loop semantics follow jax_fem_cfd utils/jax_iterative_solvers.py:
//   CG  (:87-120)  stop when (M is identity ? gamma : r.r) <= max(tol^2 b.b, atol^2)
//                  or k == maxiter; p0 = z0 = M r0.
//   BiCGSTAB (:123-167) stop when r.r <= atol2, k == maxiter or k < 0 (breakdown
//                  -10 for rho == 0, -11 for omega == 0 or alpha == 0).
#pragma once
#include "fem_ops.cuh"

#define FEM_MAX_LEVELS 14

// Reduction slot map --------------------------------------------------------
#define SL_BB 0      // b.b
#define SL_RR 1      // r.r
#define SL_RSUM 2    // sum r
#define SL_PAP 3     // p.Ap
#define SL_RZ 4      // r.z (direct)
#define SL_BSUM 5    // sum b (mean-zero rhs)
#define SL_BI 6      // BiCGSTAB: 6 rhat.r, 7 rhat.q, 8 s.s, 9 t.s, 10 t.t
#define SL_LVL0 12
#define SL_R(n) (SL_LVL0 + 6 * (n))      // 2 slots: sum R_n, sum R_n / D_n
#define SL_T(n) (SL_LVL0 + 6 * (n) + 2)  // 1 slot : sum T_n
#define SL_X(n) (SL_LVL0 + 6 * (n) + 3)  // 2 slots: sum X_n, sum colw_n X_n
#define FEM_NSLOTS (SL_LVL0 + 6 * FEM_MAX_LEVELS)

#define FEM_PREC_NONE 0
#define FEM_PREC_JACOBI 1
#define FEM_PREC_APPROX_INV 2     // solvers/standard.py:225-234 (D1L[gp] = 0)
#define FEM_PREC_APPROX_INV_PT 3  // solvers/passive_transport.py:409-418 (keeps D1x/D1L on gp)
#define FEM_PREC_MG 4

struct MgLevel {
  FemGrid g;
  FemLattice lat;
  const double* Le;
  const double* Le_off;
  const double* diag;
  const uint8_t* pin;  // gamma_p mask of this level (pinned mode), else null
  double sum_invD;     // sum 1 / diag
  double sum_colw;     // sum over nodes of the prolongation column sums (levels >= 1)
  double* x;           // level correction X_n
  double* r;           // level residual R_n (level 0: the CG residual)
  double* t;           // scratch (fine residual before restriction / prolongated x)
};

struct CgArgs {
  FemSync sync;
  int nlev;            // multigrid levels (level 0 = the problem mesh)
  int block_from;      // first level solved by CTA 0 alone (<= nlev - 1)
  int prec;
  int pinned;          // 1: set_zeroP (rows / values on gamma_p zeroed); 0: mean-zero
  int center_rhs;      // mean-zero: subtract mean(b) first (solvers/standard.py:106)
  int maxiter, coarse_maxiter;
  double tol, atol, coarse_tol;
  const double* b;     // rhs (nn)
  double* bwork;       // centred rhs copy (nn) when center_rhs
  double* x;           // in: x0, out: solution (nn)
  double *r, *z, *p0, *p1, *Ap;
  const uint8_t* ai_pin;  // approx_inv pin set (gamma_p incl. the scalar-0 default)
  int* iters;          // device out: iteration count
  int* status;         // device out: FEM_ERR_* of this solve
  double* final_rr;    // device out: final r.r (diagnostics)
  int post;            // final pin / mean fix of solvers/standard.py:119-123
  MgLevel lv[FEM_MAX_LEVELS];
};

__device__ __forceinline__ void fem_zero_partials(const FemSync& s) {
  for (int k = threadIdx.x; k < FEM_NSLOTS; k += blockDim.x) s.partials[(size_t)k * gridDim.x + blockIdx.x] = 0.0;
}

// Copy the (param-space) solver arguments into shared memory so that the
// non-inlined phase functions can take them by reference without a local copy.
template <class T>
__device__ __forceinline__ void fem_stage_args(const T& src, T* dst) {
  static_assert(sizeof(T) % 4 == 0, "args must be 4-byte sized");
  const int* s = reinterpret_cast<const int*>(&src);
  int* d = reinterpret_cast<int*>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(T) / 4); i += blockDim.x) d[i] = s[i];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Multigrid phases (core/multigrid.py:231-330)
// ---------------------------------------------------------------------------
template <class Team, class Red>
__device__ __noinline__ bool mg_down(const Team& tm, const Red& red, const CgArgs& A, int n, double* smem) {
  const MgLevel& L = A.lv[n];
  const MgLevel& C = A.lv[n + 1];
  const int nn = L.g.nn;
  const bool pinned = A.pinned;
  double mr = 0.0, mx = 0.0;
  if (!pinned) {
    double s[2];
    red.template result<2>(s, SL_R(n), smem);
    mr = s[0] / nn;
    mx = (2.0 / 3.0) * (s[1] - mr * L.sum_invD) / nn;
  }
  const double* __restrict__ rh = L.r;
  const double* __restrict__ D = L.diag;
  const uint8_t* __restrict__ pin = L.pin;
  auto xs = [&](int j) -> double {
    if (pinned) return (pin && pin[j]) ? 0.0 : (2.0 / 3.0) * rh[j] / D[j];
    return (2.0 / 3.0) * (rh[j] - mr) / D[j] - mx;
  };
  double acc[1] = {0.0};
  for (int i = tm.rank(); i < nn; i += tm.size()) {
    const double xi = xs(i);
    L.x[i] = xi;
    double rz, Lx = fem_gather_fn(L.g, i, MatShared{L.Le, 1.0}, xs);
    if (pinned) {
      const bool p = pin && pin[i];
      rz = p ? 0.0 : rh[i];
      if (p) Lx = 0.0;
    } else {
      rz = rh[i] - mr;
    }
    const double ti = rz - Lx;
    L.t[i] = ti;
    acc[0] += ti;
  }
  if (!pinned) red.template reduce<1>(acc, SL_T(n), smem);
  if (!tm.sync()) return false;
  // restriction onto the coarse level
  double mt = 0.0;
  if (!pinned) {
    double s[1];
    red.template result<1>(s, SL_T(n), smem);
    mt = s[0] / nn;
  }
  const double* __restrict__ T = L.t;
  const int cux = C.lat.ux(), cuy = C.lat.uy(), ncn = cux * cuy;
  double a2[2] = {0.0, 0.0};
  for (int I = tm.rank(); I < ncn; I += tm.size()) {
    const int R = I / cux, Cc = I % cux;
    const double v = fem_restrict_at(L.lat, R, Cc, [&](int j) { return pinned ? T[j] : T[j] - mt; });
    C.r[I] = v;
    a2[0] += v;
    a2[1] += v / C.diag[I];
  }
  if (!pinned) red.template reduce<2>(a2, SL_R(n + 1), smem);
  return tm.sync();
}

// Coarsest level. Pinned: CG to coarse_tol with maxiter coarse_maxiter on
// L with gamma_p rows zeroed (core/multigrid.py:278-287). Mean-zero: one Jacobi
// sweep from zero (core/multigrid.py:289-301). Runs in CTA 0 (BlockTeam).
template <class Red>
__device__ __noinline__ void mg_coarse(const Red& red, const CgArgs& A, double* smem, double* cg_r, double* cg_p, double* cg_q) {
  const BlockTeam tm;
  const int n = A.nlev - 1;
  const MgLevel& L = A.lv[n];
  const int nn = L.g.nn;
  if (!A.pinned) {
    double s[2];
    red.template result<2>(s, SL_R(n), smem);
    const double mr = s[0] / nn;
    const double mx = (2.0 / 3.0) * (s[1] - mr * L.sum_invD) / nn;
    // x = omega*(rN - L_off*0)/D + (1-omega)*0, then x - mean(x)
    for (int i = tm.rank(); i < nn; i += tm.size()) L.x[i] = (2.0 / 3.0) * (L.r[i] - mr) / L.diag[i] - mx;
    __syncthreads();
    return;
  }
  const uint8_t* pin = L.pin;
  // b = rN with pinned zeroed; x0 = 0 -> r = b, p = b, gamma = b.b
  double acc[1] = {0.0};
  for (int i = tm.rank(); i < nn; i += tm.size()) {
    const double bi = (pin && pin[i]) ? 0.0 : L.r[i];
    cg_r[i] = bi;
    cg_p[i] = bi;
    L.x[i] = 0.0;
    acc[0] += bi * bi;
  }
  fem_block_sum<1>(acc, smem);
  const double bs = acc[0];
  const double atol2 = fmax(A.coarse_tol * A.coarse_tol * bs, 0.0);
  double gamma = bs;
  int k = 0;
  __syncthreads();
  while (gamma > atol2 && k < A.coarse_maxiter) {
    double pq[1] = {0.0};
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      double q = fem_gather_fn(L.g, i, MatShared{L.Le, 1.0}, [&](int j) { return cg_p[j]; });
      if (pin && pin[i]) q = 0.0;
      cg_q[i] = q;
      pq[0] += cg_p[i] * q;
    }
    fem_block_sum<1>(pq, smem);
    const double alpha = gamma / pq[0];
    double rr[1] = {0.0};
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      L.x[i] = L.x[i] + alpha * cg_p[i];
      const double ri = cg_r[i] - alpha * cg_q[i];
      cg_r[i] = ri;
      rr[0] += ri * ri;
    }
    fem_block_sum<1>(rr, smem);
    const double beta = rr[0] / gamma;
    for (int i = tm.rank(); i < nn; i += tm.size()) cg_p[i] = cg_r[i] + beta * cg_p[i];
    gamma = rr[0];
    ++k;
    __syncthreads();
  }
  for (int i = tm.rank(); i < nn; i += tm.size())
    if (pin && pin[i]) L.x[i] = 0.0;
  __syncthreads();
}

// Sums of a freshly produced level correction X_n (mean-zero bookkeeping).
__device__ __forceinline__ void mg_xsums(const MgLevel& L, int i, double xi, double (&a)[2]) {
  a[0] += xi;
  const int ux = L.lat.ux();
  a[1] += fem_interp_colsum(L.lat, i / ux, i % ux) * xi;
}

// Up-sweep at level n: prolongate X_{n+1}, add to X_n, one weighted Jacobi sweep.
// For n == 0 the result is z = M r; the phase also accumulates r.z pieces.
template <class Team, class Red>
__device__ __noinline__ bool mg_up(const Team& tm, const Red& red, const CgArgs& A, int n, double* smem) {
  const MgLevel& L = A.lv[n];
  const MgLevel& C = A.lv[n + 1];
  const int nn = L.g.nn;
  const bool pinned = A.pinned;
  double mX = 0.0, mP = 0.0;
  if (!pinned) {
    double s[2];
    red.template result<2>(s, SL_X(n + 1), smem);
    mX = s[0] / C.g.nn;
    mP = (s[1] - mX * C.sum_colw) / nn;
  }
  const double* __restrict__ Xc = C.x;
  const int ux = L.lat.ux();
  for (int i = tm.rank(); i < nn; i += tm.size()) {
    const int r = i / ux, c = i % ux;
    const double xH = fem_interp_at(C.lat, r, c, [&](int I) { return pinned ? Xc[I] : Xc[I] - mX; });
    double y = L.x[i] + (pinned ? xH : xH - mP);
    if (pinned && L.pin && L.pin[i]) y = 0.0;
    L.t[i] = y;
  }
  if (!tm.sync()) return false;
  // Jacobi: x = w (rh - Loff y)/D + (1-w) y
  double mr = 0.0;
  if (!pinned && n > 0) {
    double s[2];
    red.template result<2>(s, SL_R(n), smem);
    mr = s[0] / nn;
  }
  const double* __restrict__ Y = L.t;
  const double* __restrict__ rh = L.r;
  const double w = 2.0 / 3.0;
  double a[3] = {0.0, 0.0, 0.0};
  for (int i = tm.rank(); i < nn; i += tm.size()) {
    const double off = fem_gather_fn(L.g, i, MatShared{L.Le_off, 1.0}, [&](int j) { return Y[j]; });
    const double rv = (!pinned && n > 0) ? rh[i] - mr : rh[i];
    double xn = w * (rv - off) / L.diag[i] + (1.0 - w) * Y[i];
    if (pinned && L.pin && L.pin[i]) xn = 0.0;
    L.x[i] = xn;
    if (n == 0) {
      a[0] += xn;
      a[1] += rh[i] * xn;
    } else {
      double t2[2] = {0.0, 0.0};
      mg_xsums(L, i, xn, t2);
      a[0] += t2[0];
      a[1] += t2[1];
    }
  }
  if (n == 0) {
    double v[2] = {a[0], a[1]};
    red.template reduce<2>(v, SL_X(0), smem);  // [sum z_raw, r . z_raw]
  } else if (!pinned) {
    double v[2] = {a[0], a[1]};
    red.template reduce<2>(v, SL_X(n), smem);
  }
  return tm.sync();
}

// Full V-cycle on r = lv[0].r; result in lv[0].x (raw; mean-zero subtracts
// SL_X(0)[0]/nn lazily). Levels >= block_from run in CTA 0.
static __device__ __noinline__ bool mg_vcycle(const GridTeam& gt, const GridReducer& gr, const CgArgs& A, double* smem, double* bstore,
                          double* cg_r, double* cg_p, double* cg_q) {
  const int N = A.nlev, s = A.block_from;
  for (int n = 0; n < s; ++n)
    if (!mg_down(gt, gr, A, n, smem)) return false;
  if (blockIdx.x == 0) {
    const BlockTeam bt;
    const BlockReducer br{bstore};
    // import the grid-produced sums of level s
    if (!A.pinned) {
      double v[2];
      gr.result<2>(v, SL_R(s), smem);
      if (threadIdx.x == 0) { bstore[SL_R(s)] = v[0]; bstore[SL_R(s) + 1] = v[1]; }
      __syncthreads();
    }
    for (int n = s; n < N - 1; ++n) mg_down(bt, br, A, n, smem);
    mg_coarse(br, A, smem, cg_r, cg_p, cg_q);
    if (!A.pinned) {
      // sums of the coarsest correction
      const MgLevel& L = A.lv[N - 1];
      double a[2] = {0.0, 0.0};
      for (int i = threadIdx.x; i < L.g.nn; i += blockDim.x) mg_xsums(L, i, L.x[i], a);
      br.reduce<2>(a, SL_X(N - 1), smem);
      __syncthreads();
    }
    for (int n = N - 2; n >= s; --n) mg_up(bt, br, A, n, smem);
    // export sums of level s for the grid-level prolongation (CTA 0 column only;
    // the other CTAs' columns of these slots stay zero)
    if (!A.pinned && s > 0 && threadIdx.x == 0) {
      A.sync.partials[(size_t)SL_X(s) * gridDim.x] = bstore[SL_X(s)];
      A.sync.partials[(size_t)(SL_X(s) + 1) * gridDim.x] = bstore[SL_X(s) + 1];
    }
    if (s == 0 && threadIdx.x == 0) {
      // whole hierarchy ran in CTA 0: publish r.z pieces of level 0
      A.sync.partials[(size_t)SL_X(0) * gridDim.x] = bstore[SL_X(0)];
      A.sync.partials[(size_t)(SL_X(0) + 1) * gridDim.x] = bstore[SL_X(0) + 1];
    }
  }
  if (!gt.sync()) return false;
  for (int n = s - 1; n >= 0; --n)
    if (!mg_up(gt, gr, A, n, smem)) return false;
  return true;
}
