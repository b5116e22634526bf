// Device-resident Krylov solvers: one persistent cooperative launch runs the
// whole CG / BiCGSTAB loop. Phases are separated by bounded grid barriers
// (GridTeam::sync); reductions are two-pass and deterministic; the coarse
// multigrid levels run inside CTA 0 with __syncthreads only (BlockTeam).
// Shared-matrix products (L, L_off) use the assembled stencils of
// fem_stencil.cuh; the element kind is a template parameter.
//
// Loop semantics follow jax_fem_cfd utils/jax_iterative_solvers.py:
//   CG  (:87-120)  stop when (M is identity ? gamma : r.r) <= max(tol^2 b.b, atol^2)
//                  or k == maxiter; p0 = z0 = M r0.
//   BiCGSTAB (:123-167) stop when r.r <= atol2, k == maxiter or k < 0 (breakdown
//                  -10 for rho == 0, -11 for omega == 0 or alpha == 0).
#pragma once
#include "fem_ops.cuh"
#include "fem_stencil.cuh"

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
  const double* tab;      // assembled stencil of L_e (core/element_calc.py:27)
  const double* tab_off;  // assembled stencil of L_e with zero diagonal (core/multigrid.py:66)
  const double* diag;     // assembled diag(L) (core/element_calc.py:99)
  const double* invD;     // 1 / diag
  const double* winvD;    // 1 / diag, 0 on gamma_p (pinned mode)
  const uint8_t* pin;     // gamma_p mask of this level (pinned mode), else null
  double sum_invD;        // sum 1 / diag
  double sum_colw;        // sum over nodes of the prolongation column sums (levels >= 1)
  double sum_rc;          // sum over nodes of the restriction row sums c = R 1 (levels >= 1)
  double sum_rcD;         // sum of c / diag
  double* x;              // level correction X_n
  double* r;              // level residual R_n (level 0: the CG residual)
  double* t;              // scratch (fine residual before restriction / prolongated x)
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
  int block_smem;      // doubles of dynamic smem for the CTA-0 levels (0: they stay in global memory)
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

// lattice coordinates of a node
__device__ __forceinline__ void fem_ij(const FemGrid& g, int n, int& i, int& j, int& k) {
  if (g.kind == FEM_HEX8) {
    const int pl = g.nnx * g.nny;
    k = n / pl;
    const int r = n - k * pl;
    j = r / g.nnx;
    i = r - j * g.nnx;
  } else {
    k = 0;
    j = n / g.nnx;
    i = n - j * g.nnx;
  }
}

// ---------------------------------------------------------------------------
// Multigrid phases (core/multigrid.py:231-330)
// ---------------------------------------------------------------------------
// Mean-zero bookkeeping of a level residual. Level 0 holds the CG residual r
// (rh = r - mean r). A coarser level m holds u_m = R t_{m-1} (restriction of the
// fine residual, not centred) and rh_m = u_m - alpha_m c_m - beta_m, where
// c_m = R 1, alpha_m = mean(t_{m-1}), beta_m = mean(u_m - alpha_m c_m): the
// reference's R(t - mean t) - mean(...) (core/multigrid.py:263-268) as an
// affine correction applied by every consumer.
struct LevelAffine {
  double alpha, beta, sum_rhD;
};
template <class Red>
__device__ __forceinline__ LevelAffine fem_level_affine(const Red& red, const CgArgs& A, int m, double* smem) {
  const MgLevel& L = A.lv[m];
  LevelAffine f;
  if (m == 0) {
    double u[2];
    red.template result<2>(u, SL_R(0), smem);
    f.alpha = 0.0;
    f.beta = u[0] / L.g.nn;
    f.sum_rhD = u[1] - f.beta * L.sum_invD;
  } else {
    double u[3];
    const int sl[3] = {SL_R(m), SL_R(m) + 1, SL_T(m - 1)};
    red.template result_slots<3>(u, sl, smem);
    f.alpha = u[2] / A.lv[m - 1].g.nn;
    f.beta = (u[0] - f.alpha * L.sum_rc) / L.g.nn;
    f.sum_rhD = u[1] - f.alpha * L.sum_rcD - f.beta * L.sum_invD;
  }
  return f;
}

// Down-sweep step n -> n+1 in one phase: pre-smooth from zero
// (xh = (2/3) rh / D, 0 on gamma_p or minus its mean), fine residual
// t = rh - L xh, restriction u_{n+1} = R t. Tiled over the coarse unique lattice
// (16 x blockDim/64 coarse nodes per tile): xh is staged for the tile's fine
// region plus the stencil halo, t is formed in smem on that region plus one node,
// and the tile's coarse nodes are restricted from smem. Each CTA writes x_n and
// sums t only on the fine nodes its tile owns.
template <int KIND, class Team, class Red>
__device__ __noinline__ bool mg_down(const Team& tm, const Red& red, const CgArgs& A, int n, double* smem) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF;
  const MgLevel& L = A.lv[n];
  const MgLevel& C = A.lv[n + 1];
  const FemGrid& g = L.g;
  const int nn = g.nn;
  const bool pinned = A.pinned;
  LevelAffine f{0.0, 0.0, 0.0};
  double mx = 0.0;
  if (!pinned) {
    f = fem_level_affine(red, A, n, smem);
    mx = (2.0 / 3.0) * f.sum_rhD / nn;
  }
  fem_trace_mark(A.sync, 1);
  const double* __restrict__ u = L.r;
  const double* __restrict__ iD = pinned ? L.winvD : L.invD;
  const uint8_t* __restrict__ pin = L.pin;
  const int ux = g.nnx, uy = g.nny;
  auto rhf = [&](int j) -> double {
    if (pinned || n == 0) return u[j] - f.beta;
    const int r = j / ux, c = j - r * ux;
    return u[j] - f.alpha * fem_restrict_rowsum(L.lat, r, c) - f.beta;
  };
  auto xs = [&](int j) -> double { return pinned ? (2.0 / 3.0) * u[j] * iD[j] : (2.0 / 3.0) * rhf(j) * iD[j] - mx; };
  const int nc = fem_axis_ncls(KIND, g.periodic);
  const int cux = C.lat.ux(), cuy = C.lat.uy();
  // 16 coarse columns per tile; rows chosen so one round of tiles covers the
  // level (<= one tile per CTA) within the smem staging buffer
  const int CTX = 16;
  const int ntx = (cux + CTX - 1) / CTX;
  int CTY;
  {
    int nty_t = tm.ncta() / ntx;
    if (nty_t < 1) nty_t = 1;
    CTY = (cuy + nty_t - 1) / nty_t;
  }
  {
    const int cap = (FEM_TILE_SMEM - (2 * CTX + 1 + 2 * R) * (1 + 2 * R) - (2 * CTX + 1)) /
                    (2 * (2 * CTX + 1 + 2 * R) + 2 * (2 * CTX + 1));
    if (CTY > cap) CTY = cap;
    if (CTY < 1) CTY = 1;
    if (CTY > cuy) CTY = cuy;
  }
  const int FW = 2 * CTX + 1, FH = 2 * CTY + 1;  // fine region of t
  const int SW = FW + 2 * R, SH = FH + 2 * R;    // staged xh
  double* __restrict__ sx = smem + 128;
  double* __restrict__ st = sx + SW * SH;
  const int nty = (cuy + CTY - 1) / CTY, ntile = ntx * nty;
  double acc_t[1] = {0.0}, acc_u[2] = {0.0, 0.0};
  for (int tl = tm.cta(); tl < ntile; tl += tm.ncta()) {
    const int by = tl / ntx, bx = tl - by * ntx;
    const int C0 = bx * CTX, R0 = by * CTY;
    const int fx0 = 2 * C0 - 1, fy0 = 2 * R0 - 1;  // fine coordinates of the t-region origin
    // all staged loads of a batch in flight before the first smem store
    constexpr int NB = 8;
    for (int q0 = 0; q0 < SW * SH; q0 += NB * (int)blockDim.x) {
      double v[NB];
#pragma unroll
      for (int k = 0; k < NB; ++k) {
        const int q = q0 + k * blockDim.x + threadIdx.x;
        if (q < SW * SH) {
          const int ly = q / SW, lx = q - ly * SW;
          int gx = fx0 - R + lx, gy = fy0 - R + ly;
          if (g.periodic) {
            gx = gx < 0 ? gx + ux : (gx >= ux ? gx - ux : gx);
            gy = gy < 0 ? gy + uy : (gy >= uy ? gy - uy : gy);
          } else {
            gx = gx < 0 ? 0 : (gx >= ux ? ux - 1 : gx);
            gy = gy < 0 ? 0 : (gy >= uy ? uy - 1 : gy);
          }
          v[k] = xs(gy * ux + gx);
        }
      }
#pragma unroll
      for (int k = 0; k < NB; ++k) {
        const int q = q0 + k * blockDim.x + threadIdx.x;
        if (q < SW * SH) sx[q] = v[k];
      }
    }
    __syncthreads();
    fem_trace_mark(A.sync, 2);
    for (int q = threadIdx.x; q < FW * FH; q += blockDim.x) {
      const int py = q / FW, px = q - py * FW;
      const int x = fx0 + px, y = fy0 + py;
      double tv = 0.0;
      if (x >= 0 && x < ux && y >= 0 && y < uy) {
        const int cx = fem_axis_cls(KIND, g.periodic, x, g.nex), cy = fem_axis_cls(KIND, g.periodic, y, g.ney);
        const double* __restrict__ cf = L.tab + (size_t)(cy * nc + cx) * NOFF;
        double Lx = 0.0;
#pragma unroll
        for (int dy = 0; dy < W; ++dy)
#pragma unroll
          for (int dx = 0; dx < W; ++dx) Lx += __ldg(cf + dy * W + dx) * sx[(py + dy) * SW + px + dx];
        const int j = y * ux + x;
        double rz;
        if (pinned) {
          const bool p = pin && pin[j];
          rz = p ? 0.0 : u[j];
          if (p) Lx = 0.0;
        } else {
          rz = rhf(j);
        }
        tv = rz - Lx;
        // fine nodes owned by this tile: [2 C0, 2 C0 + 2 CTX) x [2 R0, 2 R0 + 2 CTY)
        if (px >= 1 && px <= 2 * CTX && py >= 1 && py <= 2 * CTY) {
          L.x[j] = sx[(py + R) * SW + px + R];
          acc_t[0] += tv;
        }
      }
      st[q] = tv;
    }
    __syncthreads();
    fem_trace_mark(A.sync, 3);
    for (int kk = threadIdx.x; kk < CTX * CTY; kk += blockDim.x) {
      const int ky = kk / CTX, kx = kk - ky * CTX;
      const int Rr = R0 + ky, Cc = C0 + kx;
      if (Rr < cuy && Cc < cux) {
        // fine (2Rr + dr, 2Cc + dc) sits at t-region (1 + 2 ky + dr, 1 + 2 kx + dc)
        const int cy0 = 1 + 2 * ky, cx0 = 1 + 2 * kx;
        const int fyc = 2 * Rr, fxc = 2 * Cc;
        const bool up = fyc + 1 < L.lat.ny, dn = fyc - 1 >= 0, rt = fxc + 1 < L.lat.nx, lf = fxc - 1 >= 0;
        double e = 0.0, d = 0.0;
        if (up) e += st[(cy0 + 1) * FW + cx0];
        if (dn) e += st[(cy0 - 1) * FW + cx0];
        if (rt) e += st[cy0 * FW + cx0 + 1];
        if (lf) e += st[cy0 * FW + cx0 - 1];
        if (up && rt) d += st[(cy0 + 1) * FW + cx0 + 1];
        if (up && lf) d += st[(cy0 + 1) * FW + cx0 - 1];
        if (dn && rt) d += st[(cy0 - 1) * FW + cx0 + 1];
        if (dn && lf) d += st[(cy0 - 1) * FW + cx0 - 1];
        const double v = st[cy0 * FW + cx0] + 0.5 * e + 0.25 * d;
        const int I = Rr * cux + Cc;
        C.r[I] = v;
        acc_u[0] += v;
        acc_u[1] += v * C.invD[I];
      }
    }
    __syncthreads();
  }
  fem_trace_mark(A.sync, 4);
  if (!pinned) {
    red.template reduce<1>(acc_t, SL_T(n), smem);
    red.template reduce<2>(acc_u, SL_R(n + 1), smem);
  }
  fem_trace_mark(A.sync, 5);
  return tm.sync();
}

// Coarsest level (solution written to L.t). Pinned: CG to coarse_tol with maxiter coarse_maxiter on
// L with gamma_p rows zeroed (core/multigrid.py:278-287). Mean-zero: one Jacobi
// sweep from zero (core/multigrid.py:289-301). Runs in CTA 0 (BlockTeam).
template <int KIND, class Red>
__device__ __noinline__ void mg_coarse(const Red& red, const CgArgs& A, double* smem, double* cg_r, double* cg_p,
                                       double* cg_q) {
  const BlockTeam tm;
  const int n = A.nlev - 1;
  const MgLevel& L = A.lv[n];
  const FemGrid& g = L.g;
  const int nn = g.nn;
  if (!A.pinned) {
    const LevelAffine f = fem_level_affine(red, A, n, smem);
    const double mx = (2.0 / 3.0) * f.sum_rhD / nn;
    const int ux = L.lat.ux();
    // x = omega*(rN - L_off*0)/D + (1-omega)*0, then x - mean(x)
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      const double rh = (n == 0) ? L.r[i] - f.beta
                                 : L.r[i] - f.alpha * fem_restrict_rowsum(L.lat, i / ux, i % ux) - f.beta;
      L.t[i] = (2.0 / 3.0) * rh / L.diag[i] - mx;
    }
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
    L.t[i] = 0.0;
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
    fem_tiled_stencil<KIND>(tm, g, L.tab, smem + 128, [&](int j) { return cg_p[j]; },
                            [&](int i, int, int, int, double q, double pi) {
                              if (pin && pin[i]) q = 0.0;
                              cg_q[i] = q;
                              pq[0] += pi * q;
                            });
    fem_block_sum<1>(pq, smem);
    const double alpha = gamma / pq[0];
    double rr[1] = {0.0};
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      L.t[i] = L.t[i] + alpha * cg_p[i];
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
    if (pin && pin[i]) L.t[i] = 0.0;
  __syncthreads();
}

// Sums of a freshly produced level correction X_n (mean-zero bookkeeping).
__device__ __forceinline__ void mg_xsums(const MgLevel& L, int i, double xi, double (&a)[2]) {
  a[0] += xi;
  const int ux = L.lat.ux();
  a[1] += fem_interp_colsum(L.lat, i / ux, i % ux) * xi;
}

// Up-sweep at level n: prolongate X_{n+1}, add to X_n, one weighted Jacobi sweep.
// The prolongated iterate y = X_n + P X_{n+1} (- mean, or 0 on gamma_p) is
// evaluated while staging the Jacobi stencil's tile, so the sweep is a single
// phase. For n == 0 the result is z = M r; the phase also accumulates r.z pieces.
template <int KIND, class Team, class Red>
__device__ __noinline__ bool mg_up(const Team& tm, const Red& red, const CgArgs& A, int n, double* smem) {
  const MgLevel& L = A.lv[n];
  const MgLevel& C = A.lv[n + 1];
  const FemGrid& g = L.g;
  const int nn = g.nn;
  const bool pinned = A.pinned;
  double mX = 0.0, mP = 0.0;
  LevelAffine f{0.0, 0.0, 0.0};
  if (!pinned) {
    if (n > 0) {
      double v[5];
      const int sl[5] = {SL_X(n + 1), SL_X(n + 1) + 1, SL_R(n), SL_R(n) + 1, SL_T(n - 1)};
      red.template result_slots<5>(v, sl, smem);
      mX = v[0] / C.g.nn;
      mP = (v[1] - mX * C.sum_colw) / nn;
      f.alpha = v[4] / A.lv[n - 1].g.nn;
      f.beta = (v[2] - f.alpha * L.sum_rc) / nn;
    } else {
      double v[2];
      red.template result<2>(v, SL_X(n + 1), smem);
      mX = v[0] / C.g.nn;
      mP = (v[1] - mX * C.sum_colw) / nn;
    }
  }
  const double* __restrict__ Xc = C.t;  // corrected coarse iterate (after its own up-sweep / coarse solve)
  const double* __restrict__ Xf = L.x;  // pre-smoothed iterate of the down-sweep
  const uint8_t* __restrict__ pin = L.pin;
  const int ux = g.nnx;
  auto yfun = [&](int j) -> double {
    if (pinned && pin && pin[j]) return 0.0;
    const int r = j / ux, c = j - r * ux;
    const double xH = fem_interp_at(C.lat, r, c, [&](int I) { return pinned ? Xc[I] : Xc[I] - mX; });
    return Xf[j] + (pinned ? xH : xH - mP);
  };
  // Jacobi: x = w (rh - Loff y)/D + (1-w) y
  const double* __restrict__ rh = L.r;
  const double w = 2.0 / 3.0;
  double a[2] = {0.0, 0.0};
  // the staged tile reads Xf at neighbours: all threads of the team must have
  // read X_n before any writes it, so the new x goes to L.t and is swapped in below
  fem_tiled_stencil<KIND>(tm, g, L.tab_off, smem + 128, yfun, [&](int i, int, int, int, double off, double yi) {
    const double rv = (!pinned && n > 0)
                          ? rh[i] - f.alpha * fem_restrict_rowsum(L.lat, i / ux, i - (i / ux) * ux) - f.beta
                          : rh[i];
    double xn = w * (rv - off) / L.diag[i] + (1.0 - w) * yi;
    if (pinned && pin && pin[i]) xn = 0.0;
    L.t[i] = xn;
    if (n == 0) {
      a[0] += xn;
      a[1] += rh[i] * xn;
    } else {
      mg_xsums(L, i, xn, a);
    }
  });
  if (n == 0 || !pinned) red.template reduce<2>(a, SL_X(n), smem);
  if (!tm.sync()) return false;
  return true;
}

// Full V-cycle on r = lv[0].r; result in lv[0].t (raw; mean-zero subtracts
// SL_X(0)[0]/nn lazily). Levels >= block_from run in CTA 0.
template <int KIND>
__device__ __noinline__ bool mg_vcycle(const GridTeam& gt, const GridReducer& gr, const CgArgs& A, double* smem,
                                       double* bstore, double* cg_r, double* cg_p, double* cg_q) {
  const int N = A.nlev, s = A.block_from;
  for (int n = 0; n < s; ++n)
    if (!mg_down<KIND>(gt, gr, A, n, smem)) return false;
  if (blockIdx.x == 0) {
    const BlockTeam bt;
    const BlockReducer br{bstore};
    // Levels >= s: with block_smem their x / r / t vectors and the coarse-CG
    // scratch live in dynamic shared memory (no L2 round trips between the
    // CTA-local phases); the level-s residual is copied in, x_s copied out.
    __shared__ __align__(16) CgArgs sAb;
    extern __shared__ double dyn[];
    const bool in_smem = A.block_smem > 0;
    const CgArgs& B = in_smem ? sAb : A;
    if (in_smem) {
      {
        const int* src = reinterpret_cast<const int*>(&A);
        int* dst = reinterpret_cast<int*>(&sAb);
        for (int i = threadIdx.x; i < (int)(sizeof(CgArgs) / 4); i += blockDim.x) dst[i] = src[i];
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double* p = dyn + 128 + FEM_TILE_SMEM;
        for (int n = s; n < N; ++n) {
          const int m = A.lv[n].g.nn;
          sAb.lv[n].x = p;
          sAb.lv[n].r = p + m;
          sAb.lv[n].t = p + 2 * m;
          p += 3 * m;
        }
      }
      __syncthreads();
      const double* __restrict__ rsrc = A.lv[s].r;
      double* __restrict__ rdst = sAb.lv[s].r;
      for (int i = threadIdx.x; i < A.lv[s].g.nn; i += blockDim.x) rdst[i] = rsrc[i];
      const int mc = A.lv[N - 1].g.nn;
      double* p = dyn + 128 + FEM_TILE_SMEM;
      for (int n = s; n < N; ++n) p += 3 * A.lv[n].g.nn;
      cg_r = p;
      cg_p = p + mc;
      cg_q = p + 2 * mc;
      __syncthreads();
    }
    // import the grid-produced sums of level s
    if (!B.pinned) {
      double v[2], t[1] = {0.0};
      gr.result<2>(v, SL_R(s), smem);
      if (s > 0) gr.result<1>(t, SL_T(s - 1), smem);
      if (threadIdx.x == 0) {
        bstore[SL_R(s)] = v[0];
        bstore[SL_R(s) + 1] = v[1];
        if (s > 0) bstore[SL_T(s - 1)] = t[0];
      }
      __syncthreads();
    }
    for (int n = s; n < N - 1; ++n) mg_down<KIND>(bt, br, B, n, smem);
    mg_coarse<KIND>(br, B, smem, cg_r, cg_p, cg_q);
    const MgLevel& Lc = B.lv[N - 1];
    if (N == 1) {
      // single level: the coarse solve is the whole preconditioner; r.z pieces
      double a[2] = {0.0, 0.0};
      for (int i = threadIdx.x; i < Lc.g.nn; i += blockDim.x) {
        a[0] += Lc.t[i];
        a[1] += Lc.r[i] * Lc.t[i];
      }
      br.reduce<2>(a, SL_X(0), smem);
      __syncthreads();
    } else if (!B.pinned) {
      double a[2] = {0.0, 0.0};
      for (int i = threadIdx.x; i < Lc.g.nn; i += blockDim.x) mg_xsums(Lc, i, Lc.t[i], a);
      br.reduce<2>(a, SL_X(N - 1), smem);
      __syncthreads();
    }
    for (int n = N - 2; n >= s; --n) mg_up<KIND>(bt, br, B, n, smem);
    if (in_smem) {
      const double* __restrict__ xs = sAb.lv[s].t;
      double* __restrict__ xd = A.lv[s].t;
      for (int i = threadIdx.x; i < A.lv[s].g.nn; i += blockDim.x) xd[i] = xs[i];
    }
    // export the level-s sums for the grid (CTA 0 column; other columns stay zero)
    if (threadIdx.x == 0 && (s == 0 || !A.pinned)) {
      A.sync.partials[(size_t)SL_X(s) * gridDim.x] = bstore[SL_X(s)];
      A.sync.partials[(size_t)(SL_X(s) + 1) * gridDim.x] = bstore[SL_X(s) + 1];
    }
  }
  if (!gt.sync()) return false;
  for (int n = s - 1; n >= 0; --n)
    if (!mg_up<KIND>(gt, gr, A, n, smem)) return false;
  return true;
}
