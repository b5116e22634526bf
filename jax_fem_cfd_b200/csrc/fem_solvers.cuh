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
#define FEM_PREC_APPROX_INV_PT 3  // solvers/passive_transport.py:141-150 (keeps D1x/D1L on gp)
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
  double inv_nn;          // 1 / nn (means)
  double* x;              // level correction X_n
  double* r;              // level residual R_n (level 0: the CG residual)
  double* t;              // scratch (fine residual before restriction / prolongated x)
};

struct CgArgs {
  FemSync sync;
  int nlev;            // multigrid levels (level 0 = the problem mesh)
  int block_from;      // first level handled by the coarse-level team (<= nlev - 1)
  int team;            // CTAs in the coarse-level team (the first ones of the grid)
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
  int block_smem_from; // first level of the V-cycle run inside CTA 0 from shared memory (nlev: none)
  MgLevel lv[FEM_MAX_LEVELS];
  const double* bd[FEM_MAX_LEVELS];  // per-CTA shared-memory copies of those levels' 1/D (0 on gamma_p if pinned)
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

// Stencil tables of the solver levels in shared memory (FEM_TAB_SMEM doubles
// after the tile buffer): copied once per launch, in level order while they
// fit, and the shared argument copy is pointed at them. Tables that do not fit
// stay in global memory; every reader uses plain loads, so both work.
#define FEM_TAB_SMEM 2048
template <int KIND>
__device__ void fem_tables_to_smem(CgArgs& sA, double* stab) {
  constexpr int NOFF = KI<KIND>::NOFF;
  int off = 0;
  for (int l = 0; l < sA.nlev; ++l) {
    const MgLevel& L = sA.lv[l];
    if (!L.tab || !L.tab_off) break;
    const int m = fem_stencil_ncls(L.g) * NOFF;
    if (off + 2 * m > FEM_TAB_SMEM) break;
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
      stab[off + q] = L.tab[q];
      stab[off + m + q] = L.tab_off[q];
    }
    off += 2 * m;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    off = 0;
    for (int l = 0; l < sA.nlev; ++l) {
      MgLevel& L = sA.lv[l];
      if (!L.tab || !L.tab_off) break;
      const int m = fem_stencil_ncls(L.g) * NOFF;
      if (off + 2 * m > FEM_TAB_SMEM) break;
      L.tab = stab + off;
      L.tab_off = stab + off + m;
      off += 2 * m;
    }
  }
  __syncthreads();
}

// 1/D of the levels that the V-cycle runs inside CTA 0 (pinned: winvD, whose
// zeros mark gamma_p), copied into this CTA's shared memory once per launch
// (FEM_BLK_SMEM doubles); sA.bd[l] points at level l's copy.
#define FEM_BLK_SMEM 2048
__device__ __forceinline__ void fem_block_levels_to_smem(CgArgs& sA, double* sbd) {
  int off = 0;
  for (int l = sA.block_smem_from; l < sA.nlev; ++l) {
    const MgLevel& L = sA.lv[l];
    const double* src = sA.pinned ? L.winvD : L.invD;
    for (int q = threadIdx.x; q < L.g.nn; q += blockDim.x) sbd[off + q] = src[q];
    off += L.g.nn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    off = 0;
    for (int l = sA.block_smem_from; l < sA.nlev; ++l) {
      sA.bd[l] = sbd + off;
      off += sA.lv[l].g.nn;
    }
  }
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
// Per-CTA cache of each level's (alpha, beta), written by the down-sweep and
// read back by the up-sweep of the same level (same slots, same formula).
__device__ __forceinline__ double* fem_affine_cache() {
  __shared__ double c[2 * FEM_MAX_LEVELS];
  return c;
}
// Slots of the sums behind a level's affine terms (a third, ignored one at level 0).
__device__ __forceinline__ void fem_level_affine_slots(int m, int (&sl)[3]) {
  sl[0] = SL_R(m);
  sl[1] = SL_R(m) + 1;
  sl[2] = m > 0 ? SL_T(m - 1) : SL_R(m);
}
__device__ __forceinline__ LevelAffine fem_level_affine_from(const CgArgs& A, int m, const double (&u)[3]) {
  const MgLevel& L = A.lv[m];
  LevelAffine f;
  if (m == 0) {
    f.alpha = 0.0;
    f.beta = u[0] * L.inv_nn;
    f.sum_rhD = u[1] - f.beta * L.sum_invD;
  } else {
    f.alpha = u[2] * A.lv[m - 1].inv_nn;
    f.beta = (u[0] - f.alpha * L.sum_rc) * L.inv_nn;
    f.sum_rhD = u[1] - f.alpha * L.sum_rcD - f.beta * L.sum_invD;
  }
  return f;
}
template <class Red>
__device__ __forceinline__ LevelAffine fem_level_affine(const Red& red, const CgArgs& A, int m, double* smem) {
  int sl[3];
  fem_level_affine_slots(m, sl);
  double u[3];
  red.template result_slots<3>(u, sl, smem);
  return fem_level_affine_from(A, m, u);
}

// Down-sweep step n -> n+1 in one phase: pre-smooth from zero
// (xh = (2/3) rh / D, 0 on gamma_p or minus its mean), fine residual
// t = rh - L xh, restriction u_{n+1} = R t. Tiled over the coarse unique lattice
// (16 coarse columns x CTY rows, CTY chosen for one round of tiles): u and 1/D
// of the tile's fine region plus the stencil halo, and 1/D of its coarse nodes,
// are staged in one batch; xh, t (on the region plus one node) and the
// restriction are then formed from smem only. Each CTA writes x_n and sums t
// only on the fine nodes its tile owns.
template <int KIND, bool PIN, class Team, class Red>
__device__ __noinline__ bool mg_down(const Team& tm, const Red& red, const CgArgs& A, int n, double* smem) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF;
  fem_trace_mark(A.sync, 15);
  const MgLevel& L = A.lv[n];
  const MgLevel& C = A.lv[n + 1];
  const FemGrid& g = L.g;
  const int nn = g.nn;
  constexpr bool pinned = PIN;  // A.pinned, fixed per kernel instantiation
  LevelAffine f{0.0, 0.0, 0.0};
  double mx = 0.0;
  bool have_f = pinned;
  // the level's affine terms (mean-zero): partial loads issued now, combined
  // after the first tile's copies have been issued
  int asl[3];
  fem_level_affine_slots(n, asl);
  typename Red::template Pending<3> pend{};
  if (!pinned) pend = red.template result_begin<3>(asl);
  fem_trace_mark(A.sync, 16);
  auto read_affine = [&]() {
    if (have_f) return;
    double u3[3];
    fem_trace_mark(A.sync, 17);
    red.template result_end<3>(pend, u3, smem);
    fem_trace_mark(A.sync, 18);
    f = fem_level_affine_from(A, n, u3);
    mx = (2.0 / 3.0) * f.sum_rhD * L.inv_nn;
    if (threadIdx.x == 0) {
      fem_affine_cache()[2 * n] = f.alpha;
      fem_affine_cache()[2 * n + 1] = f.beta;
    }
    have_f = true;
  };
  const double* u = L.r;
  const double* iDv = pinned ? L.winvD : L.invD;
  const double* tab = L.tab;
  const int ux = g.nnx, uy = g.nny;
  const int nc = fem_axis_ncls(KIND, g.periodic);
  const int cux = C.lat.ux(), cuy = C.lat.uy();
  const int CTX = 16, ntx = (cux + CTX - 1) / CTX;
  const int FW = 2 * CTX + 1, SW = FW + 2 * R;
  // smem per tile: u and xh on SW x SH, t on FW x FH, coarse 1/D on CTX x CTY,
  // gamma_p flags (bytes) on SW x SH
  auto need = [&](int cty) {
    const int fh = 2 * cty + 1, sh = fh + 2 * R;
    return 2 * SW * sh + FW * fh + CTX * cty + (SW * sh + 7) / 8 + 1;
  };
  int CTY;
  {
    int nty_t = tm.ncta() / ntx;
    if (nty_t < 1) nty_t = 1;
    CTY = (cuy + nty_t - 1) / nty_t;
    if (CTY > cuy) CTY = cuy;
    while (CTY > 1 && need(CTY) > FEM_TILE_SMEM) --CTY;
  }
  const int FH = 2 * CTY + 1, SH = FH + 2 * R, NS = SW * SH;
  double* su = smem + 128;
  double* sx = su + NS;
  double* st = sx + NS;
  double* sci = st + FW * FH;
  unsigned char* spin = reinterpret_cast<unsigned char*>(sci + CTX * CTY);
  const int nty = (cuy + CTY - 1) / CTY, ntile = ntx * nty;
  double acc[3] = {0.0, 0.0, 0.0};  // sum t (owned fine nodes), sum u_{n+1}, sum u_{n+1} / D_{n+1}
  for (int tl = tm.cta(); tl < ntile; tl += tm.ncta()) {
    const int by = tl / ntx, bx = tl - by * ntx;
    const int C0 = bx * CTX, R0 = by * CTY;
    const int fx0 = 2 * C0 - 1, fy0 = 2 * R0 - 1;  // fine coordinates of the t-region origin
    auto fidx = [&](int q) -> int {
      const int ly = q / SW, lx = q - ly * SW;
      int gx = fx0 - R + lx, gy = fy0 - R + ly;
      if (g.periodic) {
        gx = fem_wrap(gx, ux);
        gy = fem_wrap(gy, uy);
      } else {
        gx = gx < 0 ? 0 : (gx >= ux ? ux - 1 : gx);
        gy = gy < 0 ? 0 : (gy >= uy ? uy - 1 : gy);
      }
      return gy * ux + gx;
    };
    auto rowb = [&](int r) -> int {
      int gy = fy0 - R + r;
      gy = g.periodic ? fem_wrap(gy, uy) : (gy < 0 ? 0 : (gy >= uy ? uy - 1 : gy));
      return gy * ux;
    };
    auto colx = [&](int c) -> int {
      const int gx = fx0 - R + c;
      return g.periodic ? fem_wrap(gx, ux) : (gx < 0 ? 0 : (gx >= ux ? ux - 1 : gx));
    };
    fem_stage_2d(su, u, SW, SH, rowb, colx);
    fem_stage_2d(sx, iDv, SW, SH, rowb, colx);
    fem_stage(sci, C.invD, CTX * CTY, [&](int q) -> int {
      const int ky = q / CTX, kx = q - ky * CTX;
      const int Rr = min(R0 + ky, cuy - 1), Cc = min(C0 + kx, cux - 1);
      return Rr * cux + Cc;
    });
    read_affine();
    fem_trace_mark(A.sync, 1);
    fem_stage_wait();
    fem_trace_mark(A.sync, 2);
    // xh on the staged region (pinned: winvD is 0 on gamma_p, which also marks it)
    for (int q = threadIdx.x; q < NS; q += blockDim.x) {
      const double d = sx[q];
      double v;
      if (pinned) {
        spin[q] = (d == 0.0);
        v = (2.0 / 3.0) * su[q] * d;
      } else {
        double rh = su[q] - f.beta;
        if (n > 0) {
          const int j = fidx(q), r = j / ux, c = j - r * ux;
          rh = su[q] - f.alpha * fem_restrict_rowsum(L.lat, r, c) - f.beta;
        }
        v = (2.0 / 3.0) * rh * d - mx;
      }
      sx[q] = v;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < FW * FH; q += blockDim.x) {
      const int py = q / FW, px = q - py * FW;
      const int x = fx0 + px, y = fy0 + py;
      double tv = 0.0;
      if (x >= 0 && x < ux && y >= 0 && y < uy) {
        const int cx = fem_axis_cls(KIND, g.periodic, x, g.nex), cy = fem_axis_cls(KIND, g.periodic, y, g.ney);
        const double* cf = tab + (size_t)(cy * nc + cx) * NOFF;
        double Lx = 0.0;
#pragma unroll
        for (int dy = 0; dy < W; ++dy)
#pragma unroll
          for (int dx = 0; dx < W; ++dx) Lx += cf[dy * W + dx] * sx[(py + dy) * SW + px + dx];
        const int qc = (py + R) * SW + px + R;
        double rz;
        if (pinned) {
          const bool p = spin[qc] != 0;
          rz = p ? 0.0 : su[qc];
          if (p) Lx = 0.0;
        } else {
          rz = (n == 0) ? su[qc] - f.beta : su[qc] - f.alpha * fem_restrict_rowsum(L.lat, y, x) - f.beta;
        }
        tv = rz - Lx;
        // fine nodes owned by this tile: [2 C0, 2 C0 + 2 CTX) x [2 R0, 2 R0 + 2 CTY)
        if (px >= 1 && px <= 2 * CTX && py >= 1 && py <= 2 * CTY) {
          L.x[y * ux + x] = sx[qc];
          acc[0] += tv;
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
        C.r[Rr * cux + Cc] = v;
        acc[1] += v;
        acc[2] += v * sci[kk];
      }
    }
    __syncthreads();
  }
  read_affine();  // CTAs without a tile still cache the level's terms for the up-sweep
  fem_trace_mark(A.sync, 4);
  if (!pinned) {
    const int sl[3] = {SL_T(n), SL_R(n + 1), SL_R(n + 1) + 1};
    return tm.template reduce_sync<3>(acc, sl, smem);
  }
  return tm.sync();
}

// Coarsest level (solution written to L.t). Pinned: CG to coarse_tol with maxiter coarse_maxiter on
// L with gamma_p rows zeroed (core/multigrid.py:278-287). Mean-zero: one Jacobi
// sweep from zero (core/multigrid.py:289-301). Runs in CTA 0 (BlockTeam).
template <int KIND, bool PIN, class Red>
__device__ __noinline__ void mg_coarse(const Red& red, const CgArgs& A, double* smem, double* cg_r, double* cg_p,
                                       double* cg_q) {
  const BlockTeam tm;
  const int n = A.nlev - 1;
  const MgLevel& L = A.lv[n];
  const FemGrid& g = L.g;
  const int nn = g.nn;
  if (!PIN) {
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
    const double* srcp[1] = {cg_p};
    fem_tiled_stencil<KIND, 1>(tm, g, L.tab, smem + 128, srcp, [](int, const double(&v)[1]) { return v[0]; },
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

// Coarse levels up to this many nodes are solved by one warp (mg_coarse_warp).
#define FEM_COARSE_WARP_S 4
#define FEM_COARSE_WARP_NN (32 * FEM_COARSE_WARP_S)

__device__ __forceinline__ double fem_warp_sum(double v) {
  // xor butterfly: every lane ends with the same bits (each stage adds the same
  // two values, in either order)
#pragma unroll
  for (int m = 16; m >= 1; m >>= 1) v += __shfl_xor_sync(0xffffffffu, v, m);
  return v;
}

// The pinned coarsest-level CG of mg_coarse (same start, updates and stop test)
// run by the 32 lanes of warp 0 alone, for levels of at most FEM_COARSE_WARP_NN
// nodes: node i = lane + 32 s lives in registers x[s], r[s], p[s]; p goes
// through shared memory (sp, nn doubles) for the stencil, and the dots are warp
// sums, so an iteration has no block barrier and no global-memory round trip.
template <int KIND>
__device__ __noinline__ void mg_coarse_warp(const CgArgs& A, double* sp) {
  constexpr int S = FEM_COARSE_WARP_S, R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF;
  const MgLevel& L = A.lv[A.nlev - 1];
  // the level lives in shared memory next to sp: copy what the loop reads, so
  // the stores to sp cannot force reloads
  const int nn = L.g.nn, nnx = L.g.nnx, nny = L.g.nny, nex = L.g.nex, ney = L.g.ney;
  const int per = L.g.periodic, maxit = A.coarse_maxiter;
  const double* __restrict__ tab = L.tab;
  const uint8_t* __restrict__ pin = L.pin;
  const double* __restrict__ rN = L.r;
  double* __restrict__ tN = L.t;
  const int lane = threadIdx.x & 31;
  const int nc = fem_axis_ncls(KIND, per);
  double x[S], r[S], p[S];
  constexpr bool PRE = (W == 3);        // neighbour indices kept in registers (Q1)
  constexpr int WP = PRE ? W : 1;
  int cof[S];     // table row of the node's class, -1 past nn or pinned (q = 0)
  int pos[S];     // (iy << 16) | ix
  int row[S][WP];  // neighbour rows (times nnx) and columns, wrapped or clamped
  int col[S][WP];
  double bs = 0.0;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int i = lane + 32 * s;
    const bool live = i < nn && !(pin && pin[i]);
    const double b = live ? rN[i] : 0.0;
    r[s] = b;
    p[s] = b;
    x[s] = 0.0;
    bs += b * b;
    const int ix = live ? i % nnx : 0, iy = live ? i / nnx : 0;
    cof[s] = live ? (fem_axis_cls(KIND, per, iy, ney) * nc + fem_axis_cls(KIND, per, ix, nex)) * NOFF : -1;
    pos[s] = (iy << 16) | ix;
#pragma unroll
    for (int d = 0; d < WP; ++d) {
      int w = iy + d - R, v = ix + d - R;
      w = per ? fem_wrap(w, nny) : min(max(w, 0), nny - 1);
      v = per ? fem_wrap(v, nnx) : min(max(v, 0), nnx - 1);
      row[s][d] = w * nnx;
      col[s][d] = v;
    }
  }
  bs = fem_warp_sum(bs);
  const double atol2 = fmax(A.coarse_tol * A.coarse_tol * bs, 0.0);
  double gamma = bs;
  int k = 0;
  while (gamma > atol2 && k < maxit) {
#pragma unroll
    for (int s = 0; s < S; ++s)
      if (lane + 32 * s < nn) sp[lane + 32 * s] = p[s];
    __syncwarp();
    double q[S], pq = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
      double y = 0.0;
      if (cof[s] >= 0) {
        const double* c = tab + cof[s];
        if constexpr (PRE) {
#pragma unroll
          for (int dy = 0; dy < W; ++dy)
#pragma unroll
            for (int dx = 0; dx < W; ++dx) y += c[dy * W + dx] * sp[row[s][dy] + col[s][dx]];
        } else {
          const int ix = pos[s] & 0xffff, iy = pos[s] >> 16;
#pragma unroll
          for (int dy = 0; dy < W; ++dy) {
            int w = iy + dy - R;
            w = per ? fem_wrap(w, nny) : min(max(w, 0), nny - 1);
#pragma unroll
            for (int dx = 0; dx < W; ++dx) {
              int v = ix + dx - R;
              v = per ? fem_wrap(v, nnx) : min(max(v, 0), nnx - 1);
              y += c[dy * W + dx] * sp[w * nnx + v];
            }
          }
        }
      }
      q[s] = y;
      pq += p[s] * y;
    }
    pq = fem_warp_sum(pq);
    __syncwarp();  // every read of sp before the next iteration writes it
    const double alpha = gamma / pq;
    double rr = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
      x[s] = x[s] + alpha * p[s];
      r[s] = r[s] - alpha * q[s];
      rr += r[s] * r[s];
    }
    rr = fem_warp_sum(rr);
    const double beta = rr / gamma;
#pragma unroll
    for (int s = 0; s < S; ++s) p[s] = r[s] + beta * p[s];
    gamma = rr;
    ++k;
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int i = lane + 32 * s;
    if (i < nn) tN[i] = (pin && pin[i]) ? 0.0 : x[s];
  }
}

// Sums of a freshly produced level correction X_n (mean-zero bookkeeping).
__device__ __forceinline__ void mg_xsums(const MgLevel& L, int i, double xi, double (&a)[2]) {
  a[0] += xi;
  const int ux = L.lat.ux();
  a[1] += fem_interp_colsum(L.lat, i / ux, i % ux) * xi;
}

// Up-sweep at level n: prolongate X_{n+1}, add to X_n, one weighted Jacobi sweep,
// in one phase per 32 x TY tile. Staged in one batch: X_n on the tile plus the
// stencil halo (and ω/D there in pinned mode, whose zeros mark gamma_p), the
// coarse X_{n+1} under that region, and rhs and diag of the tile's own nodes.
// The prolongated iterate y = X_n + P X_{n+1} (- means, or 0 on gamma_p) is
// formed in smem; the sweep then reads smem only. For n == 0 the result is
// z = M r and the phase also accumulates the r.z pieces.
template <int KIND, bool PIN, class Team, class Red>
__device__ __noinline__ bool mg_up(const Team& tm, const Red& red, const CgArgs& A, int n, double* smem) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF;
  fem_trace_mark(A.sync, 14);
  const MgLevel& L = A.lv[n];
  const MgLevel& C = A.lv[n + 1];
  const FemGrid& g = L.g;
  const int nn = g.nn;
  constexpr bool pinned = PIN;  // A.pinned, fixed per kernel instantiation
  double mX = 0.0, mP = 0.0;
  LevelAffine f{0.0, 0.0, 0.0};
  bool have_m = pinned;
  // the coarse correction's means (mean-zero): partial loads issued now,
  // combined after the first tile's copies have been issued
  const int msl[2] = {SL_X(n + 1), SL_X(n + 1) + 1};
  typename Red::template Pending<2> pend{};
  if (!pinned) pend = red.template result_begin<2>(msl);
  auto read_means = [&]() {
    if (have_m) return;
    double v[2];
    red.template result_end<2>(pend, v, smem);  // its __syncthreads also publishes the cache
    mX = v[0] * C.inv_nn;
    mP = (v[1] - mX * C.sum_colw) * L.inv_nn;
    if (n > 0) {
      f.alpha = fem_affine_cache()[2 * n];
      f.beta = fem_affine_cache()[2 * n + 1];
    }
    have_m = true;
  };
  const int ux = g.nnx, uy = g.nny, cux = C.lat.ux(), cuy = C.lat.uy();
  const bool per = g.periodic;
  const int nc = fem_axis_ncls(KIND, per);
  const int WR = blockDim.x >> 5, tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
  const int SX = 32 + 2 * R, CXB = SX / 2 + 3;
  const int nf = pinned ? 2 : 1;
  auto need = [&](int ty) { return nf * SX * (ty + 2 * R) + CXB * ((ty + 2 * R) / 2 + 3) + 64 * ty; };
  const int ntx = (ux + 31) >> 5;
  int TY;
  {
    int nty_t = tm.ncta() / ntx;
    if (nty_t < 1) nty_t = 1;
    TY = (uy + nty_t - 1) / nty_t;
    const int minr = WR < uy ? WR : uy;
    if (TY < minr) TY = minr;
    if (TY > uy) TY = uy;
    while (TY > 1 && need(TY) > FEM_TILE_SMEM) --TY;
  }
  const int SY = TY + 2 * R, NS = SX * SY, CYB = SY / 2 + 3;
  double* sy = smem + 128;
  double* sw = sy + NS;                     // pinned only
  double* sc = sy + nf * NS;                // coarse X_{n+1}, CXB x CYB
  double* sr = sc + CXB * CYB;              // rhs of owned nodes, 32 x TY
  double* sd = sr + 32 * TY;                // 1 / diag of owned nodes
  const int nty = (uy + TY - 1) / TY, ntile = ntx * nty;
  const double* tabo = L.tab_off;
  const double w = 2.0 / 3.0;
  double a[2] = {0.0, 0.0};
  for (int tl = tm.cta(); tl < ntile; tl += tm.ncta()) {
    const int by = tl / ntx, bx = tl - by * ntx;
    const int x0 = bx * 32, y0 = by * TY, gx0 = x0 - R, gy0 = y0 - R;
    const int cr0 = fem_floordiv2(gy0), cc0 = fem_floordiv2(gx0);
    // fine coordinates of a staged point: unwrapped (periodic) or clamped
    auto fcoord = [&](int q, int& fr, int& fc) {
      const int ly = q / SX, lx = q - ly * SX;
      fr = gy0 + ly;
      fc = gx0 + lx;
      if (!per) {
        fr = fr < 0 ? 0 : (fr >= uy ? uy - 1 : fr);
        fc = fc < 0 ? 0 : (fc >= ux ? ux - 1 : fc);
      }
    };
    auto fidx = [&](int q) -> int {
      int fr, fc;
      fcoord(q, fr, fc);
      if (per) {
        fr = fem_wrap(fr, uy);
        fc = fem_wrap(fc, ux);
      }
      return fr * ux + fc;
    };
    auto oidx = [&](int q) -> int {  // owned node q = ty * 32 + tx, clamped into the lattice
      const int ty = q >> 5, x = min(x0 + (q & 31), ux - 1), y = min(y0 + ty, uy - 1);
      return y * ux + x;
    };
    auto rowb = [&](int r) -> int {
      int fr = gy0 + r;
      fr = per ? fem_wrap(fr, uy) : (fr < 0 ? 0 : (fr >= uy ? uy - 1 : fr));
      return fr * ux;
    };
    auto colx = [&](int c) -> int {
      const int fc = gx0 + c;
      return per ? fem_wrap(fc, ux) : (fc < 0 ? 0 : (fc >= ux ? ux - 1 : fc));
    };
    fem_stage_2d(sy, L.x, SX, SY, rowb, colx);
    if (pinned) fem_stage_2d(sw, L.winvD, SX, SY, rowb, colx);
    fem_stage(sc, C.t, CXB * CYB, [&](int q) -> int {
      const int i = q / CXB, j = q - i * CXB;
      int cr = cr0 + i, cc = cc0 + j;
      if (per) {
        cr = fem_wrap(cr, cuy);
        cc = fem_wrap(cc, cux);
      } else {
        cr = cr < 0 ? 0 : (cr >= cuy ? cuy - 1 : cr);
        cc = cc < 0 ? 0 : (cc >= cux ? cux - 1 : cc);
      }
      return cr * cux + cc;
    });
    fem_stage(sr, L.r, 32 * TY, oidx);
    fem_stage(sd, L.invD, 32 * TY, oidx);
    read_means();
    fem_trace_mark(A.sync, 11);
    fem_stage_wait();
    // y = X_n + P X_{n+1} in place (the arithmetic of fem_interp_at)
    for (int q = threadIdx.x; q < NS; q += blockDim.x) {
      int fr, fc;
      fcoord(q, fr, fc);
      double y;
      if (pinned && sw[q] == 0.0) {
        y = 0.0;
      } else {
        const int Rr = fem_floordiv2(fr) - cr0, Cc = fem_floordiv2(fc) - cc0;
        auto xH = [&](int dr, int dc) -> double {
          const double v = sc[(Rr + dr) * CXB + Cc + dc];
          return pinned ? v : v - mX;
        };
        double xh;
        if (!(fr & 1) && !(fc & 1)) xh = xH(0, 0);
        else if (!(fr & 1)) xh = 0.5 * xH(0, 0) + 0.5 * xH(0, 1);
        else if (!(fc & 1)) xh = 0.5 * xH(0, 0) + 0.5 * xH(1, 0);
        else xh = 0.25 * xH(0, 0) + 0.25 * xH(0, 1) + 0.25 * xH(1, 0) + 0.25 * xH(1, 1);
        y = sy[q] + (pinned ? xh : xh - mP);
      }
      sy[q] = y;
    }
    __syncthreads();
    // Jacobi: x = w (rh - Loff y)/D + (1-w) y on the owned nodes
    for (int ty = ty0; ty < TY; ty += WR) {
      const int x = x0 + tx, yy = y0 + ty;
      if (x < ux && yy < uy) {
        const int cx = fem_axis_cls(KIND, per, x, g.nex), cy = fem_axis_cls(KIND, per, yy, g.ney);
        const double* cf = tabo + (size_t)(cy * nc + cx) * NOFF;
        double off = 0.0;
#pragma unroll
        for (int dy = 0; dy < W; ++dy)
#pragma unroll
          for (int dx = 0; dx < W; ++dx) off += cf[dy * W + dx] * sy[(ty + dy) * SX + tx + dx];
        const int qc = (ty + R) * SX + tx + R;
        const double yi = sy[qc];
        const double rhv = sr[ty * 32 + tx];
        const double rv = (!pinned && n > 0) ? rhv - f.alpha * fem_restrict_rowsum(L.lat, yy, x) - f.beta : rhv;
        double xn = w * (rv - off) * sd[ty * 32 + tx] + (1.0 - w) * yi;
        if (pinned && sw[qc] == 0.0) xn = 0.0;
        L.t[yy * ux + x] = xn;
        if (n == 0) {
          a[0] += xn;
          a[1] += rhv * xn;
        } else {
          a[0] += xn;
          a[1] += fem_interp_colsum(L.lat, yy, x) * xn;
        }
      }
    }
    __syncthreads();
  }
  fem_trace_mark(A.sync, 12);
  if (n == 0 || !pinned) {
    const int sl[2] = {SL_X(n), SL_X(n) + 1};
    return tm.template reduce_sync<2>(a, sl, smem);
  }
  return tm.sync();
}

// ---------------------------------------------------------------------------
// The coarse end of the V-cycle inside one CTA, vectors in shared memory
// ---------------------------------------------------------------------------
// Levels s = A.block_smem_from .. N-1 run in CTA 0 with __syncthreads only,
// as core/multigrid.py:231-330 writes them (explicit means, no lazy affine
// terms): no grid or team barrier and no global-memory round trip inside.
// In: u_s = R t_{s-1} (lv[s].r, raw, from the phase that restricted it) and,
// mean-zero, the sum of t_{s-1} (slot SL_T(s-1)). Out: the level's corrected
// X_s in lv[s].t and, mean-zero, its sums in SL_X(s) (CTA 0's column; the
// other columns of that slot stay zero), which the up-sweep of level s-1
// consumes as it would a team level's. Vectors r_l, x_l of every block level
// and one scratch sit in the tile region after the coarse warp CG's p buffer.

// stencil of level L (table tab) at unique node (ix, iy) on the unique-lattice
// vector v (wrapped, or clamped where the table's coefficient is zero)
template <int KIND>
__device__ __forceinline__ double mg_blk_stencil(const MgLevel& L, const double* __restrict__ tab,
                                                 const double* __restrict__ v, int ix, int iy) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF;
  const FemGrid& g = L.g;
  const int per = g.periodic, nnx = g.nnx, nny = g.nny;
  const int nc = fem_axis_ncls(KIND, per);
  const double* c = tab + (size_t)(fem_axis_cls(KIND, per, iy, g.ney) * nc + fem_axis_cls(KIND, per, ix, g.nex)) * NOFF;
  double y = 0.0;
#pragma unroll
  for (int dy = 0; dy < W; ++dy) {
    int w = iy + dy - R;
    w = per ? fem_wrap(w, nny) : min(max(w, 0), nny - 1);
#pragma unroll
    for (int dx = 0; dx < W; ++dx) {
      int u = ix + dx - R;
      u = per ? fem_wrap(u, nnx) : min(max(u, 0), nnx - 1);
      y += c[dy * W + dx] * v[w * nnx + u];
    }
  }
  return y;
}

// R t at coarse unique node (Rr, Cc) of the level below F (the sums of mg_down)
__device__ __forceinline__ double mg_blk_restrict(const FemLattice& F, const double* __restrict__ t, int Rr, int Cc) {
  const int fy = 2 * Rr, fx = 2 * Cc, ux = F.ux(), uy = F.uy();
  const bool up = fy + 1 < F.ny, dn = fy - 1 >= 0, rt = fx + 1 < F.nx, lf = fx - 1 >= 0;
  auto at = [&](int y, int x) -> double {
    y = y >= uy ? y - uy : y;
    x = x >= ux ? x - ux : x;
    return t[y * ux + x];
  };
  double e = 0.0, d = 0.0;
  if (up) e += at(fy + 1, fx);
  if (dn) e += at(fy - 1, fx);
  if (rt) e += at(fy, fx + 1);
  if (lf) e += at(fy, fx - 1);
  if (up && rt) d += at(fy + 1, fx + 1);
  if (up && lf) d += at(fy + 1, fx - 1);
  if (dn && rt) d += at(fy - 1, fx + 1);
  if (dn && lf) d += at(fy - 1, fx - 1);
  return at(fy, fx) + 0.5 * e + 0.25 * d;
}

// P x at fine unique node (fr, fc) from the coarse unique-lattice vector x
// (core/multigrid.py:90-140, the arithmetic of mg_up)
__device__ __forceinline__ double mg_blk_prolong(const FemLattice& C, const double* __restrict__ x, int fr, int fc) {
  const int cux = C.ux(), cuy = C.uy(), Rr = fr >> 1, Cc = fc >> 1;
  auto xH = [&](int dr, int dc) -> double {
    int r = Rr + dr, c = Cc + dc;
    r = r >= cuy ? r - cuy : r;
    c = c >= cux ? c - cux : c;
    return x[r * cux + c];
  };
  if (!(fr & 1) && !(fc & 1)) return xH(0, 0);
  if (!(fr & 1)) return 0.5 * xH(0, 0) + 0.5 * xH(0, 1);
  if (!(fc & 1)) return 0.5 * xH(0, 0) + 0.5 * xH(1, 0);
  return 0.25 * xH(0, 0) + 0.25 * xH(0, 1) + 0.25 * xH(1, 0) + 0.25 * xH(1, 1);
}

// mean of a block-local sum (every thread gets it)
__device__ __forceinline__ double mg_blk_mean(double v, int nn, double* smem) {
  double a[1] = {v};
  fem_block_sum<1>(a, smem);
  return a[0] / nn;
}

template <int KIND, bool PIN>
__device__ __noinline__ void mg_block_levels(const GridReducer& gr, const CgArgs& A, double* smem) {
  const BlockTeam tm;
  const int N = A.nlev, s = A.block_smem_from;
  const double w = 2.0 / 3.0;
  double* base = smem + 128 + FEM_COARSE_WARP_NN;
  // r_l at base + ro(l), x_l right after it; the scratch after the last level
  auto ro = [&](int l) {
    int o = 0;
    for (int m = s; m < l; ++m) o += 2 * A.lv[m].g.nn;
    return o;
  };
  double* tv = base + ro(N);
  // 1. the stored rhs of level s: u_s (pinned), or R(t - mean t) - its mean
  {
    const MgLevel& L = A.lv[s];
    const int nn = L.g.nn, ux = L.lat.ux();
    double* r = base + ro(s);
    double alpha = 0.0;
    if (!PIN) {
      const int sl[1] = {SL_T(s - 1)};
      double u[1];
      gr.result_slots<1>(u, sl, smem);
      alpha = u[0] * A.lv[s - 1].inv_nn;
    }
    double a = 0.0;
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      double v = L.r[i];
      if (!PIN) v -= alpha * fem_restrict_rowsum(L.lat, i / ux, i % ux);
      r[i] = v;
      a += v;
    }
    if (!PIN) {
      const double beta = mg_blk_mean(a, nn, smem);
      for (int i = tm.rank(); i < nn; i += tm.size()) r[i] -= beta;
    }
    __syncthreads();
  }
  // 2. down: pre-smooth from zero, residual, restriction
  for (int n = s; n < N - 1; ++n) {
    const MgLevel& L = A.lv[n];
    const MgLevel& C = A.lv[n + 1];
    const int nn = L.g.nn, ux = L.lat.ux(), cux = C.lat.ux(), cnn = C.g.nn;
    const double* __restrict__ d = A.bd[n];
    double* r = base + ro(n);
    double* x = r + nn;
    double* rc = base + ro(n + 1);
    const double mr = PIN ? 0.0 : mg_blk_mean([&] {
      double a = 0.0;
      for (int i = tm.rank(); i < nn; i += tm.size()) a += r[i];
      return a;
    }(), nn, smem);
    double a = 0.0;
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      const double rh = PIN ? (d[i] == 0.0 ? 0.0 : r[i]) : r[i] - mr;
      const double xh = w * rh * d[i];
      tv[i] = rh;
      x[i] = xh;
      a += xh;
    }
    if (!PIN) {
      const double mx = mg_blk_mean(a, nn, smem);
      for (int i = tm.rank(); i < nn; i += tm.size()) x[i] -= mx;
    }
    __syncthreads();
    a = 0.0;
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      double Lx = mg_blk_stencil<KIND>(L, L.tab, x, i % ux, i / ux);
      if (PIN && d[i] == 0.0) Lx = 0.0;
      const double t = tv[i] - Lx;
      tv[i] = t;
      a += t;
    }
    if (!PIN) {
      const double mt = mg_blk_mean(a, nn, smem);
      for (int i = tm.rank(); i < nn; i += tm.size()) tv[i] -= mt;
    }
    __syncthreads();
    a = 0.0;
    for (int I = tm.rank(); I < cnn; I += tm.size()) {
      const double v = mg_blk_restrict(L.lat, tv, I / cux, I % cux);
      rc[I] = v;
      a += v;
    }
    if (!PIN) {
      const double mh = mg_blk_mean(a, cnn, smem);
      for (int I = tm.rank(); I < cnn; I += tm.size()) rc[I] -= mh;
    }
    __syncthreads();
  }
  // 3. coarsest level: one Jacobi sweep from zero (mean-zero) or the warp CG (pinned)
  {
    const MgLevel& L = A.lv[N - 1];
    const int nn = L.g.nn;
    const double* __restrict__ d = A.bd[N - 1];
    double* r = base + ro(N - 1);
    double* x = r + nn;
    if (!PIN) {
      double a = 0.0;
      for (int i = tm.rank(); i < nn; i += tm.size()) a += r[i];
      const double mr = mg_blk_mean(a, nn, smem);
      a = 0.0;
      for (int i = tm.rank(); i < nn; i += tm.size()) {
        const double v = w * (r[i] - mr) * d[i];
        x[i] = v;
        a += v;
      }
      const double mx = mg_blk_mean(a, nn, smem);
      for (int i = tm.rank(); i < nn; i += tm.size()) x[i] -= mx;
    } else if constexpr (PIN && KIND != FEM_HEX8) {
      for (int i = tm.rank(); i < nn; i += tm.size()) L.r[i] = r[i];
      __syncthreads();
      if (threadIdx.x < 32) mg_coarse_warp<KIND>(A, smem + 128);
      __syncthreads();
      for (int i = tm.rank(); i < nn; i += tm.size()) x[i] = L.t[i];
    }
    __syncthreads();
  }
  // 4. up: prolongate, add, one weighted Jacobi sweep
  for (int n = N - 2; n >= s; --n) {
    const MgLevel& L = A.lv[n];
    const MgLevel& C = A.lv[n + 1];
    const int nn = L.g.nn, ux = L.lat.ux();
    const double* __restrict__ d = A.bd[n];
    double* r = base + ro(n);
    double* x = r + nn;
    const double* xc = base + ro(n + 1) + C.g.nn;
    double a = 0.0;
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      const double p = mg_blk_prolong(C.lat, xc, i / ux, i % ux);
      tv[i] = p;
      a += p;
    }
    const double mp = PIN ? 0.0 : mg_blk_mean(a, nn, smem);
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      const double y = x[i] + (tv[i] - mp);
      tv[i] = (PIN && d[i] == 0.0) ? 0.0 : y;
    }
    __syncthreads();
    a = 0.0;
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      const double off = mg_blk_stencil<KIND>(L, L.tab_off, tv, i % ux, i / ux);
      double xn = w * (r[i] - off) * d[i] + (1.0 - w) * tv[i];
      if (PIN && d[i] == 0.0) xn = 0.0;
      x[i] = xn;
      a += xn;
    }
    if (!PIN) {
      const double mj = mg_blk_mean(a, nn, smem);
      for (int i = tm.rank(); i < nn; i += tm.size()) x[i] -= mj;
    }
    __syncthreads();
  }
  // 5. X_s out, with its sums for the level above (mean-zero)
  {
    const MgLevel& L = A.lv[s];
    const int nn = L.g.nn, ux = L.lat.ux();
    const double* x = base + ro(s) + nn;
    double a[2] = {0.0, 0.0};
    for (int i = tm.rank(); i < nn; i += tm.size()) {
      const double v = x[i];
      L.t[i] = v;
      if (!PIN) {
        a[0] += v;
        a[1] += fem_interp_colsum(L.lat, i / ux, i % ux) * v;
      }
    }
    if (!PIN) gr.reduce<2>(a, SL_X(s), smem);
    __syncthreads();
  }
}

// Full V-cycle on r = lv[0].r; result in lv[0].t (raw; mean-zero subtracts
// SL_X(0)[0]/nn lazily). Levels < block_from run on the whole grid; levels from
// block_from down run on the team of the first A.team CTAs (GridTeam::team barriers,
// data in global memory), the coarsest solve in CTA 0. Grid-produced sums are
// read over all CTA columns; team phases write only the team's columns (the
// rest of those slots stay zero), so the same reads stay exact.
template <int KIND, bool PIN>
__device__ __noinline__ bool mg_vcycle(const GridTeam& gt, const GridReducer& gr, const CgArgs& A, double* smem,
                                       unsigned int* team_round, double* cg_r, double* cg_p, double* cg_q) {
  const int N = A.nlev, s = A.block_from;
  for (int n = 0; n < s; ++n)
    if (!mg_down<KIND, PIN>(gt, gr, A, n, smem)) return false;
  const int b = A.block_smem_from < N ? A.block_smem_from : N - 1;  // team levels: [s, b)
  if ((int)blockIdx.x < A.team) {
    const GridTeam tt = GridTeam::team(gt.s, team_round, A.team);
    for (int n = s; n < b; ++n)
      if (!mg_down<KIND, PIN>(tt, gr, A, n, smem)) return false;
    fem_trace_mark(A.sync, 7);
    if (b < N - 1 || A.block_smem_from == N - 1) {
      // levels b.. inside CTA 0 from shared memory (2D)
      if constexpr (KIND != FEM_HEX8) {
        if (blockIdx.x == 0) mg_block_levels<KIND, PIN>(gr, A, smem);
      }
      fem_trace_mark(A.sync, 8);
    } else if (blockIdx.x == 0) {
      bool warp_solve = false;
      if constexpr (PIN && KIND != FEM_HEX8) warp_solve = A.lv[N - 1].g.nn <= FEM_COARSE_WARP_NN;
      if (warp_solve) {
        if constexpr (PIN && KIND != FEM_HEX8) {
          if (threadIdx.x < 32) mg_coarse_warp<KIND>(A, smem + 128);
        }
        __syncthreads();
      } else {
        mg_coarse<KIND, PIN>(gr, A, smem, cg_r, cg_p, cg_q);
      }
      fem_trace_mark(A.sync, 8);
      const MgLevel& Lc = A.lv[N - 1];
      if (N == 1) {
        // single level: the coarse solve is the whole preconditioner; r.z pieces
        double a[2] = {0.0, 0.0};
        for (int i = threadIdx.x; i < Lc.g.nn; i += blockDim.x) {
          a[0] += Lc.t[i];
          a[1] += Lc.r[i] * Lc.t[i];
        }
        gr.reduce<2>(a, SL_X(0), smem);
      } else if (!PIN) {
        double a[2] = {0.0, 0.0};
        for (int i = threadIdx.x; i < Lc.g.nn; i += blockDim.x) mg_xsums(Lc, i, Lc.t[i], a);
        gr.reduce<2>(a, SL_X(N - 1), smem);
      }
    }
    if (!tt.sync()) return false;
    for (int n = b - 1; n >= s; --n)
      if (!mg_up<KIND, PIN>(tt, gr, A, n, smem)) return false;
    fem_trace_mark(A.sync, 10);
  }
  if (!gt.sync()) return false;
  for (int n = s - 1; n >= 0; --n)
    if (!mg_up<KIND, PIN>(gt, gr, A, n, smem)) return false;
  return true;
}
