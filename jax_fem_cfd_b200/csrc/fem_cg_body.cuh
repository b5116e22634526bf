// Device code of the persistent MG-PCG solve (k_cg and the packed step).
#pragma once
#include "fem_args.cuh"

// Preconditioner application z = M r; returns gamma = r . z.
template <int KIND, bool PIN>
__device__ __noinline__ bool cg_apply_prec(const GridTeam& gt, const GridReducer& gr, const CgArgs& A, double* smem,
                              unsigned int* team_round, double* cg_r, double* cg_p, double* cg_q, double rr, double r2d,
                              double& gamma, double& mz, bool defer = false) {
  const MgLevel& L0 = A.lv[0];
  const int nn = L0.g.nn;
  mz = 0.0;
  if (A.prec == FEM_PREC_NONE) {
    gamma = rr;
    return true;
  }
  if (A.prec == FEM_PREC_JACOBI) {
    gamma = r2d;
    return true;
  }
  if (A.prec == FEM_PREC_MG) {
    if (!mg_vcycle<KIND, PIN>(gt, gr, A, smem, team_round, cg_r, cg_p, cg_q)) return false;
    if (defer) return true;  // the caller reads gamma and mz (cg_mg_results) later
    if (PIN) {
      double s[2];
      gr.result<2>(s, SL_X(0), smem);
      gamma = s[1];
    } else {
      double s[3];
      const int sl[3] = {SL_X(0), SL_X(0) + 1, SL_R(0)};
      gr.result_slots<3>(s, sl, smem);
      mz = s[0] * L0.inv_nn;
      gamma = s[1] - mz * s[2];
    }
    return true;
  }
  // approximate inverse: 2-term Neumann series
  const bool pt = (A.prec == FEM_PREC_APPROX_INV_PT);
  const double* __restrict__ r = A.r;
  const double* __restrict__ D = L0.diag;
  const uint8_t* __restrict__ ap = A.ai_pin;
  double* __restrict__ T = L0.t;
  const double* __restrict__ iD = L0.invD;
  const double* src1[2] = {r, iD};
  fem_tiled_stencil<KIND, 2>(gt, L0.g, L0.tab, smem + 128, src1,
                             [](int, const double(&v)[2]) { return v[0] * v[1]; },
                             [&](int i, int, int, int, double v, double) {
                            double d1l = v / D[i];
                            if (ap && ap[i]) d1l = pt ? r[i] / D[i] : 0.0;
                            T[i] = d1l;
                          });
  if (!gt.sync()) return false;
  double acc[1] = {0.0};
  const double* src2[1] = {T};
  fem_tiled_stencil<KIND, 1>(gt, L0.g, L0.tab, smem + 128, src2, [](int, const double(&v)[1]) { return v[0]; },
                             [&](int i, int, int, int, double t, double) {
    if (ap && ap[i]) t = pt ? T[i] : 0.0;
    const double zi = 3 * (r[i] / D[i]) - 3 * T[i] + t / D[i];
    A.z[i] = zi;
    acc[0] += r[i] * zi;
  });
  gr.reduce<1>(acc, SL_RZ, smem);
  if (!gt.sync()) return false;
  double s[1];
  gr.result<1>(s, SL_RZ, smem);
  gamma = s[0];
  return true;
}

// gamma = r.z and the lazy mean mz of z after a V-cycle (mean-zero: z - mean z),
// from the slots {SL_X(0), SL_X(0) + 1, SL_R(0)}
__device__ __forceinline__ void cg_mg_slots(int (&sl)[3]) {
  sl[0] = SL_X(0);
  sl[1] = SL_X(0) + 1;
  sl[2] = SL_R(0);
}
template <bool PIN>
__device__ __forceinline__ void cg_mg_from(const CgArgs& A, const double (&s)[3], double& gamma, double& mz) {
  if (PIN) {
    gamma = s[1];
    mz = 0.0;
  } else {
    mz = s[0] * A.lv[0].inv_nn;
    gamma = s[1] - mz * s[2];
  }
}

// The MG-PCG solve of k_cg on the CTAs of one launch (or of one group of a
// packed launch: blockIdx.x / gridDim.x index the group's CTAs). A in shared
// memory; smem: [0,128) reductions, [128, +FEM_TILE_SMEM) tiles; s_round /
// s_team_round: the CTA's completed grid / team barriers on A.sync's counters,
// carried over between solves that share them.
template <int KIND, bool PIN>
__device__ __forceinline__ void cg_solve(const CgArgs& A, double* smem, unsigned int* s_round,
                                         unsigned int* s_team_round, double* cg_r, double* cg_p, double* cg_q) {
  const GridTeam gt = GridTeam::grid(&A.sync, s_round);
  const GridReducer gr{&A.sync};
  const MgLevel& L0 = A.lv[0];
  const FemGrid& g = L0.g;
  const int nn = g.nn;
  const uint8_t* pin0 = PIN ? L0.pin : nullptr;
  const double* __restrict__ D = L0.diag;
  int k = 0;
  double rr = 0.0;
  fem_zero_partials(A.sync);
  if (!gt.sync()) goto done;
  {
    const double* b = A.b;
    if (A.center_rhs) {
      double a[1] = {0.0};
      for (int i = gt.rank(); i < nn; i += gt.size()) a[0] += b[i];
      gr.reduce<1>(a, SL_BSUM, smem);
      if (!gt.sync()) goto done;
      double s[1];
      gr.result<1>(s, SL_BSUM, smem);
      const double m = s[0] / nn;
      for (int i = gt.rank(); i < nn; i += gt.size()) A.bwork[i] = b[i] - m;
      b = A.bwork;
    }
    // r0 = b - A x0
    {
      double a2[2] = {0.0, 0.0}, a3[2] = {0.0, 0.0}, a1[1] = {0.0};
      const double* srcx[1] = {A.x};
      fem_tiled_stencil<KIND, 1>(gt, g, L0.tab, smem + 128, srcx, [](int, const double(&v)[1]) { return v[0]; },
                                 [&](int i, int, int, int, double Ax, double) {
        if (pin0 && pin0[i]) Ax = 0.0;
        const double bi = b[i], ri = bi - Ax;
        A.r[i] = ri;
        a2[0] += bi * bi;
        a2[1] += ri * ri;
        a3[0] += ri;
        a3[1] += ri * L0.invD[i];
        a1[0] += ri * ri * L0.invD[i];
      });
      gr.reduce<2>(a2, SL_BB, smem);
      gr.reduce<2>(a3, SL_R(0), smem);
      gr.reduce<1>(a1, SL_RZ, smem);
      if (!gt.sync()) goto done;
    }
    double bb_rr[2], r2d[1];
    gr.result<2>(bb_rr, SL_BB, smem);
    gr.result<1>(r2d, SL_RZ, smem);
    rr = bb_rr[1];
    const double atol2 = fmax(A.tol * A.tol * bb_rr[0], A.atol * A.atol);
    double gamma, mz;
    if (!cg_apply_prec<KIND, PIN>(gt, gr, A, smem, s_team_round, cg_r, cg_p, cg_q, rr, r2d[0], gamma, mz)) goto done;
    double beta = 0.0;
    bool have_p = false;
    bool pending = false;  // MG: gamma / mz of the last V-cycle are read in the next phase A
    int cur = 0;
    double rs = (A.prec == FEM_PREC_NONE) ? gamma : rr;
    const unsigned long long t_start = fem_globaltimer_early();
    while (rs > atol2 && k < A.maxiter) {
      if (fem_watchdog_fired(A.sync.err)) break;
      double* __restrict__ pold = cur ? A.p1 : A.p0;
      double* __restrict__ pnew = cur ? A.p0 : A.p1;
      const int prec = A.prec;
      const double* __restrict__ r = A.r;
      const double* __restrict__ zs = (prec == FEM_PREC_MG) ? L0.t : A.z;
      {
        // p = z + beta p_old staged and combined in smem; Ap on the owned nodes
        const double* srcA[3] = {(prec == FEM_PREC_NONE || prec == FEM_PREC_JACOBI) ? r : zs,
                                 have_p ? pold : nullptr, prec == FEM_PREC_JACOBI ? D : nullptr};
        auto comb = [&](int, const double(&v)[3]) -> double {
          double zv;
          if (prec == FEM_PREC_JACOBI) zv = v[0] / v[2];
          else if (prec == FEM_PREC_MG) zv = v[0] - mz;
          else zv = v[0];
          return have_p ? zv + beta * v[1] : zv;
        };
        // pending V-cycle sums: loads issued here, combined while the copies fly
        int msl[3];
        cg_mg_slots(msl);
        GridReducer::Pending<3> mpend{};
        if (pending) mpend = gr.result_begin<3>(msl);
        auto pre = [&]() {
          if (!pending) return;
          double s3[3], gamma_;
          gr.result_end<3>(mpend, s3, smem);
          cg_mg_from<PIN>(A, s3, gamma_, mz);
          beta = gamma_ / gamma;
          gamma = gamma_;
          pending = false;
        };
        double a[1] = {0.0};
        fem_tiled_stencil<KIND, 3>(gt, g, L0.tab, smem + 128, srcA, comb,
                                   [&](int i, int, int, int, double q, double pn) {
                                     pnew[i] = pn;
                                     if (pin0 && pin0[i]) q = 0.0;
                                     A.Ap[i] = q;
                                     a[0] += pn * q;
                                   },
                                   pre);
        const int slp[1] = {SL_PAP};
        if (!gt.reduce_sync<1>(a, slp, smem)) goto done;
      }
      double pap[1];
      gr.result<1>(pap, SL_PAP, smem);
      const double alpha = gamma / pap[0];
      {
        // x += alpha p, r -= alpha Ap; loads of a batch of nodes first
        double a4[4] = {0.0, 0.0, 0.0, 0.0};  // r.r, sum r, sum r / D (via 1/D), sum r^2 / D
        constexpr int U = 2;
        const int stride = gt.size();
        const double* __restrict__ iD0 = L0.invD;
        for (int i0 = gt.rank(); i0 < nn; i0 += U * stride) {
          double xv[U], pv[U], rv[U], av[U], iv[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i < nn) {
              xv[u] = A.x[i];
              pv[u] = pnew[i];
              rv[u] = A.r[i];
              av[u] = A.Ap[i];
              iv[u] = iD0[i];
            }
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            if (i < nn) {
              A.x[i] = xv[u] + alpha * pv[u];
              const double ri = rv[u] - alpha * av[u];
              A.r[i] = ri;
              a4[0] += ri * ri;
              a4[1] += ri;
              a4[2] += ri * iv[u];
              a4[3] += ri * ri * iv[u];
            }
          }
        }
        const int sl4[4] = {SL_RR, SL_R(0), SL_R(0) + 1, SL_RZ};
        fem_watchdog_arm(A.sync.err, t_start);
        if (!gt.reduce_sync<4>(a4, sl4, smem)) goto done;
      }
      ++k;
      double t2[2];
      const int slrz[2] = {SL_RR, SL_RZ};
      gr.result_slots<2>(t2, slrz, smem);
      rr = t2[0];
      double t1[1] = {t2[1]};
      double gamma_;
      if (prec == FEM_PREC_NONE) {
        gamma_ = rr;
      } else if (prec == FEM_PREC_JACOBI) {
        gamma_ = t1[0];
      } else {
        if (!(rr > atol2 && k < A.maxiter)) break;  // z of a final iteration is never used
        const bool defer = (prec == FEM_PREC_MG);
        if (!cg_apply_prec<KIND, PIN>(gt, gr, A, smem, s_team_round, cg_r, cg_p, cg_q, rr, t1[0], gamma_, mz, defer))
          goto done;
        pending = defer;
      }
      if (!pending) {
        beta = gamma_ / gamma;
        gamma = gamma_;
      }
      have_p = true;
      cur ^= 1;
      rs = (prec == FEM_PREC_NONE) ? gamma : rr;
      if (!isfinite(rs)) break;
    }
    // final modification of solvers/standard.py:119-123
    if (A.post) {
      if (PIN) {
        for (int i = gt.rank(); i < nn; i += gt.size())
          if (pin0 && pin0[i]) A.x[i] = 0.0;
      } else {
        double a[1] = {0.0};
        for (int i = gt.rank(); i < nn; i += gt.size()) a[0] += A.x[i];
        gr.reduce<1>(a, SL_BSUM, smem);
        if (!gt.sync()) goto done;
        double s[1];
        gr.result<1>(s, SL_BSUM, smem);
        const double m = s[0] / nn;
        for (int i = gt.rank(); i < nn; i += gt.size()) A.x[i] = A.x[i] - m;
      }
    }
  }
done:
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int st = *(volatile int*)A.sync.err & (FEM_ERR_BARRIER_TIMEOUT | FEM_ERR_WATCHDOG);
    if (!isfinite(rr)) st |= FEM_ERR_NONFINITE;
    if (k >= A.maxiter) st |= FEM_ERR_MAXITER;
    *A.iters = k;
    *A.status = st;
    if (A.final_rr) *A.final_rr = rr;
  }
}

