// Device code of the persistent BiCGSTAB solve (k_bicgstab and the packed step).
#pragma once
#include "fem_b200.h"
#include "fem_args.cuh"

template <int KIND, int NC, class Src>
__device__ __forceinline__ void bi_apply(const BiArgs& A, const MatCombo& op, int i, const Src& src, double (&y)[NC]) {
  int ix, iy, iz;
  fem_ij(A.g, i, ix, iy, iz);
  fem_gather_k<KIND, NC>(A.g, ix, iy, iz, op, src, y);
  if (A.mask) {
#pragma unroll
    for (int c = 0; c < NC; ++c)
      if (A.mask[i + (size_t)c * A.g.nn]) y[c] = src(i, c);
  }
}

// The operator apply of the solver: the element-by-element product of op on
// load(j, c), or (OTF) op.alpha op.A + cv_coef Ce from Gauss-point factors on
// comb of the staged sources (Ce never materialised).
template <int KIND, int NC, bool OTF, int NSRC, class Team, class Load, class Comb, class Body>
__device__ __forceinline__ void bi_tiled_apply(const Team& tm, const BiArgs& A, const MatCombo& op, double* tsm,
                                               const FemC3Tma& tma, const Load& load,
                                               const double* const (&src)[NSRC], const Comb& comb,
                                               const Body& body) {
  if constexpr (OTF && KIND == FEM_HEX8) {
    fem_tiled_conv3<NC, NSRC>(tm, A.g, tsm, tma, src, comb, A.cvf, A.qt, A.cv_coef, op.alpha, op.A, body);
  } else if constexpr (OTF) {
    fem_tiled_conv<KIND, NC, NSRC>(tm, A.g, tsm, src, comb, A.cvf, A.qt, A.cv_coef, op.alpha, op.A, body);
  } else if constexpr (KIND == FEM_HEX8) {
    // explicit per-element matrices: element-centric (fem_tiled_ebe3e); other
    // combinations (transposed B, a third matrix) node-centric
    if (op.B && !op.transB && !op.C) fem_tiled_ebe3e<NC>(tm, A.g, tsm, load, op, body);
    else fem_tiled_ebe<KIND, NC>(tm, A.g, tsm, load, op, body);
  } else {
    fem_tiled_ebe<KIND, NC>(tm, A.g, tsm, load, op, body);
  }
}

// The BiCGSTAB solve of k_bicgstab on the CTAs of one launch (or of one group of
// a packed launch). op: the operator with its shared matrix (if any) already in
// shared memory; smem: 128 doubles of reduction scratch; tsm: the tiled
// operator's staging; s_round: the CTA's completed barriers on A.sync's counter.
template <int KIND, int NC, bool OTF>
__device__ __forceinline__ void bicgstab_solve(const BiArgs& A, const MatCombo& op, double* smem, double* tsm,
                                               const FemC3Tma& tma, unsigned int* s_round) {
  const GridTeam gt = GridTeam::grid(&A.sync, s_round);
  const GridReducer gr{&A.sync};
  const int nn = A.g.nn;
  const size_t N = nn;
  int k = 0;
  double rr = 0.0;
  fem_zero_partials(A.sync);
  if (!gt.sync()) goto done;
  {
    {
      double a[2] = {0.0, 0.0};
      const double* sx0[1] = {A.x};
      bi_tiled_apply<KIND, NC, OTF>(gt, A, op, tsm, tma, [&](int j, int c) { return A.x[j + c * N]; }, sx0,
                                    [](int, const double(&v)[1]) { return v[0]; },
                              [&](int i, const double(&Ax)[NC], const double(&xc)[NC]) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          const size_t o = i + c * N;
          const double ax = (A.mask && A.mask[o]) ? xc[c] : Ax[c];
          const double bi = A.b[o], ri = bi - ax;
          A.r[o] = ri;
          A.rhat[o] = ri;
          A.p0[o] = ri;
          A.q0[o] = ri;
          a[0] += bi * bi;
          a[1] += ri * ri;
        }
      });
      gr.reduce<2>(a, SL_BB, smem);
      if (!gt.sync()) goto done;
    }
    double bb[2];
    gr.result<2>(bb, SL_BB, smem);
    rr = bb[1];
    double rhr = bb[1];
    const double atol2 = fmax(A.tol * A.tol * bb[0], A.atol * A.atol);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    int cur = 0;
    const unsigned long long t_start = fem_globaltimer_early();
    while (rr > atol2 && k < A.maxiter && k >= 0) {
      if (fem_watchdog_fired(A.sync.err)) break;
      const double rho_ = rhr;
      const double beta = rho_ / rho * alpha / omega;
      double* __restrict__ pold = cur ? A.p1 : A.p0;
      double* __restrict__ pnew = cur ? A.p0 : A.p1;
      double* __restrict__ qold = cur ? A.q1 : A.q0;
      double* __restrict__ qnew = cur ? A.q0 : A.q1;
      const double* __restrict__ r = A.r;
      {
        auto pn = [&](int j, int c) {
          const size_t o = j + c * N;
          return r[o] + beta * (pold[o] - omega * qold[o]);
        };
        double a[1] = {0.0};
        const double* spn[3] = {r, pold, qold};
        bi_tiled_apply<KIND, NC, OTF>(gt, A, op, tsm, tma, pn, spn,
                                      [&](int, const double(&v)[3]) { return v[0] + beta * (v[1] - omega * v[2]); },
                                      [&](int i, const double(&qv)[NC], const double(&pc)[NC]) {
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            const size_t o = i + c * N;
            const double q = (A.mask && A.mask[o]) ? pc[c] : qv[c];
            pnew[o] = pc[c];
            qnew[o] = q;
            a[0] += A.rhat[o] * q;
          }
        });
        gr.reduce<1>(a, SL_BI + 1, smem);
        if (!gt.sync()) goto done;
      }
      double rq[1];
      gr.result<1>(rq, SL_BI + 1, smem);
      const double alpha_ = rho_ / rq[0];
      auto sv = [&](int j, int c) {
        const size_t o = j + c * N;
        return r[o] - alpha_ * qnew[o];
      };
      {
        double a[3] = {0.0, 0.0, 0.0};
        const double* ssv[2] = {r, qnew};
        bi_tiled_apply<KIND, NC, OTF>(gt, A, op, tsm, tma, sv, ssv,
                                      [&](int, const double(&v)[2]) { return v[0] - alpha_ * v[1]; }, [&](int i, const double(&tvv)[NC], const double(&sc)[NC]) {
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            const size_t o = i + c * N;
            const double tvc = (A.mask && A.mask[o]) ? sc[c] : tvv[c];
            const double s = sc[c];
            A.t[o] = tvc;
            a[0] += s * s;
            a[1] += tvc * s;
            a[2] += tvc * tvc;
          }
        });
        gr.reduce<3>(a, SL_BI + 2, smem);
        if (!gt.sync()) goto done;
      }
      double st[3];
      gr.result<3>(st, SL_BI + 2, smem);
      const double omega_ = st[1] / st[2];
      const bool exit_early = st[0] < atol2;
      {
        double a[2] = {0.0, 0.0};
        for (int i = gt.rank(); i < nn; i += gt.size()) {
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            const size_t o = i + c * N;
            const double s = sv(i, c);
            double xn, rn;
            if (exit_early) {
              xn = A.x[o] + alpha_ * pnew[o];
              rn = s;
            } else {
              xn = A.x[o] + (alpha_ * pnew[o] + omega_ * s);
              rn = s - omega_ * A.t[o];
            }
            A.x[o] = xn;
            A.r[o] = rn;
            a[0] += rn * rn;
            a[1] += A.rhat[o] * rn;
          }
        }
        gr.reduce<2>(a, SL_RR, smem);  // SL_RR, SL_RSUM (= rhat.r)
        fem_watchdog_arm(A.sync.err, t_start);
        if (!gt.sync()) goto done;
      }
      double nr[2];
      gr.result<2>(nr, SL_RR, smem);
      rr = nr[0];
      rhr = nr[1];
      int k_ = (omega_ == 0.0 || alpha_ == 0.0) ? -11 : k + 1;
      if (rho_ == 0.0) k_ = -10;
      k = k_;
      rho = rho_;
      alpha = alpha_;
      omega = omega_;
      cur ^= 1;
    }
  }
done:
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int st = *(volatile int*)A.sync.err & (FEM_ERR_BARRIER_TIMEOUT | FEM_ERR_WATCHDOG);
    if (!isfinite(rr)) st |= FEM_ERR_NONFINITE;
    if (k >= A.maxiter) st |= FEM_ERR_MAXITER;
    if (k < 0) st |= FEM_ERR_BREAKDOWN;
    *A.iters = k;
    *A.status = st;
  }
}

