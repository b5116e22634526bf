// 4-step projection stage kernels and the scalar-transport rhs.
#include "fem_args.cuh"


// rhs of solvers/standard.py:31-37 and the initial guess x0; also keeps G P_n.
template <int KIND>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_mom_rhs(StepArgs S, const double* __restrict__ Un,
                                                            const double* __restrict__ Pn,
                                                            const double* __restrict__ Ud,
                                                            const double* __restrict__ F, double* __restrict__ rhs,
                                                            double* __restrict__ x0, double* __restrict__ gPn) {
  const FemGrid& g = S.g;
  const size_t N = g.nn;
  constexpr int ND = KI<KIND>::DIM;
  const MatCombo vc{S.Le, S.mu, S.Ce, S.rho, 0, nullptr, 0.0};
  const MatShared ms_m{S.Me, 1.0};
  auto src = [&](int j, int c) { return Un[j + c * N]; };
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    double ms[ND], v[ND], gp[ND];
    fem_gather_k<KIND, ND>(g, ix, iy, iz, ms_m, src, ms);
    if (S.vcv) {
#pragma unroll
      for (int c = 0; c < ND; ++c) v[c] = S.vcv[n + c * N];
    } else {
      fem_gather_k<KIND, ND>(g, ix, iy, iz, vc, src, v);
    }
    fem_gather_grad_k<KIND, ND>(g, ix, iy, iz, S.Ge, [&](int j) { return Pn[j]; }, gp);
#pragma unroll
    for (int c = 0; c < ND; ++c) {
      const size_t o = n + c * N;
      double r = ((S.rho / S.dt) * ms[c] - gp[c]) - (1 - S.theta) * v[c];
      if (F) r = r + F[o];
      gPn[o] = gp[c];
      const bool d = S.dmask && S.dmask[o];
      rhs[o] = d ? Ud[o] : r;
      x0[o] = d ? Ud[o] : Un[o];
    }
  }
}

// U* = U_hat + (dt/rho) G P_n / M   (solvers/standard.py:156)
__global__ void k_ustar(int n, double c, const double* __restrict__ Uh, const double* __restrict__ gPn,
                        const double* __restrict__ M, double* __restrict__ Us) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    Us[i] = Uh[i] + ((c * gPn[i]) / M[i]);
}

// PPE rhs (rho/dt)(D U* - F_p) with pinned rows zeroed, and x0 (solvers/standard.py:97-107).
template <int KIND>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_p_rhs(StepArgs S, const double* __restrict__ Us,
                                                          const double* __restrict__ Fp,
                                                          const double* __restrict__ Pn, double* __restrict__ rhs,
                                                          double* __restrict__ x0) {
  const FemGrid& g = S.g;
  constexpr int ND = KI<KIND>::DIM;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    const double du = fem_gather_div_k<KIND, ND>(g, ix, iy, iz, S.Ge, Us);
    double r = (S.rho / S.dt) * (Fp ? du - Fp[n] : du);
    double x = Pn[n];
    if (S.pinned && S.pmask && S.pmask[n]) {
      r = 0.0;
      x = 0.0;
    }
    rhs[n] = r;
    x0[n] = x;
  }
}

// U = U* - (dt/rho) G P / M ; U[gamma_d] = U_d   (solvers/standard.py:160-163)
template <int KIND>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_ufinal(StepArgs S, const double* __restrict__ Us,
                                                           const double* __restrict__ P,
                                                           const double* __restrict__ Ud, double* __restrict__ U) {
  const FemGrid& g = S.g;
  const size_t N = g.nn;
  const double c = S.dt / S.rho;
  constexpr int ND = KI<KIND>::DIM;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    double gp[ND];
    fem_gather_grad_k<KIND, ND>(g, ix, iy, iz, S.Ge, [&](int j) { return P[j]; }, gp);
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const size_t o = n + d * N;
      const double u = Us[o] - ((c * gp[d]) / S.M[o]);
      U[o] = (S.dmask && S.dmask[o]) ? Ud[o] : u;
    }
  }
}

// Scalar transport rhs (solvers/passive_transport.py:26-33 / 50-57):
// rhs = (1/dt)(Me + Mtau_e) phi_n - 0.5 (Ce_n + D Le + Ctau_e) phi_n, with the
// per-element parts pre-combined into Erhs_e; Dirichlet rows -> phi_d.
template <int KIND>
__global__ void k_phi_rhs(FemGrid g, const double* __restrict__ Me, const double* __restrict__ Le, double dt, double D,
                          const double* __restrict__ Mt, const double* __restrict__ Cn, const double* __restrict__ Ct,
                          const double* __restrict__ phin, const uint8_t* __restrict__ mask,
                          const double* __restrict__ phid, double* __restrict__ rhs, double* __restrict__ x0) {
  const MatCombo mm{Me, 1.0, Mt, 1.0, 0, nullptr, 0.0};
  const MatCombo vm{Le, D, Cn, 1.0, 0, Ct, 1.0};
  auto src = [&](int j, int) { return phin[j]; };
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    double ms[1], vc[1];
    fem_gather_k<KIND, 1>(g, ix, iy, iz, mm, src, ms);
    fem_gather_k<KIND, 1>(g, ix, iy, iz, vm, src, vc);
    const double r = (1 / dt) * ms[0] - 0.5 * vc[0];
    const bool m = mask && mask[n];
    rhs[n] = m ? phid[n] : r;
    x0[n] = m ? phid[n] : phin[n];
  }
}

int fem_launch_mom_rhs(const StepArgs& S, const double* Un, const double* Pn, const double* Ud, const double* F,
                       double* rhs, double* x0, double* gPn, cudaStream_t s) {
  const int nb = fem_nblocks(S.g.nn, FEM_OP_THREADS);
  FEM_KIND_DISPATCH(S.g.kind, K, (k_mom_rhs<K><<<nb, FEM_OP_THREADS, 0, s>>>(S, Un, Pn, Ud, F, rhs, x0, gPn)));
  return fem_after_launch("k_mom_rhs");
}
int fem_launch_ustar(int n, double c, const double* Uh, const double* gPn, const double* M, double* Us,
                     cudaStream_t s) {
  k_ustar<<<fem_nblocks(n, 256), 256, 0, s>>>(n, c, Uh, gPn, M, Us);
  return fem_after_launch("k_ustar");
}
int fem_launch_p_rhs(const StepArgs& S, const double* Us, const double* Fp, const double* Pn, double* rhs, double* x0,
                     cudaStream_t s) {
  const int nb = fem_nblocks(S.g.nn, FEM_OP_THREADS);
  FEM_KIND_DISPATCH(S.g.kind, K, (k_p_rhs<K><<<nb, FEM_OP_THREADS, 0, s>>>(S, Us, Fp, Pn, rhs, x0)));
  return fem_after_launch("k_p_rhs");
}
int fem_launch_ufinal(const StepArgs& S, const double* Us, const double* P, const double* Ud, double* U,
                      cudaStream_t s) {
  const int nb = fem_nblocks(S.g.nn, FEM_OP_THREADS);
  FEM_KIND_DISPATCH(S.g.kind, K, (k_ufinal<K><<<nb, FEM_OP_THREADS, 0, s>>>(S, Us, P, Ud, U)));
  return fem_after_launch("k_ufinal");
}
int fem_launch_phi_rhs(const FemGrid& g, const double* Me, const double* Le, double dt, double D, const double* Mt,
                       const double* Cn, const double* Ct, const double* phin, const uint8_t* mask,
                       const double* phid, double* rhs, double* x0, cudaStream_t s) {
  const int nb = fem_nblocks(g.nn, FEM_OP_THREADS);
  FEM_KIND_DISPATCH(g.kind, K,
                    (k_phi_rhs<K><<<nb, FEM_OP_THREADS, 0, s>>>(g, Me, Le, dt, D, Mt, Cn, Ct, phin, mask, phid, rhs,
                                                               x0)));
  return fem_after_launch("k_phi_rhs");
}
