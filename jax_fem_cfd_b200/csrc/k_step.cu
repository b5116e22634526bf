// 4-step projection stage kernels and the scalar-transport rhs.
#include "fem_step_body.cuh"


template <int KIND>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_mom_rhs(StepArgs S, const double* __restrict__ Un,
                                                            const double* __restrict__ Pn,
                                                            const double* __restrict__ Ud,
                                                            const double* __restrict__ F, double* __restrict__ rhs,
                                                            double* __restrict__ x0, double* __restrict__ gPn) {
  step_mom_rhs<KIND>(S, Un, Pn, Ud, F, rhs, x0, gPn);
}
__global__ void k_ustar(int n, double c, const double* __restrict__ Uh, const double* __restrict__ gPn,
                        const double* __restrict__ M, double* __restrict__ Us) {
  step_ustar(n, c, Uh, gPn, M, Us);
}
template <int KIND>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_p_rhs(StepArgs S, const double* __restrict__ Us,
                                                          const double* __restrict__ Fp,
                                                          const double* __restrict__ Pn, double* __restrict__ rhs,
                                                          double* __restrict__ x0) {
  step_p_rhs<KIND>(S, Us, Fp, Pn, rhs, x0);
}
template <int KIND>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_ufinal(StepArgs S, const double* __restrict__ Us,
                                                           const double* __restrict__ P,
                                                           const double* __restrict__ Ud, double* __restrict__ U) {
  step_ufinal<KIND>(S, Us, P, Ud, U);
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
