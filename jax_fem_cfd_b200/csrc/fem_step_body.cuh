// Stage bodies of the 4-step projection (solvers/standard.py:148-165): grid-
// stride loops over blockIdx.x / gridDim.x, so they run as kernels of their own
// (k_step.cu) and as stages of the packed step (k_pack.cu), one group of CTAs
// per request.
#pragma once
#include "fem_args.cuh"

// hex8: y_t = sum over the 27 lattice offsets of T_t[class][offset] src(node +
// offset) for NT assembled tables T_t on one source (neighbour values loaded
// once); the tables are the assembled rows of shared element matrices
// (fem_stencil_entry), zero where an offset leaves the lattice.
template <int NT, class Src>
__device__ __forceinline__ void step_stencil3(const FemGrid& g, const double* const (&tab)[NT], int i, int j, int k,
                                              const Src& src, double (&y)[NT]) {
  const int cx = fem_axis_cls(FEM_HEX8, 0, i, g.nex), cy = fem_axis_cls(FEM_HEX8, 0, j, g.ney);
  const int cz = fem_axis_cls(FEM_HEX8, 0, k, g.nez);
  const int base = ((cz * 3 + cy) * 3 + cx) * 27;
  int col[3], row[3], pl[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int v = i + d - 1, w = j + d - 1, z = k + d - 1;
    col[d] = v < 0 ? 0 : (v >= g.nnx ? g.nnx - 1 : v);
    row[d] = (w < 0 ? 0 : (w >= g.nny ? g.nny - 1 : w)) * g.nnx;
    pl[d] = (z < 0 ? 0 : (z >= g.nnz ? g.nnz - 1 : z)) * g.nnx * g.nny;
  }
#pragma unroll
  for (int t = 0; t < NT; ++t) y[t] = 0.0;
#pragma unroll
  for (int dz = 0; dz < 3; ++dz)
#pragma unroll
    for (int dy = 0; dy < 3; ++dy)
#pragma unroll
      for (int dx = 0; dx < 3; ++dx) {
        const int o = (dz * 3 + dy) * 3 + dx;
        const double v = src(pl[dz] + row[dy] + col[dx]);
#pragma unroll
        for (int t = 0; t < NT; ++t) y[t] += __ldg(tab[t] + base + o) * v;
      }
}
#define STEP_TAB(S, t) ((S).tab3 + (size_t)(t) * FEM_TAB_MAX)  // 0: Me, 1-3: Ge_d, 4-6: Ge_d^T

// rhs of solvers/standard.py:31-37 and the initial guess x0; also keeps G P_n.
template <int KIND>
__device__ __forceinline__ void step_mom_rhs(const StepArgs& S, const double* __restrict__ Un,
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
    bool tabs = false;
    if constexpr (KIND == FEM_HEX8) {
      if (S.tab3) {
        const double* tm[1] = {STEP_TAB(S, 0)};
#pragma unroll
        for (int c = 0; c < ND; ++c) {
          double y1[1];
          step_stencil3<1>(g, tm, ix, iy, iz, [&](int j) { return Un[j + c * N]; }, y1);
          ms[c] = y1[0];
        }
        const double* tg[3] = {STEP_TAB(S, 1), STEP_TAB(S, 2), STEP_TAB(S, 3)};
        double g3[3];
        step_stencil3<3>(g, tg, ix, iy, iz, [&](int j) { return Pn[j]; }, g3);
#pragma unroll
        for (int c = 0; c < ND; ++c) gp[c] = g3[c];
        tabs = true;
      }
    }
    if (!tabs) fem_gather_k<KIND, ND>(g, ix, iy, iz, ms_m, src, ms);
    if (S.vcv) {
#pragma unroll
      for (int c = 0; c < ND; ++c) v[c] = S.vcv[n + c * N];
    } else {
      fem_gather_k<KIND, ND>(g, ix, iy, iz, vc, src, v);
    }
    if (!tabs) fem_gather_grad_k<KIND, ND>(g, ix, iy, iz, S.Ge, [&](int j) { return Pn[j]; }, gp);
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
__device__ __forceinline__ void step_ustar(int n, double c, const double* __restrict__ Uh, const double* __restrict__ gPn,
                        const double* __restrict__ M, double* __restrict__ Us) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    Us[i] = Uh[i] + ((c * gPn[i]) / M[i]);
}

// PPE rhs (rho/dt)(D U* - F_p) with pinned rows zeroed, and x0 (solvers/standard.py:97-107).
template <int KIND>
__device__ __forceinline__ void step_p_rhs(const StepArgs& S, const double* __restrict__ Us,
                                                          const double* __restrict__ Fp,
                                                          const double* __restrict__ Pn, double* __restrict__ rhs,
                                                          double* __restrict__ x0) {
  const FemGrid& g = S.g;
  constexpr int ND = KI<KIND>::DIM;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    double du;
    bool tabs = false;
    if constexpr (KIND == FEM_HEX8) {
      if (S.tab3) {
        // per-component divergence parts, added in component order as the gather does
        const size_t N = g.nn;
        double acc[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double* td[1] = {STEP_TAB(S, 4 + d)};
          double y1[1];
          step_stencil3<1>(g, td, ix, iy, iz, [&](int j) { return Us[j + d * N]; }, y1);
          acc[d] = y1[0];
        }
        du = acc[0] + acc[1] + acc[2];
        tabs = true;
      }
    }
    if (!tabs) du = fem_gather_div_k<KIND, ND>(g, ix, iy, iz, S.Ge, Us);
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
__device__ __forceinline__ void step_ufinal(const StepArgs& S, const double* __restrict__ Us,
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
    bool tabs = false;
    if constexpr (KIND == FEM_HEX8) {
      if (S.tab3) {
        const double* tg[3] = {STEP_TAB(S, 1), STEP_TAB(S, 2), STEP_TAB(S, 3)};
        double g3[3];
        step_stencil3<3>(g, tg, ix, iy, iz, [&](int j) { return P[j]; }, g3);
#pragma unroll
        for (int d = 0; d < ND; ++d) gp[d] = g3[d];
        tabs = true;
      }
    }
    if (!tabs) fem_gather_grad_k<KIND, ND>(g, ix, iy, iz, S.Ge, [&](int j) { return P[j]; }, gp);
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const size_t o = n + d * N;
      const double u = Us[o] - ((c * gp[d]) / S.M[o]);
      U[o] = (S.dmask && S.dmask[o]) ? Ud[o] : u;
    }
  }
}


// Gauss-point factors of Ce(U) (fem_conv_factors), one thread per element,
// structure of arrays fq[k * ne + e].
template <int KIND>
__device__ __forceinline__ void step_conv_factors(const FemGrid& g, const FemQuadTab& qt,
                                                  const double* __restrict__ U, double bd,
                                                  double* __restrict__ fq) {
  constexpr int NEN = KI<KIND>::NEN, NQ = KQ<KIND>::NQ, S = KI<KIND>::S;
  const size_t nn = g.nn, ne = g.ne;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.ne; e += gridDim.x * blockDim.x) {
    const int ey = e / g.nex, ex = e - ey * g.nex;
    double ux[NEN], uy[NEN];
#pragma unroll
    for (int b = 0; b < NEN; ++b) {
      int i = S * ex + kdi<KIND>(b), j = S * ey + kdj<KIND>(b);
      if (g.periodic) {
        i = i >= g.nnx ? i - g.nnx : i;
        j = j >= g.nny ? j - g.nny : j;
      }
      const size_t n = (size_t)j * g.nnx + i;
      ux[b] = U[n];
      uy[b] = U[n + nn];
    }
    double f[3 * NQ];
    fem_conv_factors<KIND>(qt, ux, uy, bd, f);
#pragma unroll
    for (int k = 0; k < 3 * NQ; ++k) fq[k * ne + e] = f[k];
  }
}

// y = alpha Ash x + cc Ce x over the whole lattice, the tiles dealt over the CTAs
// (sA: Ash in shared memory or null; sm: FEM_CONV_SMEM doubles).
template <int KIND, int NC>
__device__ __forceinline__ void step_conv_apply(const FemGrid& g, const FemQuadTab& qt, const double* __restrict__ fq,
                                                double cc, double alpha, const double* sA,
                                                const double* __restrict__ x, double* __restrict__ y, double* sm) {
  const size_t nn = g.nn;
  struct Tiles {
    __device__ __forceinline__ int cta() const { return blockIdx.x; }
    __device__ __forceinline__ int ncta() const { return gridDim.x; }
  } tm;
  const double* src[1] = {x};
  fem_tiled_conv<KIND, NC, 1>(tm, g, sm, src, [](int, const double(&v)[1]) { return v[0]; }, fq, qt, cc, alpha, sA,
                              [&](int i, const double(&v)[NC], const double(&)[NC]) {
#pragma unroll
                                for (int c = 0; c < NC; ++c) y[i + c * nn] = v[c];
                              });
}

