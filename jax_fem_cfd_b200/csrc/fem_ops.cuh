// Element-by-element operators, evaluated node-centrically (see fem_common.cuh).
//
// Reference semantics (jax_fem_cfd core/element_mult.py): y = segment_sum over
// elements of A_e x[nconn[e]]. Here the owner thread of node n computes
// y[n] = sum_{(e,a) incident to n} sum_b A_e[a][b] x[node(e,b)].
#pragma once
#include "fem_common.cuh"

// Element-matrix coefficient providers --------------------------------------
// All matrices are row-major nen x nen.
struct MatShared {
  const double* A;  // shared element matrix (smem or global)
  double alpha;
  __device__ __forceinline__ double operator()(int, int a, int b, int nen) const { return alpha * A[a * nen + b]; }
};
struct MatSharedT {  // transpose of a shared matrix (divergence: Ge_i^T)
  const double* A;
  __device__ __forceinline__ double operator()(int, int a, int b, int nen) const { return A[b * nen + a]; }
};
// alpha*A + beta*B_e (+ gamma*C_e), B_e / C_e per element, optionally transposed.
struct MatCombo {
  const double* A;
  double alpha;
  const double* B;
  double beta;
  int transB;
  const double* C;
  double gamma;
  __device__ __forceinline__ double operator()(int e, int a, int b, int nen) const {
    double v = 0.0;
    if (A) v = alpha * A[a * nen + b];
    if (B) {
      const size_t off = (size_t)e * nen * nen;
      v += beta * (transB ? B[off + b * nen + a] : B[off + a * nen + b]);
    }
    if (C) v += gamma * C[(size_t)e * nen * nen + a * nen + b];
    return v;
  }
};

// y_c[n] for NC components sharing one coefficient provider (x_c = x + c*stride).
template <int NC, class Mat>
__device__ __forceinline__ void fem_gather(const FemGrid& g, int n, const Mat& m, const double* __restrict__ x,
                                           int stride, double (&y)[NC]) {
#pragma unroll
  for (int c = 0; c < NC; ++c) y[c] = 0.0;
  const int nen = g.nen;
  fem_for_incident(g, n, [&](int ie, int je, int ke, int e, int a) {
    double part[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) part[c] = 0.0;
    for (int b = 0; b < nen; ++b) {
      const double coef = m(e, a, b, nen);
      const int j = fem_elem_node(g, ie, je, ke, b);
#pragma unroll
      for (int c = 0; c < NC; ++c) part[c] += coef * x[j + (size_t)c * stride];
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) y[c] += part[c];
  });
}

// Same as fem_gather, but the input value at node j is produced by a functor
// (used to fuse a pointwise producer into the stencil: x_j = f(j)).
template <class Mat, class Src>
__device__ __forceinline__ double fem_gather_fn(const FemGrid& g, int n, const Mat& m, const Src& src) {
  double y = 0.0;
  const int nen = g.nen;
  fem_for_incident(g, n, [&](int ie, int je, int ke, int e, int a) {
    double part = 0.0;
    for (int b = 0; b < nen; ++b) {
      const int j = fem_elem_node(g, ie, je, ke, b);
      part += m(e, a, b, nen) * src(j);
    }
    y += part;
  });
  return y;
}

// Gradient: y_d[n] = sum Ge_d rows * P (ND outputs from one input).
template <int ND>
__device__ __forceinline__ void fem_gather_grad(const FemGrid& g, int n, const double* Ge, const double* __restrict__ P,
                                                double (&y)[ND]) {
#pragma unroll
  for (int d = 0; d < ND; ++d) y[d] = 0.0;
  const int nen = g.nen, nen2 = nen * nen;
  fem_for_incident(g, n, [&](int ie, int je, int ke, int e, int a) {
    double part[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) part[d] = 0.0;
    for (int b = 0; b < nen; ++b) {
      const double pj = P[fem_elem_node(g, ie, je, ke, b)];
#pragma unroll
      for (int d = 0; d < ND; ++d) part[d] += Ge[d * nen2 + a * nen + b] * pj;
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) y[d] += part[d];
  });
}

// Divergence: y[n] = sum_d sum Ge_d^T rows * U_d (reference sums the per-component
// assembled vectors, core/element_mult.py:147-155).
template <int ND>
__device__ __forceinline__ double fem_gather_div(const FemGrid& g, int n, const double* Ge, const double* __restrict__ U,
                                                 int nn) {
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  const int nen = g.nen, nen2 = nen * nen;
  fem_for_incident(g, n, [&](int ie, int je, int ke, int e, int a) {
    double part[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) part[d] = 0.0;
    for (int b = 0; b < nen; ++b) {
      const int j = fem_elem_node(g, ie, je, ke, b);
#pragma unroll
      for (int d = 0; d < ND; ++d) part[d] += Ge[d * nen2 + b * nen + a] * U[j + (size_t)d * nn];
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) acc[d] += part[d];
  });
  double y = acc[0];
#pragma unroll
  for (int d = 1; d < ND; ++d) y += acc[d];
  return y;
}

// ---------------------------------------------------------------------------
// Element matrices from quadrature data (core/element_calc.py:165-200).
// Quadrature layout: wq[q], N[q*nen + I], dN[(q*ndim + d)*nen + I].
// ---------------------------------------------------------------------------
struct FemQuad {
  const double* wq;
  const double* N;
  const double* dN;
  int nq, nen, ndim;
};

// Ce_e[a][b] = sum_q w N[q][a] (u_q . dN_q[b]) + beta * sum_q w N[q][a] divu_q N[q][b]
// One CTA handles EPB elements; requires blockDim >= EPB * nq.
#define FEM_CE_EPB 8
__device__ __forceinline__ void fem_convection_block(const FemGrid& g, const FemQuad Q, const double* __restrict__ U,
                                                     double beta, double* __restrict__ Ce, int e0, int mode,
                                                     double* s_uq /* EPB*nq*3 */, double* s_div /* EPB*nq */,
                                                     double* s_T /* EPB*nq*nen */) {
  // mode 0: conservative convection (beta), mode 1: Ctau_tilde = sum_q w dN^T (u u^T) dN
  const int nen = Q.nen, nq = Q.nq, nd = Q.ndim;
  const int nloc = min(FEM_CE_EPB, g.ne - e0);
  // stage 1: velocity and divergence at each quadrature point
  for (int t = threadIdx.x; t < nloc * nq; t += blockDim.x) {
    const int le = t / nq, q = t % nq, e = e0 + le;
    int ie = e % g.nex, r = e / g.nex, je = r % g.ney, ke = r / g.ney;
    double u[3] = {0, 0, 0}, dv = 0.0;
    for (int I = 0; I < nen; ++I) {
      const int j = fem_elem_node(g, ie, je, ke, I);
      const double NI = Q.N[q * nen + I];
      for (int d = 0; d < nd; ++d) {
        const double uj = U[j + (size_t)d * g.nn];
        u[d] += NI * uj;
        dv += Q.dN[(q * nd + d) * nen + I] * uj;
      }
    }
    for (int d = 0; d < 3; ++d) s_uq[(le * nq + q) * 3 + d] = u[d];
    s_div[le * nq + q] = dv;
  }
  __syncthreads();
  if (mode == 0) {
    // stage 2: T[q][b] = w_q (u_q . dN_q[b] + beta divu_q N_q[b])
    for (int t = threadIdx.x; t < nloc * nq * nen; t += blockDim.x) {
      const int le = t / (nq * nen), rem = t % (nq * nen), q = rem / nen, b = rem % nen;
      double v = 0.0;
      for (int d = 0; d < nd; ++d) v += s_uq[(le * nq + q) * 3 + d] * Q.dN[(q * nd + d) * nen + b];
      v += beta * s_div[le * nq + q] * Q.N[q * nen + b];
      s_T[(le * nq + q) * nen + b] = v;
    }
    __syncthreads();
    // stage 3: Ce[a][b] = sum_q (w_q N[q][a]) T[q][b]; flat, coalesced writes
    const int per = nen * nen;
    for (int t = threadIdx.x; t < nloc * per; t += blockDim.x) {
      const int le = t / per, ab = t % per, a = ab / nen, b = ab % nen;
      double v = 0.0;
      for (int q = 0; q < nq; ++q) v += (Q.N[q * nen + a] * Q.wq[q]) * s_T[(le * nq + q) * nen + b];
      Ce[(size_t)e0 * per + t] = v;
    }
  } else {
    // Ctau_tilde[a][b] = sum_q w_q (dN_q[:,a] . u_q)(u_q . dN_q[:,b])
    for (int t = threadIdx.x; t < nloc * nq * nen; t += blockDim.x) {
      const int le = t / (nq * nen), rem = t % (nq * nen), q = rem / nen, b = rem % nen;
      double v = 0.0;
      for (int d = 0; d < nd; ++d) v += s_uq[(le * nq + q) * 3 + d] * Q.dN[(q * nd + d) * nen + b];
      s_T[(le * nq + q) * nen + b] = v;
    }
    __syncthreads();
    const int per = nen * nen;
    for (int t = threadIdx.x; t < nloc * per; t += blockDim.x) {
      const int le = t / per, ab = t % per, a = ab / nen, b = ab % nen;
      double v = 0.0;
      for (int q = 0; q < nq; ++q) v += Q.wq[q] * s_T[(le * nq + q) * nen + a] * s_T[(le * nq + q) * nen + b];
      Ce[(size_t)e0 * per + t] = v;
    }
  }
  __syncthreads();
}

// The same build with the element's table sizes known at compile time (loops
// unrolled, every sum in the order above) and the quadrature tables (w, N, dN)
// in shared memory: EPB elements per round of three stages.
template <int NQ, int NEN, int ND, int EPB>
struct FemCeBlockSmem {
  double uq[EPB * NQ * 3], div[EPB * NQ], T[EPB * NQ * NEN];
  double w[NQ], N[NQ * NEN], dN[NQ * ND * NEN];
};
template <int NQ, int NEN, int ND, int EPB>
__device__ __forceinline__ void fem_convection_block_k(const FemGrid& g, const double* __restrict__ U, double beta,
                                                       double* __restrict__ Ce, int e0, int mode,
                                                       FemCeBlockSmem<NQ, NEN, ND, EPB>& S) {
  const int nloc = min(EPB, g.ne - e0);
  for (int t = threadIdx.x; t < nloc * NQ; t += blockDim.x) {
    const int le = t / NQ, q = t - le * NQ, e = e0 + le;
    const int ie = e % g.nex, r = e / g.nex, je = r % g.ney, ke = r / g.ney;
    double u[3] = {0, 0, 0}, dv = 0.0;
#pragma unroll
    for (int I = 0; I < NEN; ++I) {
      const int j = fem_elem_node(g, ie, je, ke, I);
      const double NI = S.N[q * NEN + I];
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        const double uj = U[j + (size_t)d * g.nn];
        u[d] += NI * uj;
        dv += S.dN[(q * ND + d) * NEN + I] * uj;
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) S.uq[(le * NQ + q) * 3 + d] = u[d];
    S.div[le * NQ + q] = dv;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nloc * NQ * NEN; t += blockDim.x) {
    const int le = t / (NQ * NEN), rem = t - le * (NQ * NEN), q = rem / NEN, b = rem - q * NEN;
    double v = 0.0;
#pragma unroll
    for (int d = 0; d < ND; ++d) v += S.uq[(le * NQ + q) * 3 + d] * S.dN[(q * ND + d) * NEN + b];
    if (mode == 0) v += beta * S.div[le * NQ + q] * S.N[q * NEN + b];
    S.T[(le * NQ + q) * NEN + b] = v;
  }
  __syncthreads();
  constexpr int per = NEN * NEN;
  for (int t = threadIdx.x; t < nloc * per; t += blockDim.x) {
    const int le = t / per, ab = t - le * per, a = ab / NEN, b = ab - a * NEN;
    double v = 0.0;
    if (mode == 0) {
#pragma unroll
      for (int q = 0; q < NQ; ++q) v += (S.N[q * NEN + a] * S.w[q]) * S.T[(le * NQ + q) * NEN + b];
    } else {
#pragma unroll
      for (int q = 0; q < NQ; ++q) v += S.w[q] * S.T[(le * NQ + q) * NEN + a] * S.T[(le * NQ + q) * NEN + b];
    }
    Ce[(size_t)e0 * per + t] = v;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Multigrid lattice transfers (core/multigrid.py:90-212). Arrays are indexed
// [row = y][col = x]; "full" extents include the periodic duplicate row/column.
// ---------------------------------------------------------------------------
struct FemLattice {
  int nx, ny;      // full lattice extents (lvl_nums nnx, nny)
  int periodic;
  __device__ __forceinline__ int ux() const { return periodic ? nx - 1 : nx; }
  __device__ __forceinline__ int uy() const { return periodic ? ny - 1 : ny; }
  // unique-node index of full-lattice (r, c)
  __device__ __forceinline__ int idx(int r, int c) const {
    if (periodic) {
      if (c == nx - 1) c = 0;
      if (r == ny - 1) r = 0;
      return r * (nx - 1) + c;
    }
    return r * nx + c;
  }
};

// Bilinear prolongation value at fine unique node (r, c) from coarse values xH(I).
template <class Src>
__device__ __forceinline__ double fem_interp_at(const FemLattice& H, int r, int c, const Src& xH) {
  const int R = r >> 1, C = c >> 1;
  if (!(r & 1) && !(c & 1)) return xH(H.idx(R, C));
  if (!(r & 1)) return 0.5 * xH(H.idx(R, C)) + 0.5 * xH(H.idx(R, C + 1));
  if (!(c & 1)) return 0.5 * xH(H.idx(R, C)) + 0.5 * xH(H.idx(R + 1, C));
  return 0.25 * xH(H.idx(R, C)) + 0.25 * xH(H.idx(R, C + 1)) + 0.25 * xH(H.idx(R + 1, C)) +
         0.25 * xH(H.idx(R + 1, C + 1));
}

// R = I^T on the full fine lattice: coarse full node (R, C) gathers fine full
// nodes (2R+dr, 2C+dc) inside the full lattice with weights 1, 1/2, 1/4.
template <class Src>
__device__ __forceinline__ double fem_restrict_at(const FemLattice& h, int R, int C, const Src& xh) {
  const int r0 = 2 * R, c0 = 2 * C;
  const bool up = r0 + 1 < h.ny, dn = r0 - 1 >= 0, rt = c0 + 1 < h.nx, lf = c0 - 1 >= 0;
  double e = 0.0, d = 0.0;
  if (up) e += xh(h.idx(r0 + 1, c0));
  if (dn) e += xh(h.idx(r0 - 1, c0));
  if (rt) e += xh(h.idx(r0, c0 + 1));
  if (lf) e += xh(h.idx(r0, c0 - 1));
  if (up && rt) d += xh(h.idx(r0 + 1, c0 + 1));
  if (up && lf) d += xh(h.idx(r0 + 1, c0 - 1));
  if (dn && rt) d += xh(h.idx(r0 - 1, c0 + 1));
  if (dn && lf) d += xh(h.idx(r0 - 1, c0 - 1));
  return xh(h.idx(r0, c0)) + 0.5 * e + 0.25 * d;
}

// Row sum of the restriction at coarse unique node (R, C): (R 1)_I on the full
// fine lattice (neighbours outside it are skipped, periodic too).
__device__ __forceinline__ double fem_restrict_rowsum(const FemLattice& H, int R, int C) {
  const double wr = 1.0 + (R > 0 ? 0.5 : 0.0) + (R < H.ny - 1 ? 0.5 : 0.0);
  const double wc = 1.0 + (C > 0 ? 0.5 : 0.0) + (C < H.nx - 1 ? 0.5 : 0.0);
  return wr * wc;
}

// Column sum of the prolongation at coarse unique node (R, C): sum_i P_iI.
__device__ __forceinline__ double fem_interp_colsum(const FemLattice& H, int R, int C) {
  if (H.periodic) return 4.0;
  const double wr = 1.0 + (R > 0 ? 0.5 : 0.0) + (R < H.ny - 1 ? 0.5 : 0.0);
  const double wc = 1.0 + (C > 0 ? 0.5 : 0.0) + (C < H.nx - 1 ? 0.5 : 0.0);
  return wr * wc;
}
