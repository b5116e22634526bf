// Element-product, element-matrix, transfer, boundary and blas-1 kernels.
#include <mutex>
#include "fem_b200.h"
#include "fem_step_body.cuh"


template <int KIND, int NC>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_ebe_apply(FemGrid g, MatCombo m, const double* __restrict__ x,
                                                              double* __restrict__ y) {
  const size_t N = g.nn;
  auto src = [&](int j, int c) { return x[j + c * N]; };
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    double v[NC];
    fem_gather_k<KIND, NC>(g, ix, iy, iz, m, src, v);
#pragma unroll
    for (int c = 0; c < NC; ++c) y[n + c * N] = v[c];
  }
}

template <int KIND>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_grad(FemGrid g, const double* __restrict__ Ge,
                                                         const double* __restrict__ P, double* __restrict__ y) {
  constexpr int ND = KI<KIND>::DIM;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    double v[ND];
    fem_gather_grad_k<KIND, ND>(g, ix, iy, iz, Ge, [&](int j) { return P[j]; }, v);
#pragma unroll
    for (int d = 0; d < ND; ++d) y[n + (size_t)d * g.nn] = v[d];
  }
}

template <int KIND>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_div(FemGrid g, const double* __restrict__ Ge,
                                                        const double* __restrict__ U, double* __restrict__ y) {
  constexpr int ND = KI<KIND>::DIM;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    y[n] = fem_gather_div_k<KIND, ND>(g, ix, iy, iz, Ge, U);
  }
}

// Ce / Ctau_tilde build, FEM_CE_EPB elements per CTA.
__global__ void __launch_bounds__(FEM_OP_THREADS) k_convection(FemGrid g, FemQuad Q, const double* __restrict__ U,
                                                               double beta, int mode, double* __restrict__ Ce) {
  __shared__ double s_uq[FEM_CE_EPB * 9 * 3];
  __shared__ double s_div[FEM_CE_EPB * 9];
  __shared__ double s_T[FEM_CE_EPB * 9 * 9];
  for (int e0 = blockIdx.x * FEM_CE_EPB; e0 < g.ne; e0 += gridDim.x * FEM_CE_EPB)
    fem_convection_block(g, Q, U, beta, Ce, e0, mode, s_uq, s_div, s_T);
}

// y = (alpha A + beta B_e) x on hex8, 3 components, by the element-centric
// tiles of fem_tiled_ebe3e (one run of z-planes per CTA; no grid barrier).
struct FemCtaTeam {
  __device__ __forceinline__ int cta() const { return blockIdx.x; }
  __device__ __forceinline__ int ncta() const { return gridDim.x; }
};
__global__ void __launch_bounds__(FEM_THREADS, 1) k_ebe3e_apply(FemGrid g, MatCombo m, const double* __restrict__ x,
                                                                double* __restrict__ y) {
  extern __shared__ __align__(128) double sm[];
  __shared__ double sA[64];
  if (m.A) {
    for (int t = threadIdx.x; t < 64; t += blockDim.x) sA[t] = m.A[t];
    __syncthreads();
    m.A = sA;
  }
  const size_t N = g.nn;
  fem_tiled_ebe3e<3>(FemCtaTeam{}, g, sm, [&](int j, int c) { return x[j + c * N]; }, m,
                     [&](int n, const double(&v)[3], const double(&)[3]) {
#pragma unroll
                       for (int c = 0; c < 3; ++c) y[n + c * N] = v[c];
                     });
}
int fem_launch_ebe3e(const FemGrid& g, const MatCombo& m, const double* x, double* y, int grid, cudaStream_t s) {
  if (g.kind != FEM_HEX8 || !m.B || m.transB || m.C || grid < 1) return FEM_E_ARG;
  const int dyn = fem_ebe3e_smem(3) * (int)sizeof(double);
  // the shared-memory limit is a per-device function attribute: set once per device
  static std::mutex mu;
  static unsigned long long done = 0ull;  // bit d: set on device d (devices 0..63)
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fem_after_launch("cudaGetDevice");
  {
    std::lock_guard<std::mutex> lock(mu);
    const unsigned long long bit = dev < 64 ? (1ull << dev) : 0ull;
    if (!(done & bit)) {
      if (cudaFuncSetAttribute(k_ebe3e_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess)
        return fem_after_launch("k_ebe3e_apply attribute");
      done |= bit;
    }
  }
  k_ebe3e_apply<<<grid, FEM_THREADS, dyn, s>>>(g, m, x, y);
  return fem_after_launch("k_ebe3e_apply");
}

// The same build for one element kind (fem_convection_block_k): 32 elements
// per round, quadrature tables staged in shared memory once per CTA.
#define FEM_CE_EPB_K 32
template <int NQ, int NEN, int ND>
__global__ void __launch_bounds__(FEM_OP_THREADS) k_convection_k(FemGrid g, FemQuad Q, const double* __restrict__ U,
                                                                 double beta, int mode, double* __restrict__ Ce) {
  __shared__ FemCeBlockSmem<NQ, NEN, ND, FEM_CE_EPB_K> S;
  for (int t = threadIdx.x; t < NQ; t += blockDim.x) S.w[t] = Q.wq[t];
  for (int t = threadIdx.x; t < NQ * NEN; t += blockDim.x) S.N[t] = Q.N[t];
  for (int t = threadIdx.x; t < NQ * ND * NEN; t += blockDim.x) S.dN[t] = Q.dN[t];
  __syncthreads();
  for (int e0 = blockIdx.x * FEM_CE_EPB_K; e0 < g.ne; e0 += gridDim.x * FEM_CE_EPB_K)
    fem_convection_block_k<NQ, NEN, ND, FEM_CE_EPB_K>(g, U, beta, Ce, e0, mode, S);
}

// hex8 form of the same build (8 Gauss points, 8 nodes, 3 dimensions), two
// stages per round of 32 elements: thread (element, q) interpolates u and div u
// at Gauss point q and writes T[q][b] for its 8 nodes b; thread (element, block)
// then forms a 2 x 4 block of Ce[a][b] = sum_q (N[q][a] w[q]) T[q][b], loading
// each factor once per Gauss point for its 8 entries. Every sum has the terms and
// order of fem_convection_block; the rows of T are padded (66 doubles per
// element) so the block loads of different elements fall in different banks.
#define FEM_CE8_EPB 32
#define FEM_CE8_TS 66
__global__ void __launch_bounds__(256) k_convection_hex8(FemGrid g, FemQuad Q, const double* __restrict__ U,
                                                         double beta, int mode, double* __restrict__ Ce) {
  __shared__ __align__(16) double T[FEM_CE8_EPB * FEM_CE8_TS];
  __shared__ double sN[64], sNW[64], sdN[192];
  for (int t = threadIdx.x; t < 64; t += blockDim.x) {
    sN[t] = Q.N[t];
    sNW[t] = Q.N[t] * Q.wq[t >> 3];
  }
  for (int t = threadIdx.x; t < 192; t += blockDim.x) sdN[t] = Q.dN[t];
  __syncthreads();
  const size_t nn = g.nn;
  for (int e0 = blockIdx.x * FEM_CE8_EPB; e0 < g.ne; e0 += gridDim.x * FEM_CE8_EPB) {
    const int nloc = min(FEM_CE8_EPB, g.ne - e0);
    for (int t = threadIdx.x; t < nloc * 8; t += blockDim.x) {
      const int le = t >> 3, q = t & 7, e = e0 + le;
      const int ie = e % g.nex, r = e / g.nex, je = r % g.ney, ke = r / g.ney;
      double u[3] = {0, 0, 0}, dv = 0.0;
#pragma unroll
      for (int I = 0; I < 8; ++I) {
        const int j = fem_elem_node(g, ie, je, ke, I);
        const double NI = sN[q * 8 + I];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double uj = U[j + (size_t)d * nn];
          u[d] += NI * uj;
          dv += sdN[(q * 3 + d) * 8 + I] * uj;
        }
      }
      double* Tq = T + le * FEM_CE8_TS + q * 8;
#pragma unroll
      for (int b = 0; b < 8; ++b) {
        double v = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) v += u[d] * sdN[(q * 3 + d) * 8 + b];
        if (mode == 0) v += beta * dv * sN[q * 8 + b];
        Tq[b] = v;
      }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < nloc * 8; t += blockDim.x) {
      const int le = t >> 3, blk = t & 7, a0 = 2 * (blk >> 1), b0 = 4 * (blk & 1);
      const double* Te = T + le * FEM_CE8_TS + b0;
      double v[2][4];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int k = 0; k < 4; ++k) v[i][k] = 0.0;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const double2 t01 = *reinterpret_cast<const double2*>(Te + q * 8);
        const double2 t23 = *reinterpret_cast<const double2*>(Te + q * 8 + 2);
        const double tb[4] = {t01.x, t01.y, t23.x, t23.y};
        if (mode == 0) {
          const double f0 = sNW[q * 8 + a0], f1 = sNW[q * 8 + a0 + 1];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            v[0][k] += f0 * tb[k];
            v[1][k] += f1 * tb[k];
          }
        } else {
          // Ctau_tilde: w_q T[q][a] T[q][b]
          const double wq = Q.wq[q];
          const double ta0 = T[le * FEM_CE8_TS + q * 8 + a0], ta1 = T[le * FEM_CE8_TS + q * 8 + a0 + 1];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            v[0][k] += wq * ta0 * tb[k];
            v[1][k] += wq * ta1 * tb[k];
          }
        }
      }
      double2* out = reinterpret_cast<double2*>(Ce + (size_t)(e0 + le) * 64 + a0 * 8 + b0);
      out[0] = make_double2(v[0][0], v[0][1]);
      out[1] = make_double2(v[0][2], v[0][3]);
      out[4] = make_double2(v[1][0], v[1][1]);
      out[5] = make_double2(v[1][2], v[1][3]);
    }
    __syncthreads();
  }
}

// core/element_calc.py:202-229 (per-element tau, r-norm blend).
__global__ void k_supg_tau(FemGrid g, FemQuad Q, const double* __restrict__ U, const double* __restrict__ Ce,
                           const double* __restrict__ Ct, double D, double dt, double r, double* __restrict__ tau) {
  const int nen = g.nen, nq = Q.nq, nd = Q.ndim, per = nen * nen;
  D = D + 1e-6;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.ne; e += gridDim.x * blockDim.x) {
    const int ie = e % g.nex, rr = e / g.nex, je = rr % g.ney, ke = rr / g.ney;
    double ce2 = 0.0, kt2 = 0.0;
    for (int t = 0; t < per; ++t) {
      const double c = Ce[(size_t)e * per + t], k = Ct[(size_t)e * per + t];
      ce2 += c * c;
      kt2 += k * k;
    }
    const double ce_n = sqrt(ce2), kt_n = sqrt(kt2);
    double un2 = 0.0;
    for (int q = 0; q < nq; ++q) {
      double s = 0.0;
      for (int d = 0; d < nd; ++d) {
        double uq = 0.0;
        for (int I = 0; I < nen; ++I) uq += Q.N[q * nen + I] * U[fem_elem_node(g, ie, je, ke, I) + (size_t)d * g.nn];
        s += uq * uq;
      }
      un2 += s;
    }
    un2 /= nq;
    const double Re = (un2 * ce_n) / (D * kt_n);
    const double t1 = ce_n / kt_n, t2 = dt / 2, t3 = t1 * Re;
    tau[e] = pow(1 / pow(t1, r) + 1 / pow(t2, r) + 1 / pow(t3, r), -1 / r);
  }
}

// Combined per-element matrix for the SUPG scalar operator:
// out_e = s_m * tau_e * Cn_e^T + s_c * (C_e + tau_e * Ct_e)   (transport lhs/rhs).
__global__ void k_supg_combine(int ne, int nen, const double* __restrict__ tau, const double* __restrict__ Cn,
                               const double* __restrict__ C, const double* __restrict__ Ct, double s_m, double s_c,
                               double* __restrict__ out) {
  const int per = nen * nen;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)ne * per; t += gridDim.x * blockDim.x) {
    const size_t e = t / per;
    const int ab = (int)(t % per), a = ab / nen, b = ab % nen;
    out[t] = s_m * (tau[e] * Cn[e * per + b * nen + a]) + s_c * (C[t] + tau[e] * Ct[t]);
  }
}

// ------------------------------------------------------------- transfers ----
__global__ void k_interp(FemLattice H, FemLattice h, const double* __restrict__ xH, double* __restrict__ xh) {
  const int ux = h.ux(), n = ux * h.uy();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    xh[i] = fem_interp_at(H, i / ux, i % ux, [&](int I) { return xH[I]; });
}

__global__ void k_restrict(FemLattice h, FemLattice H, const double* __restrict__ xh, double* __restrict__ xH) {
  const int ux = H.ux(), n = ux * H.uy();
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < n; I += gridDim.x * blockDim.x)
    xH[I] = fem_restrict_at(h, I / ux, I % ux, [&](int j) { return xh[j]; });
}

// ------------------------------------------------------------- boundary flux --
// Per boundary face: Fe_I = sum_q (N w)[q][I] (n . U_q) (core/element_calc.py:
// 111-163); the per-node sums in face order follow (the segment_sum order of
// core/element_calc.py:131-133). A face that names a node outside [0, nn) is
// skipped: its entries get Fe = 0, nothing of it is read, and *skipped counts it.
__global__ void k_boundary_fe(const double* __restrict__ coords, int dim, const int32_t* __restrict__ bconn,
                              const double* __restrict__ nvec, int nb, int npf, const double* __restrict__ U, int nn,
                              double* __restrict__ Fe, int* __restrict__ skipped) {
  const double s3 = 1.0 / sqrt(3.0), g35 = sqrt(3.0 / 5.0);
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nb; f += gridDim.x * blockDim.x) {
    const int32_t* nd = bconn + (size_t)f * npf;
    bool bad = false;
    for (int I = 0; I < npf; ++I) bad |= (unsigned)nd[I] >= (unsigned)nn;
    if (bad) {
      for (int I = 0; I < npf; ++I) Fe[(size_t)f * npf + I] = 0.0;
      atomicAdd(skipped, 1);
      continue;
    }
    double nrm[3] = {nvec[f * dim], nvec[f * dim + 1], dim == 3 ? nvec[f * dim + 2] : 0.0};
    double Ub[4][3];
    for (int I = 0; I < npf; ++I)
      for (int d = 0; d < 3; ++d) Ub[I][d] = (d < dim) ? U[nd[I] + (size_t)d * nn] : 0.0;
    double out[4] = {0, 0, 0, 0};
    if (npf == 2) {  // lin2
      const double ddx = coords[nd[1] * dim] - coords[nd[0] * dim], ddy = coords[nd[1] * dim + 1] - coords[nd[0] * dim + 1];
      const double h = sqrt(ddx * ddx + ddy * ddy);
      for (int q = 0; q < 2; ++q) {
        const double xi = (q == 0 ? -1.0 : 1.0) * s3;
        const double Nq[2] = {(1 - xi) / 2, (1 + xi) / 2};
        const double w = 1.0 * (h / 2);
        double un = 0.0;
        for (int d = 0; d < 2; ++d) un += nrm[d] * (Nq[0] * Ub[0][d] + Nq[1] * Ub[1][d]);
        for (int I = 0; I < 2; ++I) out[I] += (Nq[I] * w) * un;
      }
    } else if (npf == 3) {  // lin3
      const double gp[3] = {-g35, 0.0, g35}, w1[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
      for (int q = 0; q < 3; ++q) {
        const double xi = gp[q];
        const double Nq[3] = {xi * (xi - 1) / 2, 1 - xi * xi, xi * (xi + 1) / 2};
        const double dv[3] = {(2 * xi - 1) / 2, -2 * xi, (2 * xi + 1) / 2};
        double jx = 0, jy = 0;
        for (int a = 0; a < 3; ++a) {
          jx += dv[a] * coords[nd[a] * dim];
          jy += dv[a] * coords[nd[a] * dim + 1];
        }
        const double w = w1[q] * sqrt(jx * jx + jy * jy);
        double un = 0.0;
        for (int d = 0; d < 2; ++d) un += nrm[d] * (Nq[0] * Ub[0][d] + Nq[1] * Ub[1][d] + Nq[2] * Ub[2][d]);
        for (int I = 0; I < 3; ++I) out[I] += (Nq[I] * w) * un;
      }
    } else {  // quad4 face of an axis-aligned hex: the in-plane axes are the two
              // other than the normal's dominant component
      int dn = 0;
      for (int d = 1; d < 3; ++d)
        if (fabs(nrm[d]) > fabs(nrm[dn])) dn = d;
      const int ax[2] = {dn == 0 ? 1 : 0, dn == 2 ? 1 : 2};
      const double sx[4] = {-1, 1, 1, -1}, sy[4] = {-1, -1, 1, 1};
      for (int q = 0; q < 4; ++q) {
        const double xi = sx[q] * s3, eta = sy[q] * s3;
        double Nq[4], dxi[4], deta[4];
        for (int a = 0; a < 4; ++a) {
          Nq[a] = (1 + sx[a] * xi) * (1 + sy[a] * eta) / 4;
          dxi[a] = sx[a] * (1 + sy[a] * eta) / 4;
          deta[a] = sy[a] * (1 + sx[a] * xi) / 4;
        }
        double J[2][2] = {{0, 0}, {0, 0}};
        for (int a = 0; a < 4; ++a)
          for (int d = 0; d < 2; ++d) {
            J[0][d] += dxi[a] * coords[nd[a] * dim + ax[d]];
            J[1][d] += deta[a] * coords[nd[a] * dim + ax[d]];
          }
        const double w = fabs(J[0][0] * J[1][1] - J[0][1] * J[1][0]);
        double un = 0.0;
        for (int d = 0; d < 3; ++d) {
          double uq = 0.0;
          for (int a = 0; a < 4; ++a) uq += Nq[a] * Ub[a][d];
          un += nrm[d] * uq;
        }
        for (int I = 0; I < 4; ++I) out[I] += (Nq[I] * w) * un;
      }
    }
    for (int I = 0; I < npf; ++I) Fe[(size_t)f * npf + I] = out[I];
  }
}

// Node-parallel assembly with the result of a serial scatter in face order,
// bit for bit: each node sums its entries t (bconn[t] == node) in increasing t,
// through a node -> entry CSR built on the device (count, one-CTA exclusive
// scan, fill, then an insertion sort of each node's short list). Entries whose
// node is outside [0, nn) are left out.
__global__ void k_bs_count(const int32_t* __restrict__ bconn, int m, int nn, int* __restrict__ cnt) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    const int n = bconn[t];
    if ((unsigned)n < (unsigned)nn) atomicAdd(cnt + n, 1);
  }
}
// off[i] = sum_{i' < i} cnt[i'] for i in [0, nn]; one CTA, each thread a contiguous chunk
__global__ void k_bs_scan(const int* __restrict__ cnt, int nn, int* __restrict__ off) {
  __shared__ int part[1024];
  const int T = blockDim.x, tid = threadIdx.x;
  const int chunk = (nn + T - 1) / T;
  const int b = min(nn, tid * chunk), e = min(nn, b + chunk);
  int sum = 0;
  for (int i = b; i < e; ++i) sum += cnt[i];
  part[tid] = sum;
  __syncthreads();
  for (int d = 1; d < T; d <<= 1) {
    const int v = tid >= d ? part[tid - d] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  int run = part[tid] - sum;
  for (int i = b; i < e; ++i) {
    off[i] = run;
    run += cnt[i];
  }
  if (tid == T - 1) off[nn] = part[T - 1];
}
// The same prefix sum over many CTAs, in three passes of FEM_SCAN_CHUNK elements
// per CTA: chunk sums, their exclusive scan in one CTA, then each chunk scanned
// from its offset. Integer sums, so off is the single-CTA result exactly.
#define FEM_SCAN_CHUNK 4096  // 256 threads x 16 consecutive elements
__device__ __forceinline__ int fem_block_sum_int(int v, int* ws) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) ws[warp] = v;
  __syncthreads();
  int t = 0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
  return t;
}
__global__ void k_scan_chunk_sums(const int* __restrict__ cnt, int n, int* __restrict__ bsum) {
  __shared__ int ws[32];
  const int base = blockIdx.x * FEM_SCAN_CHUNK, end = min(n, base + FEM_SCAN_CHUNK);
  int v = 0;
  for (int i = base + threadIdx.x; i < end; i += blockDim.x) v += cnt[i];
  v = fem_block_sum_int(v, ws);
  if (threadIdx.x == 0) bsum[blockIdx.x] = v;
}
// exclusive scan of bsum[0, nb) in place by one CTA; *total = the sum of all
__global__ void k_scan_chunk_offsets(int* __restrict__ bsum, int nb, int* __restrict__ total) {
  __shared__ int ws[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nb; b0 += blockDim.x) {
    const int i = b0 + threadIdx.x;
    const int v = i < nb ? bsum[i] : 0;
    int x = v;  // inclusive warp scan
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    int before = carry;
    for (int w = 0; w < warp; ++w) before += ws[w];
    if (i < nb) bsum[i] = before + x - v;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int w = 0; w < nw; ++w) t += ws[w];
      carry += t;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}
// off[i] for the chunk of this CTA: thread t scans its 16 consecutive elements
__global__ void k_scan_chunk_apply(const int* __restrict__ cnt, int n, const int* __restrict__ bsum,
                                   int* __restrict__ off) {
  __shared__ int ws[32];
  constexpr int V = FEM_SCAN_CHUNK / 256;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int i0 = blockIdx.x * FEM_SCAN_CHUNK + threadIdx.x * V;
  int v[V], s = 0;
#pragma unroll
  for (int k = 0; k < V; ++k) {
    v[k] = (i0 + k < n) ? cnt[i0 + k] : 0;
    s += v[k];
  }
  int x = s;  // inclusive warp scan of the thread sums
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  int run = bsum[blockIdx.x] + x - s;
  for (int w = 0; w < warp; ++w) run += ws[w];
#pragma unroll
  for (int k = 0; k < V; ++k) {
    if (i0 + k < n) off[i0 + k] = run;
    run += v[k];
  }
}
// off[0, n] (n + 1 entries) from cnt[0, n): bsum holds fem_scan_chunks(n) ints
static inline int fem_scan_chunks(int n) { return (n + FEM_SCAN_CHUNK - 1) / FEM_SCAN_CHUNK; }
static int fem_launch_scan(const int* cnt, int n, int* off, int* bsum, cudaStream_t s) {
  if (n <= 0) {
    if (cudaMemsetAsync(off, 0, sizeof(int), s) != cudaSuccess) return fem_after_launch("memset");
    return FEM_OK;
  }
  const int nb = fem_scan_chunks(n);
  k_scan_chunk_sums<<<nb, 256, 0, s>>>(cnt, n, bsum);
  if (int rc = fem_after_launch("k_scan_chunk_sums")) return rc;
  k_scan_chunk_offsets<<<1, 1024, 0, s>>>(bsum, nb, off + n);
  if (int rc = fem_after_launch("k_scan_chunk_offsets")) return rc;
  k_scan_chunk_apply<<<nb, 256, 0, s>>>(cnt, n, bsum, off);
  return fem_after_launch("k_scan_chunk_apply");
}
__global__ void k_bs_fill(const int32_t* __restrict__ bconn, int m, int nn, const int* __restrict__ off,
                          int* __restrict__ cur, int* __restrict__ list) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    const int n = bconn[t];
    if ((unsigned)n < (unsigned)nn) list[off[n] + atomicAdd(cur + n, 1)] = t;
  }
}
__global__ void k_bs_gather(const int* __restrict__ off, int* __restrict__ list, const double* __restrict__ Fe, int nn,
                            double* __restrict__ F) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < nn; n += gridDim.x * blockDim.x) {
    const int b = off[n], e = off[n + 1];
    for (int i = b + 1; i < e; ++i) {
      const int v = list[i];
      int j = i - 1;
      while (j >= b && list[j] > v) {
        list[j + 1] = list[j];
        --j;
      }
      list[j + 1] = v;
    }
    double acc = 0.0;
    for (int i = b; i < e; ++i) acc += Fe[list[i]];
    F[n] = acc;
  }
}

// The same assembly with tables of a fixed size, independent of nn (the
// no-allocation entry point): the CSR is indexed by slots of an open-addressing
// hash table of `cap` (a power of two, at least twice the entry count) node ids
// instead of by node. Slot assignment depends on the order of the atomics, but
// every slot holds one node and sums its entries in increasing t, so F is the
// same as the per-node CSR's. keys must be -1 and cnt, cur zero on entry.
__global__ void k_bh_count(const int32_t* __restrict__ bconn, int m, int nn, int cap, int* __restrict__ keys,
                           int* __restrict__ slot, int* __restrict__ cnt) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    const int n = bconn[t];
    int h = -1;
    if ((unsigned)n < (unsigned)nn) {
      // linear probing; the table is at most half full, so a free slot or the
      // node's own slot is met within cap probes
      unsigned p = ((unsigned)n * 2654435761u) & (unsigned)(cap - 1);
      for (int k = 0; k < cap; ++k, p = (p + 1) & (unsigned)(cap - 1)) {
        const int prev = atomicCAS(keys + p, -1, n);
        if (prev == -1 || prev == n) {
          h = (int)p;
          break;
        }
      }
      if (h >= 0) atomicAdd(cnt + h, 1);
    }
    slot[t] = h;
  }
}
__global__ void k_bh_fill(const int* __restrict__ slot, int m, const int* __restrict__ off, int* __restrict__ cur,
                          int* __restrict__ list) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
    const int h = slot[t];
    if (h >= 0) list[off[h] + atomicAdd(cur + h, 1)] = t;
  }
}
__global__ void k_bh_gather(const int* __restrict__ keys, int cap, const int* __restrict__ off, int* __restrict__ list,
                            const double* __restrict__ Fe, double* __restrict__ F) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < cap; h += gridDim.x * blockDim.x) {
    const int n = keys[h];
    if (n < 0) continue;
    const int b = off[h], e = off[h + 1];
    for (int i = b + 1; i < e; ++i) {
      const int v = list[i];
      int j = i - 1;
      while (j >= b && list[j] > v) {
        list[j + 1] = list[j];
        --j;
      }
      list[j + 1] = v;
    }
    double acc = 0.0;
    for (int i = b; i < e; ++i) acc += Fe[list[i]];
    F[n] = acc;
  }
}
__global__ void k_fill_zero(double* __restrict__ F, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) F[i] = 0.0;
}

// ---------------------------------------------------------------- blas-1 ----
__global__ void k_dot_partial(const double* __restrict__ x, const double* __restrict__ y, int n,
                              double* __restrict__ part) {
  __shared__ double smem[96];
  double a[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[0] += x[i] * y[i];
  fem_block_sum<1>(a, smem);
  if (threadIdx.x == 0) part[blockIdx.x] = a[0];
}
__global__ void k_dot_final(const double* __restrict__ part, int np, double* __restrict__ out) {
  __shared__ double smem[96];
  double a[1] = {0.0};
  for (int i = threadIdx.x; i < np; i += blockDim.x) a[0] += part[i];
  fem_block_sum<1>(a, smem);
  if (threadIdx.x == 0) out[0] = a[0];
}
__global__ void k_axpby(double a, const double* __restrict__ x, double b, double* __restrict__ y, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a * x[i] + b * y[i];
}


__global__ void k_lincomb(int n, double a, const double* __restrict__ X, double b, const double* __restrict__ Y,
                          double* __restrict__ out) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) out[i] = a * X[i] + b * Y[i];
}

__global__ void k_scale_elem(int ne, int nen, const double* __restrict__ tau, const double* __restrict__ X, int trans,
                             double* __restrict__ out) {
  const int per = nen * nen;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)ne * per; t += gridDim.x * blockDim.x) {
    const size_t e = t / per;
    const int ab = (int)(t % per), a = ab / nen, b = ab % nen;
    out[t] = tau[e] * (trans ? X[e * per + b * nen + a] : X[t]);
  }
}

// out = s_m * Mt + s_c * (C + Ct)   (per element, flat)
// out = s_m Mt + s_c (C + Ct) per element entry; with tn = nen > 0 each element's
// nen x nen block is written transposed
__global__ void k_elem_combine(size_t n, double s_m, const double* __restrict__ Mt, double s_c,
                               const double* __restrict__ C, const double* __restrict__ Ct, int tn,
                               double* __restrict__ out) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    size_t o = t;
    if (tn > 0) {
      const size_t per = (size_t)tn * tn, e = t / per, ab = t % per;
      o = e * per + (ab % tn) * tn + ab / tn;
    }
    out[o] = s_m * Mt[t] + s_c * (C[t] + Ct[t]);
  }
}

// y = alpha S x for an assembled stencil table S (fem_stencil.cuh), one tile of
// 32 x (blockDim/32) nodes per CTA (3D: one plane), x staged in smem by cp.async.
template <int KIND>
__global__ void __launch_bounds__(512) k_stencil_apply(FemGrid g, const double* __restrict__ tab, double alpha,
                                                       const double* __restrict__ x, double* __restrict__ y,
                                                       int cap_doubles) {
  extern __shared__ double sm[];
  __shared__ double stab[FEM_TAB_MAX];
  const int nt = fem_stencil_ncls(g) * KI<KIND>::NOFF;
  for (int t = threadIdx.x; t < nt; t += blockDim.x) stab[t] = tab[t];
  __syncthreads();
  struct Tiles {
    __device__ __forceinline__ int cta() const { return blockIdx.x; }
    __device__ __forceinline__ int ncta() const { return gridDim.x; }
  } tm;
  const double* src[1] = {x};
  fem_tiled_stencil<KIND, 1>(tm, g, stab, sm, src, [](int, const double(&v)[1]) { return v[0]; },
                             [&](int n, int, int, int, double acc, double) { y[n] = alpha * acc; }, FemNoHook(),
                             cap_doubles);
}

// Streaming y = alpha S x (2D kinds) in register strips: a warp owns 32 - 2R
// node columns and M rows. Its 32 lanes load columns x0 - R .. x0 + 31 - R of
// rows y0 - R .. y0 + M - 1 + R straight into registers (one coalesced load per
// row and lane, all issued before any use), the horizontal neighbours come
// from warp shuffles and each row feeds the W output rows it touches. Strips
// clear of the top and bottom boundary rows of a Q1 lattice keep their column's
// 9 coefficients in registers; the others read the table per row. The sum runs
// over dy, then dx, in ascending order for every node. Each CTA assembles the
// stencil table of A in shared memory (fem_stencil_table_block) on entry.
template <int KIND, int M>
__global__ void __launch_bounds__(256, 2) k_stencil_strip(FemGrid g, const double* __restrict__ A, double alpha,
                                                          const double* __restrict__ x, double* __restrict__ y) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF, OW = 32 - 2 * R, NR = M + 2 * R;
  __shared__ double stab[16 * NOFF];
  fem_stencil_table_block<KIND>(g, A, 0, 0, stab);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int nc = fem_axis_ncls(KIND, g.periodic);
  const int ntx = (g.nnx + OW - 1) / OW, nty = (g.nny + M - 1) / M;
  const int nitem = ntx * nty;  // below nn: fits an int
  const int wstep = (gridDim.x * blockDim.x) >> 5;
  for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < nitem; it += wstep) {
    const int by = it / ntx, bx = it - by * ntx;
    const int xg = bx * OW + lane - R, y0 = by * M;
    const int gx = g.periodic ? fem_wrap(xg, g.nnx) : (xg < 0 ? 0 : (xg >= g.nnx ? g.nnx - 1 : xg));
    double v[NR];
    if (y0 >= R && y0 + M + R <= g.nny) {  // all rows inside the lattice: no wrap or clamp
      const double* p = x + (size_t)(y0 - R) * g.nnx + gx;
#pragma unroll
      for (int r = 0; r < NR; ++r) v[r] = __ldg(p + (size_t)r * g.nnx);
    } else {
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        int gy = y0 - R + r;
        gy = g.periodic ? fem_wrap(gy, g.nny) : (gy < 0 ? 0 : (gy >= g.nny ? g.nny - 1 : gy));
        v[r] = __ldg(x + (size_t)gy * g.nnx + gx);
      }
    }
    const bool own = lane >= R && lane < 32 - R && xg < g.nnx;
    const int cx = own ? fem_axis_cls(KIND, g.periodic, xg, g.nex) : 0;
    double acc[M];
#pragma unroll
    for (int m = 0; m < M; ++m) acc[m] = 0.0;
    const bool fast = KIND == FEM_Q1_2D && (g.periodic || (y0 >= 1 && y0 + M <= g.ney));
    if (fast) {
      const double* c = stab + ((g.periodic ? 0 : 1) * nc + cx) * NOFF;
      double cf[NOFF];
#pragma unroll
      for (int o = 0; o < NOFF; ++o) cf[o] = c[o];
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        double sh[W];
        sh[R] = v[r];
#pragma unroll
        for (int d = 1; d <= R; ++d) {
          sh[R + d] = __shfl_down_sync(0xffffffffu, v[r], d);
          sh[R - d] = __shfl_up_sync(0xffffffffu, v[r], d);
        }
#pragma unroll
        for (int dy = 0; dy < W; ++dy) {
          const int m = r - dy;
          if (m >= 0 && m < M) {
#pragma unroll
            for (int dx = 0; dx < W; ++dx) acc[m] += cf[dy * W + dx] * sh[dx];
          }
        }
      }
    } else {
      int crow[M];
#pragma unroll
      for (int m = 0; m < M; ++m) {
        const int yg = y0 + m < g.nny ? y0 + m : g.nny - 1;
        crow[m] = (fem_axis_cls(KIND, g.periodic, yg, g.ney) * nc + cx) * NOFF;
      }
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        double sh[W];
        sh[R] = v[r];
#pragma unroll
        for (int d = 1; d <= R; ++d) {
          sh[R + d] = __shfl_down_sync(0xffffffffu, v[r], d);
          sh[R - d] = __shfl_up_sync(0xffffffffu, v[r], d);
        }
#pragma unroll
        for (int dy = 0; dy < W; ++dy) {
          const int m = r - dy;
          if (m >= 0 && m < M) {
            const double* c = stab + crow[m] + dy * W;
#pragma unroll
            for (int dx = 0; dx < W; ++dx) acc[m] += c[dx] * sh[dx];
          }
        }
      }
    }
    if (own) {
#pragma unroll
      for (int m = 0; m < M; ++m)
        if (y0 + m < g.nny) y[(size_t)(y0 + m) * g.nnx + xg] = alpha * acc[m];
    }
  }
}

int fem_launch_shared_apply(int ncomp, const FemGrid& g, const double* A, double* tab, double alpha, const double* x,
                            double* y, int sms, cudaStream_t s) {
  if (g.kind == FEM_HEX8) {
    if (int rc = fem_launch_stencil_build(g, A, 0, 0, tab, s)) return rc;
  }
  for (int c = 0; c < ncomp; ++c) {
    const size_t o = (size_t)c * g.nn;
    if (g.kind == FEM_HEX8) {
      constexpr int T = 512, TY = T / 32;
      const int grid = ((g.nnx + 31) / 32) * ((g.nny + TY - 1) / TY) * g.nnz;
      // fem_tiled_stencil_3d with one source: 1 staged plane + a ring of 3
      const int dyn = (32 + 2) * (TY + 2) * 4 * (int)sizeof(double);
      k_stencil_apply<FEM_HEX8><<<grid, T, dyn, s>>>(g, tab, alpha, x + o, y + o, dyn / (int)sizeof(double));
    } else {
      constexpr int M = 16;
      const int ow = (g.kind == FEM_Q2_2D) ? 28 : 30;
      const long long nwarp = (long long)((g.nnx + ow - 1) / ow) * ((g.nny + M - 1) / M);
      const long long need = (nwarp + 7) / 8;
      const int grid = (int)(need < 2LL * sms ? need : 2LL * sms);
      if (g.kind == FEM_Q1_2D)
        k_stencil_strip<FEM_Q1_2D, M><<<grid, 256, 0, s>>>(g, A, alpha, x + o, y + o);
      else
        k_stencil_strip<FEM_Q2_2D, M><<<grid, 256, 0, s>>>(g, A, alpha, x + o, y + o);
    }
    if (int rc = fem_after_launch("k_stencil_apply")) return rc;
  }
  return 0;
}

int fem_launch_ebe(int ncomp, const FemGrid& g, const MatCombo& m, const double* x, double* y, cudaStream_t s) {
  const int nb = fem_nblocks(g.nn, FEM_OP_THREADS);
  FEM_KIND_DISPATCH(g.kind, K, {
    if (ncomp == 1) k_ebe_apply<K, 1><<<nb, FEM_OP_THREADS, 0, s>>>(g, m, x, y);
    else if (ncomp == 2) k_ebe_apply<K, 2><<<nb, FEM_OP_THREADS, 0, s>>>(g, m, x, y);
    else k_ebe_apply<K, 3><<<nb, FEM_OP_THREADS, 0, s>>>(g, m, x, y);
  });
  return fem_after_launch("k_ebe_apply");
}
int fem_launch_grad(int ndim, const FemGrid& g, const double* Ge, const double* P, double* y, cudaStream_t s) {
  const int nb = fem_nblocks(g.nn, FEM_OP_THREADS);
  FEM_KIND_DISPATCH(g.kind, K, (k_grad<K><<<nb, FEM_OP_THREADS, 0, s>>>(g, Ge, P, y)));
  return fem_after_launch("k_grad");
}
int fem_launch_div(int ndim, const FemGrid& g, const double* Ge, const double* U, double* y, cudaStream_t s) {
  const int nb = fem_nblocks(g.nn, FEM_OP_THREADS);
  FEM_KIND_DISPATCH(g.kind, K, (k_div<K><<<nb, FEM_OP_THREADS, 0, s>>>(g, Ge, U, y)));
  return fem_after_launch("k_div");
}
int fem_launch_convection(const FemGrid& g, const FemQuad& Q, const double* U, double beta, int mode, double* out,
                          cudaStream_t s) {
  const int nbk = fem_nblocks((g.ne + FEM_CE_EPB_K - 1) / FEM_CE_EPB_K, 1, 148 * 16);
  if (Q.nq == 8 && Q.nen == 8 && Q.ndim == 3 && g.kind == FEM_HEX8) {
    const int nb8 = fem_nblocks((g.ne + FEM_CE8_EPB - 1) / FEM_CE8_EPB, 1, 148 * 16);
    k_convection_hex8<<<nb8, 256, 0, s>>>(g, Q, U, beta, mode, out);
    return fem_after_launch("k_convection_hex8");
  }
  if (Q.nq == 9 && Q.nen == 9 && Q.ndim == 2) {
    k_convection_k<9, 9, 2><<<nbk, FEM_OP_THREADS, 0, s>>>(g, Q, U, beta, mode, out);
    return fem_after_launch("k_convection_k");
  }
  if (Q.nq == 4 && Q.nen == 4 && Q.ndim == 2) {
    k_convection_k<4, 4, 2><<<nbk, FEM_OP_THREADS, 0, s>>>(g, Q, U, beta, mode, out);
    return fem_after_launch("k_convection_k");
  }
  const int nb = fem_nblocks((g.ne + FEM_CE_EPB - 1) / FEM_CE_EPB, 1, 148 * 32);
  k_convection<<<nb, FEM_OP_THREADS, 0, s>>>(g, Q, U, beta, mode, out);
  return fem_after_launch("k_convection");
}
int fem_launch_supg_tau(const FemGrid& g, const FemQuad& Q, const double* U, const double* Ce, const double* Ct,
                        double D, double dt, double r, double* tau, cudaStream_t s) {
  k_supg_tau<<<fem_nblocks(g.ne, 128), 128, 0, s>>>(g, Q, U, Ce, Ct, D, dt, r, tau);
  return fem_after_launch("k_supg_tau");
}
int fem_launch_scale_elem(int ne, int nen, const double* tau, const double* X, int trans, double* out, cudaStream_t s) {
  k_scale_elem<<<fem_nblocks((long long)ne * nen * nen, 256), 256, 0, s>>>(ne, nen, tau, X, trans, out);
  return fem_after_launch("k_scale_elem");
}
int fem_launch_elem_combine(size_t n, double s_m, const double* Mt, double s_c, const double* C, const double* Ct,
                            double* out, int transpose_nen, cudaStream_t s) {
  k_elem_combine<<<fem_nblocks((long long)n, 256), 256, 0, s>>>(n, s_m, Mt, s_c, C, Ct, transpose_nen, out);
  return fem_after_launch("k_elem_combine");
}
int fem_launch_lincomb(int n, double a, const double* X, double b, const double* Y, double* out, cudaStream_t s) {
  k_lincomb<<<1, 128, 0, s>>>(n, a, X, b, Y, out);
  return fem_after_launch("k_lincomb");
}
int fem_launch_interp(const FemLattice& H, const FemLattice& h, const double* xH, double* xh, cudaStream_t s) {
  k_interp<<<fem_nblocks((long long)h.nx * h.ny, 256), 256, 0, s>>>(H, h, xH, xh);
  return fem_after_launch("k_interp");
}
int fem_launch_restrict(const FemLattice& h, const FemLattice& H, const double* xh, double* xH, cudaStream_t s) {
  k_restrict<<<fem_nblocks((long long)H.nx * H.ny, 256), 256, 0, s>>>(h, H, xh, xH);
  return fem_after_launch("k_restrict");
}
int fem_launch_boundary_hash(const double* coords, int dim, const int32_t* bconn, const double* nvec, int nb, int npf,
                             const double* U, int nn, const FemBoundaryHash& H, double* Fp, cudaStream_t s) {
  const int m = nb * npf;
  if (cudaMemsetAsync(H.skipped, 0, sizeof(int), s) != cudaSuccess) return fem_after_launch("memset");
  if (nb > 0) {
    k_boundary_fe<<<fem_nblocks(nb, 128), 128, 0, s>>>(coords, dim, bconn, nvec, nb, npf, U, nn, H.Fe, H.skipped);
    if (int rc = fem_after_launch("k_boundary_fe")) return rc;
  }
  k_fill_zero<<<fem_nblocks(nn, 256), 256, 0, s>>>(Fp, nn);
  if (int rc = fem_after_launch("k_fill_zero")) return rc;
  if (m == 0) return FEM_OK;
  if (cudaMemsetAsync(H.keys, 0xff, (size_t)H.cap * sizeof(int), s) != cudaSuccess ||
      cudaMemsetAsync(H.cnt, 0, (size_t)H.cap * sizeof(int), s) != cudaSuccess)
    return fem_after_launch("memset");
  k_bh_count<<<fem_nblocks(m, 256), 256, 0, s>>>(bconn, m, nn, H.cap, H.keys, H.slot, H.cnt);
  if (int rc = fem_after_launch("k_bh_count")) return rc;
  k_bs_scan<<<1, 1024, 0, s>>>(H.cnt, H.cap, H.off);
  if (int rc = fem_after_launch("k_bs_scan")) return rc;
  if (cudaMemsetAsync(H.cnt, 0, (size_t)H.cap * sizeof(int), s) != cudaSuccess) return fem_after_launch("memset");
  k_bh_fill<<<fem_nblocks(m, 256), 256, 0, s>>>(H.slot, m, H.off, H.cnt, H.list);
  if (int rc = fem_after_launch("k_bh_fill")) return rc;
  k_bh_gather<<<fem_nblocks(H.cap, 256), 256, 0, s>>>(H.keys, H.cap, H.off, H.list, H.Fe, Fp);
  return fem_after_launch("k_bh_gather");
}
int fem_launch_boundary_csr(const double* coords, int dim, const int32_t* bconn, const double* nvec, int nb, int npf,
                            const double* U, int nn, double* Fe, int* cnt, int* off, int* list, int* skipped,
                            double* Fp, cudaStream_t s) {
  const int m = nb * npf;
  if (cudaMemsetAsync(skipped, 0, sizeof(int), s) != cudaSuccess) return fem_after_launch("memset");
  if (nb > 0) {
    k_boundary_fe<<<fem_nblocks(nb, 128), 128, 0, s>>>(coords, dim, bconn, nvec, nb, npf, U, nn, Fe, skipped);
    if (int rc = fem_after_launch("k_boundary_fe")) return rc;
  }
  if (cudaMemsetAsync(cnt, 0, (size_t)nn * sizeof(int), s) != cudaSuccess) return fem_after_launch("memset");
  if (m > 0) {
    k_bs_count<<<fem_nblocks(m, 256), 256, 0, s>>>(bconn, m, nn, cnt);
    if (int rc = fem_after_launch("k_bs_count")) return rc;
  }
  // off holds nn + 1 offsets, then fem_scan_chunks(nn) chunk sums of the scan
  if (int rc = fem_launch_scan(cnt, nn, off, off + nn + 1, s)) return rc;
  if (cudaMemsetAsync(cnt, 0, (size_t)nn * sizeof(int), s) != cudaSuccess) return fem_after_launch("memset");
  if (m > 0) {
    k_bs_fill<<<fem_nblocks(m, 256), 256, 0, s>>>(bconn, m, nn, off, cnt, list);
    if (int rc = fem_after_launch("k_bs_fill")) return rc;
  }
  k_bs_gather<<<fem_nblocks(nn, 256), 256, 0, s>>>(off, list, Fe, nn, Fp);
  return fem_after_launch("k_bs_gather");
}
int fem_launch_dot(const double* x, const double* y, int n, double* part, double* out, cudaStream_t s) {
  const int nb = fem_nblocks(n, 256, 1024);
  k_dot_partial<<<nb, 256, 0, s>>>(x, y, n, part);
  if (int rc = fem_after_launch("k_dot_partial")) return rc;
  k_dot_final<<<1, 256, 0, s>>>(part, nb, out);
  return fem_after_launch("k_dot_final");
}
int fem_launch_axpby(double a, const double* x, double b, double* y, int n, cudaStream_t s) {
  k_axpby<<<fem_nblocks(n, 256), 256, 0, s>>>(a, x, b, y, n);
  return fem_after_launch("k_axpby");
}

__global__ void k_scatter(const int64_t* __restrict__ idx, const double* __restrict__ vals, double value, int n,
                          double* __restrict__ out) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[idx[k]] = vals ? vals[k] : value;
}
__global__ void k_make_mask(const int64_t* __restrict__ idx, int n, int len, uint8_t* __restrict__ mask) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int64_t i = idx[k];
    if (i >= 0 && i < len) mask[i] = 1;
  }
}
int fem_launch_scatter(const int64_t* idx, const double* vals, double value, int n, double* out, cudaStream_t s) {
  k_scatter<<<fem_nblocks(n, 256), 256, 0, s>>>(idx, vals, value, n, out);
  return fem_after_launch("k_scatter");
}
int fem_launch_make_mask(const int64_t* idx, int n, int len, uint8_t* mask, cudaStream_t s) {
  k_make_mask<<<fem_nblocks(n, 256), 256, 0, s>>>(idx, n, len, mask);
  return fem_after_launch("k_make_mask");
}

// ------------------------------------------------- on-the-fly convection ----
template <int KIND>
__global__ void __launch_bounds__(256) k_conv_factors(FemGrid g, const __grid_constant__ FemQuadTab qt,
                                                      const double* __restrict__ U, double bd,
                                                      double* __restrict__ fq) {
  step_conv_factors<KIND>(g, qt, U, bd, fq);
}

// y = alpha Ash x + cc Ce x over the whole lattice, one tile per CTA.
template <int KIND, int NC>
__global__ void __launch_bounds__(FEM_THREADS) k_conv_apply(FemGrid g, const __grid_constant__ FemQuadTab qt,
                                                            const double* __restrict__ fq, double cc, double alpha,
                                                            const double* __restrict__ Ash,
                                                            const double* __restrict__ x, double* __restrict__ y) {
  extern __shared__ double sm[];
  __shared__ double sA[81];
  constexpr int NEN = KI<KIND>::NEN;
  if (Ash)
    for (int t = threadIdx.x; t < NEN * NEN; t += blockDim.x) sA[t] = Ash[t];
  __syncthreads();
  step_conv_apply<KIND, NC>(g, qt, fq, cc, alpha, Ash ? sA : nullptr, x, y, sm);
}

int fem_launch_conv_factors(const FemGrid& g, const FemQuadTab& qt, const double* U, double bd, double* fq,
                            cudaStream_t s) {
  if (g.kind == FEM_HEX8) return FEM_E_ARG;
  const int nb = fem_nblocks(g.ne, 256);
  if (g.kind == FEM_Q1_2D)
    k_conv_factors<FEM_Q1_2D><<<nb, 256, 0, s>>>(g, qt, U, bd, fq);
  else
    k_conv_factors<FEM_Q2_2D><<<nb, 256, 0, s>>>(g, qt, U, bd, fq);
  return fem_after_launch("k_conv_factors");
}

int fem_launch_conv_apply(int ncomp, const FemGrid& g, const FemQuadTab& qt, const double* fq, double cc,
                          double alpha, const double* Ash, const double* x, double* y, int grid, cudaStream_t s) {
  if (g.kind == FEM_HEX8 || ncomp != 2 || grid < 1) return FEM_E_ARG;
  const int ntile = grid;  // one tile per CTA (tile height adapts to the grid)
  const int dyn = FEM_CONV_SMEM * (int)sizeof(double);
  if (g.kind == FEM_Q1_2D) {
    cudaFuncSetAttribute(k_conv_apply<FEM_Q1_2D, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    k_conv_apply<FEM_Q1_2D, 2><<<ntile, FEM_THREADS, dyn, s>>>(g, qt, fq, cc, alpha, Ash, x, y);
  } else {
    cudaFuncSetAttribute(k_conv_apply<FEM_Q2_2D, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    k_conv_apply<FEM_Q2_2D, 2><<<ntile, FEM_THREADS, dyn, s>>>(g, qt, fq, cc, alpha, Ash, x, y);
  }
  return fem_after_launch("k_conv_apply");
}

// hex8: Gauss-point factors of Ce(U), element-major fq[e * 32 + 4 q + k]
// (fem_conv3_factors), one thread per element
__global__ void __launch_bounds__(256) k_conv_factors3(FemGrid g, const __grid_constant__ FemQuadTab qt,
                                                       const double* __restrict__ U, double bd,
                                                       double* __restrict__ fq) {
  const size_t nn = g.nn;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.ne; e += gridDim.x * blockDim.x) {
    const int ex = e % g.nex, eyz = e / g.nex, ey = eyz % g.ney, ez = eyz / g.ney;
    double u[3][8];
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      const size_t n = fem_enode<FEM_HEX8, 0>(g, ex, ey, ez) + (size_t)kdk<FEM_HEX8>(b) * g.nnx * g.nny +
                       (size_t)kdj<FEM_HEX8>(b) * g.nnx + kdi<FEM_HEX8>(b);
#pragma unroll
      for (int c = 0; c < 3; ++c) u[c][b] = U[n + c * nn];
    }
    fem_conv3_factors(qt, u, bd, fq + (size_t)e * FEM_C3_NF);
  }
}

// hex8: y = alpha Ash x + cc Ce x (3 components) from the factors, one tile
// loop per CTA over the lattice
__global__ void __launch_bounds__(FEM_THREADS, 1) k_conv_apply3(FemGrid g, const __grid_constant__ FemQuadTab qt,
                                                                const double* __restrict__ fq, double cc,
                                                                double alpha, const double* __restrict__ Ash,
                                                                const double* __restrict__ x, double* __restrict__ y,
                                                                int* err) {
  extern __shared__ __align__(128) double sm3[];
  __shared__ double sA[64];
  __shared__ __align__(8) uint64_t bar;
  __shared__ unsigned phase;
  if (Ash)
    for (int t = threadIdx.x; t < 64; t += blockDim.x) sA[t] = Ash[t];
  if (threadIdx.x == 0) {
    fem_mbar_init(&bar, 1);
    phase = 0u;
  }
  __syncthreads();
  const size_t nn = g.nn;
  struct Tiles {
    __device__ __forceinline__ int cta() const { return blockIdx.x; }
    __device__ __forceinline__ int ncta() const { return gridDim.x; }
  } tm;
  const double* src[1] = {x};
  const FemC3Tma tma{&bar, &phase, err};
  fem_tiled_conv3<3, 1>(tm, g, sm3, tma, src, [](int, const double(&v)[1]) { return v[0]; }, fq, qt, cc, alpha,
                        Ash ? sA : nullptr, [&](int i, const double(&v)[3], const double(&)[3]) {
#pragma unroll
                          for (int c = 0; c < 3; ++c) y[i + c * nn] = v[c];
                        });
}

int fem_launch_conv_factors3(const FemGrid& g, const FemQuadTab& qt, const double* U, double bd, double* fq,
                             cudaStream_t s) {
  if (g.kind != FEM_HEX8) return FEM_E_ARG;
  k_conv_factors3<<<fem_nblocks(g.ne, 256), 256, 0, s>>>(g, qt, U, bd, fq);
  return fem_after_launch("k_conv_factors3");
}

int fem_launch_conv_apply3(const FemGrid& g, const FemQuadTab& qt, const double* fq, double cc, double alpha,
                           const double* Ash, const double* x, double* y, int grid, int* err, cudaStream_t s) {
  if (g.kind != FEM_HEX8 || grid < 1) return FEM_E_ARG;
  const int dyn = FEM_C3_SMEM(3, 1) * (int)sizeof(double);
  cudaFuncSetAttribute(k_conv_apply3, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
  k_conv_apply3<<<grid, FEM_THREADS, dyn, s>>>(g, qt, fq, cc, alpha, Ash, x, y, err);
  return fem_after_launch("k_conv_apply3");
}

// ---------------------------------------------------- convection VJP ----
// d/dU <a, Ce(U) b> (Ce of core/element_calc.py:165-185 acting on each of ncomp
// components): per element and local node k,
//   ge[e][d][k] = sum_q w_q (N_k(q) s_d(q) + beta dN_k/dx_d(q) t(q)),
//   s_d = sum_c A_c d_d B_c,  t = sum_c A_c B_c,
// A_c, B_c, d_d B_c being a_c, b_c and the derivatives of b_c at the Gauss point;
// then each node sums its incident elements' entries in a fixed order.
template <int KIND>
__global__ void __launch_bounds__(256) k_conv_vjp_elem(FemGrid g, const __grid_constant__ FemQuadTab qt, int ncomp,
                                                       const double* __restrict__ a, const double* __restrict__ b,
                                                       double beta, double* __restrict__ ge) {
  constexpr int NEN = KI<KIND>::NEN, DIM = KI<KIND>::DIM, NQ = (KIND == FEM_Q2_2D) ? 9 : (KIND == FEM_HEX8 ? 8 : 4);
  const size_t nn = g.nn;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.ne; e += gridDim.x * blockDim.x) {
    const int ex = e % g.nex, eyz = e / g.nex, ey = eyz % g.ney, ez = eyz / g.ney;
    int nd[NEN];
#pragma unroll
    for (int k = 0; k < NEN; ++k) nd[k] = fem_elem_node(g, ex, ey, ez, k);
    double out[DIM][NEN];
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
      for (int k = 0; k < NEN; ++k) out[d][k] = 0.0;
    for (int q = 0; q < NQ; ++q) {
      double sd[DIM], t = 0.0;
#pragma unroll
      for (int d = 0; d < DIM; ++d) sd[d] = 0.0;
      for (int c = 0; c < ncomp; ++c) {
        double Ac = 0.0, Bc = 0.0, dB[DIM];
#pragma unroll
        for (int d = 0; d < DIM; ++d) dB[d] = 0.0;
#pragma unroll
        for (int k = 0; k < NEN; ++k) {
          const double av = a[nd[k] + c * nn], bv = b[nd[k] + c * nn];
          Ac += qt.N[q][k] * av;
          Bc += qt.N[q][k] * bv;
          dB[0] += qt.dx[q][k] * bv;
          dB[1] += qt.dy[q][k] * bv;
          if (DIM == 3) dB[DIM - 1] += qt.dz[q][k] * bv;
        }
#pragma unroll
        for (int d = 0; d < DIM; ++d) sd[d] += Ac * dB[d];
        t += Ac * Bc;
      }
#pragma unroll
      for (int k = 0; k < NEN; ++k) {
        out[0][k] += qt.w[q] * (qt.N[q][k] * sd[0] + beta * qt.dx[q][k] * t);
        out[1][k] += qt.w[q] * (qt.N[q][k] * sd[1] + beta * qt.dy[q][k] * t);
        if (DIM == 3) out[DIM - 1][k] += qt.w[q] * (qt.N[q][k] * sd[DIM - 1] + beta * qt.dz[q][k] * t);
      }
    }
#pragma unroll
    for (int d = 0; d < DIM; ++d)
#pragma unroll
      for (int k = 0; k < NEN; ++k) ge[((size_t)e * DIM + d) * NEN + k] = out[d][k];
  }
}
template <int KIND>
__global__ void __launch_bounds__(256) k_conv_vjp_gather(FemGrid g, const double* __restrict__ ge,
                                                         double* __restrict__ y) {
  constexpr int NEN = KI<KIND>::NEN, DIM = KI<KIND>::DIM;
  const size_t nn = g.nn;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    double v[DIM];
#pragma unroll
    for (int d = 0; d < DIM; ++d) v[d] = 0.0;
    fem_incident_k<KIND>(g, ix, iy, iz, [&](int, int, int, int e, int k) {
#pragma unroll
      for (int d = 0; d < DIM; ++d) v[d] += ge[((size_t)e * DIM + d) * NEN + k];
    });
#pragma unroll
    for (int d = 0; d < DIM; ++d) y[n + d * nn] = v[d];
  }
}

// ------------------------------------------------------- transport VJP ----
// Velocity side of the passive-scalar step's adjoint (solvers/passive_transport.py:
// 14-97 with the matrices of :80-88): for s = sum_e lam_e^T (B(U_n) phi_n - E(U_n, U) phi)_e,
// ge_n = ds/dU_n and ge_u = ds/dU per element and local node, with
//   E = Mtau/dt + (Ce(U) + Ctau)/2,  B = Mtau/dt - (Ce(U_n) + Ctau)/2   (SUPG)
//   E = Ce(U)/2,                     B = -Ce(U_n)/2                     (plain)
// Ce with beta = 1 (core/element_calc.py:165-185), Ct = sum_q w dN^T (u u^T) dN
// (:188-200), tau the r = 2 blend of ce = |Ce(U)|_F, kt = |Ct|_F and the mean
// |u|^2 over the Gauss points (:202-229), Ctau = tau Ct, Mtau = tau Ce(U_n)^T.
// The derivative goes through the element matrices: with G = ds/d(matrix),
// <G, Ce(V)> and <G, Ct(u)> are differentiated at the Gauss points and
// interpolated back to the nodes.
template <int KIND>
__global__ void __launch_bounds__(128) k_transport_vjp_elem(FemGrid g, const __grid_constant__ FemQuadTab qt,
                                                            const double* __restrict__ Un, const double* __restrict__ U,
                                                            const double* __restrict__ lam,
                                                            const double* __restrict__ phin,
                                                            const double* __restrict__ phi, double dt, double D,
                                                            int supg, double* __restrict__ gen,
                                                            double* __restrict__ geu) {
  constexpr int NEN = KI<KIND>::NEN, NQ = (KIND == FEM_Q2_2D) ? 9 : 4;
  const size_t nn = g.nn;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.ne; e += gridDim.x * blockDim.x) {
    const int ex = e % g.nex, ey = e / g.nex;
    int nd[NEN];
    double l[NEN], fn[NEN], f[NEN], un[2][NEN], uu[2][NEN];
#pragma unroll
    for (int k = 0; k < NEN; ++k) {
      nd[k] = fem_elem_node(g, ex, ey, 0, k);
      l[k] = lam[nd[k]];
      fn[k] = phin[nd[k]];
      f[k] = phi[nd[k]];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        un[c][k] = Un[nd[k] + c * nn];
        uu[c][k] = U[nd[k] + c * nn];
      }
    }
    // Ce(U) and Ct(U_n) (the ones whose norms enter tau); lam^T Ce(U_n)^T (phi_n - phi)
    // and lam^T Ct (phi_n + phi) at the Gauss points, without forming Ce(U_n)
    double Cu[NEN][NEN], Ct[NEN][NEN];
    for (int a = 0; a < NEN; ++a)
      for (int b = 0; b < NEN; ++b) Cu[a][b] = Ct[a][b] = 0.0;
    double un2 = 0.0, sCnT = 0.0, sCt = 0.0;
    for (int q = 0; q < NQ; ++q) {
      double vn[2] = {0.0, 0.0}, vu[2] = {0.0, 0.0}, divn = 0.0, divu = 0.0;
      double dq = 0.0, lq = 0.0, gl = 0.0, gs = 0.0;
      for (int k = 0; k < NEN; ++k) {
        for (int c = 0; c < 2; ++c) {
          vn[c] += qt.N[q][k] * un[c][k];
          vu[c] += qt.N[q][k] * uu[c][k];
        }
        divn += qt.dx[q][k] * un[0][k] + qt.dy[q][k] * un[1][k];
        divu += qt.dx[q][k] * uu[0][k] + qt.dy[q][k] * uu[1][k];
        dq += qt.N[q][k] * (fn[k] - f[k]);
        lq += qt.N[q][k] * l[k];
      }
      for (int k = 0; k < NEN; ++k) {
        const double gk = qt.dx[q][k] * vn[0] + qt.dy[q][k] * vn[1];
        gl += gk * l[k];
        gs += gk * (fn[k] + f[k]);
      }
      un2 += vn[0] * vn[0] + vn[1] * vn[1];
      const double w = qt.w[q];
      // sum_ab d_a Ce(U_n)_ab l_b and sum_ab l_a Ct_ab s_b at this point
      sCnT += w * dq * (gl + divn * lq);
      sCt += w * gl * gs;
      if (supg)
        for (int a = 0; a < NEN; ++a) {
          const double na = qt.N[q][a], ga = qt.dx[q][a] * vn[0] + qt.dy[q][a] * vn[1];
          for (int b = 0; b < NEN; ++b) {
            const double gb = qt.dx[q][b] * vn[0] + qt.dy[q][b] * vn[1];
            Cu[a][b] += w * na * ((vu[0] * qt.dx[q][b] + vu[1] * qt.dy[q][b]) + divu * qt.N[q][b]);
            Ct[a][b] += w * ga * gb;
          }
        }
    }
    un2 /= NQ;
    // ds/d(matrix), applied without storing it:
    //   G_u = -lam phi^T / 2 + cu Ce(U)        (Ce(U) through ce in tau)
    //   G_n = -lam phi_n^T / 2 + (tau/dt) (phi_n - phi) lam^T
    //   G_t = -(tau/2) lam (phi_n + phi)^T + ct Ct
    // and gu2 = ds/d(mean |u|^2)
    double tdt = 0.0, th = 0.0, cu = 0.0, ct = 0.0, gu2 = 0.0;
    if (supg) {
      double ce = 0.0, kt = 0.0;
      for (int a = 0; a < NEN; ++a)
        for (int b = 0; b < NEN; ++b) {
          ce += Cu[a][b] * Cu[a][b];
          kt += Ct[a][b] * Ct[a][b];
        }
      ce = sqrt(ce);
      kt = sqrt(kt);
      const double De = D + 1e-6, c = dt / 2;
      const double t1 = ce / kt, t3 = t1 * (un2 * ce) / (De * kt);
      const double tau = 1.0 / sqrt(1.0 / (t1 * t1) + 1.0 / (c * c) + 1.0 / (t3 * t3));
      // d tau = tau^3 (t1^-3 d t1 + t3^-3 d t3), t1 = ce / kt, t3 = un2 ce^2 / (De kt^2)
      const double tau3 = tau * tau * tau, i1 = 1.0 / (t1 * t1 * t1), i3 = 1.0 / (t3 * t3 * t3);
      const double dce = tau3 * (i1 / kt + i3 * 2.0 * un2 * ce / (De * kt * kt));
      const double dkt = tau3 * (-i1 * ce / (kt * kt) - i3 * 2.0 * un2 * ce * ce / (De * kt * kt * kt));
      const double dun2 = tau3 * i3 * ce * ce / (De * kt * kt);
      const double gtau = sCnT / dt - 0.5 * sCt;
      tdt = tau / dt;
      th = 0.5 * tau;
      cu = gtau * dce / ce;
      ct = gtau * dkt / kt;
      gu2 = gtau * dun2;
    }
    // back to the nodes: <G, Ce(V)> and <G_t, Ct(u)> differentiated at the Gauss points
    double on[2][NEN], ou[2][NEN];
    for (int c = 0; c < 2; ++c)
      for (int k = 0; k < NEN; ++k) on[c][k] = ou[c][k] = 0.0;
    for (int q = 0; q < NQ; ++q) {
      const double w = qt.w[q];
      double vn[2] = {0.0, 0.0};
      double lq = 0.0, fq = 0.0, fnq = 0.0, dq = 0.0, dl[2] = {0.0, 0.0}, df[2] = {0.0, 0.0}, dfn[2] = {0.0, 0.0};
      double gl = 0.0, gs = 0.0, ss[2] = {0.0, 0.0};
      for (int k = 0; k < NEN; ++k) {
        const double nk = qt.N[q][k], xk = qt.dx[q][k], yk = qt.dy[q][k];
        vn[0] += nk * un[0][k];
        vn[1] += nk * un[1][k];
        lq += nk * l[k];
        fq += nk * f[k];
        fnq += nk * fn[k];
        dq += nk * (fn[k] - f[k]);
        dl[0] += xk * l[k];
        dl[1] += yk * l[k];
        df[0] += xk * f[k];
        df[1] += yk * f[k];
        dfn[0] += xk * fn[k];
        dfn[1] += yk * fn[k];
        ss[0] += xk * (fn[k] + f[k]);
        ss[1] += yk * (fn[k] + f[k]);
      }
      gl = dl[0] * vn[0] + dl[1] * vn[1];
      gs = ss[0] * vn[0] + ss[1] * vn[1];
      // S_d = sum_ab G_ab N_a dN_b/dx_d, T = sum_ab G_ab N_a N_b (rank-one parts in closed form)
      double Su[2] = {-0.5 * lq * df[0], -0.5 * lq * df[1]}, Tu = -0.5 * lq * fq;
      double Sn[2] = {-0.5 * lq * dfn[0] + tdt * dq * dl[0], -0.5 * lq * dfn[1] + tdt * dq * dl[1]};
      double Tn = -0.5 * lq * fnq + tdt * dq * lq;
      // d/du of sum_ab G_t,ab (dN_a . u)(dN_b . u) = sum_ab G_t,ab (dN_a (dN_b . u) + (dN_a . u) dN_b)
      double Gq[2] = {-th * (dl[0] * gs + gl * ss[0]), -th * (dl[1] * gs + gl * ss[1])};
      if (supg)
        for (int a = 0; a < NEN; ++a) {
          const double na = qt.N[q][a], ga = qt.dx[q][a] * vn[0] + qt.dy[q][a] * vn[1];
          for (int b = 0; b < NEN; ++b) {
            const double dxb = qt.dx[q][b], dyb = qt.dy[q][b], gb = dxb * vn[0] + dyb * vn[1];
            const double cua = cu * Cu[a][b] * na, cta = ct * Ct[a][b];
            Su[0] += cua * dxb;
            Su[1] += cua * dyb;
            Tu += cua * qt.N[q][b];
            Gq[0] += cta * (qt.dx[q][a] * gb + ga * dxb);
            Gq[1] += cta * (qt.dy[q][a] * gb + ga * dyb);
          }
        }
      for (int k = 0; k < NEN; ++k) {
        const double nk = qt.N[q][k];
        ou[0][k] += w * (nk * Su[0] + qt.dx[q][k] * Tu);
        ou[1][k] += w * (nk * Su[1] + qt.dy[q][k] * Tu);
        if (supg) {
          on[0][k] += w * (nk * Sn[0] + qt.dx[q][k] * Tn) + nk * (w * Gq[0] + gu2 * 2.0 * vn[0] / NQ);
          on[1][k] += w * (nk * Sn[1] + qt.dy[q][k] * Tn) + nk * (w * Gq[1] + gu2 * 2.0 * vn[1] / NQ);
        } else {
          on[0][k] += w * (nk * Sn[0] + qt.dx[q][k] * Tn);
          on[1][k] += w * (nk * Sn[1] + qt.dy[q][k] * Tn);
        }
      }
    }
    for (int c = 0; c < 2; ++c)
      for (int k = 0; k < NEN; ++k) {
        gen[((size_t)e * 2 + c) * NEN + k] = on[c][k];
        geu[((size_t)e * 2 + c) * NEN + k] = ou[c][k];
      }
  }
}

int fem_launch_transport_vjp(const FemGrid& g, const FemQuadTab& qt, const double* Un, const double* U,
                             const double* lam, const double* phin, const double* phi, double dt, double D, int supg,
                             double* gen, double* geu, double* yn, double* yu, cudaStream_t s) {
  if (g.kind == FEM_HEX8) return FEM_E_ARG;
  const int be = fem_nblocks(g.ne, 128), bn = fem_nblocks(g.nn, 256);
  if (g.kind == FEM_Q1_2D) {
    k_transport_vjp_elem<FEM_Q1_2D><<<be, 128, 0, s>>>(g, qt, Un, U, lam, phin, phi, dt, D, supg, gen, geu);
    k_conv_vjp_gather<FEM_Q1_2D><<<bn, 256, 0, s>>>(g, gen, yn);
    k_conv_vjp_gather<FEM_Q1_2D><<<bn, 256, 0, s>>>(g, geu, yu);
  } else {
    k_transport_vjp_elem<FEM_Q2_2D><<<be, 128, 0, s>>>(g, qt, Un, U, lam, phin, phi, dt, D, supg, gen, geu);
    k_conv_vjp_gather<FEM_Q2_2D><<<bn, 256, 0, s>>>(g, gen, yn);
    k_conv_vjp_gather<FEM_Q2_2D><<<bn, 256, 0, s>>>(g, geu, yu);
  }
  return fem_after_launch("k_transport_vjp");
}

int fem_launch_conv_vjp(const FemGrid& g, const FemQuadTab& qt, int ncomp, const double* a, const double* b,
                        double beta, double* ge, double* y, cudaStream_t s) {
  const int be = fem_nblocks(g.ne, 256), bn = fem_nblocks(g.nn, 256);
  FEM_KIND_DISPATCH(g.kind, KIND, {
    k_conv_vjp_elem<KIND><<<be, 256, 0, s>>>(g, qt, ncomp, a, b, beta, ge);
    k_conv_vjp_gather<KIND><<<bn, 256, 0, s>>>(g, ge, y);
  });
  return fem_after_launch("k_conv_vjp");
}

// Self-test of the grid barrier's time limit: one CTA waits at a counter
// barrier for one more party than the launch has, so the wait can only end
// through the FEM_BARRIER_TIMEOUT_NS limit. It then sets FEM_ERR_BARRIER_TIMEOUT
// in the error word and returns, as a solver kernel does; status receives the
// error word (0 if the barrier had completed).
__global__ void k_selftest_barrier(FemSync sync, int* __restrict__ status) {
  __shared__ unsigned int round;
  if (threadIdx.x == 0) round = 0u;
  __syncthreads();
  const bool ok = fem_counter_barrier(&sync, sync.count, &round, (int)gridDim.x + 1, 31u);
  if (blockIdx.x == 0 && threadIdx.x == 0) *status = ok ? 0 : (*(volatile int*)sync.err & FEM_ERR_BARRIER_TIMEOUT);
}

int fem_launch_selftest_barrier(const FemSync& sync, int* status, cudaStream_t s) {
  k_selftest_barrier<<<1, 64, 0, s>>>(sync, status);
  return fem_after_launch("k_selftest_barrier");
}
