// Setup kernels: mesh lattice, shape functions, element matrices, assembled diagonals.
#include "fem_args.cuh"


// setup/regular_mesh.py: node coordinates (i*dx, j*dy[, k*dz]) (quad9: i*dx/2)
// and connectivity in the generator's local node order.
__global__ void k_mesh_generate(FemGrid g, double dx, double dy, double dz, double* __restrict__ coords,
                                int64_t* __restrict__ nconn) {
  const int dim = (g.kind == FEM_HEX8) ? 3 : 2;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int n = tid; n < g.nn; n += stride) {
    int i, j, k;
    fem_node_ijk(g, n, i, j, k);
    if (g.kind == FEM_Q2_2D) {
      coords[n * 2 + 0] = i * dx / 2;
      coords[n * 2 + 1] = j * dy / 2;
    } else {
      coords[n * dim + 0] = i * dx;
      coords[n * dim + 1] = j * dy;
      if (dim == 3) coords[n * 3 + 2] = k * dz;
    }
  }
  if (nconn)
    for (int e = tid; e < g.ne; e += stride) {
      const int ie = e % g.nex, r = e / g.nex, je = r % g.ney, ke = r / g.ney;
      for (int b = 0; b < g.nen; ++b) nconn[(size_t)e * g.nen + b] = fem_elem_node(g, ie, je, ke, b);
    }
}

__device__ __forceinline__ void fem_inv2(const double J[2][2], double inv[2][2], double& det) {
  det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
  inv[0][0] = J[1][1] / det;
  inv[0][1] = -J[0][1] / det;
  inv[1][0] = -J[1][0] / det;
  inv[1][1] = J[0][0] / det;
}

__device__ __forceinline__ void fem_inv3(const double J[3][3], double inv[3][3], double& det) {
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  inv[0][0] = c00 / det;
  inv[1][0] = c01 / det;
  inv[2][0] = c02 / det;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
}

// core/shape_functions.py: one thread per Gauss point.
// family: 0 quad4, 1 quad9, 2 hex8, 3 lin2, 4 lin3.
__global__ void k_shape_functions(int family, const double* __restrict__ coords, double* __restrict__ wq,
                                  double* __restrict__ N, double* __restrict__ dN) {
  const int q = threadIdx.x;
  const double r3 = sqrt(3.0), g35 = sqrt(3.0 / 5.0);
  if (family == 0 || family == 2) {
    const int nen = family == 0 ? 4 : 8, dim = family == 0 ? 2 : 3;
    if (q >= nen) return;
    const double sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1},
                 sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    const double xi = sx[q] / r3, eta = sy[q] / r3, ze = (dim == 3) ? sz[q] / r3 : 0.0;
    double dref[3][8];
    for (int a = 0; a < nen; ++a) {
      if (dim == 2) {
        N[q * nen + a] = (1 + sx[a] * xi) * (1 + sy[a] * eta) / 4;
        dref[0][a] = sx[a] * (1 + sy[a] * eta) / 4;
        dref[1][a] = sy[a] * (1 + sx[a] * xi) / 4;
      } else {
        N[q * nen + a] = (1 + sx[a] * xi) * (1 + sy[a] * eta) * (1 + sz[a] * ze) / 8;
        dref[0][a] = sx[a] * (1 + sy[a] * eta) * (1 + sz[a] * ze) / 8;
        dref[1][a] = sy[a] * (1 + sx[a] * xi) * (1 + sz[a] * ze) / 8;
        dref[2][a] = sz[a] * (1 + sx[a] * xi) * (1 + sy[a] * eta) / 8;
      }
    }
    if (dim == 2) {
      double J[2][2] = {{0, 0}, {0, 0}}, inv[2][2], det;
      for (int r = 0; r < 2; ++r)
        for (int d = 0; d < 2; ++d)
          for (int a = 0; a < nen; ++a) J[r][d] += dref[r][a] * coords[a * 2 + d];
      fem_inv2(J, inv, det);
      wq[q] = det;
      for (int d = 0; d < 2; ++d)
        for (int a = 0; a < nen; ++a) dN[(q * 2 + d) * nen + a] = inv[d][0] * dref[0][a] + inv[d][1] * dref[1][a];
    } else {
      double J[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, inv[3][3], det;
      for (int r = 0; r < 3; ++r)
        for (int d = 0; d < 3; ++d)
          for (int a = 0; a < nen; ++a) J[r][d] += dref[r][a] * coords[a * 3 + d];
      fem_inv3(J, inv, det);
      wq[q] = det;
      for (int d = 0; d < 3; ++d)
        for (int a = 0; a < nen; ++a)
          dN[(q * 3 + d) * nen + a] = inv[d][0] * dref[0][a] + inv[d][1] * dref[1][a] + inv[d][2] * dref[2][a];
    }
  } else if (family == 1) {
    if (q >= 9) return;
    const double gp[3] = {-g35, 0.0, g35}, w1[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    const double xi = gp[q % 3], eta = gp[q / 3], w = w1[q / 3] * w1[q % 3];
    double Nv[9], dx[9], dy[9];
    Nv[0] = xi * eta * (xi - 1) * (eta - 1) / 4;
    Nv[1] = (1 - xi * xi) * eta * (eta - 1) / 2;
    Nv[2] = xi * eta * (xi + 1) * (eta - 1) / 4;
    Nv[3] = xi * (xi + 1) * (1 - eta * eta) / 2;
    Nv[4] = xi * eta * (xi + 1) * (eta + 1) / 4;
    Nv[5] = (1 - xi * xi) * eta * (eta + 1) / 2;
    Nv[6] = xi * eta * (xi - 1) * (eta + 1) / 4;
    Nv[7] = xi * (xi - 1) * (1 - eta * eta) / 2;
    Nv[8] = (1 - xi * xi) * (1 - eta * eta);
    dx[0] = eta * (2 * xi - 1) * (eta - 1) / 4;
    dx[1] = -2 * xi * eta * (eta - 1) / 2;
    dx[2] = eta * (2 * xi + 1) * (eta - 1) / 4;
    dx[3] = (2 * xi + 1) * (1 - eta * eta) / 2;
    dx[4] = eta * (2 * xi + 1) * (eta + 1) / 4;
    dx[5] = -2 * xi * eta * (eta + 1) / 2;
    dx[6] = eta * (2 * xi - 1) * (eta + 1) / 4;
    dx[7] = (2 * xi - 1) * (1 - eta * eta) / 2;
    dx[8] = -2 * xi * (1 - eta * eta);
    dy[0] = xi * (xi - 1) * (2 * eta - 1) / 4;
    dy[1] = (1 - xi * xi) * (2 * eta - 1) / 2;
    dy[2] = xi * (xi + 1) * (2 * eta - 1) / 4;
    dy[3] = xi * (xi + 1) * (-2 * eta) / 2;
    dy[4] = xi * (xi + 1) * (2 * eta + 1) / 4;
    dy[5] = (1 - xi * xi) * (2 * eta + 1) / 2;
    dy[6] = xi * (xi - 1) * (2 * eta + 1) / 4;
    dy[7] = xi * (xi - 1) * (-2 * eta) / 2;
    dy[8] = -2 * eta * (1 - xi * xi);
    double J[2][2] = {{0, 0}, {0, 0}}, inv[2][2], det;
    for (int a = 0; a < 9; ++a) {
      N[q * 9 + a] = Nv[a];
      for (int d = 0; d < 2; ++d) {
        J[0][d] += dx[a] * coords[a * 2 + d];
        J[1][d] += dy[a] * coords[a * 2 + d];
      }
    }
    fem_inv2(J, inv, det);
    wq[q] = w * det;
    for (int d = 0; d < 2; ++d)
      for (int a = 0; a < 9; ++a) dN[(q * 2 + d) * 9 + a] = inv[d][0] * dx[a] + inv[d][1] * dy[a];
  } else if (family == 3) {
    if (q >= 2) return;
    const double xi = (q == 0 ? -1.0 : 1.0) / r3;
    const double ddx = coords[2] - coords[0], ddy = coords[3] - coords[1];
    const double h = sqrt(ddx * ddx + ddy * ddy);
    N[q * 2 + 0] = (1 - xi) / 2;
    N[q * 2 + 1] = (1 + xi) / 2;
    dN[q * 2 + 0] = -0.5 * (2 / h);
    dN[q * 2 + 1] = 0.5 * (2 / h);
    wq[q] = 1.0 * (h / 2);
  } else if (family == 4) {
    if (q >= 3) return;
    const double gp[3] = {-g35, 0.0, g35}, w1[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    const double xi = gp[q];
    const double Nv[3] = {xi * (xi - 1) / 2, 1 - xi * xi, xi * (xi + 1) / 2};
    const double dv[3] = {(2 * xi - 1) / 2, -2 * xi, (2 * xi + 1) / 2};
    double jx = 0, jy = 0;
    for (int a = 0; a < 3; ++a) {
      jx += dv[a] * coords[a * 2 + 0];
      jy += dv[a] * coords[a * 2 + 1];
    }
    const double J = sqrt(jx * jx + jy * jy);
    for (int a = 0; a < 3; ++a) {
      N[q * 3 + a] = Nv[a];
      dN[q * 3 + a] = dv[a] / J;
    }
    wq[q] = w1[q] * J;
  }
}

// core/element_calc.py:9-40: Me, Le, Ge from Gauss-point data (one CTA).
__global__ void k_element_matrices(int nq, int nen, int dim, const double* __restrict__ wq,
                                   const double* __restrict__ N, const double* __restrict__ dN,
                                   double* __restrict__ Me, double* __restrict__ Le, double* __restrict__ Leoff,
                                   double* __restrict__ Ge) {
  for (int t = threadIdx.x; t < nen * nen; t += blockDim.x) {
    const int a = t / nen, b = t % nen;
    double m = 0.0, l = 0.0;
    for (int q = 0; q < nq; ++q) {
      m += (N[q * nen + a] * wq[q]) * N[q * nen + b];
      double lq = 0.0;
      for (int d = 0; d < dim; ++d) lq += (dN[(q * dim + d) * nen + a] * wq[q]) * dN[(q * dim + d) * nen + b];
      l += lq;
    }
    Me[t] = m;
    Le[t] = l;
    Leoff[t] = (a == b) ? 0.0 : l;
    for (int d = 0; d < dim; ++d) {
      double gsum = 0.0;
      for (int q = 0; q < nq; ++q) gsum += (N[q * nen + a] * wq[q]) * dN[(q * dim + d) * nen + b];
      Ge[d * nen * nen + t] = gsum;
    }
  }
}

// Assembled lumped mass (rowsum Me) and diag(Le) (core/element_calc.py:9-25, 99-109).
__global__ void k_assemble_diag(FemGrid g, int ndim, const double* __restrict__ Me, const double* __restrict__ Le,
                                double* __restrict__ M, double* __restrict__ Ldiag) {
  const int nen = g.nen;
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    double m = 0.0, l = 0.0;
    fem_for_incident(g, n, [&](int, int, int, int, int a) {
      if (Me) {
        double rs = 0.0;
        for (int b = 0; b < nen; ++b) rs += Me[a * nen + b];
        m += rs;
      }
      if (Le) l += Le[a * nen + a];
    });
    if (M && Me)
      for (int c = 0; c < ndim; ++c) M[n + (size_t)c * g.nn] = m;
    if (Ldiag && Le) Ldiag[n] = l;
  }
}



__global__ void k_level_sums(FemGrid g, FemLattice lat, const double* __restrict__ diag, double* out) {
  __shared__ double smem[128];
  double a[4] = {0.0, 0.0, 0.0, 0.0};
  const int ux = lat.ux();
  for (int i = threadIdx.x; i < g.nn; i += blockDim.x) {
    const double iv = 1.0 / diag[i];
    const int R = i / ux, C = i % ux;
    const double rc = fem_restrict_rowsum(lat, R, C);
    a[0] += iv;
    a[1] += fem_interp_colsum(lat, R, C);
    a[2] += rc;
    a[3] += rc * iv;
  }
  fem_block_sum<4>(a, smem);
  if (threadIdx.x == 0)
    for (int q = 0; q < 4; ++q) out[q] = a[q];
}

int fem_launch_mesh_generate(const FemGrid& g, double dx, double dy, double dz, double* coords, int64_t* nconn,
                             cudaStream_t s) {
  k_mesh_generate<<<fem_nblocks(g.nn > g.ne ? g.nn : g.ne, 256), 256, 0, s>>>(g, dx, dy, dz, coords, nconn);
  return fem_after_launch("k_mesh_generate");
}
int fem_launch_shape_functions(int family, const double* coords, double* wq, double* N, double* dN, cudaStream_t s) {
  k_shape_functions<<<1, 32, 0, s>>>(family, coords, wq, N, dN);
  return fem_after_launch("k_shape_functions");
}
int fem_launch_element_matrices(int nq, int nen, int dim, const double* wq, const double* N, const double* dN,
                                double* Me, double* Le, double* Leoff, double* Ge, cudaStream_t s) {
  k_element_matrices<<<1, 128, 0, s>>>(nq, nen, dim, wq, N, dN, Me, Le, Leoff, Ge);
  return fem_after_launch("k_element_matrices");
}
int fem_launch_assemble_diag(const FemGrid& g, int ndim, const double* Me, const double* Le, double* M, double* Ldiag,
                             cudaStream_t s) {
  k_assemble_diag<<<fem_nblocks(g.nn, 256), 256, 0, s>>>(g, ndim, Me, Le, M, Ldiag);
  return fem_after_launch("k_assemble_diag");
}
int fem_launch_level_sums(const FemGrid& g, const FemLattice& lat, const double* diag, double* out, cudaStream_t s) {
  k_level_sums<<<1, 512, 0, s>>>(g, lat, diag, out);
  return fem_after_launch("k_level_sums");
}

__global__ void k_invdiag(int n, const double* __restrict__ D, const uint8_t* __restrict__ pin, double* __restrict__ invD,
                          double* __restrict__ winvD) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = 1.0 / D[i];
    invD[i] = v;
    winvD[i] = (pin && pin[i]) ? 0.0 : v;
  }
}

int fem_launch_stencil_build(const FemGrid& g, const double* A, int transpose, int skip_diag, double* out,
                             cudaStream_t s) {
  const int ncls = fem_stencil_ncls(g);
  FEM_KIND_DISPATCH(g.kind, K, (k_stencil_build<K><<<1, 512, 0, s>>>(g, A, transpose, skip_diag, out)));
  (void)ncls;
  return fem_after_launch("k_stencil_build");
}

int fem_launch_invdiag(int n, const double* D, const uint8_t* pin, double* invD, double* winvD, cudaStream_t s) {
  k_invdiag<<<fem_nblocks(n, 256), 256, 0, s>>>(n, D, pin, invD, winvD);
  return fem_after_launch("k_invdiag");
}
