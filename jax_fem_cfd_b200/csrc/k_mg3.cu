// Geometric multigrid for the hex8 pressure Poisson problem and the solves
// built on it: a multigrid-preconditioned CG in FP64 (the reference's CG,
// utils/jax_iterative_solvers.py:87-120, with its stop rule and iteration
// count) and a mixed-precision solve (FP64 iterative refinement around a
// fixed number of FP32 multigrid-PCG iterations).
//
// The reference refuses 3D multigrid (setup/simulation.py:75-76). This is the
// 3D form of its 2D scheme (core/multigrid.py): every axis halved per level,
// the Laplacian re-discretised on each level, lattice-trilinear prolongation
// P and R = P^T, gamma_p rows zeroed (the set_zeroP branch), and, instead of
// one weighted-Jacobi sweep, a degree-3 Chebyshev smoother on D^-1 A (interval
// [0.2, 1.1] x a power-iteration estimate of its largest eigenvalue, the same
// polynomial before and after the coarse correction, so the V-cycle is
// symmetric). The coarsest level is solved exactly in FP64 by its inverse,
// formed on the device at setup (Gauss-Jordan; the matrix is SPD).
//
// The operator is applied in the tensor-product form of the trilinear
// Laplacian on a uniform box, A = Kx(x)My(x)Mz + Mx(x)Ky(x)Mz + Mx(x)My(x)Kz,
// with K and M the assembled 1D stiffness and mass rows (exact for the
// 2x2x2 Gauss-rule Le). A warp owns 30 x-columns of one lattice row and marches
// up a run of z-planes: per plane each lane loads 3 values (rows y-1, y, y+1),
// the x-neighbours come by shuffles, and two plane partials per node
// ((Kx My + Mx Ky) v and (Mx My) v) are combined across three planes with the
// z rows. That is 3 loads and 33 FMAs per node, with every sum in FP64 whatever
// the storage type T of the vectors.
//
// Each solve is one CUDA graph, built once per context and parameter set: a
// prologue, a conditional WHILE node whose body is one PCG iteration (FP64
// solve) or one refinement cycle (mixed solve), and an epilogue. The loop
// condition is computed on the device, so a solve never waits for the host.
// Every loop is bounded by its iteration cap and by a 10 s device-side wall
// budget, checked where the condition is set.
#include <cmath>
#include <cstdio>
#include <cstring>

#include "fem_b200.h"
#include "fem_args.cuh"
#include "fem_mg3.cuh"

#define MG3_THREADS 256
// The sweep kernels are bound by memory latency: at most 64 registers, so 4
// CTAs (32 warps) fit on an SM. Against 77 registers and 3 CTAs, the channel's
// V-cycle went from 0.298 to 0.275 ms.
#define MG3_MIN_BLOCKS 4
#define MG3_OW 30            // owned x-columns per warp
#define MG3_PARTS 4096       // capacity of one partial-sum slot (blocks of a launch)
#define MG3_WATCHDOG_NS 10000000000ull

// ------------------------------------------------------------------ device ----

// Class of lattice coordinate c on an axis of n nodes: 0 first, 2 last, 1 inside.
__device__ __forceinline__ int mg3_cls(int c, int n) { return c <= 0 ? 0 : (c >= n - 1 ? 2 : 1); }

// y(i) = (A v)(i) for every node, epi(i, y(i)) for the nodes a lane owns; src(j)
// returns v(j) as a double. All 32 lanes of a warp run the same trip counts (the
// shuffles need them); only epi is guarded.
template <class Src, class Epi>
__device__ __forceinline__ void mg3_sweep(const Mg3Geo& G, const Src& src, const Epi& epi) {
  const int lane = threadIdx.x & 31;
  const int nx = G.nx, ny = G.ny, nz = G.nz, zs = G.zs, pl = nx * ny;
  const int ntx = (nx + MG3_OW - 1) / MG3_OW, nseg = (nz + zs - 1) / zs;
  const int nitem = ntx * ny * nseg;
  const int wstep = (gridDim.x * blockDim.x) >> 5;
  for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < nitem; it += wstep) {
    const int bx = it % ntx, rest = it / ntx, y = rest % ny, seg = rest / ny;
    const int xg = bx * MG3_OW + lane - 1;
    const int gx = xg < 0 ? 0 : (xg >= nx ? nx - 1 : xg);
    const bool own = lane >= 1 && lane <= MG3_OW && xg < nx;
    const int cx = mg3_cls(xg, nx), cy = mg3_cls(y, ny);
    const double kx0 = G.k[0][cx][0], kx1 = G.k[0][cx][1], kx2 = G.k[0][cx][2];
    const double mx0 = G.m[0][cx][0], mx1 = G.m[0][cx][1], mx2 = G.m[0][cx][2];
    const double ky0 = G.k[1][cy][0], ky1 = G.k[1][cy][1], ky2 = G.k[1][cy][2];
    const double my0 = G.m[1][cy][0], my1 = G.m[1][cy][1], my2 = G.m[1][cy][2];
    const int rm = (y > 0 ? y - 1 : 0) * nx + gx, r0 = y * nx + gx, rp = (y + 1 < ny ? y + 1 : y) * nx + gx;
    // a = ((Kx My + Mx Ky) v)(x, y, p), b = ((Mx My) v)(x, y, p)
    auto plane = [&](int p, double& a, double& b) {
      const int o = p * pl;
      const double v0 = src(o + rm), v1 = src(o + r0), v2 = src(o + rp);
      const double l0 = __shfl_up_sync(0xffffffffu, v0, 1), h0 = __shfl_down_sync(0xffffffffu, v0, 1);
      const double l1 = __shfl_up_sync(0xffffffffu, v1, 1), h1 = __shfl_down_sync(0xffffffffu, v1, 1);
      const double l2 = __shfl_up_sync(0xffffffffu, v2, 1), h2 = __shfl_down_sync(0xffffffffu, v2, 1);
      const double k0 = kx0 * l0 + kx1 * v0 + kx2 * h0, m0 = mx0 * l0 + mx1 * v0 + mx2 * h0;
      const double k1 = kx0 * l1 + kx1 * v1 + kx2 * h1, m1 = mx0 * l1 + mx1 * v1 + mx2 * h1;
      const double k2 = kx0 * l2 + kx1 * v2 + kx2 * h2, m2 = mx0 * l2 + mx1 * v2 + mx2 * h2;
      a = my0 * k0 + ky0 * m0 + my1 * k1 + ky1 * m1 + my2 * k2 + ky2 * m2;
      b = my0 * m0 + my1 * m1 + my2 * m2;
    };
    const int z0 = seg * zs, z1 = min(z0 + zs, nz);
    double a0 = 0.0, b0 = 0.0, a1, b1, a2, b2;
    if (z0 > 0) plane(z0 - 1, a0, b0);
    plane(z0, a1, b1);
    for (int z = z0; z < z1; ++z) {
      if (z + 1 < nz) {
        plane(z + 1, a2, b2);
      } else {
        a2 = 0.0;
        b2 = 0.0;
      }
      const int cz = mg3_cls(z, nz);
      const double v = G.m[2][cz][0] * a0 + G.k[2][cz][0] * b0 + G.m[2][cz][1] * a1 + G.k[2][cz][1] * b1 +
                       G.m[2][cz][2] * a2 + G.k[2][cz][2] * b2;
      if (own) epi(z * pl + y * nx + xg, v);
      a0 = a1;
      b0 = b1;
      a1 = a2;
      b1 = b2;
    }
  }
}

// 2D lattice levels: one thread per node, the level's assembled stencil table
// (fem_stencil_apply, sums in FP64).
template <class Src, class Epi>
__device__ __forceinline__ void mg3_sweep(const Mg2Geo& G, const Src& src, const Epi& epi) {
  const FemGrid& g = G.g;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.nn; i += gridDim.x * blockDim.x) {
    const int ix = i % g.nnx, iy = i / g.nnx;
    const double y = g.kind == FEM_Q1_2D ? fem_stencil_apply<FEM_Q1_2D>(g, G.tab, ix, iy, 0, src)
                                         : fem_stencil_apply<FEM_Q2_2D>(g, G.tab, ix, iy, 0, src);
    epi(i, y);
  }
}

// Block sums of NV doubles (fixed shuffle tree, warps in order); thread 0 writes
// part[k][blockIdx.x], part[k] = parts + k * MG3_PARTS. Every thread must call it.
template <int NV>
__device__ __forceinline__ void mg3_block_parts(double (&v)[NV], double* parts) {
  __shared__ double s[NV][32];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) s[k][threadIdx.x >> 5] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[k][w];
      parts[k * MG3_PARTS + blockIdx.x] = t;
    }
  }
}

// Sum of part[0..np) in a fixed order, the same value in every block that calls
// it (all threads must call it; the result is returned to every thread).
__device__ __forceinline__ double mg3_sum_parts(const double* __restrict__ part, int np) {
  __shared__ double s[32];
  __shared__ double tot;
  double v = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) v += part[k];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    tot = t;
  }
  __syncthreads();
  return tot;
}

template <class T>
__device__ __forceinline__ double ld(const T* p, int i) {
  return (double)p[i];
}

// Chebyshev steps 1 and 2 from x = 0 (pre-smoothing): x1 = b1 D^-1 r is formed
// on the fly at the neighbours, d2 = a2 x1 + b2 D^-1 (r - A x1), x2 = x1 + d2.
template <class T, class G>
__global__ void __launch_bounds__(MG3_THREADS, MG3_MIN_BLOCKS) k_mg3_first(Mg3Lev<T, G> L, double b1, double a2, double b2) {
  mg3_sweep(L.geo, [&](int j) { return b1 * ld(L.invD, j) * ld(L.r, j); }, [&](int i, double ax) {
    const double iD = ld(L.invD, i), x1 = b1 * iD * ld(L.r, i);
    const double d = a2 * x1 + b2 * iD * (ld(L.r, i) - ax);
    L.d[i] = (T)d;
    L.xa[i] = (T)(x1 + d);
  });
}

// One Chebyshev step d = a d + b D^-1 (r - A x_in), x_out = x_in + d (FIRST: a d
// is absent, d is not read). NDOT = 1 adds the block partials of r . x_out;
// NDOT = 3 also those of sum x_out and sum r (mean-zero problems).
template <class T, class G, bool FIRST, int NDOT>
__global__ void __launch_bounds__(MG3_THREADS, MG3_MIN_BLOCKS)
    k_mg3_step(Mg3Lev<T, G> L, const T* __restrict__ xin, T* __restrict__ xout, double a, double b, double* parts) {
  double acc[NDOT > 0 ? NDOT : 1];
#pragma unroll
  for (int k = 0; k < (NDOT > 0 ? NDOT : 1); ++k) acc[k] = 0.0;
  mg3_sweep(L.geo, [&](int j) { return ld(xin, j); }, [&](int i, double ax) {
    const double res = ld(L.r, i) - ax;
    const double d = (FIRST ? 0.0 : a * ld(L.d, i)) + b * ld(L.invD, i) * res;
    const double x = ld(xin, i) + d;
    L.d[i] = (T)d;
    xout[i] = (T)x;
    if (NDOT > 0) acc[0] += ld(L.r, i) * (double)(T)x;
    if (NDOT > 1) {
      acc[1] += (double)(T)x;
      acc[2] += ld(L.r, i);
    }
  });
  if constexpr (NDOT > 0) mg3_block_parts<NDOT>(acc, parts);
}

// t = r - A x, zero on gamma_p (D^-1 = 0 marks a gamma_p node)
template <class T, class G>
__global__ void __launch_bounds__(MG3_THREADS, MG3_MIN_BLOCKS) k_mg3_resid(Mg3Lev<T, G> L, const T* __restrict__ x) {
  mg3_sweep(L.geo, [&](int j) { return ld(x, j); }, [&](int i, double ax) {
    L.t[i] = L.invD[i] == (T)0 ? (T)0 : (T)(ld(L.r, i) - ax);
  });
}

// r_C = R t_F with R = P^T of the trilinear prolongation (weights 1, 1/2 per axis)
template <class T>
__global__ void k_mg3_restrict(Mg3Lev<T, Mg3Geo> F, Mg3Lev<T, Mg3Geo> C) {
  const int NX = C.geo.nx, NY = C.geo.ny, NZ = C.geo.nz, nx = F.geo.nx, ny = F.geo.ny, nz = F.geo.nz;
  const int n = NX * NY * NZ;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < n; I += gridDim.x * blockDim.x) {
    const int X = I % NX, YZ = I / NX, Y = YZ % NY, Z = YZ / NY;
    double acc = 0.0;
    for (int dz = -1; dz <= 1; ++dz) {
      const int z = 2 * Z + dz;
      if (z < 0 || z >= nz) continue;
      const double wz = dz ? 0.5 : 1.0;
      for (int dy = -1; dy <= 1; ++dy) {
        const int y = 2 * Y + dy;
        if (y < 0 || y >= ny) continue;
        const double wy = wz * (dy ? 0.5 : 1.0);
        const T* row = F.t + ((size_t)z * ny + y) * nx;
        for (int dx = -1; dx <= 1; ++dx) {
          const int x = 2 * X + dx;
          if (x < 0 || x >= nx) continue;
          acc += wy * (dx ? 0.5 : 1.0) * (double)row[x];
        }
      }
    }
    C.r[I] = (T)acc;
  }
}

// x_out = x_pre + P x_C, zero on gamma_p
template <class T>
__global__ void k_mg3_prolong(Mg3Lev<T, Mg3Geo> F, Mg3Lev<T, Mg3Geo> C, const T* __restrict__ xpre,
                              const T* __restrict__ xc, T* __restrict__ xout) {
  const int NX = C.geo.nx, NY = C.geo.ny, nx = F.geo.nx, ny = F.geo.ny;
  const int n = F.geo.nx * F.geo.ny * F.geo.nz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (F.invD[i] == (T)0) {
      xout[i] = (T)0;
      continue;
    }
    const int x = i % nx, yz = i / nx, y = yz % ny, z = yz / ny;
    const int X0 = x >> 1, Y0 = y >> 1, Z0 = z >> 1;
    const int X1 = X0 + (x & 1), Y1 = Y0 + (y & 1), Z1 = Z0 + (z & 1);
    const double wx = (x & 1) ? 0.5 : 1.0, wy = (y & 1) ? 0.5 : 1.0, wz = (z & 1) ? 0.5 : 1.0;
    auto c = [&](int X, int Y, int Z) { return (double)xc[((size_t)Z * NY + Y) * NX + X]; };
    double s = 0.0;
    // odd coordinates take both neighbours with weight 1/2, even ones the one node
    s += wx * wy * wz * c(X0, Y0, Z0);
    if (x & 1) s += wx * wy * wz * c(X1, Y0, Z0);
    if (y & 1) s += wx * wy * wz * c(X0, Y1, Z0);
    if ((x & 1) && (y & 1)) s += wx * wy * wz * c(X1, Y1, Z0);
    if (z & 1) {
      s += wx * wy * wz * c(X0, Y0, Z1);
      if (x & 1) s += wx * wy * wz * c(X1, Y0, Z1);
      if (y & 1) s += wx * wy * wz * c(X0, Y1, Z1);
      if ((x & 1) && (y & 1)) s += wx * wy * wz * c(X1, Y1, Z1);
    }
    xout[i] = (T)(ld(xpre, i) + s);
  }
}

// 2D levels: r_C = P^T t_F on the unique-node lattices (weights 1, 1/2 per
// axis; periodic neighbours wrap), the transpose of fem_interp_at
template <class T>
__global__ void k_mg2_restrict(Mg3Lev<T, Mg2Geo> F, Mg3Lev<T, Mg2Geo> C) {
  const FemLattice &h = F.geo.lat, &H = C.geo.lat;
  const int ux = h.ux(), uy = h.uy(), Ux = H.ux(), n = C.geo.g.nn;
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < n; I += gridDim.x * blockDim.x) {
    const int R = I / Ux, Cc = I % Ux;
    double acc = 0.0;
    for (int dr = -1; dr <= 1; ++dr) {
      int r = 2 * R + dr;
      if (h.periodic) {
        r = r < 0 ? r + uy : (r >= uy ? r - uy : r);
      } else if (r < 0 || r >= uy) {
        continue;
      }
      const double wr = dr ? 0.5 : 1.0;
      for (int dc = -1; dc <= 1; ++dc) {
        int c = 2 * Cc + dc;
        if (h.periodic) {
          c = c < 0 ? c + ux : (c >= ux ? c - ux : c);
        } else if (c < 0 || c >= ux) {
          continue;
        }
        acc += wr * (dc ? 0.5 : 1.0) * (double)F.t[r * ux + c];
      }
    }
    C.r[I] = (T)acc;
  }
}
// x_out = x_pre + P x_C (lattice-bilinear, fem_interp_at), zero on gamma_p
template <class T>
__global__ void k_mg2_prolong(Mg3Lev<T, Mg2Geo> F, Mg3Lev<T, Mg2Geo> C, const T* __restrict__ xpre,
                              const T* __restrict__ xc, T* __restrict__ xout, int mean_zero) {
  const int ux = F.geo.lat.ux(), n = F.geo.g.nn;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (!mean_zero && F.invD[i] == (T)0) {
      xout[i] = (T)0;
      continue;
    }
    xout[i] = (T)(ld(xpre, i) + fem_interp_at(C.geo.lat, i / ux, i % ux, [&](int J) { return (double)xc[J]; }));
  }
}

// Coarsest level: x = Ainv r' in FP64 (r' = r with gamma_p zeroed), one warp per row
template <class T, class G>
__global__ void k_mg3_coarse(Mg3Lev<T, G> C, int n, int mean_zero, const double* __restrict__ Ainv,
                             T* __restrict__ xout) {
  __shared__ double rs[MG3_COARSE_MAX];
  for (int j = threadIdx.x; j < n; j += blockDim.x)
    rs[j] = (!mean_zero && C.invD[j] == (T)0) ? 0.0 : (double)C.r[j];
  __syncthreads();
  const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
  for (int i = blockIdx.x * wpb + (threadIdx.x >> 5); i < n; i += gridDim.x * wpb) {
    const double* row = Ainv + (size_t)i * n;
    double s = 0.0;
    for (int j = lane; j < n; j += 32) s += row[j] * rs[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) xout[i] = (!mean_zero && C.invD[i] == (T)0) ? (T)0 : (T)s;
  }
}

// --------------------------------------------------------------- CG pieces ----

// p = z + beta p_old (beta = sc->beta), Ap (zero on gamma_p), block partials of p . Ap
// (mean-zero problems: z is taken minus its mean sc->zbar, the projection of
// the preconditioned residual onto the mean-zero subspace)
template <class T, class G>
__global__ void __launch_bounds__(MG3_THREADS, MG3_MIN_BLOCKS)
    k_mg3_ap(Mg3Lev<T, G> L, const T* __restrict__ z, const T* __restrict__ pold, T* __restrict__ pnew,
             T* __restrict__ Ap, const Mg3Scal* sc, int inner, int mean_zero, double* parts) {
  const double beta = inner ? sc->beta_i : sc->beta;
  const double zb = mean_zero ? sc->zbar : 0.0;
  double acc[1] = {0.0};
  mg3_sweep(L.geo, [&](int j) { return (double)(T)((ld(z, j) - zb) + beta * ld(pold, j)); }, [&](int i, double ax) {
    const T p = (T)((ld(z, i) - zb) + beta * ld(pold, i));
    const T q = (!mean_zero && L.invD[i] == (T)0) ? (T)0 : (T)ax;
    pnew[i] = p;
    Ap[i] = q;
    acc[0] += (double)p * (double)q;
  });
  mg3_block_parts<1>(acc, parts);
}

// alpha = gamma / sum(pAp parts); x += alpha p; r -= alpha Ap; p_old = p; partials of r . r
template <class T>
__global__ void k_mg3_xr(int n, T* __restrict__ x, T* __restrict__ r, const T* __restrict__ pnew,
                         T* __restrict__ pold, const T* __restrict__ Ap, const Mg3Scal* sc, int inner,
                         const double* __restrict__ pap, int np, double* parts) {
  const double pq = mg3_sum_parts(pap, np);
  const double alpha = (inner ? sc->gamma_i : sc->gamma) / pq;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double p = ld(pnew, i);
    x[i] = (T)(ld(x, i) + alpha * p);
    const T rn = (T)(ld(r, i) - alpha * ld(Ap, i));
    r[i] = rn;
    pold[i] = pnew[i];
    acc[0] += (double)rn * (double)rn;
  }
  mg3_block_parts<1>(acc, parts);
}

// FP64 residual r = b - A x (gamma_p rows of A x zeroed) stored as T, with the
// block partials of r . r and b . b
template <class T, class G>
__global__ void __launch_bounds__(MG3_THREADS, MG3_MIN_BLOCKS)
    k_mg3_res64(G geo, const uint8_t* __restrict__ pin, const double* __restrict__ b, const double* __restrict__ x,
                T* __restrict__ r, double* parts) {
  double acc[2] = {0.0, 0.0};
  mg3_sweep(geo, [&](int j) { return x[j]; }, [&](int i, double ax) {
    const double ri = b[i] - ((pin && pin[i]) ? 0.0 : ax);
    r[i] = (T)ri;
    acc[0] += ri * ri;
    acc[1] += b[i] * b[i];
  });
  mg3_block_parts<2>(acc, parts);
}

// x += d; x = 0 on gamma_p when pin is given
template <class T>
__global__ void k_mg3_add(int n, double* __restrict__ x, const T* __restrict__ d, const uint8_t* __restrict__ pin) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = x[i] + (d ? (double)d[i] : 0.0);
    x[i] = (pin && pin[i]) ? 0.0 : v;
  }
}

// partials of sum x (FP64), and x -= mean(x) from them (every block sums them
// in the same order)
__global__ void k_mg3_sum(int n, const double* __restrict__ x, double* parts) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[0] += x[i];
  mg3_block_parts<1>(acc, parts);
}
__global__ void k_mg3_center(int n, double* __restrict__ x, const double* __restrict__ parts, int np) {
  const double m = mg3_sum_parts(parts, np) / n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] -= m;
}

__device__ __forceinline__ unsigned long long mg3_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Loop control, one block. Modes:
//  MG3_CTL_PCG0  prologue of the FP64 PCG: gamma = r.z, rr, bb, atol2, k = 0
//  MG3_CTL_PCG   end of a PCG iteration: k++, gamma, beta, rr; condition
//  MG3_CTL_IN0 / MG3_CTL_IN  the same for the inner FP32 PCG (no condition)
//  MG3_CTL_MX0   prologue of the refinement: rr, bb, cycles = 0; condition
//  MG3_CTL_MX    end of a refinement cycle: cycles++, rr; condition
// The condition (WHILE node) is set in the modes that carry it; it is false
// once the cap, the tolerance, a non-finite value or the wall budget stops
// the loop, and the reason goes to sc->status.
// inv_n > 0 (mean-zero problems): prz + MG3_PARTS and + 2 MG3_PARTS hold the
// partials of sum z and sum r; z is projected to mean zero (zbar = sum z / n)
// and gamma = r . (z - zbar).
__global__ void k_mg3_ctl(Mg3Scal* sc, int mode, const double* __restrict__ prz, int nrz,
                          const double* __restrict__ prr, int nrr, double inv_n, cudaGraphConditionalHandle h) {
  double rz = prz ? mg3_sum_parts(prz, nrz) : 0.0;
  if (prz && inv_n > 0.0) {
    const double sz = mg3_sum_parts(prz + MG3_PARTS, nrz), sr = mg3_sum_parts(prz + 2 * MG3_PARTS, nrz);
    const double zb = sz * inv_n;
    rz -= zb * sr;
    if (threadIdx.x == 0) sc->zbar = zb;
  }
  const double rr = prr ? mg3_sum_parts(prr, nrr) : 0.0;
  const double bb = (mode == MG3_CTL_PCG0 || mode == MG3_CTL_MX0) ? mg3_sum_parts(prr + MG3_PARTS, nrr) : 0.0;
  if (threadIdx.x != 0) return;
  unsigned int cond = 0;
  if (mode == MG3_CTL_PCG0 || mode == MG3_CTL_MX0) {
    sc->t0 = mg3_now();
    sc->status = 0;
    sc->rr = rr;
    sc->bb = bb;
    sc->rr0 = rr;
    const double a2 = sc->tol * sc->tol * bb, b2 = sc->atol * sc->atol;
    sc->atol2 = a2 > b2 ? a2 : b2;
    sc->k = 0;
    sc->cycles = 0;
    if (mode == MG3_CTL_PCG0) {
      sc->gamma = rz;
      sc->beta = 0.0;
    }
    cond = (rr > sc->atol2 && (mode == MG3_CTL_PCG0 ? sc->k < sc->maxiter : sc->cycles < sc->max_cycles)) ? 1u : 0u;
    if (!isfinite(rr) || !isfinite(bb) || (mode == MG3_CTL_PCG0 && !isfinite(rz))) {
      sc->status |= FEM_STATUS_NONFINITE;
      cond = 0;
    }
  } else if (mode == MG3_CTL_PCG) {
    sc->k += 1;
    sc->beta = rz / sc->gamma;
    sc->gamma = rz;
    sc->rr = rr;
    cond = (rr > sc->atol2 && sc->k < sc->maxiter) ? 1u : 0u;
    if (!isfinite(rr) || !isfinite(rz)) {
      sc->status |= FEM_STATUS_NONFINITE;
      cond = 0;
    }
  } else if (mode == MG3_CTL_IN0) {
    sc->gamma_i = rz;
    sc->beta_i = 0.0;
  } else if (mode == MG3_CTL_IN) {
    sc->beta_i = rz / sc->gamma_i;
    sc->gamma_i = rz;
  } else if (mode == MG3_CTL_MX) {
    sc->cycles += 1;
    sc->rr = rr;
    cond = (rr > sc->atol2 && sc->cycles < sc->max_cycles) ? 1u : 0u;
    if (!isfinite(rr)) {
      sc->status |= FEM_STATUS_NONFINITE;
      cond = 0;
    }
  }
  if (mode == MG3_CTL_PCG0 || mode == MG3_CTL_PCG || mode == MG3_CTL_MX0 || mode == MG3_CTL_MX) {
    if (cond && mg3_now() - sc->t0 > MG3_WATCHDOG_NS) {
      sc->status |= FEM_STATUS_WATCHDOG;
      cond = 0;
    }
    cudaGraphSetConditional(h, cond);
  }
}

// Epilogue: iteration count (PCG) or cycles (mixed) and status into sc->out_*
__global__ void k_mg3_finish(Mg3Scal* sc, int mode) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int st = sc->status;
  const bool conv = sc->rr <= sc->atol2;
  if (!conv && !(st & (FEM_STATUS_NONFINITE | FEM_STATUS_WATCHDOG))) st |= FEM_STATUS_MAXITER;
  sc->relres = sc->bb > 0.0 ? sqrt(sc->rr / sc->bb) : 0.0;
  sc->out_iters = mode == MG3_MODE_PCG ? sc->k : sc->cycles;
  sc->out_status = st;
}

// Per-call inputs of a solve (kernel parameters, so the call stays asynchronous)
__global__ void k_mg3_set(Mg3Scal* sc, double tol, double atol, int maxiter, int max_cycles) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sc->tol = tol;
  sc->atol = atol;
  sc->maxiter = maxiter;
  sc->max_cycles = max_cycles;
}

// ------------------------------------------------------------------- setup ----

// 1/D (D = the centre coefficient of the tensor-product row), 0 on gamma_p
__global__ void k_mg3_invdiag(Mg3Geo G, const uint8_t* __restrict__ pin, double* __restrict__ invD64,
                              float* __restrict__ invD32) {
  const int n = G.nx * G.ny * G.nz;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int x = i % G.nx, yz = i / G.nx, y = yz % G.ny, z = yz / G.ny;
    const int cx = mg3_cls(x, G.nx), cy = mg3_cls(y, G.ny), cz = mg3_cls(z, G.nz);
    const double D = G.k[0][cx][1] * G.m[1][cy][1] * G.m[2][cz][1] + G.m[0][cx][1] * G.k[1][cy][1] * G.m[2][cz][1] +
                     G.m[0][cx][1] * G.m[1][cy][1] * G.k[2][cz][1];
    const double v = (pin && pin[i]) ? 0.0 : 1.0 / D;
    invD64[i] = v;
    invD32[i] = (float)v;
  }
}

// start vector of the power iteration: hash(i) / 2^32 - 1/2, 0 on gamma_p
__global__ void k_mg3_pw_init(int n, const double* __restrict__ invD, double* __restrict__ v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = invD[i] == 0.0 ? 0.0 : (double)((unsigned)i * 2654435761u) / 4294967296.0 - 0.5;
}
// w = D^-1 A v, partials of w . w and v . v
template <class G>
__global__ void __launch_bounds__(MG3_THREADS, MG3_MIN_BLOCKS)
    k_mg3_pw(G geo, const double* __restrict__ invD, const double* __restrict__ v, double* __restrict__ w,
             double* parts) {
  double acc[2] = {0.0, 0.0};
  mg3_sweep(geo, [&](int j) { return v[j]; }, [&](int i, double ax) {
    const double wi = invD[i] * ax;
    w[i] = wi;
    acc[0] += wi * wi;
    acc[1] += v[i] * v[i];
  });
  mg3_block_parts<2>(acc, parts);
}
// v = w / ||w||; block 0 keeps (w.w, v.v) in out[0..1]
__global__ void k_mg3_pw_scale(int n, const double* __restrict__ w, double* __restrict__ v,
                               const double* __restrict__ parts, int np, double* out) {
  const double ww = mg3_sum_parts(parts, np);
  const double vv = mg3_sum_parts(parts + MG3_PARTS, np);
  const double s = 1.0 / sqrt(ww);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = w[i] * s;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    out[0] = ww;
    out[1] = vv;
  }
}

// dense coarse matrix: A with gamma_p rows and columns replaced by the identity
__global__ void k_mg3_dense(Mg3Geo G, const uint8_t* __restrict__ pin, double* __restrict__ A) {
  const int n = G.nx * G.ny * G.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / n), j = (int)(t % n);
    const bool pi = pin && pin[i], pj = pin && pin[j];
    double v = 0.0;
    if (pi || pj) {
      v = (i == j) ? 1.0 : 0.0;
    } else {
      const int xi = i % G.nx, yi = (i / G.nx) % G.ny, zi = i / (G.nx * G.ny);
      const int xj = j % G.nx, yj = (j / G.nx) % G.ny, zj = j / (G.nx * G.ny);
      const int dx = xj - xi, dy = yj - yi, dz = zj - zi;
      if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1) {
        const int cx = mg3_cls(xi, G.nx), cy = mg3_cls(yi, G.ny), cz = mg3_cls(zi, G.nz);
        v = G.k[0][cx][dx + 1] * G.m[1][cy][dy + 1] * G.m[2][cz][dz + 1] +
            G.m[0][cx][dx + 1] * G.k[1][cy][dy + 1] * G.m[2][cz][dz + 1] +
            G.m[0][cx][dx + 1] * G.m[1][cy][dy + 1] * G.k[2][cz][dz + 1];
      }
    }
    A[t] = v;
  }
}
// 2D levels: 1/diag(A), 0 on gamma_p (pinned problems)
__global__ void k_mg2_invdiag(int n, const double* __restrict__ diag, const uint8_t* __restrict__ pin,
                              double* __restrict__ invD64, float* __restrict__ invD32) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = (pin && pin[i]) ? 0.0 : 1.0 / diag[i];
    invD64[i] = v;
    invD32[i] = (float)v;
  }
}
// dense coarse matrix of a 2D level from its stencil table: row i gets the
// coefficient of every offset at the neighbour it names (one thread per row,
// so coinciding neighbours of a tiny periodic lattice add up as in the
// stencil apply); the matrix is zeroed before. Then either the gamma_p rows
// and columns become the identity, or (mean-zero) c 1 1^T is added, which makes
// it SPD and leaves A^-1 r mean-zero and exact for every mean-zero r.
template <int KIND>
__global__ void k_mg2_dense_rows(FemGrid g, const double* __restrict__ tab, double* __restrict__ A) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF;
  const int n = g.nn, nc = fem_axis_ncls(KIND, g.periodic);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int ix = i % g.nnx, iy = i / g.nnx;
    const double* c = tab + (size_t)(fem_axis_cls(KIND, g.periodic, iy, g.ney) * nc +
                                     fem_axis_cls(KIND, g.periodic, ix, g.nex)) * NOFF;
    for (int dy = 0; dy < W; ++dy)
      for (int dx = 0; dx < W; ++dx) {
        int v = ix + dx - R, w = iy + dy - R;
        if (g.periodic) {
          v = fem_wrap(v, g.nnx);
          w = fem_wrap(w, g.nny);
        } else {
          v = v < 0 ? 0 : (v >= g.nnx ? g.nnx - 1 : v);
          w = w < 0 ? 0 : (w >= g.nny ? g.nny - 1 : w);
        }
        A[(size_t)i * n + w * g.nnx + v] += c[dy * W + dx];
      }
  }
}
__global__ void k_mg2_dense_fix(int n, const uint8_t* __restrict__ pin, int mean_zero, double shift,
                                double* __restrict__ A) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / n), j = (int)(t % n);
    if (mean_zero)
      A[t] += shift;
    else if ((pin && pin[i]) || (pin && pin[j]))
      A[t] = (i == j) ? 1.0 : 0.0;
  }
}

// Gauss-Jordan step k of the in-place inversion (no pivoting: A is SPD)
__global__ void k_mg3_gj_pivot(int n, int k, const double* __restrict__ A, double* __restrict__ rowk,
                               double* __restrict__ colk) {
  const double p = 1.0 / A[(size_t)k * n + k];
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    rowk[j] = (j == k) ? p : A[(size_t)k * n + j] * p;
    colk[j] = (j == k) ? 0.0 : A[(size_t)j * n + k];
  }
}
__global__ void k_mg3_gj_update(int n, int k, double* __restrict__ A, const double* __restrict__ rowk,
                                const double* __restrict__ colk) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * n;
       t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t / n), j = (int)(t % n);
    if (i == k)
      A[t] = rowk[j];
    else
      A[t] = (j == k ? 0.0 : A[t]) - colk[i] * rowk[j];
  }
}

// -------------------------------------------------------------------- host ----

#define MG3_TRY(...)          \
  do {                        \
    int _r = (__VA_ARGS__);   \
    if (_r) return _r;        \
  } while (0)
#define MG3_CUDA(call)                                              \
  do {                                                              \
    cudaError_t _e = (call);                                        \
    if (_e != cudaSuccess) return fem_cuda_error(#call, _e);        \
  } while (0)
#define MG3_NSLOTS 6

static int mg3_blocks_elem(long long n, int cap) { return fem_nblocks(n, MG3_THREADS, cap); }
static int mg3_items(const Mg3Geo& G) {
  return ((G.nx + MG3_OW - 1) / MG3_OW) * G.ny * ((G.nz + G.zs - 1) / G.zs);
}
static int mg3_blocks_sweep(const Mg3Geo& G, int cap) {
  const int warps = mg3_items(G), b = (warps + (MG3_THREADS / 32) - 1) / (MG3_THREADS / 32);
  return b < 1 ? 1 : (b > cap ? cap : b);
}
static int mg3_blocks_sweep(const Mg2Geo& G, int cap) { return mg3_blocks_elem(G.g.nn, cap); }
static int mg3_nn(const Mg3Geo& G) { return G.nx * G.ny * G.nz; }
static int mg3_nn(const Mg2Geo& G) { return G.g.nn; }

// 1D assembled rows of one axis: K = (1/h)[-1 2 -1], M = (h/6)[1 4 1] inside,
// the one-element halves at the first and last node.
static void mg3_axis(double h, double (&k)[3][3], double (&m)[3][3]) {
  const double ki = 1.0 / h, mi = h / 6.0;
  const double K[3][3] = {{0.0, ki, -ki}, {-ki, 2 * ki, -ki}, {-ki, ki, 0.0}};
  const double M[3][3] = {{0.0, 2 * mi, mi}, {mi, 4 * mi, mi}, {mi, 2 * mi, 0.0}};
  memcpy(k, K, sizeof(K));
  memcpy(m, M, sizeof(M));
}

static Mg3Geo mg3_geo(int nex, int ney, int nez, double lx, double ly, double lz, int cap_warps) {
  Mg3Geo G;
  memset(&G, 0, sizeof(G));
  G.nx = nex + 1;
  G.ny = ney + 1;
  G.nz = nez + 1;
  mg3_axis(lx / nex, G.k[0], G.m[0]);
  mg3_axis(ly / ney, G.k[1], G.m[1]);
  mg3_axis(lz / nez, G.k[2], G.m[2]);
  // planes per work item: the longest run that still gives every SM several warps
  G.zs = 8;
  while (G.zs > 1 && mg3_items(G) < cap_warps) G.zs >>= 1;
  return G;
}

template <class T, class G>
static void mg3_bind(Mg3Lev<T, G>& L, const G& geo, T* base, const T* invD) {
  const size_t n = (size_t)mg3_nn(geo);
  L.geo = geo;
  L.invD = invD;
  L.r = base;
  L.t = base + n;
  L.xa = base + 2 * n;
  L.xb = base + 3 * n;
  L.d = base + 4 * n;
}

void mg3_destroy(Mg3* M) {
  if (!M) return;
  for (auto& gc : M->graphs)
    if (gc.exec) cudaGraphExecDestroy(gc.exec);
  void* ps[] = {M->pin, M->invD64, M->invD32, M->v64, M->v32, M->Ainv, M->parts, M->sc, M->x64, M->b64,
                M->work64, M->work32, M->gj};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (M->s2) cudaStreamDestroy(M->s2);
  delete M;
}

template <class T>
static int dalloc_t(T** p, size_t n) {
  if (cudaMalloc((void**)p, (n ? n : 1) * sizeof(T)) != cudaSuccess) {
    *p = nullptr;
    return fem_cuda_error("cudaMalloc", cudaGetLastError());
  }
  return FEM_OK;
}

// Buffers of a hierarchy whose level sizes (M->nn, M->off, M->total) are set.
static int mg3_alloc(Mg3* M) {
  const size_t tot = M->total, n0 = M->nn[0], nc = M->nn[M->nlev - 1];
  int rc = FEM_OK;
  rc = rc ? rc : dalloc_t(&M->pin, tot);
  rc = rc ? rc : dalloc_t(&M->invD64, tot);
  rc = rc ? rc : dalloc_t(&M->invD32, tot);
  rc = rc ? rc : dalloc_t(&M->work64, 5 * tot);
  rc = rc ? rc : dalloc_t(&M->work32, 5 * tot);
  rc = rc ? rc : dalloc_t(&M->v64, 4 * n0);  // p_old, p_new, Ap, spare (FP64 PCG)
  rc = rc ? rc : dalloc_t(&M->v32, 4 * n0);  // p_old, p_new, Ap, d (FP32 inner)
  rc = rc ? rc : dalloc_t(&M->x64, n0);
  rc = rc ? rc : dalloc_t(&M->b64, n0);
  rc = rc ? rc : dalloc_t(&M->Ainv, nc * nc);
  rc = rc ? rc : dalloc_t(&M->parts, MG3_NSLOTS * (size_t)MG3_PARTS);
  rc = rc ? rc : dalloc_t(&M->sc, 1);
  rc = rc ? rc : dalloc_t(&M->gj, 2 * nc + 2);
  if (rc == FEM_OK && cudaStreamCreateWithFlags(&M->s2, cudaStreamNonBlocking) != cudaSuccess)
    rc = fem_cuda_error("cudaStreamCreateWithFlags", cudaGetLastError());
  return rc;
}

// lambda_max of D^-1 A per smoothed level (power iteration, FP64) and the
// Chebyshev coefficients over [lo, hi] lambda (Saad, Algorithm 12.1)
template <class G>
static int mg3_chebyshev(Mg3* M, const G* geo, cudaStream_t s) {
  double hs[2] = {0.0, 0.0};
  for (int l = 0; l < M->nlev - 1; ++l) {
    const int n = M->nn[l], gb = mg3_blocks_sweep(geo[l], M->cap), ge = mg3_blocks_elem(n, M->cap);
    double *v = M->work64 + 5 * M->off[l], *w = v + n;  // the level's r and t serve as scratch
    k_mg3_pw_init<<<ge, MG3_THREADS, 0, s>>>(n, M->invD64 + M->off[l], v);
    for (int it = 0; it < MG3_POWER_ITERS; ++it) {
      k_mg3_pw<G><<<gb, MG3_THREADS, 0, s>>>(geo[l], M->invD64 + M->off[l], v, w, M->parts);
      k_mg3_pw_scale<<<ge, MG3_THREADS, 0, s>>>(n, w, v, M->parts, gb, M->gj);
    }
    MG3_TRY(fem_after_launch("k_mg3_pw"));
    MG3_CUDA(cudaMemcpyAsync(hs, M->gj, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    MG3_CUDA(cudaStreamSynchronize(s));
    const double lam = std::sqrt(hs[0]) / std::sqrt(hs[1]);
    M->lam[l] = lam;
    const double lo = MG3_CHEB_LO * lam, hi = MG3_CHEB_HI * lam;
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    double rho_old = 1.0 / sigma;
    M->ca[l][0] = 0.0;
    M->cb[l][0] = 1.0 / theta;
    for (int k = 1; k < MG3_DEGREE; ++k) {
      const double rho = 1.0 / (2.0 * sigma - rho_old);
      M->ca[l][k] = rho * rho_old;
      M->cb[l][k] = 2.0 * rho / delta;
      rho_old = rho;
    }
  }
  return FEM_OK;
}

// In-place Gauss-Jordan inversion of the n x n coarse matrix in M->Ainv
static int mg3_invert(Mg3* M, int n, cudaStream_t s) {
  const long long nn2 = (long long)n * n;
  const int gb = (int)std::min<long long>((nn2 + 255) / 256, (long long)M->cap * 4);
  for (int k = 0; k < n; ++k) {
    k_mg3_gj_pivot<<<1, 1024, 0, s>>>(n, k, M->Ainv, M->gj, M->gj + n);
    k_mg3_gj_update<<<gb, 256, 0, s>>>(n, k, M->Ainv, M->gj, M->gj + n);
    if ((k & 255) == 255 || k == n - 1) MG3_TRY(fem_after_launch("k_mg3_gj"));
  }
  MG3_CUDA(cudaStreamSynchronize(s));
  return FEM_OK;
}

int mg3_setup(Mg3** out, int nex, int ney, int nez, double lx, double ly, double lz, int nlev,
              const uint8_t* level_pins, int sms, cudaStream_t s) {
  *out = nullptr;
  if (nlev < 2 || nlev > FEM_MAX_LEVELS) return FEM_E_ARG;
  const int f = 1 << (nlev - 1);
  if (nex % f || ney % f || nez % f) return FEM_E_ARG;
  Mg3* M = new Mg3();
  M->nlev = nlev;
  M->sms = sms;
  M->cap = sms * 8;
  const int cap_warps = sms * 32;
  size_t tot = 0;
  for (int l = 0; l < nlev; ++l) {
    M->geo[l] = mg3_geo(nex >> l, ney >> l, nez >> l, lx, ly, lz, cap_warps);
    const size_t n = (size_t)mg3_nn(M->geo[l]);
    M->off[l] = tot;
    M->nn[l] = (int)n;
    tot += n;
  }
  M->total = tot;
  const int nc = M->nn[nlev - 1];
  if (nc > MG3_COARSE_MAX) {
    snprintf(fem_err_buf(), 256, "hex8 multigrid: coarsest level of %d nodes exceeds %d (add levels)", nc,
             MG3_COARSE_MAX);
    mg3_destroy(M);
    return FEM_E_ARG;
  }
  int rc = mg3_alloc(M);
  for (int l = 0; l < nlev && rc == FEM_OK; ++l) {
    const size_t o = M->off[l];
    if (level_pins) {
      if (cudaMemcpyAsync(M->pin + o, level_pins + o, M->nn[l], cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        rc = fem_cuda_error("cudaMemcpyAsync", cudaGetLastError());
    } else {
      if (cudaMemsetAsync(M->pin + o, 0, M->nn[l], s) != cudaSuccess ||
          cudaMemsetAsync(M->pin + o, 1, 1, s) != cudaSuccess)
        rc = fem_cuda_error("cudaMemsetAsync", cudaGetLastError());
    }
    if (rc) break;
    k_mg3_invdiag<<<mg3_blocks_elem(M->nn[l], M->cap), MG3_THREADS, 0, s>>>(M->geo[l], M->pin + o, M->invD64 + o,
                                                                            M->invD32 + o);
    rc = fem_after_launch("k_mg3_invdiag");
    mg3_bind(M->l64[l], M->geo[l], M->work64 + 5 * o, (const double*)(M->invD64 + o));
    mg3_bind(M->l32[l], M->geo[l], M->work32 + 5 * o, (const float*)(M->invD32 + o));
  }
  if (rc == FEM_OK) rc = mg3_chebyshev(M, M->geo, s);
  // coarsest level: its dense inverse, in place
  if (rc == FEM_OK) {
    const long long nn2 = (long long)nc * nc;
    const int gb = (int)std::min<long long>((nn2 + 255) / 256, (long long)M->cap * 4);
    k_mg3_dense<<<gb, 256, 0, s>>>(M->geo[nlev - 1], M->pin + M->off[nlev - 1], M->Ainv);
    rc = fem_after_launch("k_mg3_dense");
  }
  if (rc == FEM_OK) rc = mg3_invert(M, nc, s);
  if (rc) {
    mg3_destroy(M);
    return rc;
  }
  *out = M;
  return FEM_OK;
}

int mg2_setup(Mg3** out, int nlev, const FemGrid* grids, const double* const* tabs, const double* const* diags,
              const uint8_t* const* pins, int mean_zero, int sms, cudaStream_t s) {
  *out = nullptr;
  if (nlev < 2 || nlev > FEM_MAX_LEVELS) return FEM_E_ARG;
  Mg3* M = new Mg3();
  M->nlev = nlev;
  M->sms = sms;
  M->cap = sms * 8;
  M->d2 = 1;
  M->mz = mean_zero ? 1 : 0;
  size_t tot = 0;
  for (int l = 0; l < nlev; ++l) {
    const FemGrid& g = grids[l];
    Mg2Geo& G = M->geo2[l];
    G.g = g;
    const int sc = (g.kind == FEM_Q2_2D) ? 2 : 1;
    G.lat = FemLattice{sc * g.nex + 1, sc * g.ney + 1, g.periodic};
    G.tab = tabs[l];
    M->off[l] = tot;
    M->nn[l] = g.nn;
    tot += g.nn;
  }
  M->total = tot;
  const int nc = M->nn[nlev - 1];
  if (nc > MG3_COARSE_MAX) {
    snprintf(fem_err_buf(), 256, "mixed multigrid: coarsest level of %d nodes exceeds %d", nc, MG3_COARSE_MAX);
    mg3_destroy(M);
    return FEM_E_ARG;
  }
  int rc = mg3_alloc(M);
  for (int l = 0; l < nlev && rc == FEM_OK; ++l) {
    const size_t o = M->off[l];
    const uint8_t* pin = mean_zero ? nullptr : pins[l];
    if (pin) {
      if (cudaMemcpyAsync(M->pin + o, pin, M->nn[l], cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        rc = fem_cuda_error("cudaMemcpyAsync", cudaGetLastError());
    } else if (cudaMemsetAsync(M->pin + o, 0, M->nn[l], s) != cudaSuccess) {
      rc = fem_cuda_error("cudaMemsetAsync", cudaGetLastError());
    }
    if (rc) break;
    k_mg2_invdiag<<<mg3_blocks_elem(M->nn[l], M->cap), MG3_THREADS, 0, s>>>(M->nn[l], diags[l],
                                                                            mean_zero ? nullptr : M->pin + o,
                                                                            M->invD64 + o, M->invD32 + o);
    rc = fem_after_launch("k_mg2_invdiag");
    mg3_bind(M->m64[l], M->geo2[l], M->work64 + 5 * o, (const double*)(M->invD64 + o));
    mg3_bind(M->m32[l], M->geo2[l], M->work32 + 5 * o, (const float*)(M->invD32 + o));
  }
  if (rc == FEM_OK) rc = mg3_chebyshev(M, M->geo2, s);
  if (rc == FEM_OK) {
    const Mg2Geo& C = M->geo2[nlev - 1];
    const long long nn2 = (long long)nc * nc;
    const int gb = (int)std::min<long long>((nn2 + 255) / 256, (long long)M->cap * 4);
    if (cudaMemsetAsync(M->Ainv, 0, sizeof(double) * nn2, s) != cudaSuccess)
      rc = fem_cuda_error("cudaMemsetAsync", cudaGetLastError());
    if (rc == FEM_OK) {
      if (C.g.kind == FEM_Q1_2D)
        k_mg2_dense_rows<FEM_Q1_2D><<<mg3_blocks_elem(nc, M->cap), MG3_THREADS, 0, s>>>(C.g, C.tab, M->Ainv);
      else
        k_mg2_dense_rows<FEM_Q2_2D><<<mg3_blocks_elem(nc, M->cap), MG3_THREADS, 0, s>>>(C.g, C.tab, M->Ainv);
      rc = fem_after_launch("k_mg2_dense_rows");
    }
    if (rc == FEM_OK) {
      // the shift of the mean-zero coarse matrix: about its mean diagonal entry / n
      double d[2] = {0.0, 0.0};
      if (cudaMemcpyAsync(d, M->Ainv, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
          cudaStreamSynchronize(s) != cudaSuccess)
        rc = fem_cuda_error("coarse diagonal", cudaGetLastError());
      if (rc == FEM_OK) {
        k_mg2_dense_fix<<<gb, 256, 0, s>>>(nc, M->mz ? nullptr : M->pin + M->off[nlev - 1], M->mz, d[0] / nc,
                                           M->Ainv);
        rc = fem_after_launch("k_mg2_dense_fix");
      }
    }
  }
  if (rc == FEM_OK) rc = mg3_invert(M, nc, s);
  if (rc) {
    mg3_destroy(M);
    return rc;
  }
  *out = M;
  return FEM_OK;
}

// transfers per level geometry
template <class T>
static void mg3_restrict(const Mg3* M, const Mg3Lev<T, Mg3Geo>& F, const Mg3Lev<T, Mg3Geo>& C, int nC,
                         cudaStream_t s) {
  k_mg3_restrict<T><<<mg3_blocks_elem(nC, M->cap), MG3_THREADS, 0, s>>>(F, C);
}
template <class T>
static void mg3_restrict(const Mg3* M, const Mg3Lev<T, Mg2Geo>& F, const Mg3Lev<T, Mg2Geo>& C, int nC,
                         cudaStream_t s) {
  k_mg2_restrict<T><<<mg3_blocks_elem(nC, M->cap), MG3_THREADS, 0, s>>>(F, C);
}
template <class T>
static void mg3_prolong(const Mg3* M, const Mg3Lev<T, Mg3Geo>& F, const Mg3Lev<T, Mg3Geo>& C, int nF,
                        cudaStream_t s) {
  k_mg3_prolong<T><<<mg3_blocks_elem(nF, M->cap), MG3_THREADS, 0, s>>>(F, C, F.xb, C.xb, F.xa);
}
template <class T>
static void mg3_prolong(const Mg3* M, const Mg3Lev<T, Mg2Geo>& F, const Mg3Lev<T, Mg2Geo>& C, int nF,
                        cudaStream_t s) {
  k_mg2_prolong<T><<<mg3_blocks_elem(nF, M->cap), MG3_THREADS, 0, s>>>(F, C, F.xb, C.xb, F.xa, M->mz);
}

// V-cycle on the level vectors of precision T: input lv[0].r, output lv[0].xb.
// dot: block partials of r . z (and, mean-zero, sum z and sum r) into
// dot_parts, written by the last smoothing step.
template <class T, class G>
static int mg3_vcycle(const Mg3* M, Mg3Lev<T, G>* lv, double* dot_parts, cudaStream_t s) {
  const int N = M->nlev, cap = M->cap;
  for (int l = 0; l < N - 1; ++l) {
    const Mg3Lev<T, G>& L = lv[l];
    const int gb = mg3_blocks_sweep(L.geo, cap);
    k_mg3_first<T, G><<<gb, MG3_THREADS, 0, s>>>(L, M->cb[l][0], M->ca[l][1], M->cb[l][1]);
    const T* x = L.xa;
    T* y = L.xb;
    for (int k = 2; k < MG3_DEGREE; ++k) {  // pre-smoothing steps 3.. (ping-pong ending in xb)
      k_mg3_step<T, G, false, 0><<<gb, MG3_THREADS, 0, s>>>(L, x, y, M->ca[l][k], M->cb[l][k], nullptr);
      const T* tmp = y;
      y = const_cast<T*>(x);
      x = tmp;
    }
    // x holds the pre-smoothed iterate; keep it in xb
    if (x != L.xb) MG3_CUDA(cudaMemcpyAsync(L.xb, x, sizeof(T) * M->nn[l], cudaMemcpyDeviceToDevice, s));
    k_mg3_resid<T, G><<<gb, MG3_THREADS, 0, s>>>(L, L.xb);
    mg3_restrict(M, L, lv[l + 1], M->nn[l + 1], s);
    MG3_TRY(fem_after_launch("k_mg3_down"));
  }
  const Mg3Lev<T, G>& C = lv[N - 1];
  const int nc = M->nn[N - 1];
  k_mg3_coarse<T, G><<<(nc + 7) / 8, 256, 0, s>>>(C, nc, M->mz, M->Ainv, C.xb);
  MG3_TRY(fem_after_launch("k_mg3_coarse"));
  for (int l = N - 2; l >= 0; --l) {
    const Mg3Lev<T, G>& L = lv[l];
    const int gb = mg3_blocks_sweep(L.geo, cap);
    mg3_prolong(M, L, lv[l + 1], M->nn[l], s);
    // post-smoothing: steps xa -> xb -> xa -> xb (degree 3 ends in xb)
    T* bufs[2] = {L.xa, L.xb};
    for (int k = 0; k < MG3_DEGREE; ++k) {
      const bool last = (k == MG3_DEGREE - 1);
      double* dp = (l == 0 && last) ? dot_parts : nullptr;
      const T* xi = bufs[k & 1];
      T* xo = bufs[(k + 1) & 1];
      if (k == 0)
        k_mg3_step<T, G, true, 0><<<gb, MG3_THREADS, 0, s>>>(L, xi, xo, 0.0, M->cb[l][0], nullptr);
      else if (dp && M->mz)
        k_mg3_step<T, G, false, 3><<<gb, MG3_THREADS, 0, s>>>(L, xi, xo, M->ca[l][k], M->cb[l][k], dp);
      else if (dp)
        k_mg3_step<T, G, false, 1><<<gb, MG3_THREADS, 0, s>>>(L, xi, xo, M->ca[l][k], M->cb[l][k], dp);
      else
        k_mg3_step<T, G, false, 0><<<gb, MG3_THREADS, 0, s>>>(L, xi, xo, M->ca[l][k], M->cb[l][k], nullptr);
    }
    MG3_TRY(fem_after_launch("k_mg3_up"));
  }
  return FEM_OK;
}

int mg3_vcycle64(Mg3* M, const double* r, double* z, cudaStream_t s) {
  if (M->d2) return FEM_E_STATE;
  Mg3Lev<double>& L0 = M->l64[0];
  MG3_CUDA(cudaMemcpyAsync(L0.r, r, sizeof(double) * M->nn[0], cudaMemcpyDeviceToDevice, s));
  MG3_TRY(mg3_vcycle<double>(M, M->l64, nullptr, s));
  MG3_CUDA(cudaMemcpyAsync(z, L0.xb, sizeof(double) * M->nn[0], cudaMemcpyDeviceToDevice, s));
  return FEM_OK;
}

// ------------------------------------------------------------- graph build ----

// Captures prologue, WHILE(body) and epilogue on M's streams into one graph.
template <class Pro, class Body, class Epi>
static int mg3_capture(Mg3* M, cudaStream_t cs, Pro pro, Body body, Epi epi, cudaGraphExec_t* exec) {
  *exec = nullptr;
  MG3_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int rc = FEM_OK;
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cudaGraphConditionalHandle h = 0;
  if (cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &ndeps) != cudaSuccess ||
      cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess)
    rc = fem_cuda_error("conditional handle", cudaGetLastError());
  if (rc == FEM_OK) rc = pro(cs, h);
  cudaGraphNode_t cnode = nullptr;
  if (rc == FEM_OK) {
    if (cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &ndeps) != cudaSuccess) {
      rc = fem_cuda_error("cudaStreamGetCaptureInfo", cudaGetLastError());
    } else {
      cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      if (cudaGraphAddNode(&cnode, g, deps, ndeps, &cp) != cudaSuccess) {
        rc = fem_cuda_error("cudaGraphAddNode(conditional)", cudaGetLastError());
      } else {
        cudaGraph_t bg = cp.conditional.phGraph_out[0];
        if (cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) {
          rc = fem_cuda_error("cudaStreamUpdateCaptureDependencies", cudaGetLastError());
        } else if (cudaStreamBeginCaptureToGraph(M->s2, bg, nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
          rc = fem_cuda_error("cudaStreamBeginCaptureToGraph", cudaGetLastError());
        } else {
          rc = body(M->s2, h);
          cudaGraph_t bout = nullptr;
          const cudaError_t e = cudaStreamEndCapture(M->s2, &bout);
          if (rc == FEM_OK && e != cudaSuccess) rc = fem_cuda_error("cudaStreamEndCapture(body)", e);
        }
      }
    }
  }
  if (rc == FEM_OK) rc = epi(cs);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(cs, &graph);
  if (rc == FEM_OK && e != cudaSuccess) rc = fem_cuda_error("cudaStreamEndCapture", e);
  if (rc == FEM_OK && cudaGraphInstantiate(exec, graph, 0) != cudaSuccess) {
    rc = fem_cuda_error("cudaGraphInstantiate", cudaGetLastError());
    *exec = nullptr;
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
  return rc;
}

// One PCG iteration's vectors on level 0, of type T.
template <class T>
struct Mg3Cg {
  T *x, *r, *z, *pold, *pnew, *Ap;
};

template <class T, class G>
static int mg3_cg_iter(const Mg3* M, Mg3Lev<T, G>* lv, const Mg3Cg<T>& V, int inner, bool vcycle, int ctl_mode,
                       cudaGraphConditionalHandle h, cudaStream_t s) {
  const Mg3Lev<T, G>& L0 = lv[0];
  const int n = M->nn[0], gb = mg3_blocks_sweep(L0.geo, M->cap), ge = mg3_blocks_elem(n, M->cap);
  double *pA = M->parts, *pB = M->parts + MG3_PARTS, *pC = M->parts + 3 * MG3_PARTS;
  k_mg3_ap<T, G><<<gb, MG3_THREADS, 0, s>>>(L0, V.z, V.pold, V.pnew, V.Ap, M->sc, inner, M->mz, pA);
  k_mg3_xr<T><<<ge, MG3_THREADS, 0, s>>>(n, V.x, V.r, V.pnew, V.pold, V.Ap, M->sc, inner, pA, gb, pB);
  MG3_TRY(fem_after_launch("k_mg3_cg"));
  if (vcycle) {
    MG3_TRY(mg3_vcycle<T, G>(M, lv, pC, s));
    k_mg3_ctl<<<1, 256, 0, s>>>(M->sc, ctl_mode, pC, gb, pB, ge, M->mz ? 1.0 / n : 0.0, h);
    MG3_TRY(fem_after_launch("k_mg3_ctl"));
  }
  return FEM_OK;
}

static bool mg3_key_eq(const Mg3GraphKey& a, const Mg3GraphKey& b) { return memcmp(&a, &b, sizeof(a)) == 0; }

static Mg3GraphCache* mg3_cache_slot(Mg3* M, const Mg3GraphKey& key) {
  for (auto& g : M->graphs)
    if (g.exec && mg3_key_eq(g.key, key)) return &g;
  for (auto& g : M->graphs)
    if (!g.exec) {
      g.key = key;
      return &g;
    }
  // evict the first
  cudaGraphExecDestroy(M->graphs[0].exec);
  M->graphs[0].exec = nullptr;
  M->graphs[0].key = key;
  return &M->graphs[0];
}

// FP64 MG-PCG (utils/jax_iterative_solvers.py:87-120 with M = the V-cycle):
// b, x (x0 in, solution out) device FP64; iters/status device ints. hex8.
int mg3_pcg(Mg3* M, const double* b, double* x, double tol, double atol, int maxiter, int* iters, int* status,
            cudaStream_t s, cudaStream_t cs) {
  if (M->d2) return FEM_E_STATE;
  Mg3GraphKey key;
  memset(&key, 0, sizeof(key));
  key.mode = MG3_MODE_PCG;
  Mg3GraphCache* gc = mg3_cache_slot(M, key);
  const int n = M->nn[0];
  Mg3Lev<double>* lv = M->l64;
  if (!gc->exec) {
    const Mg3Cg<double> V{M->x64, lv[0].r, lv[0].xb, M->v64, M->v64 + n, M->v64 + 2 * n};
    const int gb = mg3_blocks_sweep(lv[0].geo, M->cap);
    double *pB = M->parts + MG3_PARTS, *pC = M->parts + 3 * MG3_PARTS;
    auto pro = [&](cudaStream_t cs_, cudaGraphConditionalHandle h) -> int {
      MG3_CUDA(cudaMemsetAsync(V.pold, 0, sizeof(double) * n, cs_));
      k_mg3_res64<double, Mg3Geo><<<gb, MG3_THREADS, 0, cs_>>>(lv[0].geo, M->pin, M->b64, M->x64, lv[0].r, pB);
      MG3_TRY(fem_after_launch("k_mg3_res64"));
      MG3_TRY(mg3_vcycle<double>(M, lv, pC, cs_));
      k_mg3_ctl<<<1, 256, 0, cs_>>>(M->sc, MG3_CTL_PCG0, pC, gb, pB, gb, 0.0, h);
      return fem_after_launch("k_mg3_ctl");
    };
    auto body = [&](cudaStream_t bs, cudaGraphConditionalHandle h) -> int {
      return mg3_cg_iter<double>(M, lv, V, 0, true, MG3_CTL_PCG, h, bs);
    };
    auto epi = [&](cudaStream_t cs_) -> int {
      k_mg3_add<double><<<mg3_blocks_elem(n, M->cap), MG3_THREADS, 0, cs_>>>(n, M->x64, (const double*)nullptr,
                                                                             M->pin);
      k_mg3_finish<<<1, 32, 0, cs_>>>(M->sc, MG3_MODE_PCG);
      return fem_after_launch("k_mg3_finish");
    };
    MG3_TRY(mg3_capture(M, cs, pro, body, epi, &gc->exec));
  }
  // per-call values: tolerances and the cap live in the device scalars
  k_mg3_set<<<1, 32, 0, s>>>(M->sc, tol, atol, maxiter, 0);
  MG3_TRY(fem_after_launch("k_mg3_set"));
  MG3_CUDA(cudaMemcpyAsync(M->b64, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  MG3_CUDA(cudaMemcpyAsync(M->x64, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  MG3_CUDA(cudaGraphLaunch(gc->exec, s));
  MG3_CUDA(cudaMemcpyAsync(x, M->x64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  MG3_CUDA(cudaMemcpyAsync(iters, &M->sc->out_iters, sizeof(int), cudaMemcpyDeviceToDevice, s));
  MG3_CUDA(cudaMemcpyAsync(status, &M->sc->out_status, sizeof(int), cudaMemcpyDeviceToDevice, s));
  return FEM_OK;
}

// The mixed-precision refinement graph for level vectors of geometry G.
template <class G>
static int mg3_mixed_graph(Mg3* M, Mg3Lev<float, G>* lv, int inner, cudaStream_t cs, cudaGraphExec_t* exec) {
  const int n = M->nn[0];
  float* d32 = M->v32 + 3 * n;
  const Mg3Cg<float> V{d32, lv[0].r, lv[0].xb, M->v32, M->v32 + n, M->v32 + 2 * n};
  const int gb = mg3_blocks_sweep(lv[0].geo, M->cap), ge = mg3_blocks_elem(n, M->cap);
  double *pA = M->parts, *pB = M->parts + MG3_PARTS, *pC = M->parts + 3 * MG3_PARTS;
  const uint8_t* pin0 = M->mz ? nullptr : M->pin;
  const double inv_n = M->mz ? 1.0 / n : 0.0;
  auto pro = [&](cudaStream_t cs_, cudaGraphConditionalHandle h) -> int {
    if (M->mz) {  // centre b (mean-zero problems solve on the mean-zero subspace)
      k_mg3_sum<<<ge, MG3_THREADS, 0, cs_>>>(n, M->b64, pA);
      k_mg3_center<<<ge, MG3_THREADS, 0, cs_>>>(n, M->b64, pA, ge);
    }
    k_mg3_res64<float, G><<<gb, MG3_THREADS, 0, cs_>>>(lv[0].geo, pin0, M->b64, M->x64, lv[0].r, pB);
    k_mg3_ctl<<<1, 256, 0, cs_>>>(M->sc, MG3_CTL_MX0, nullptr, 0, pB, gb, 0.0, h);
    return fem_after_launch("k_mg3_ctl");
  };
  auto body = [&](cudaStream_t bs, cudaGraphConditionalHandle h) -> int {
    MG3_CUDA(cudaMemsetAsync(d32, 0, sizeof(float) * n, bs));
    MG3_CUDA(cudaMemsetAsync(V.pold, 0, sizeof(float) * n, bs));
    MG3_TRY(mg3_vcycle<float, G>(M, lv, pC, bs));
    k_mg3_ctl<<<1, 256, 0, bs>>>(M->sc, MG3_CTL_IN0, pC, gb, nullptr, 0, inv_n, h);
    for (int k = 0; k < inner; ++k) MG3_TRY(mg3_cg_iter<float, G>(M, lv, V, 1, k + 1 < inner, MG3_CTL_IN, h, bs));
    k_mg3_add<float><<<ge, MG3_THREADS, 0, bs>>>(n, M->x64, d32, nullptr);
    k_mg3_res64<float, G><<<gb, MG3_THREADS, 0, bs>>>(lv[0].geo, pin0, M->b64, M->x64, lv[0].r, pB);
    k_mg3_ctl<<<1, 256, 0, bs>>>(M->sc, MG3_CTL_MX, nullptr, 0, pB, gb, 0.0, h);
    return fem_after_launch("k_mg3_mixed");
  };
  auto epi = [&](cudaStream_t cs_) -> int {
    if (M->mz) {
      k_mg3_sum<<<ge, MG3_THREADS, 0, cs_>>>(n, M->x64, pA);
      k_mg3_center<<<ge, MG3_THREADS, 0, cs_>>>(n, M->x64, pA, ge);
    } else {
      k_mg3_add<float><<<ge, MG3_THREADS, 0, cs_>>>(n, M->x64, (const float*)nullptr, M->pin);
    }
    k_mg3_finish<<<1, 32, 0, cs_>>>(M->sc, MG3_MODE_MIXED);
    return fem_after_launch("k_mg3_finish");
  };
  return mg3_capture(M, cs, pro, body, epi, exec);
}

// Mixed precision: FP64 refinement x += d until ||b - A x|| <= tol ||b|| or
// max_cycles, d from `inner` FP32 MG-PCG iterations on A d = r from d = 0.
int mg3_mixed(Mg3* M, const double* b, double* x, double tol, int inner, int max_cycles, int* cycles, int* status,
              cudaStream_t s, cudaStream_t cs) {
  Mg3GraphKey key;
  memset(&key, 0, sizeof(key));
  key.mode = MG3_MODE_MIXED;
  key.inner = inner;
  Mg3GraphCache* gc = mg3_cache_slot(M, key);
  const int n = M->nn[0];
  if (!gc->exec) {
    if (M->d2)
      MG3_TRY(mg3_mixed_graph<Mg2Geo>(M, M->m32, inner, cs, &gc->exec));
    else
      MG3_TRY(mg3_mixed_graph<Mg3Geo>(M, M->l32, inner, cs, &gc->exec));
  }
  k_mg3_set<<<1, 32, 0, s>>>(M->sc, tol, 0.0, 0, max_cycles);
  MG3_TRY(fem_after_launch("k_mg3_set"));
  MG3_CUDA(cudaMemcpyAsync(M->b64, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  MG3_CUDA(cudaMemcpyAsync(M->x64, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  MG3_CUDA(cudaGraphLaunch(gc->exec, s));
  MG3_CUDA(cudaMemcpyAsync(x, M->x64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  if (cycles) MG3_CUDA(cudaMemcpyAsync(cycles, &M->sc->out_iters, sizeof(int), cudaMemcpyDeviceToDevice, s));
  if (status) MG3_CUDA(cudaMemcpyAsync(status, &M->sc->out_status, sizeof(int), cudaMemcpyDeviceToDevice, s));
  return FEM_OK;
}

// Final relative residual of the last solve (host; waits for s).
int mg3_last_relres(Mg3* M, double* relres, cudaStream_t s) {
  Mg3Scal h;
  MG3_CUDA(cudaMemcpyAsync(&h, M->sc, sizeof(h), cudaMemcpyDeviceToHost, s));
  MG3_CUDA(cudaStreamSynchronize(s));
  if (relres) *relres = h.relres;
  return FEM_OK;
}
