// Mixed-precision pressure-Poisson solve (Q1 2D, pinned gamma_p rows): FP64
// iterative refinement around an FP32 multigrid-preconditioned CG.
//
// Outer (FP64): r = b - A x with A's gamma_p rows zeroed (the operator of
// solvers/standard.py:85-125), its norm, x += d. Inner (FP32 vectors; the
// stencil sums are accumulated in FP64, because A p of a smooth p is about h^2
// |p| and an FP32 sum of the 9 terms loses most of its digits on fine
// lattices): a fixed number of PCG iterations on A d = r
// from d = 0, preconditioned by the V-cycle of core/multigrid.py:231-330 in its
// pinned form (one weighted Jacobi pre- and post-sweep, R = I^T, lattice
// bilinear P, gamma_p zeroed); the coarsest level is solved in FP64 by CG to
// the hierarchy's coarse tolerance. Dot products accumulate in FP64 through
// per-block partials summed in a fixed order (deterministic). The CG scalars
// live in device memory, so the inner loop never waits for the host.
//
// Every phase is its own streaming kernel over the lattice (one thread per
// node, neighbours through L1), which keeps the FP32 vectors' halved bytes.
#include "fem_b200.h"
#include "fem_args.cuh"

struct MxLevel {
  FemGrid g;
  FemLattice lat;
  const double* tab;      // assembled stencil of L_e
  const double* tab_off;  // the same with a zero diagonal
  const double* invD;     // 1 / diag(L)
  const double* winvD;    // 1 / diag(L), 0 on gamma_p
  const uint8_t* pin;     // gamma_p mask (or null)
  float *r, *x, *t, *u;    // residual, pre-smoothed x, scratch, prolongated iterate
  float *iD, *wiD;        // FP32 copies of invD and winvD
};

#define MX_THREADS 256

__device__ __forceinline__ int mx_clamp(const FemGrid& g, int v, int n) {
  return g.periodic ? fem_wrap(v, n) : (v < 0 ? 0 : (v >= n ? n - 1 : v));
}
// sum_off coef(i)[off] * src(node i + off) on a Q1 lattice, accumulated in FP64
template <class Src>
__device__ __forceinline__ double mx_sten(const FemGrid& g, const double* __restrict__ tab, int i, const Src& src) {
  const int ix = i % g.nnx, iy = i / g.nnx, nc = fem_axis_ncls(FEM_Q1_2D, g.periodic);
  const double* c = tab + (fem_axis_cls(FEM_Q1_2D, g.periodic, iy, g.ney) * nc +
                           fem_axis_cls(FEM_Q1_2D, g.periodic, ix, g.nex)) * 9;
  double y = 0.0;
#pragma unroll
  for (int dy = 0; dy < 3; ++dy) {
    const int row = mx_clamp(g, iy + dy - 1, g.nny) * g.nnx;
#pragma unroll
    for (int dx = 0; dx < 3; ++dx) y += c[dy * 3 + dx] * (double)src(row + mx_clamp(g, ix + dx - 1, g.nnx));
  }
  return y;
}
__device__ __forceinline__ bool mx_pin(const MxLevel& L, int i) { return L.pin && L.pin[i]; }


// Q1 stencil sums in warp strips (the scheme of k_stencil_strip): a warp owns
// 30 node columns and MX_M rows; each lane loads its column's MX_M + 2 source
// values src(j) (all loads in flight before use), the horizontal neighbours
// come by shuffles, the sum runs over dy then dx in FP64, and epi(i, acc) is
// called for each owned node i (lanes 1..30). Strips clear of the first and
// last lattice rows (every strip of a periodic lattice) keep their column's 9
// coefficients in registers; the others read them per row.
#define MX_M 8
template <class Src, class Epi>
__device__ __forceinline__ void mx_strips(const FemGrid& g, const double* __restrict__ tab, const Src& src,
                                          const Epi& epi) {
  constexpr int OW = 30, NR = MX_M + 2;
  const int lane = threadIdx.x & 31, nc = fem_axis_ncls(FEM_Q1_2D, g.periodic);
  const int ntx = (g.nnx + OW - 1) / OW, nty = (g.nny + MX_M - 1) / MX_M, nitem = ntx * nty;
  const int wstep = (gridDim.x * blockDim.x) >> 5;
  for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < nitem; it += wstep) {
    const int by = it / ntx, bx = it - by * ntx;
    const int xg = bx * OW + lane - 1, y0 = by * MX_M;
    const int gx = mx_clamp(g, xg, g.nnx);
    double v[NR];
    if (y0 >= 1 && y0 + MX_M + 1 <= g.nny) {
#pragma unroll
      for (int r = 0; r < NR; ++r) v[r] = src((y0 - 1 + r) * g.nnx + gx);
    } else {
#pragma unroll
      for (int r = 0; r < NR; ++r) v[r] = src(mx_clamp(g, y0 - 1 + r, g.nny) * g.nnx + gx);
    }
    const bool own = lane >= 1 && lane <= OW && xg < g.nnx;
    const int cx = own ? fem_axis_cls(FEM_Q1_2D, g.periodic, xg, g.nex) : 0;
    double acc[MX_M];
#pragma unroll
    for (int m = 0; m < MX_M; ++m) acc[m] = 0.0;
    if (g.periodic || (y0 >= 1 && y0 + MX_M <= g.ney)) {
      const double* c = tab + ((g.periodic ? 0 : 1) * nc + cx) * 9;
      double cf[9];
#pragma unroll
      for (int o = 0; o < 9; ++o) cf[o] = c[o];
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const double sl = __shfl_up_sync(0xffffffffu, v[r], 1), sr = __shfl_down_sync(0xffffffffu, v[r], 1);
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
          const int m = r - dy;
          if (m >= 0 && m < MX_M) {
            acc[m] += cf[dy * 3] * sl;
            acc[m] += cf[dy * 3 + 1] * v[r];
            acc[m] += cf[dy * 3 + 2] * sr;
          }
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const double sl = __shfl_up_sync(0xffffffffu, v[r], 1), sr = __shfl_down_sync(0xffffffffu, v[r], 1);
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
          const int m = r - dy;
          if (m >= 0 && m < MX_M) {
            const int yy = y0 + m < g.nny ? y0 + m : g.nny - 1;
            const double* c = tab + (fem_axis_cls(FEM_Q1_2D, g.periodic, yy, g.ney) * nc + cx) * 9 + dy * 3;
            acc[m] += c[0] * sl;
            acc[m] += c[1] * v[r];
            acc[m] += c[2] * sr;
          }
        }
      }
    }
    if (own) {
#pragma unroll
      for (int m = 0; m < MX_M; ++m)
        if (y0 + m < g.nny) epi((y0 + m) * g.nnx + xg, acc[m]);
    }
  }
}

// The same sums one node per thread (neighbours through L1): the better form on
// lattices below MX_STRIP_NN nodes, where a strip leaves most lanes idle.
#define MX_STRIP_NN (1 << 23)
template <bool STRIP, class Src, class Epi>
__device__ __forceinline__ void mx_apply(const FemGrid& g, const double* __restrict__ tab, const Src& src,
                                         const Epi& epi) {
  if constexpr (STRIP) {
    mx_strips(g, tab, src, epi);
  } else {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.nn; i += gridDim.x * blockDim.x)
      epi(i, mx_sten(g, tab, i, src));
  }
}

// block sum of a double into part[blockIdx.x] (fixed shuffle tree, warps in order)
__device__ __forceinline__ void mx_block_part(double v, double* part) {
  __shared__ double s[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    part[blockIdx.x] = t;
  }
}

// down-sweep at level L: x = (2/3) rh / D (rh = r, 0 on gamma_p), t = rh - L x
// (L x = 0 on gamma_p); x at the neighbours is formed on the fly from r
template <bool STRIP>
__global__ void k_mx_down(MxLevel L) {
  const double w = 2.0 / 3.0;
  mx_apply<STRIP>(L.g, L.tab, [&](int j) { return w * (double)L.r[j] * (double)L.wiD[j]; }, [&](int i, double lx) {
    const bool p = mx_pin(L, i);
    const double rh = p ? 0.0 : (double)L.r[i];
    L.x[i] = (float)(w * rh * (double)L.wiD[i]);
    L.t[i] = (float)(rh - (p ? 0.0 : lx));
  });
}
// r_C = R t_L
__global__ void k_mx_restrict(MxLevel L, MxLevel C) {
  const int cux = C.lat.ux();
  for (int I = blockIdx.x * blockDim.x + threadIdx.x; I < C.g.nn; I += gridDim.x * blockDim.x)
    C.r[I] = (float)fem_restrict_at(L.lat, I / cux, I % cux, [&](int j) { return (double)L.t[j]; });
}
// up-sweep at level L, prolongation: u = x_L + P xc (0 on gamma_p)
__global__ void k_mx_prolong(MxLevel L, MxLevel C, const float* __restrict__ xc) {
  const int ux = L.lat.ux();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < L.g.nn; i += gridDim.x * blockDim.x)
    L.u[i] = mx_pin(L, i) ? 0.0f
                          : (float)((double)L.x[i] +
                                    fem_interp_at(C.lat, i / ux, i % ux, [&](int J) { return (double)xc[J]; }));
}
// up-sweep at level L, post-smoothing: out = (2/3)(r - Loff u) / D + (1/3) u (0 on gamma_p)
template <bool STRIP>
__global__ void k_mx_jacobi(MxLevel L, float* __restrict__ out) {
  const double w = 2.0 / 3.0;
  mx_apply<STRIP>(L.g, L.tab_off, [&](int j) { return (double)L.u[j]; }, [&](int i, double off) {
    out[i] = mx_pin(L, i) ? 0.0f
                          : (float)(w * ((double)L.r[i] - off) * (double)L.iD[i] + (1.0 - w) * (double)L.u[i]);
  });
}
__global__ void k_mx_cvt(int n, const double* __restrict__ a, float* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (float)a[i];
}
// coarsest level: FP64 CG on L x = r with gamma_p rows zeroed (core/multigrid.py:278-287), one warp,
// at most 128 nodes (4 per lane in registers, p through smem)
__global__ void k_mx_coarse(MxLevel L, double tol, int maxit) {
  constexpr int S = 4;
  __shared__ double sp[32 * S];
  const int lane = threadIdx.x, nn = L.g.nn;
  double x[S], r[S], p[S];
  double bs = 0.0;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int i = lane + 32 * s;
    const double b = (i < nn && !mx_pin(L, i)) ? (double)L.r[i] : 0.0;
    r[s] = b;
    p[s] = b;
    x[s] = 0.0;
    bs += b * b;
  }
  bs = fem_warp_sum(bs);
  const double atol2 = tol * tol * bs;
  double gamma = bs;
  for (int k = 0; gamma > atol2 && k < maxit; ++k) {
#pragma unroll
    for (int s = 0; s < S; ++s)
      if (lane + 32 * s < nn) sp[lane + 32 * s] = p[s];
    __syncwarp();
    double q[S], pq = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int i = lane + 32 * s;
      q[s] = 0.0;
      if (i < nn && !mx_pin(L, i)) {
        const int ix = i % L.g.nnx, iy = i / L.g.nnx, nc = fem_axis_ncls(FEM_Q1_2D, L.g.periodic);
        const double* c = L.tab + (fem_axis_cls(FEM_Q1_2D, L.g.periodic, iy, L.g.ney) * nc +
                                   fem_axis_cls(FEM_Q1_2D, L.g.periodic, ix, L.g.nex)) * 9;
        for (int dy = 0; dy < 3; ++dy)
          for (int dx = 0; dx < 3; ++dx)
            q[s] += c[dy * 3 + dx] * sp[mx_clamp(L.g, iy + dy - 1, L.g.nny) * L.g.nnx +
                                        mx_clamp(L.g, ix + dx - 1, L.g.nnx)];
      }
      pq += p[s] * q[s];
    }
    pq = fem_warp_sum(pq);
    __syncwarp();
    const double alpha = gamma / pq;
    double rr = 0.0;
#pragma unroll
    for (int s = 0; s < S; ++s) {
      x[s] += alpha * p[s];
      r[s] -= alpha * q[s];
      rr += r[s] * r[s];
    }
    rr = fem_warp_sum(rr);
    const double beta = rr / gamma;
#pragma unroll
    for (int s = 0; s < S; ++s) p[s] = r[s] + beta * p[s];
    gamma = rr;
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int i = lane + 32 * s;
    if (i < nn) L.x[i] = mx_pin(L, i) ? 0.0f : (float)x[s];
  }
}

// CG pieces (level 0). sc[0] = r.z, sc[1] = previous r.z, sc[2] = p.Ap
__global__ void k_mx_p(int n, const float* __restrict__ z, float* __restrict__ p, const double* sc, int first) {
  const float beta = first ? 0.0f : (float)(sc[0] / sc[1]);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = first ? z[i] : z[i] + beta * p[i];  // p is not read before the first iteration
}
template <bool STRIP>
__global__ void k_mx_ap(MxLevel L, const float* __restrict__ p, float* __restrict__ Ap, double* part) {
  double a = 0.0;
  mx_apply<STRIP>(L.g, L.tab, [&](int j) { return (double)p[j]; }, [&](int i, double s) {
    const float q = mx_pin(L, i) ? 0.0f : (float)s;
    Ap[i] = q;
    a += (double)p[i] * (double)q;
  });
  mx_block_part(a, part);
}
__global__ void k_mx_xr(int n, float* __restrict__ x, float* __restrict__ r, const float* __restrict__ p,
                        const float* __restrict__ Ap, const double* sc) {
  const float alpha = (float)(sc[0] / sc[2]);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    x[i] += alpha * p[i];
    r[i] -= alpha * Ap[i];
  }
}
__global__ void k_mx_dot(int n, const float* __restrict__ a, const float* __restrict__ b, double* part) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += (double)a[i] * (double)b[i];
  mx_block_part(s, part);
}
// sc[slot] = sum of part[0..np) in a fixed order; shift: sc[1] = sc[0] first
__global__ void k_mx_final(const double* __restrict__ part, int np, double* sc, int slot, int shift) {
  double s = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) s += part[k];
  __shared__ double w[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += w[k];
    if (shift) sc[1] = sc[0];
    sc[slot] = t;
  }
}
// FP64 residual r = b - A x (gamma_p rows of A x zeroed) into FP32, its squared norm parts
template <bool STRIP>
__global__ void k_mx_res64(MxLevel L, const double* __restrict__ b, const double* __restrict__ x,
                           float* __restrict__ r32, double* part) {
  double a = 0.0;
  mx_apply<STRIP>(L.g, L.tab, [&](int j) { return x[j]; }, [&](int i, double ax) {
    const double ri = b[i] - (mx_pin(L, i) ? 0.0 : ax);
    r32[i] = (float)ri;
    a += ri * ri;
  });
  mx_block_part(a, part);
}
__global__ void k_mx_dot64(int n, const double* __restrict__ a, double* part) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * a[i];
  mx_block_part(s, part);
}
// x += d (d FP32); with pin: x = 0 on gamma_p (the final modification of solvers/standard.py:119-123)
__global__ void k_mx_add(int n, double* __restrict__ x, const float* __restrict__ d, const uint8_t* pin) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = x[i] + (d ? (double)d[i] : 0.0);
    x[i] = (pin && pin[i]) ? 0.0 : v;
  }
}

// ------------------------------------------------------------------ host ----

struct MxPlan {
  MxLevel lv[FEM_MAX_LEVELS];
  int nlev, grid;
  float *p, *Ap, *d;
  double *part, *sc;
  double coarse_tol;
};

static int mx_grid(long long n, int grid) {
  long long b = (n + MX_THREADS - 1) / MX_THREADS;
  return (int)(b < 1 ? 1 : (b > grid ? grid : b));
}

static void mx_res64(const MxLevel& L0, int gb, const double* b, const double* x, double* part, cudaStream_t s) {
  if (L0.g.nn >= MX_STRIP_NN)
    k_mx_res64<true><<<gb, MX_THREADS, 0, s>>>(L0, b, x, L0.r, part);
  else
    k_mx_res64<false><<<gb, MX_THREADS, 0, s>>>(L0, b, x, L0.r, part);
}

static int mx_vcycle(const MxPlan& P, cudaStream_t s) {
  const int N = P.nlev;
  for (int l = 0; l < N - 1; ++l) {
    if (P.lv[l].g.nn >= MX_STRIP_NN)
      k_mx_down<true><<<mx_grid(P.lv[l].g.nn, P.grid), MX_THREADS, 0, s>>>(P.lv[l]);
    else
      k_mx_down<false><<<mx_grid(P.lv[l].g.nn, P.grid), MX_THREADS, 0, s>>>(P.lv[l]);
    if (int rc = fem_after_launch("k_mx_down")) return rc;
    k_mx_restrict<<<mx_grid(P.lv[l + 1].g.nn, P.grid), MX_THREADS, 0, s>>>(P.lv[l], P.lv[l + 1]);
    if (int rc = fem_after_launch("k_mx_restrict")) return rc;
  }
  k_mx_coarse<<<1, 32, 0, s>>>(P.lv[N - 1], P.coarse_tol, 1000);
  if (int rc = fem_after_launch("k_mx_coarse")) return rc;
  for (int l = N - 2; l >= 0; --l) {
    const float* xc = (l == N - 2) ? P.lv[N - 1].x : P.lv[l + 1].t;
    const int gl = mx_grid(P.lv[l].g.nn, P.grid);
    k_mx_prolong<<<gl, MX_THREADS, 0, s>>>(P.lv[l], P.lv[l + 1], xc);
    if (P.lv[l].g.nn >= MX_STRIP_NN)
      k_mx_jacobi<true><<<gl, MX_THREADS, 0, s>>>(P.lv[l], P.lv[l].t);
    else
      k_mx_jacobi<false><<<gl, MX_THREADS, 0, s>>>(P.lv[l], P.lv[l].t);
    if (int rc = fem_after_launch("k_mx_up")) return rc;
  }
  return 0;  // z in lv[0].t
}

// One outer cycle's inner solve: `inner` PCG iterations on A d = r32 from d = 0.
static int mx_inner(const MxPlan& P, int inner, cudaStream_t s) {
  const MxLevel& L0 = P.lv[0];
  const int n = L0.g.nn, gb = mx_grid(n, P.grid);
  if (cudaMemsetAsync(P.d, 0, sizeof(float) * n, s) != cudaSuccess) return fem_after_launch("cudaMemsetAsync");
  if (int rc = mx_vcycle(P, s)) return rc;
  k_mx_dot<<<gb, MX_THREADS, 0, s>>>(n, L0.r, L0.t, P.part);
  k_mx_final<<<1, 256, 0, s>>>(P.part, gb, P.sc, 0, 0);
  for (int k = 0; k < inner; ++k) {
    k_mx_p<<<gb, MX_THREADS, 0, s>>>(n, L0.t, P.p, P.sc, k == 0);
    if (n >= MX_STRIP_NN)
      k_mx_ap<true><<<gb, MX_THREADS, 0, s>>>(L0, P.p, P.Ap, P.part);
    else
      k_mx_ap<false><<<gb, MX_THREADS, 0, s>>>(L0, P.p, P.Ap, P.part);
    k_mx_final<<<1, 256, 0, s>>>(P.part, gb, P.sc, 2, 0);
    k_mx_xr<<<gb, MX_THREADS, 0, s>>>(n, P.d, L0.r, P.p, P.Ap, P.sc);
    if (k + 1 < inner) {
      if (int rc = mx_vcycle(P, s)) return rc;
      k_mx_dot<<<gb, MX_THREADS, 0, s>>>(n, L0.r, L0.t, P.part);
      k_mx_final<<<1, 256, 0, s>>>(P.part, gb, P.sc, 0, 1);
    }
    if (int rc = fem_after_launch("k_mx_inner")) return rc;
  }
  return 0;
}

int fem_mixed_poisson(const CgArgs& A, int grid, float* work, double* dwork, const double* b, double* x, double tol,
                      int inner, int max_cycles, int* cycles, double* relres, cudaStream_t s, MxGraphCache* gc,
                      cudaStream_t cap) {
  MxPlan P;
  P.nlev = A.nlev;
  P.grid = grid;
  P.coarse_tol = A.coarse_tol;
  float* f = work;
  for (int l = 0; l < A.nlev; ++l) {
    const MgLevel& M = A.lv[l];
    MxLevel& L = P.lv[l];
    L.g = M.g;
    L.lat = M.lat;
    L.tab = M.tab;
    L.tab_off = M.tab_off;
    L.invD = M.invD;
    L.winvD = M.winvD;
    L.pin = M.pin;
    L.r = f;
    L.x = f + M.g.nn;
    L.t = f + 2 * M.g.nn;
    L.u = f + 3 * M.g.nn;
    L.iD = f + 4 * M.g.nn;
    L.wiD = f + 5 * M.g.nn;
    f += 6 * (size_t)M.g.nn;
    const int gl = mx_grid(M.g.nn, grid);
    k_mx_cvt<<<gl, MX_THREADS, 0, s>>>(M.g.nn, M.invD, L.iD);
    k_mx_cvt<<<gl, MX_THREADS, 0, s>>>(M.g.nn, M.winvD, L.wiD);
  }
  const int n = A.lv[0].g.nn, gb = mx_grid(n, grid);
  P.p = f;
  P.Ap = f + n;
  P.d = f + 2 * n;
  P.part = dwork;
  P.sc = dwork + grid;  // sc[0..3], norms at sc[4], sc[5]
  const MxLevel& L0 = P.lv[0];
  k_mx_dot64<<<gb, MX_THREADS, 0, s>>>(n, b, P.part);
  k_mx_final<<<1, 256, 0, s>>>(P.part, gb, P.sc, 5, 0);
  mx_res64(L0, gb, b, x, P.part, s);
  k_mx_final<<<1, 256, 0, s>>>(P.part, gb, P.sc, 4, 0);
  if (int rc = fem_after_launch("k_mx_res64")) return rc;
  double nrm[2];
  if (cudaMemcpyAsync(nrm, P.sc + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return fem_after_launch("norms");
  const double bb = nrm[1];
  double rr = nrm[0];
  // the inner solve only touches the context's buffers: captured once into a
  // CUDA graph (per inner count) and replayed every cycle
  if (gc && cap && (!gc->exec || gc->inner != inner)) {
    if (gc->exec) cudaGraphExecDestroy(gc->exec);
    gc->exec = nullptr;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      const int rc = mx_inner(P, inner, cap);
      const cudaError_t e = cudaStreamEndCapture(cap, &graph);
      if (rc == 0 && e == cudaSuccess && cudaGraphInstantiate(&gc->exec, graph, 0) == cudaSuccess) gc->inner = inner;
      else gc->exec = nullptr;
      if (graph) cudaGraphDestroy(graph);
    }
    cudaGetLastError();  // a failed capture falls back to direct launches
  }
  int k = 0;
  while (rr > tol * tol * bb && k < max_cycles) {
    if (gc && gc->exec) {
      if (cudaGraphLaunch(gc->exec, s) != cudaSuccess) return fem_after_launch("cudaGraphLaunch");
    } else if (int rc = mx_inner(P, inner, s)) {
      return rc;
    }
    k_mx_add<<<gb, MX_THREADS, 0, s>>>(n, x, P.d, nullptr);
    mx_res64(L0, gb, b, x, P.part, s);
    k_mx_final<<<1, 256, 0, s>>>(P.part, gb, P.sc, 4, 0);
    if (int rc = fem_after_launch("k_mx_res64")) return rc;
    if (cudaMemcpyAsync(nrm, P.sc + 4, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return fem_after_launch("norms");
    rr = nrm[0];
    ++k;
  }
  k_mx_add<<<gb, MX_THREADS, 0, s>>>(n, x, nullptr, L0.pin);
  if (int rc = fem_after_launch("k_mx_add")) return rc;
  if (cycles) *cycles = k;
  if (relres) *relres = bb > 0.0 ? sqrt(rr / bb) : 0.0;
  return 0;
}
