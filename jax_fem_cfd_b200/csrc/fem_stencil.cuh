// Element-kind specialised lattice machinery.
//
// 1. fem_incident_k<KIND>: the node-centric incidence loop with the element
//    kind known at compile time (unrolled candidates, compile-time local-node
//    offsets) for operators with per-element matrices (Ce, SUPG terms).
//
// 2. Assembled stencils: for a SHARED element matrix A on the uniform lattice,
//    the node-centric sum y_n = sum_{(e,a) ~ n} sum_b A[a][b] x[node(e,b)] only
//    depends on which incident elements exist, i.e. on the node's class along
//    each axis (boundary position and, for quad9, parity). A table holds, per
//    class, the coefficient of every lattice offset (3^d or 5^2 offsets), built
//    on the device from A with the same incidence rules; applying it is an
//    unrolled constant-offset stencil. Values equal the element-by-element sum
//    up to summation order.
#pragma once
#include "fem_common.cuh"

template <int KIND>
struct KI;
template <>
struct KI<FEM_Q1_2D> {
  static constexpr int R = 1, W = 3, NOFF = 9, S = 1, NEN = 4, DIM = 2;
};
template <>
struct KI<FEM_Q2_2D> {
  static constexpr int R = 2, W = 5, NOFF = 25, S = 2, NEN = 9, DIM = 2;
};
template <>
struct KI<FEM_HEX8> {
  static constexpr int R = 1, W = 3, NOFF = 27, S = 1, NEN = 8, DIM = 3;
};

template <int KIND>
__device__ __forceinline__ constexpr int kdi(int b) {
  return KIND == FEM_Q2_2D ? (int)((FEM_Q2_DI >> (2 * b)) & 3u) : (int)((FEM_Q1_DI >> (2 * (b & 3))) & 3u);
}
template <int KIND>
__device__ __forceinline__ constexpr int kdj(int b) {
  return KIND == FEM_Q2_2D ? (int)((FEM_Q2_DJ >> (2 * b)) & 3u) : (int)((FEM_Q1_DJ >> (2 * (b & 3))) & 3u);
}
template <int KIND>
__device__ __forceinline__ constexpr int kdk(int b) {
  return KIND == FEM_HEX8 ? (b >> 2) : 0;
}

// Candidates along one axis: (e0, d0) valid if v0, (e1, d1) valid if v1.
template <int KIND>
__device__ __forceinline__ void fem_axis_pair(int periodic, int c, int nel, int& e0, int& d0, bool& v0, int& e1,
                                              int& d1, bool& v1) {
  if (KIND == FEM_Q2_2D && (c & 1)) {
    e0 = (c - 1) >> 1;
    d0 = 1;
    v0 = true;
    e1 = 0;
    d1 = 0;
    v1 = false;
    return;
  }
  const int h = (KIND == FEM_Q2_2D) ? (c >> 1) : c;
  v0 = (h >= 1) || periodic;
  e0 = (h >= 1) ? h - 1 : nel - 1;
  d0 = (KIND == FEM_Q2_2D) ? 2 : 1;
  v1 = h < nel;
  e1 = h;
  d1 = 0;
}

// f(ie, je, ke, e, a) for every element incident to lattice node (i, j, k).
template <int KIND, class F>
__device__ __forceinline__ void fem_incident_k(const FemGrid& g, int i, int j, int k, F&& f) {
  int ei0, di0, ei1, di1, ej0, dj0, ej1, dj1, ek0 = 0, dk0 = 0, ek1 = 0, dk1 = 0;
  bool vi0, vi1, vj0, vj1, vk0 = true, vk1 = false;
  fem_axis_pair<KIND>(g.periodic, i, g.nex, ei0, di0, vi0, ei1, di1, vi1);
  fem_axis_pair<KIND>(g.periodic, j, g.ney, ej0, dj0, vj0, ej1, dj1, vj1);
  if (KIND == FEM_HEX8) fem_axis_pair<FEM_HEX8>(0, k, g.nez, ek0, dk0, vk0, ek1, dk1, vk1);
#pragma unroll
  for (int zk = 0; zk < (KIND == FEM_HEX8 ? 2 : 1); ++zk) {
    if (!(zk ? vk1 : vk0)) continue;
    const int ek = zk ? ek1 : ek0, dk = zk ? dk1 : dk0;
#pragma unroll
    for (int zj = 0; zj < 2; ++zj) {
      if (!(zj ? vj1 : vj0)) continue;
      const int ej = zj ? ej1 : ej0, dj = zj ? dj1 : dj0;
#pragma unroll
      for (int zi = 0; zi < 2; ++zi) {
        if (!(zi ? vi1 : vi0)) continue;
        const int ei = zi ? ei1 : ei0, di = zi ? di1 : di0;
        const int e = (ek * g.ney + ej) * g.nex + ei;
        f(ei, ej, ek, e, fem_local_index(KIND, di, dj, dk));
      }
    }
  }
}

// Node index of local node B (compile-time) of element (ie, je, ke).
template <int KIND, int B>
__device__ __forceinline__ int fem_enode(const FemGrid& g, int ie, int je, int ke) {
  constexpr int S = KI<KIND>::S;
  int c = S * ie + kdi<KIND>(B), r = S * je + kdj<KIND>(B);
  if (g.periodic) {
    if (c >= g.nnx) c -= g.nnx;
    if (r >= g.nny) r -= g.nny;
  }
  return ((ke + kdk<KIND>(B)) * g.nny + r) * g.nnx + c;
}

template <int KIND, int B = 0>
struct ElemNodes {
  template <class F>
  __device__ __forceinline__ static void run(const FemGrid& g, int ie, int je, int ke, F&& f) {
    if constexpr (B < KI<KIND>::NEN) {
      f(B, fem_enode<KIND, B>(g, ie, je, ke));
      ElemNodes<KIND, B + 1>::run(g, ie, je, ke, f);
    }
  }
};

// Gather with a per-element coefficient functor m(e, a, b) and NC sources src(j, c).
template <int KIND, int NC, class Mat, class Src>
__device__ __forceinline__ void fem_gather_k(const FemGrid& g, int i, int j, int k, const Mat& m, const Src& src,
                                             double (&y)[NC]) {
#pragma unroll
  for (int c = 0; c < NC; ++c) y[c] = 0.0;
  fem_incident_k<KIND>(g, i, j, k, [&](int ie, int je, int ke, int e, int a) {
    double part[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) part[c] = 0.0;
    ElemNodes<KIND>::run(g, ie, je, ke, [&](int b, int jn) {
      const double coef = m(e, a, b, KI<KIND>::NEN);
#pragma unroll
      for (int c = 0; c < NC; ++c) part[c] += coef * src(jn, c);
    });
#pragma unroll
    for (int c = 0; c < NC; ++c) y[c] += part[c];
  });
}

// ---------------------------------------------------------------- stencils --

__host__ __device__ __forceinline__ int fem_axis_ncls(int kind, int periodic) {
  if (kind == FEM_Q2_2D) return periodic ? 2 : 4;
  return periodic ? 1 : 3;
}
__device__ __forceinline__ int fem_axis_cls(int kind, int periodic, int c, int nel) {
  if (kind == FEM_Q2_2D) {
    if (periodic) return c & 1;
    if (c & 1) return 3;
    return c == 0 ? 0 : (c == 2 * nel ? 2 : 1);
  }
  if (periodic) return 0;
  return c == 0 ? 0 : (c == nel ? 2 : 1);
}
// representative lattice coordinate of a class, -1 if the lattice has none
__device__ __forceinline__ int fem_axis_rep(int kind, int periodic, int cls, int nel) {
  if (kind == FEM_Q2_2D) {
    if (periodic) return cls;
    if (cls == 0) return 0;
    if (cls == 1) return nel >= 2 ? 2 : -1;
    if (cls == 2) return 2 * nel;
    return 1;
  }
  if (periodic) return 0;
  if (cls == 0) return 0;
  if (cls == 1) return nel >= 2 ? 1 : -1;
  return nel;
}

// largest stencil table (doubles): 3D hex8, 27 classes x 27 offsets, with room to spare
#define FEM_TAB_MAX (64 * 27)
__host__ __device__ __forceinline__ int fem_stencil_ncls(const FemGrid& g) {
  const int n = fem_axis_ncls(g.kind, g.periodic);
  return g.kind == FEM_HEX8 ? n * n * n : n * n;
}
__host__ __device__ __forceinline__ int fem_stencil_noff(int kind) {
  return kind == FEM_Q2_2D ? 25 : (kind == FEM_HEX8 ? 27 : 9);
}

// offset of lattice coordinate v relative to c, periodic-aware, in [-R, R]
__device__ __forceinline__ int fem_rel(int v, int c, int n, int periodic) {
  int d = v - c;
  if (periodic) {
    d %= n;
    if (d < 0) d += n;
    if (2 * d > n) d -= n;
  }
  return d;
}

// Entry t = cls * NOFF + off of the table of the assembled form of shared
// matrix A (nen x nen): the sum, over the incident elements of the class's
// representative node (incidence order) and then b ascending, of the A[a][b]
// whose node b lies at offset off. transpose: use A^T; skip_diag: omit b == a.
template <int KIND>
__device__ __forceinline__ double fem_stencil_entry(const FemGrid& g, const double* __restrict__ A, int transpose,
                                                    int skip_diag, int t) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF, NEN = KI<KIND>::NEN, S = KI<KIND>::S;
  const int nc = fem_axis_ncls(KIND, g.periodic);
  const int cls = t / NOFF, want = t - cls * NOFF;
  const int cx = cls % nc, cy = (cls / nc) % nc, cz = cls / (nc * nc);
  const int i = fem_axis_rep(KIND, g.periodic, cx, g.nex), j = fem_axis_rep(KIND, g.periodic, cy, g.ney);
  const int k = (KIND == FEM_HEX8) ? fem_axis_rep(KIND, 0, cz, g.nez) : 0;
  double acc = 0.0;
  if (i >= 0 && j >= 0 && k >= 0) {
    fem_incident_k<KIND>(g, i, j, k, [&](int ie, int je, int ke, int e, int a) {
      for (int b = 0; b < NEN; ++b) {
        if (skip_diag && b == a) continue;
        const int bi = S * ie + kdi<KIND>(b), bj = S * je + kdj<KIND>(b), bk = ke + kdk<KIND>(b);
        const int dx = fem_rel(bi, i, g.nnx, g.periodic) + R, dy = fem_rel(bj, j, g.nny, g.periodic) + R;
        const int dz = (KIND == FEM_HEX8) ? (bk - k + R) : 0;
        if ((dz * W + dy) * W + dx == want) acc += transpose ? A[b * NEN + a] : A[a * NEN + b];
      }
    });
  }
  return acc;
}
// The whole table by the threads of one CTA (out: global or shared memory).
template <int KIND>
__device__ __forceinline__ void fem_stencil_table_block(const FemGrid& g, const double* __restrict__ A, int transpose,
                                                        int skip_diag, double* out) {
  const int n = fem_stencil_ncls(g) * KI<KIND>::NOFF;
  for (int t = threadIdx.x; t < n; t += blockDim.x) out[t] = fem_stencil_entry<KIND>(g, A, transpose, skip_diag, t);
}
template <int KIND>
__global__ void k_stencil_build(FemGrid g, const double* __restrict__ A, int transpose, int skip_diag,
                                double* __restrict__ out) {
  fem_stencil_table_block<KIND>(g, A, transpose, skip_diag, out);
}

// y = sum_off coef[cls(i,j,k)][off] * src(node(i,j,k) + off)
template <int KIND, class Src>
__device__ __forceinline__ double fem_stencil_apply(const FemGrid& g, const double* __restrict__ tab, int i, int j,
                                                    int k, const Src& src) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF;
  const int nc = fem_axis_ncls(KIND, g.periodic);
  const int cx = fem_axis_cls(KIND, g.periodic, i, g.nex), cy = fem_axis_cls(KIND, g.periodic, j, g.ney);
  const int cz = (KIND == FEM_HEX8) ? fem_axis_cls(KIND, 0, k, g.nez) : 0;
  const double* __restrict__ c = tab + (size_t)((cz * nc + cy) * nc + cx) * NOFF;
  int col[W], row[W], pl[KIND == FEM_HEX8 ? W : 1];
#pragma unroll
  for (int d = 0; d < W; ++d) {
    int v = i + d - R, w = j + d - R;
    if (g.periodic) {
      v = v < 0 ? v + g.nnx : (v >= g.nnx ? v - g.nnx : v);
      w = w < 0 ? w + g.nny : (w >= g.nny ? w - g.nny : w);
    } else {
      v = v < 0 ? 0 : (v >= g.nnx ? g.nnx - 1 : v);
      w = w < 0 ? 0 : (w >= g.nny ? g.nny - 1 : w);
    }
    col[d] = v;
    row[d] = w * g.nnx;
  }
  if (KIND == FEM_HEX8) {
#pragma unroll
    for (int d = 0; d < W; ++d) {
      int z = k + d - R;
      z = z < 0 ? 0 : (z >= g.nnz ? g.nnz - 1 : z);
      pl[d] = z * g.nnx * g.nny;
    }
  } else {
    pl[0] = 0;
  }
  double y = 0.0;
#pragma unroll
  for (int dz = 0; dz < (KIND == FEM_HEX8 ? W : 1); ++dz)
#pragma unroll
    for (int dy = 0; dy < W; ++dy)
#pragma unroll
      for (int dx = 0; dx < W; ++dx) {
        const int o = (dz * W + dy) * W + dx;
        y += __ldg(c + o) * src(pl[dz] + row[dy] + col[dx]);
      }
  return y;
}

// Gradient: y_d = sum Ge_d rows * P (ND outputs from one input).
template <int KIND, int ND, class Src>
__device__ __forceinline__ void fem_gather_grad_k(const FemGrid& g, int i, int j, int k, const double* Ge,
                                                  const Src& P, double (&y)[ND]) {
  constexpr int NEN = KI<KIND>::NEN, NEN2 = NEN * NEN;
#pragma unroll
  for (int d = 0; d < ND; ++d) y[d] = 0.0;
  fem_incident_k<KIND>(g, i, j, k, [&](int ie, int je, int ke, int e, int a) {
    double part[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) part[d] = 0.0;
    ElemNodes<KIND>::run(g, ie, je, ke, [&](int b, int jn) {
      const double pj = P(jn);
#pragma unroll
      for (int d = 0; d < ND; ++d) part[d] += Ge[d * NEN2 + a * NEN + b] * pj;
    });
#pragma unroll
    for (int d = 0; d < ND; ++d) y[d] += part[d];
  });
}

// Divergence: sum_d sum Ge_d^T rows * U_d (per-component sums added at the end,
// as the reference adds the assembled component vectors).
template <int KIND, int ND>
__device__ __forceinline__ double fem_gather_div_k(const FemGrid& g, int i, int j, int k, const double* Ge,
                                                   const double* __restrict__ U) {
  constexpr int NEN = KI<KIND>::NEN, NEN2 = NEN * NEN;
  double acc[ND];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d] = 0.0;
  const size_t nn = g.nn;
  fem_incident_k<KIND>(g, i, j, k, [&](int ie, int je, int ke, int e, int a) {
    double part[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) part[d] = 0.0;
    ElemNodes<KIND>::run(g, ie, je, ke, [&](int b, int jn) {
#pragma unroll
      for (int d = 0; d < ND; ++d) part[d] += Ge[d * NEN2 + b * NEN + a] * U[jn + d * nn];
    });
#pragma unroll
    for (int d = 0; d < ND; ++d) acc[d] += part[d];
  });
  double y = acc[0];
#pragma unroll
  for (int d = 1; d < ND; ++d) y += acc[d];
  return y;
}

// Kernel dispatch on the element kind (the grid's kind must match KIND).
#define FEM_KIND_DISPATCH(kind, KIND_NAME, ...)        \
  do {                                                 \
    if ((kind) == FEM_Q1_2D) {                         \
      constexpr int KIND_NAME = FEM_Q1_2D;             \
      __VA_ARGS__;                                     \
    } else if ((kind) == FEM_Q2_2D) {                  \
      constexpr int KIND_NAME = FEM_Q2_2D;             \
      __VA_ARGS__;                                     \
    } else {                                           \
      constexpr int KIND_NAME = FEM_HEX8;              \
      __VA_ARGS__;                                     \
    }                                                  \
  } while (0)

// Tiled stencil with shared-memory staging. For each 32 x TY tile of the
// lattice owned by this CTA (TY from fem_tile_rows), the NSRC source vectors
// over the tile plus an R-wide halo (3 planes in 3D) are staged into smem in
// one batch (fem_stage), combined in place into the stencil's input
// v = comb(q, s_0[q], .., s_{NSRC-1}[q]) (q = staged index), and every thread
// applies the assembled stencil of its nodes from smem and calls
// body(n, x, y, z, value, v_center). The tables `tab` may live in shared or
// global memory (plain loads). Needs NSRC * (32+2R) * (TY+2R) * (3 in 3D)
// doubles of smem at sm.
#define FEM_TILE_SMEM 8192

// Tile height (lattice rows) so that one round of tiles covers the level with
// at most ncta tiles (one tile per CTA), capped by the smem staging buffer.
__device__ __forceinline__ int fem_tile_rows(int nx, int ny, int nplanes, int halo, int ncta, int cap_doubles,
                                             int planes_staged) {
  const int ntx = (nx + 31) >> 5;
  int nty = ncta / (ntx * nplanes);
  if (nty < 1) nty = 1;
  int th = (ny + nty - 1) / nty;
  const int rows_per_tile_cap = cap_doubles / ((32 + 2 * halo) * planes_staged) - 2 * halo;
  const int minr = blockDim.x >> 5;
  if (th < minr) th = minr;
  if (th > rows_per_tile_cap) th = rows_per_tile_cap;
  if (th > ny) th = ny < minr ? minr : ny;
  return th;
}

struct FemNoHook {
  __device__ __forceinline__ void operator()() const {}
};

// 3D form of fem_tiled_stencil. A CTA owns a column tile (32 x TY nodes of an
// x-y plane) and a run of z-planes, and marches up the run. Each step stages
// plane z+1 of the NSRC sources (halo included) into `stg`, combines it into a
// ring of three planes (z-1, z, z+1; clamped at the lattice ends) and applies
// the stencil on plane z. Every source value is staged and combined once per
// column tile and run (plus two planes at the run's start) instead of once for
// each of the planes above, at and below it. The stencil sum of a node (terms,
// order, coefficients) is the one of the plane-by-plane form. The tile is as
// tall as the cap_doubles of smem at sm allow ((NSRC + 3) * (32+2R) * (TY+2R)
// doubles), and the CTAs are spread over runs of z.
template <int KIND, int NSRC, class Team, class Comb, class Body, class Pre>
__device__ __forceinline__ void fem_tiled_stencil_3d(const Team& tm, const FemGrid& g, const double* tab,
                                                     double* __restrict__ sm, const double* const (&src)[NSRC],
                                                     const Comb& comb, const Body& body, const Pre& pre,
                                                     int cap_doubles) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF;
  const int WR = blockDim.x >> 5;
  // the tallest tile the smem allows, then the rows split evenly over as many tiles
  const int TYmax = fem_tile_rows(g.nnx, g.nny, 1, R, 1, cap_doubles, NSRC + 3);
  const int nty = (g.nny + TYmax - 1) / TYmax, TY = (g.nny + nty - 1) / nty;
  const int SX = 32 + 2 * R, SY = TY + 2 * R, SXY = SX * SY;
  const int ntx = (g.nnx + 31) >> 5, nt2 = ntx * nty;
  int nzc = tm.ncta() / nt2;
  if (nzc < 1) nzc = 1;
  if (nzc > g.nnz) nzc = g.nnz;
  const int zl = (g.nnz + nzc - 1) / nzc;
  const int nunit = nt2 * ((g.nnz + zl - 1) / zl);
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
  const int nc = fem_axis_ncls(KIND, g.periodic);
  const size_t plane = (size_t)g.nnx * g.nny;
  double* __restrict__ stg = sm;                // NSRC * SXY: the plane being staged
  double* __restrict__ ring = sm + NSRC * SXY;  // 3 * SXY: combined planes
  bool first = true;
  for (int u = tm.cta(); u < nunit; u += tm.ncta()) {
    const int zc = u / nt2, rr = u - zc * nt2, by = rr / ntx, bx = rr - by * ntx;
    const int z0 = zc * zl, z1 = min(g.nnz, z0 + zl);
    const int x0 = bx * 32 - R, y0 = by * TY - R;
    auto rowb = [&](int r) -> int {
      int gy = y0 + r;
      gy = g.periodic ? fem_wrap(gy, g.nny) : (gy < 0 ? 0 : (gy >= g.nny ? g.nny - 1 : gy));
      return gy * g.nnx;
    };
    auto colx = [&](int c) -> int {
      const int gx = x0 + c;
      return g.periodic ? fem_wrap(gx, g.nnx) : (gx < 0 ? 0 : (gx >= g.nnx ? g.nnx - 1 : gx));
    };
    for (int q = z0 - 1; q <= z1; ++q) {
      const int gz = q < 0 ? 0 : (q >= g.nnz ? g.nnz - 1 : q);
#pragma unroll
      for (int k = 0; k < NSRC; ++k)
        if (src[k] != nullptr) fem_stage_2d(stg + k * SXY, src[k] + gz * plane, SX, SY, rowb, colx);
      if (first) {
        pre();
        first = false;
      }
      fem_stage_wait();
      double* __restrict__ slot = ring + ((q - z0 + 1) % 3) * SXY;
      for (int s = threadIdx.x; s < SXY; s += blockDim.x) {
        double v[NSRC];
#pragma unroll
        for (int k = 0; k < NSRC; ++k) v[k] = stg[k * SXY + s];
        slot[s] = comb(s, v);
      }
      __syncthreads();
      if (q > z0) {
        const int z = q - 1;
        const double* pl[3] = {ring + ((q - z0 - 1) % 3) * SXY, ring + ((q - z0) % 3) * SXY, slot};
        const int cz = fem_axis_cls(KIND, 0, z, g.nez);
        for (int ty = ty0; ty < TY; ty += WR) {
          const int x = bx * 32 + tx, y = by * TY + ty;
          if (x < g.nnx && y < g.nny) {
            const int cx = fem_axis_cls(KIND, g.periodic, x, g.nex), cy = fem_axis_cls(KIND, g.periodic, y, g.ney);
            const double* c = tab + (size_t)((cz * nc + cy) * nc + cx) * NOFF;
            double acc = 0.0;
#pragma unroll
            for (int dz = 0; dz < W; ++dz)
#pragma unroll
              for (int dy = 0; dy < W; ++dy)
#pragma unroll
                for (int dx = 0; dx < W; ++dx)
                  acc += c[(dz * W + dy) * W + dx] * pl[dz][(ty + dy) * SX + tx + dx];
            const int n = (z * g.nny + y) * g.nnx + x;
            body(n, x, y, z, acc, pl[1][(ty + R) * SX + tx + R]);
          }
        }
      }
    }
    __syncthreads();
  }
  if (first) pre();
}

// pre() runs once per CTA while its first tile's copies are in flight (every
// thread, before comb is used; a CTA without a tile runs it after the loop).
// cap_doubles: the smem at sm (the 3D form sizes its tiles by it; the 2D
// form uses FEM_TILE_SMEM).
template <int KIND, int NSRC, class Team, class Comb, class Body, class Pre = FemNoHook>
__device__ __forceinline__ void fem_tiled_stencil(const Team& tm, const FemGrid& g, const double* tab,
                                                  double* __restrict__ sm, const double* const (&src)[NSRC],
                                                  const Comb& comb, const Body& body, const Pre& pre = Pre(),
                                                  int cap_doubles = FEM_TILE_SMEM) {
  constexpr int R = KI<KIND>::R, W = KI<KIND>::W, NOFF = KI<KIND>::NOFF;
  constexpr bool D3 = (KIND == FEM_HEX8);
  if constexpr (D3) {
    fem_tiled_stencil_3d<KIND, NSRC>(tm, g, tab, sm, src, comb, body, pre, cap_doubles);
    return;
  }
  const int WR = blockDim.x >> 5;  // warps = rows per pass
  const int TY = fem_tile_rows(g.nnx, g.nny, g.nnz, R, tm.ncta(), FEM_TILE_SMEM, (D3 ? 3 : 1) * NSRC);
  const int SX = 32 + 2 * R, SY = TY + 2 * R, SXY = SX * SY, NS = SXY * (D3 ? 3 : 1);
  const int ntx = (g.nnx + 31) >> 5, nty = (g.nny + TY - 1) / TY, nt2 = ntx * nty, ntile = nt2 * g.nnz;
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
  const int nc = fem_axis_ncls(KIND, g.periodic);
  for (int t = tm.cta(); t < ntile; t += tm.ncta()) {
    const int z = t / nt2, rr = t - z * nt2, by = rr / ntx, bx = rr - by * ntx;
    const int x0 = bx * 32 - R, y0 = by * TY - R;
    auto rowb = [&](int r) -> int {
      int gy = y0 + r;
      gy = g.periodic ? fem_wrap(gy, g.nny) : (gy < 0 ? 0 : (gy >= g.nny ? g.nny - 1 : gy));
      return gy * g.nnx;
    };
    auto colx = [&](int c) -> int {
      const int gx = x0 + c;
      return g.periodic ? fem_wrap(gx, g.nnx) : (gx < 0 ? 0 : (gx >= g.nnx ? g.nnx - 1 : gx));
    };
    if constexpr (D3) {
      // planes z-1, z, z+1 (clamped) one after another, each staged row-wise:
      // sm[k * NS + lz * SXY + ly * SX + lx]
      const size_t plane = (size_t)g.nnx * g.nny;
#pragma unroll
      for (int k = 0; k < NSRC; ++k) {
        if (src[k] == nullptr) continue;
#pragma unroll
        for (int lz = 0; lz < 3; ++lz) {
          int gz = z + lz - 1;
          gz = gz < 0 ? 0 : (gz >= g.nnz ? g.nnz - 1 : gz);
          fem_stage_2d(sm + k * NS + lz * SXY, src[k] + gz * plane, SX, SY, rowb, colx);
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < NSRC; ++k) fem_stage_2d(sm + k * NS, src[k], SX, SY, rowb, colx);
    }
    if (t == tm.cta()) pre();
    fem_stage_wait();
    for (int s = threadIdx.x; s < NS; s += blockDim.x) {
      double v[NSRC];
#pragma unroll
      for (int k = 0; k < NSRC; ++k) v[k] = sm[k * NS + s];
      sm[s] = comb(s, v);
    }
    __syncthreads();
    for (int ty = ty0; ty < TY; ty += WR) {
      const int x = bx * 32 + tx, y = by * TY + ty;
      if (x < g.nnx && y < g.nny) {
        const int cx = fem_axis_cls(KIND, g.periodic, x, g.nex), cy = fem_axis_cls(KIND, g.periodic, y, g.ney);
        const int cz = D3 ? fem_axis_cls(KIND, 0, z, g.nez) : 0;
        const double* c = tab + (size_t)((cz * nc + cy) * nc + cx) * NOFF;
        double acc = 0.0;
#pragma unroll
        for (int dz = 0; dz < (D3 ? W : 1); ++dz)
#pragma unroll
          for (int dy = 0; dy < W; ++dy)
#pragma unroll
            for (int dx = 0; dx < W; ++dx)
              acc += c[(dz * W + dy) * W + dx] * sm[dz * SXY + (ty + dy) * SX + tx + dx];
        const int n = (z * g.nny + y) * g.nnx + x;
        body(n, x, y, z, acc, sm[(D3 ? SXY : 0) + (ty + R) * SX + tx + R]);
      }
    }
    __syncthreads();
  }
  if (tm.cta() >= ntile) pre();
}

// Tiled element-by-element product with per-element coefficients m(e, a, b, nen)
// and NC source components staged in smem (layout sm[c * NS + s]). For each
// owned node: y_c = sum_{(e,a)} sum_b m(e,a,b) * src_c(node(e,b)); then
// body(n, y[NC], center[NC]). Needs NC * (32+2R)(blockDim/32+2R)(3 in 3D) doubles.
template <int KIND, int NC, class Team, class Load, class Mat, class Body>
__device__ __forceinline__ void fem_tiled_ebe(const Team& tm, const FemGrid& g, double* __restrict__ sm,
                                              const Load& load, const Mat& m, const Body& body) {
  constexpr int R = KI<KIND>::R, NEN = KI<KIND>::NEN;
  constexpr bool D3 = (KIND == FEM_HEX8);
  const int TY = blockDim.x >> 5;
  const int SX = 32 + 2 * R, SY = TY + 2 * R, SXY = SX * SY, NS = SXY * (D3 ? 3 : 1);
  const int ntx = (g.nnx + 31) >> 5, nty = (g.nny + TY - 1) / TY, nt2 = ntx * nty, ntile = nt2 * g.nnz;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int t = tm.cta(); t < ntile; t += tm.ncta()) {
    const int z = t / nt2, rr = t - z * nt2, by = rr / ntx, bx = rr - by * ntx;
    const int x0 = bx * 32 - R, y0 = by * TY - R;
#pragma unroll 2
    for (int s = threadIdx.x; s < NS; s += blockDim.x) {
      const int lz = D3 ? s / SXY : 0, r2 = s - lz * SXY, ly = r2 / SX, lx = r2 - ly * SX;
      int gx = x0 + lx, gy = y0 + ly, gz = D3 ? z + lz - 1 : 0;
      if (g.periodic) {
        gx = fem_wrap(gx, g.nnx);
        gy = fem_wrap(gy, g.nny);
      } else {
        gx = gx < 0 ? 0 : (gx >= g.nnx ? g.nnx - 1 : gx);
        gy = gy < 0 ? 0 : (gy >= g.nny ? g.nny - 1 : gy);
      }
      if (D3) gz = gz < 0 ? 0 : (gz >= g.nnz ? g.nnz - 1 : gz);
      const int j = (gz * g.nny + gy) * g.nnx + gx;
#pragma unroll
      for (int c = 0; c < NC; ++c) sm[c * NS + s] = load(j, c);
    }
    __syncthreads();
    const int x = bx * 32 + tx, y = by * TY + ty;
    if (x < g.nnx && y < g.nny) {
      const int cen = (D3 ? SXY : 0) + (ty + R) * SX + tx + R;
      double v[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) v[c] = 0.0;
      fem_incident_k<KIND>(g, x, y, z, [&](int, int, int, int e, int a) {
        int dia, dja, dka;
        fem_local_offset(KIND, a, dia, dja, dka);
        const int base = cen - dia - dja * SX - dka * SXY;
        double part[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) part[c] = 0.0;
#pragma unroll
        for (int b = 0; b < NEN; ++b) {
          const int sidx = base + kdi<KIND>(b) + kdj<KIND>(b) * SX + kdk<KIND>(b) * SXY;
          const double coef = m(e, a, b, NEN);
#pragma unroll
          for (int c = 0; c < NC; ++c) part[c] += coef * sm[c * NS + sidx];
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) v[c] += part[c];
      });
      double ctr[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) ctr[c] = sm[c * NS + cen];
      body((z * g.nny + y) * g.nnx + x, v, ctr);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Element-centric hex8 product with per-element matrices (the explicit Ce of
// the momentum operator): y = sum_e P_e^T (alpha A + beta B_e) P_e x for NC
// components, B_e row-major per element (transB == 0, no C).
//
// The CTA owns a tile of EX x EY elements (and the nodes at their low corners;
// the last tile of each axis also owns the closing node line) and marches a
// run of z. For each element layer L it forms every row of every element of
// the tile plus a one-element halo in -x and -y: a warp takes four elements at
// a time, lane l forms row l % 8 of element l / 8 from its 64-byte row of B_e
// (four 16-byte loads; each element's 512 bytes are read whole by its 8 lanes)
// and the staged node values, summing over the element's nodes in order, as
// the node-centric fem_tiled_ebe does. Rows 0-3 (bottom nodes) serve node
// plane L, rows 4-7 (top nodes) are kept for plane L + 1. Each node then sums
// its incident elements' rows in the order of fem_incident_k (layer below,
// then above; y - 1 before y; x - 1 before x), so results are deterministic.
// The next node plane's values are loaded into registers while a layer
// computes.
//
// Shared memory (doubles): fem_ebe3e_smem(NC). load(j, c): the source value at
// node j; body(n, y[NC], x_n[NC]) as in fem_tiled_ebe.
#define FEM_E3_EX 32
#define FEM_E3_EY 8
#define FEM_E3_FX (FEM_E3_EX + 1)         // element footprint (halo in -x, -y)
#define FEM_E3_FY (FEM_E3_EY + 1)
#define FEM_E3_PX (FEM_E3_EX + 2)         // staged node plane (34 x 10)
#define FEM_E3_PY (FEM_E3_EY + 2)
#define FEM_E3_NE (FEM_E3_FX * FEM_E3_FY)  // 297 elements per layer
__host__ __device__ constexpr int fem_ebe3e_smem(int nc) {
  return 3 * nc * FEM_E3_PX * FEM_E3_PY + 3 * nc * 4 * FEM_E3_NE;
}
template <int NC, class Team, class Load, class Body>
__device__ __forceinline__ void fem_tiled_ebe3e(const Team& tm, const FemGrid& g, double* __restrict__ sm,
                                                const Load& load, const MatCombo& op, const Body& body) {
  constexpr int PX = FEM_E3_PX, PXY = FEM_E3_PX * FEM_E3_PY, FX = FEM_E3_FX, NE = FEM_E3_NE;
  constexpr int RS = 4 * NE;                   // 4 rows per element, per component
  double* __restrict__ stg = sm;               // node planes: [slot (z % 3)][c][PXY]
  double* __restrict__ bot = sm + 3 * NC * PXY;  // rows 0-3 of the current layer: [c][fe * 4 + row]
  double* __restrict__ top = bot + NC * RS;      // rows 4-7 of layers L & 1: [L & 1][c][fe * 4 + row - 4]
  const int nex = g.nex, ney = g.ney, nez = g.nez, nnz = nez + 1;
  const int tnx = (nex + FEM_E3_EX - 1) / FEM_E3_EX, tny = (ney + FEM_E3_EY - 1) / FEM_E3_EY, nt2 = tnx * tny;
  int nzc = tm.ncta() / nt2;
  if (nzc < 1) nzc = 1;
  if (nzc > nnz) nzc = nnz;
  const int zl = (nnz + nzc - 1) / nzc, nunit = nt2 * ((nnz + zl - 1) / zl);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  // lane l forms row a = l % 8 of the warp's element slot l / 8 (four elements per warp step)
  const int a = lane & 7, slot = lane >> 3;
  double sA[8];
#pragma unroll
  for (int b = 0; b < 8; ++b) sA[b] = op.A ? op.alpha * op.A[a * 8 + b] : 0.0;
  const double beta = op.beta;
  const double* __restrict__ B = op.B;
  for (int u = tm.cta(); u < nunit; u += tm.ncta()) {
    const int zc = u / nt2, rr = u - zc * nt2, by = rr / tnx, bx = rr - by * tnx;
    const int ex0 = bx * FEM_E3_EX, ey0 = by * FEM_E3_EY;
    const int nx1 = (bx == tnx - 1) ? nex + 1 : ex0 + FEM_E3_EX, ny1 = (by == tny - 1) ? ney + 1 : ey0 + FEM_E3_EY;
    const int z0 = zc * zl, z1 = min(nnz, z0 + zl);
    const int Lb = max(z0 - 1, 0), Le = min(z1 - 1, nez - 1);
    // node (x, y) of plane z at staged cell q of the 34 x 10 window (clamped into the lattice)
    auto stage_cell = [&](int q, int z, double (&v)[NC]) {
      const int py = q / PX, px = q - py * PX;
      int gx = ex0 - 1 + px, gy = ey0 - 1 + py;
      gx = gx < 0 ? 0 : (gx > nex ? nex : gx);
      gy = gy < 0 ? 0 : (gy > ney ? ney : gy);
      const int j = (z * g.nny + gy) * g.nnx + gx;
#pragma unroll
      for (int c = 0; c < NC; ++c) v[c] = load(j, c);
    };
    // y of node plane z from the rows kept for it (below: layer z - 1, above: layer z)
    auto finalize = [&](int z) {
      const int wx = nx1 - ex0, cnt = wx * (ny1 - ey0);
      const double* __restrict__ tb = top + ((z - 1) & 1) * NC * RS;
      for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
        const int qy = q / wx, x = ex0 + (q - qy * wx), y = ey0 + qy;
        double acc[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] = 0.0;
#pragma unroll
        for (int zk = 0; zk < 2; ++zk) {
          if (zk == 0 ? z < 1 : z >= nez) continue;
          const double* __restrict__ buf = zk == 0 ? tb : bot;
#pragma unroll
          for (int zj = 0; zj < 2; ++zj) {
            const int ey = zj ? y : y - 1;
            if (ey < 0 || ey >= ney) continue;
#pragma unroll
            for (int zi = 0; zi < 2; ++zi) {
              const int ex = zi ? x : x - 1;
              if (ex < 0 || ex >= nex) continue;
              // row of this node in element (ex, ey): quad4 index of (x - ex, y - ey)
              const int r = fem_local_index(FEM_HEX8, 1 - zi, 1 - zj, 0);
              const int fe = (ey - ey0 + 1) * FX + (ex - ex0 + 1);
#pragma unroll
              for (int c = 0; c < NC; ++c) acc[c] += buf[c * RS + fe * 4 + r];
            }
          }
        }
        double ctr[NC];
        const int cq = (y - ey0 + 1) * PX + (x - ex0 + 1);
#pragma unroll
        for (int c = 0; c < NC; ++c) ctr[c] = stg[((z % 3) * NC + c) * PXY + cq];
        body((z * g.nny + y) * g.nnx + x, acc, ctr);
      }
    };
    if (threadIdx.x < PXY) {
#pragma unroll
      for (int pl = 0; pl < 2; ++pl) {
        double v[NC];
        stage_cell(threadIdx.x, Lb + pl, v);
#pragma unroll
        for (int c = 0; c < NC; ++c) stg[(((Lb + pl) % 3) * NC + c) * PXY + threadIdx.x] = v[c];
      }
    }
    __syncthreads();
    for (int L = Lb; L <= Le; ++L) {
      const int s0 = L % 3, s1 = (L + 1) % 3;
      // plane L + 2 into registers while the layer computes
      double pv[NC];
      const bool pf = L + 2 <= nez && threadIdx.x < PXY;
      if (pf) stage_cell(threadIdx.x, L + 2, pv);
      double* __restrict__ tw = top + (L & 1) * NC * RS;
      const size_t lay = (size_t)L * ney;
      // row a of element fe: sum_b (alpha A[a][b] + beta B_e[a][b]) x(node b), b in order
      for (int f0 = warp; f0 < NE; f0 += 4 * nwarp) {
        const int fe = f0 + slot * nwarp, ly = fe / FX, lx = fe - ly * FX;
        const int ex = ex0 - 1 + lx, ey = ey0 - 1 + ly;
        if (fe < NE && ex >= 0 && ex < nex && ey >= 0 && ey < ney) {
          const double2* __restrict__ row = reinterpret_cast<const double2*>(B + ((lay + ey) * nex + ex) * 64 + a * 8);
          double2 cb[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) cb[q] = __ldg(row + q);
          double v[8];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            v[2 * q] = sA[2 * q];
            v[2 * q] += beta * cb[q].x;
            v[2 * q + 1] = sA[2 * q + 1];
            v[2 * q + 1] += beta * cb[q].y;
          }
          const int w = ly * PX + lx;
          const double* __restrict__ xl = stg + s0 * NC * PXY + w;  // node plane L at the element's low corner
          const double* __restrict__ xh = stg + s1 * NC * PXY + w;  // node plane L + 1
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            double p = 0.0;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
              const double* __restrict__ xp = kdk<FEM_HEX8>(b) ? xh : xl;
              p += v[b] * xp[c * PXY + kdj<FEM_HEX8>(b) * PX + kdi<FEM_HEX8>(b)];
            }
            if (a < 4) bot[c * RS + fe * 4 + a] = p;
            else tw[c * RS + fe * 4 + a - 4] = p;
          }
        }
      }
      if (pf) {
#pragma unroll
        for (int c = 0; c < NC; ++c) stg[(((L + 2) % 3) * NC + c) * PXY + threadIdx.x] = pv[c];
      }
      __syncthreads();
      if (L >= z0 && L < z1) finalize(L);
      __syncthreads();
    }
    // the closing node plane z = nez has elements only below
    if (z0 <= nez && nez < z1) {
      finalize(nez);
      __syncthreads();
    }
  }
}
