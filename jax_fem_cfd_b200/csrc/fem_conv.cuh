// Convection operator applied without materialising Ce. The conservative
// convection element matrix of core/element_calc.py:165-185,
//   Ce_e[a][b] = sum_q w_q N_a(q) (u_q . grad N_b(q)) + beta sum_q w_q N_a(q) (div u)_q N_b(q),
// acts on an element vector x_e as
//   (Ce_e x_e)_a = sum_q w_q N_a(q) [ u_q . grad x_q + beta (div u)_q x_q ],
// with u_q, (div u)_q, x_q and grad x_q interpolated at the Gauss points from the
// element's nodal values. u is fixed for a whole solve, so its Gauss-point
// factors (27 doubles per Q2 element instead of Ce's 81) are formed once and every
// operator apply interpolates only x. The mesh is uniform, so one table of Gauss
// weights, shape functions and physical derivatives serves every element; it is
// passed by value in the kernel parameters.
#pragma once
#include "fem_stencil.cuh"

#define FEM_QT_MAX 9
struct FemQuadTab {
  double w[FEM_QT_MAX];
  double N[FEM_QT_MAX][FEM_QT_MAX];   // [q][node]
  double dx[FEM_QT_MAX][FEM_QT_MAX];  // d N_node / dx at q
  double dy[FEM_QT_MAX][FEM_QT_MAX];  // d N_node / dy at q
  double dz[FEM_QT_MAX][FEM_QT_MAX];  // d N_node / dz at q (hex8)
  // Q2 tensor factors (filled and checked on the host): N[q][b] = nx[qx][i] ny[qy][j],
  // dx[q][b] = ddx[qx][i] ny[qy][j], dy[q][b] = nx[qx][i] ddy[qy][j] for node b at
  // element-local lattice offset (i, j) and Gauss point q = qi[qy][qx]
  double nx[3][3], ny[3][3], ddx[3][3], ddy[3][3];
  int qi[3][3];
};

template <int KIND>
struct KQ;
template <>
struct KQ<FEM_Q1_2D> {
  static constexpr int NQ = 4;
};
template <>
struct KQ<FEM_Q2_2D> {
  static constexpr int NQ = 9;
};

// Gauss-point factors of Ce(u) for one element (2D kinds): for each point q,
// f[3q] = w_q u_q, f[3q+1] = w_q v_q, f[3q+2] = w_q beta (div u)_q, so that
// (Ce x)_a = sum_q N_a(q) (f[3q] dx x_q + f[3q+1] dy x_q + f[3q+2] x_q).
template <int KIND>
__device__ __forceinline__ void fem_conv_factors(const FemQuadTab& T, const double (&ux)[KI<KIND>::NEN],
                                                 const double (&uy)[KI<KIND>::NEN], double bd,
                                                 double (&f)[3 * KQ<KIND>::NQ]) {
  constexpr int NEN = KI<KIND>::NEN, NQ = KQ<KIND>::NQ;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double uqx = 0.0, uqy = 0.0, div = 0.0;
#pragma unroll
    for (int b = 0; b < NEN; ++b) {
      uqx += T.N[q][b] * ux[b];
      uqy += T.N[q][b] * uy[b];
      div += T.dx[q][b] * ux[b] + T.dy[q][b] * uy[b];
    }
    f[3 * q] = T.w[q] * uqx;
    f[3 * q + 1] = T.w[q] * uqy;
    f[3 * q + 2] = T.w[q] * (bd * div);
  }
}

// y_a = cc (Ce x)_a + alpha (Ash x)_a for one element from its Gauss-point
// factors (fac(k) = factor k of this element). The Gauss-point loop is not
// unrolled (indexed table reads): that keeps only x, the accumulators and one
// point's temporaries live, which the 128-register budget of the persistent
// solver allows without spills.
template <int KIND, class Fac>
__device__ __forceinline__ void fem_conv_element(const FemQuadTab& T, const double (&xl)[KI<KIND>::NEN],
                                                 const Fac& fac, double cc, double alpha, const double* Ash,
                                                 double (&y)[KI<KIND>::NEN]);

template <int KIND, class Fac>
__device__ __forceinline__ void fem_conv_element_loop(const FemQuadTab& T, const double (&xl)[KI<KIND>::NEN],
                                                      const Fac& fac, double cc, double alpha, const double* Ash,
                                                      double (&y)[KI<KIND>::NEN]) {
  constexpr int NEN = KI<KIND>::NEN, NQ = KQ<KIND>::NQ;
  double acc[NEN];
#pragma unroll
  for (int a = 0; a < NEN; ++a) acc[a] = 0.0;
  // the factors of Gauss point q + 1 are loaded while point q is evaluated (the
  // loop stays rolled, so the loads would otherwise wait inside each iteration)
  double f0 = fac(0), f1 = fac(1), f2 = fac(2);
#pragma unroll 1
  for (int q = 0; q < NQ; ++q) {
    double n0 = 0.0, n1 = 0.0, n2 = 0.0;
    if (q + 1 < NQ) {
      n0 = fac(3 * q + 3);
      n1 = fac(3 * q + 4);
      n2 = fac(3 * q + 5);
    }
    double xq = 0.0, gx = 0.0, gy = 0.0;
#pragma unroll
    for (int b = 0; b < NEN; ++b) {
      xq += T.N[q][b] * xl[b];
      gx += T.dx[q][b] * xl[b];
      gy += T.dy[q][b] * xl[b];
    }
    const double sq = (f0 * gx + f1 * gy) + f2 * xq;
    f0 = n0;
    f1 = n1;
    f2 = n2;
#pragma unroll
    for (int a = 0; a < NEN; ++a) acc[a] += T.N[q][a] * sq;
  }
#pragma unroll
  for (int a = 0; a < NEN; ++a) {
    double sh = 0.0;
    if (Ash) {
#pragma unroll
      for (int b = 0; b < NEN; ++b) sh += Ash[a * NEN + b] * xl[b];
    }
    y[a] = alpha * sh + cc * acc[a];
  }
}

// The same product for Q2 by sum factorisation over the tensor-product basis
// (the factors in T.nx / T.ny / T.ddx / T.ddy): x is interpolated along x for
// each node row (values and x-derivatives), then along y at each Gauss point,
// and the test functions are applied along x and then y. 216 FMAs per element
// row instead of 351, and a few table reads instead of ~320; the order of the
// sums differs from fem_conv_element's, the values agree to rounding.
template <class Fac>
__device__ __forceinline__ void fem_conv_element_q2(const FemQuadTab& T, const double (&xl)[9], const Fac& fac,
                                                    double cc, double alpha, const double* Ash, double (&y)[9]) {
#pragma unroll
  for (int a = 0; a < 9; ++a) {
    double sh = 0.0;
    if (Ash) {
#pragma unroll
      for (int b = 0; b < 9; ++b) sh += Ash[a * 9 + b] * xl[b];
    }
    y[a] = alpha * sh;
  }
  double U[3][3], V[3][3];  // [node row j][Gauss column qx]: values and x-derivatives
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double X[3];
#pragma unroll
    for (int b = 0; b < 9; ++b)
      if (kdj<FEM_Q2_2D>(b) == j) X[kdi<FEM_Q2_2D>(b)] = xl[b];
#pragma unroll
    for (int qx = 0; qx < 3; ++qx) {
      U[j][qx] = (T.nx[qx][0] * X[0] + T.nx[qx][1] * X[1]) + T.nx[qx][2] * X[2];
      V[j][qx] = (T.ddx[qx][0] * X[0] + T.ddx[qx][1] * X[1]) + T.ddx[qx][2] * X[2];
    }
  }
  double acc[3][3];  // [i][j]
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) acc[i][j] = 0.0;
#pragma unroll 1
  for (int qy = 0; qy < 3; ++qy) {
    const double y0 = T.ny[qy][0], y1 = T.ny[qy][1], y2 = T.ny[qy][2];
    const double e0 = T.ddy[qy][0], e1 = T.ddy[qy][1], e2 = T.ddy[qy][2];
    double wv[3] = {0.0, 0.0, 0.0};  // sum over qx of nx[qx][i] s(qx, qy)
#pragma unroll
    for (int qx = 0; qx < 3; ++qx) {
      const double xq = (y0 * U[0][qx] + y1 * U[1][qx]) + y2 * U[2][qx];
      const double gy = (e0 * U[0][qx] + e1 * U[1][qx]) + e2 * U[2][qx];
      const double gx = (y0 * V[0][qx] + y1 * V[1][qx]) + y2 * V[2][qx];
      const int q = T.qi[qy][qx];
      const double sq = (fac(3 * q) * gx + fac(3 * q + 1) * gy) + fac(3 * q + 2) * xq;
#pragma unroll
      for (int i = 0; i < 3; ++i) wv[i] += T.nx[qx][i] * sq;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      acc[i][0] += y0 * wv[i];
      acc[i][1] += y1 * wv[i];
      acc[i][2] += y2 * wv[i];
    }
  }
#pragma unroll
  for (int b = 0; b < 9; ++b) y[b] += cc * acc[kdi<FEM_Q2_2D>(b)][kdj<FEM_Q2_2D>(b)];
}

template <int KIND, class Fac>
__device__ __forceinline__ void fem_conv_element(const FemQuadTab& T, const double (&xl)[KI<KIND>::NEN],
                                                 const Fac& fac, double cc, double alpha, const double* Ash,
                                                 double (&y)[KI<KIND>::NEN]) {
  if constexpr (KIND == FEM_Q2_2D) {
    fem_conv_element_q2(T, xl, fac, cc, alpha, Ash, y);
  } else {
    fem_conv_element_loop<KIND>(T, xl, fac, cc, alpha, Ash, y);
  }
}

// Local node index of element-local lattice offset (i, j) (inverse of kdi/kdj).
template <int KIND>
__device__ __forceinline__ int fem_local_node(int i, int j) {
  if (KIND == FEM_Q2_2D) {
    // quad9 order: (0,0) (1,0) (2,0) (2,1) (2,2) (1,2) (0,2) (0,1) (1,1)
    constexpr int t[9] = {0, 1, 2, 7, 8, 3, 6, 5, 4};
    return t[j * 3 + i];
  }
  constexpr int t[4] = {0, 1, 3, 2};  // quad4: (0,0) (1,0) (1,1) (0,1)
  return t[j * 2 + i];
}

// Dynamic smem of fem_tiled_conv (doubles); the tile height adapts to it.
#define FEM_CONV_SMEM 16384

// Tiled application of y = alpha Ash x + cc Ce x (2D, NC components). x is
// comb(s, v) of NSRC source vectors (v[k] = src[k][c*nn + node] at staged point
// s), Ce enters through its Gauss-point factors fq (structure of arrays
// fq[k * ne + e], k < 3 NQ). Each CTA takes one tile of 32 x TY owned nodes (TY
// even, chosen so one round of tiles covers the lattice, capped by
// FEM_CONV_SMEM): the sources on the tile plus its halo are staged by cp.async
// and combined in smem, every element touching the tile computes its rows for
// all components once (border elements are computed by both tiles), and each
// owned node sums the rows of its incident elements in a fixed order:
// body(n, y[NC], x_center[NC]). Deterministic, no atomics. pre() runs once per
// CTA while the first tile's copies are in flight.
template <int KIND, int NC, int NSRC, class Team, class Comb, class Body, class Pre = FemNoHook>
__device__ __forceinline__ void fem_tiled_conv(const Team& tm, const FemGrid& g, double* __restrict__ sm,
                                               const double* const (&src)[NSRC], const Comb& comb,
                                               const double* __restrict__ fq, const FemQuadTab& T, double cc,
                                               double alpha, const double* Ash, const Body& body,
                                               const Pre& pre = Pre()) {
  static_assert(KIND != FEM_HEX8, "2D kinds only");
  constexpr int R = KI<KIND>::R, S = KI<KIND>::S, NEN = KI<KIND>::NEN;
  constexpr int SX = 32 + 2 * R, EX = 31 / S + 2;
  const int WR = blockDim.x >> 5;
  const int ntx = (g.nnx + 31) >> 5;
  // tile height: a multiple of S, one round of tiles, within FEM_CONV_SMEM
  auto need = [&](int ty) {
    const int ns = SX * (ty + 2 * R), ne_t = EX * ((ty - 1) / S + 2);
    const int a = NSRC * NC * ns, b = NC * ns + ne_t * NC * NEN;
    return a > b ? a : b;
  };
  int TY;
  {
    int nty_t = tm.ncta() / ntx;
    if (nty_t < 1) nty_t = 1;
    TY = (g.nny + nty_t - 1) / nty_t;
    TY = ((TY + S - 1) / S) * S;
    while (TY > S && need(TY) > FEM_CONV_SMEM) TY -= S;
  }
  const int SY = TY + 2 * R, NS = SX * SY;
  const int EY = (TY - 1) / S + 2, NE = EX * EY;
  double* sx = sm;              // NC * NS: the combined x (over the first source's slots)
  double* sy = sx + NC * NS;    // NE * NC * NEN element rows (over the other sources' slots)
  const size_t nn = g.nn, ne = g.ne;
  const int nty = (g.nny + TY - 1) / TY, ntile = ntx * nty;
  const int tx = threadIdx.x & 31, ty0 = threadIdx.x >> 5;
  for (int t = tm.cta(); t < ntile; t += tm.ncta()) {
    const int by = t / ntx, bx = t - by * ntx;
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
#pragma unroll
    for (int k = 0; k < NSRC; ++k)
#pragma unroll
      for (int c = 0; c < NC; ++c)
        fem_stage_2d(sm + (k * NC + c) * NS, src[k] ? src[k] + c * nn : nullptr, SX, SY, rowb, colx);
    if (t == tm.cta()) pre();
    fem_stage_wait();
    for (int s = threadIdx.x; s < NC * NS; s += blockDim.x) {
      double v[NSRC];
#pragma unroll
      for (int k = 0; k < NSRC; ++k) v[k] = sm[k * NC * NS + s];
      sx[s] = comb(s, v);
    }
    __syncthreads();
    // element rows: element (ex0 + lex, ey0 + ley), its node (i, j) at staged
    // (R - S + S lex + i, R - S + S ley + j)
    const int ex0 = bx * 32 / S - 1, ey0 = by * TY / S - 1;
    for (int w = threadIdx.x; w < NE * NC; w += blockDim.x) {
      const int el = w % NE, c = w / NE;
      const int ley = el / EX, lex = el - ley * EX;
      const int ex = ex0 + lex, ey = ey0 + ley;
      double y[NEN];
      if (g.periodic || (ex >= 0 && ex < g.nex && ey >= 0 && ey < g.ney)) {
        const size_t e = (size_t)fem_wrap(ey, g.ney) * g.nex + fem_wrap(ex, g.nex);
        const int base = (R - S + S * ley) * SX + (R - S + S * lex);
        double xl[NEN];
#pragma unroll
        for (int b = 0; b < NEN; ++b) xl[b] = sx[c * NS + base + kdj<KIND>(b) * SX + kdi<KIND>(b)];
        fem_conv_element<KIND>(T, xl, [&](int k) { return __ldg(fq + k * ne + e); }, cc, alpha, Ash, y);
      } else {
#pragma unroll
        for (int a = 0; a < NEN; ++a) y[a] = 0.0;
      }
#pragma unroll
      for (int a = 0; a < NEN; ++a) sy[(el * NC + c) * NEN + a] = y[a];
    }
    __syncthreads();
    for (int ty = ty0; ty < TY; ty += WR) {
      const int x = bx * 32 + tx, yy = by * TY + ty;
      if (x < g.nnx && yy < g.nny) {
        double v[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) v[c] = 0.0;
        // incident elements: node local (tx, ty) is element-local (i, j) of element
        // lex = (tx + S - i) / S, ley = (ty + S - j) / S when divisible
#pragma unroll
        for (int j = 0; j <= S; ++j) {
          if ((ty + S - j) % S) continue;
          const int ley = (ty + S - j) / S, ey = ey0 + ley;
          if (!g.periodic && (ey < 0 || ey >= g.ney)) continue;
#pragma unroll
          for (int i = 0; i <= S; ++i) {
            if ((tx + S - i) % S) continue;
            const int lex = (tx + S - i) / S, ex = ex0 + lex;
            if (!g.periodic && (ex < 0 || ex >= g.nex)) continue;
            const int el = ley * EX + lex, a = fem_local_node<KIND>(i, j);
#pragma unroll
            for (int c = 0; c < NC; ++c) v[c] += sy[(el * NC + c) * NEN + a];
          }
        }
        double ctr[NC];
        const int cen = (ty + R) * SX + tx + R;
#pragma unroll
        for (int c = 0; c < NC; ++c) ctr[c] = sx[c * NS + cen];
        body(yy * g.nnx + x, v, ctr);
      }
    }
    __syncthreads();
  }
  if (tm.cta() >= ntile) pre();
}
