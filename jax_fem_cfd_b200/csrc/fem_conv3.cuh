// hex8 convection applied without materialising Ce (the 3D form of fem_conv.cuh).
//
// (Ce_e x_e)_a = sum_q w_q N_a(q) [ u_q . grad x_q + beta (div u)_q x_q ]
// (core/element_calc.py:165-185). Per element and Gauss point the factors
// f[4q..4q+3] = w_q (u_q, v_q, w_q, beta (div u)_q) are formed once per solve,
// element-major (32 doubles per element), so one lattice row of elements is one
// contiguous run of memory.
//
// fem_tiled_conv3 applies y = alpha Ash x + cc Ce x node-centrically: a CTA owns
// a column tile of 32 x 8 node columns and a run of z-planes and marches up the
// element layers. Per layer the factors of the tile's 33 x 9 elements arrive
// by TMA bulk copies (cp.async.bulk, one per element row, completing on an
// mbarrier; the next layer's copies are issued as soon as the current layer's
// element rows are computed, so they overlap the node sums and the staging of
// the next node plane), the source vectors of the new node plane are staged
// by cp.async and combined, every element of the layer computes its 8 rows for
// all components into shared memory, and each node adds the rows of its 4
// incident elements of the layer. A node's sum is (its 4 elements below, then
// its 4 elements above) in a fixed order, so results are deterministic.
#pragma once
#include "fem_conv.cuh"

#define FEM_C3_TX 32                 // node columns of a tile (one warp row)
#define FEM_C3_TY 8                  // node rows of a tile
#define FEM_C3_EX (FEM_C3_TX + 1)    // element columns touching a tile
#define FEM_C3_EY (FEM_C3_TY + 1)    // element rows touching a tile
#define FEM_C3_SX (FEM_C3_TX + 2)    // staged node columns
#define FEM_C3_SY (FEM_C3_TY + 2)    // staged node rows
#define FEM_C3_NF 32                 // factors per element
// dynamic smem (doubles) of fem_tiled_conv3 for NC components and NSRC sources
#define FEM_C3_SMEM(NC, NSRC)                                                                          \
  (FEM_C3_EY * FEM_C3_EX * FEM_C3_NF + (NSRC) * (NC) * FEM_C3_SX * FEM_C3_SY + 2 * (NC) * FEM_C3_SX * FEM_C3_SY + \
   FEM_C3_EY * FEM_C3_EX * (NC) * 8)
#define FEM_C3_SMEM_MAX FEM_C3_SMEM(3, 3)
// bounded mbarrier wait (try_wait rounds, each suspends the thread for a while)
#define FEM_C3_WAIT_ROUNDS (1 << 22)

// ------------------------------------------------------------ mbarrier / TMA ----
__device__ __forceinline__ void fem_mbar_init(uint64_t* bar, unsigned count) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fem_mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
// 1D bulk copy global -> shared completing on bar (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void fem_bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst), b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
               "l"(src), "r"(bytes), "r"(b)
               : "memory");
}
// Waits for phase `parity` of bar; false if it did not complete within the bound.
__device__ __forceinline__ bool fem_mbar_wait(uint64_t* bar, unsigned parity) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  for (int it = 0; it < FEM_C3_WAIT_ROUNDS; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// TMA state of one CTA: its mbarrier and the parity of the next phase to wait for.
struct FemC3Tma {
  uint64_t* bar;
  unsigned* phase;  // shared
  int* err;         // error word (FEM_ERR_BARRIER_TIMEOUT on a copy that does not land)
};

// ------------------------------------------------------------- element rows ----

// Gauss-point factors of one hex8 element: f[4q + k] = w_q (u, v, w, bd div)_q
__device__ __forceinline__ void fem_conv3_factors(const FemQuadTab& T, const double (&u)[3][8], double bd,
                                                  double* __restrict__ f) {
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    double uq[3] = {0.0, 0.0, 0.0}, div = 0.0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
#pragma unroll
      for (int c = 0; c < 3; ++c) uq[c] += T.N[q][b] * u[c][b];
      div += T.dx[q][b] * u[0][b] + T.dy[q][b] * u[1][b] + T.dz[q][b] * u[2][b];
    }
    f[4 * q] = T.w[q] * uq[0];
    f[4 * q + 1] = T.w[q] * uq[1];
    f[4 * q + 2] = T.w[q] * uq[2];
    f[4 * q + 3] = T.w[q] * (bd * div);
  }
}

// y_a = alpha (Ash x)_a + cc (Ce x)_a of one element from its factors f (shared)
__device__ __forceinline__ void fem_conv3_element(const FemQuadTab& T, const double (&xl)[8],
                                                  const double* __restrict__ f, double cc, double alpha,
                                                  const double* Ash, double (&y)[8]) {
  double acc[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) acc[a] = 0.0;
#pragma unroll 1
  for (int q = 0; q < 8; ++q) {
    double xq = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      xq += T.N[q][b] * xl[b];
      gx += T.dx[q][b] * xl[b];
      gy += T.dy[q][b] * xl[b];
      gz += T.dz[q][b] * xl[b];
    }
    const double sq = ((f[4 * q] * gx + f[4 * q + 1] * gy) + f[4 * q + 2] * gz) + f[4 * q + 3] * xq;
#pragma unroll
    for (int a = 0; a < 8; ++a) acc[a] += T.N[q][a] * sq;
  }
#pragma unroll
  for (int a = 0; a < 8; ++a) {
    double sh = 0.0;
    if (Ash) {
#pragma unroll
      for (int b = 0; b < 8; ++b) sh += Ash[a * 8 + b] * xl[b];
    }
    y[a] = alpha * sh + cc * acc[a];
  }
}

// z-run length of the tiles: the number of runs per column tile that fills the
// CTAs in whole rounds best (each run also reads the layer below its first plane)
__host__ __device__ __forceinline__ int fem_c3_zrun(const FemGrid& g, int ncta) {
  const int ncol = ((g.nnx + FEM_C3_TX - 1) / FEM_C3_TX) * ((g.nny + FEM_C3_TY - 1) / FEM_C3_TY);
  int best = g.nnz;
  double best_eff = -1.0;
  for (int nr = 1; nr <= 16 && nr <= g.nnz; ++nr) {
    const int zr = (g.nnz + nr - 1) / nr;
    const int runs = (g.nnz + zr - 1) / zr, tiles = ncol * runs;
    const int rounds = (tiles + ncta - 1) / ncta;
    const double eff = (double)g.nnz / (double)(zr + 1) * (double)zr / g.nnz * (double)tiles / (rounds * ncta);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = zr;
    }
  }
  return best;
}

// Issue the factor rows of element layer ke of the tile (x0, y0) into sf.
__device__ __forceinline__ void fem_c3_issue(const FemGrid& g, const double* __restrict__ fq, int x0, int y0, int ke,
                                             double* sf, const FemC3Tma& tma) {
  const int ielo = max(x0 - 1, 0), iehi = min(x0 + FEM_C3_TX - 1, g.nex - 1);
  const int jelo = max(y0 - 1, 0), jehi = min(y0 + FEM_C3_TY - 1, g.ney - 1);
  const unsigned rowbytes = (unsigned)(iehi - ielo + 1) * FEM_C3_NF * 8u;
  const unsigned total = (iehi >= ielo && jehi >= jelo) ? rowbytes * (unsigned)(jehi - jelo + 1) : 0u;
  // async-proxy writes follow this CTA's generic reads of sf (ordered by the
  // preceding __syncthreads)
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  fem_mbar_expect_tx(tma.bar, total);
  if (total == 0u) return;
  for (int je = jelo; je <= jehi; ++je) {
    const size_t e0 = ((size_t)ke * g.ney + je) * g.nex + ielo;
    double* dst = sf + ((je - (y0 - 1)) * FEM_C3_EX + (ielo - (x0 - 1))) * FEM_C3_NF;
    fem_bulk_g2s(dst, fq + e0 * FEM_C3_NF, rowbytes, tma.bar);
  }
}

// The tiled operator (see the file comment). src[k] + c nn is source k of
// component c; comb(s, v) combines the NSRC staged values at staged point s;
// body(n, y[NC], x_center[NC]) for every node of the lattice. Team: cta()/ncta()
// of the tile loop. Every thread of the CTA must call it.
template <int NC, int NSRC, class Team, class Comb, class Body>
__device__ __forceinline__ void fem_tiled_conv3(const Team& tm, const FemGrid& g, double* __restrict__ sm,
                                                const FemC3Tma& tma, const double* const (&src)[NSRC],
                                                const Comb& comb, const double* __restrict__ fq, const FemQuadTab& T,
                                                double cc, double alpha, const double* Ash, const Body& body) {
  constexpr int EX = FEM_C3_EX, EY = FEM_C3_EY, SX = FEM_C3_SX, SY = FEM_C3_SY, NS = SX * SY;
  constexpr int NE = EX * EY;
  double* sf = sm;                                  // EY * EX * 32 factors (TMA destination)
  double* sraw = sf + NE * FEM_C3_NF;               // NSRC * NC * NS raw staging of one plane
  double* sx = sraw + NSRC * NC * NS;               // 2 planes * NC * NS combined sources
  double* er = sx + 2 * NC * NS;                    // NE * NC * 8 element rows
  const size_t nn = g.nn;
  const int ntx = (g.nnx + FEM_C3_TX - 1) / FEM_C3_TX, nty = (g.nny + FEM_C3_TY - 1) / FEM_C3_TY;
  const int zr = fem_c3_zrun(g, tm.ncta());
  const int nzr = (g.nnz + zr - 1) / zr, ntile = ntx * nty * nzr;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const bool gather = ty < FEM_C3_TY;  // the first 8 warps own the tile's nodes
  for (int t = tm.cta(); t < ntile; t += tm.ncta()) {
    const int zi = t / (ntx * nty), rr = t - zi * (ntx * nty), by = rr / ntx, bx = rr - by * ntx;
    const int x0 = bx * FEM_C3_TX, y0 = by * FEM_C3_TY;
    const int z0 = zi * zr, z1 = min(z0 + zr, g.nnz);
    const int kfirst = max(z0 - 1, 0), klast = min(z1 - 1, g.nez - 1);
    auto colx = [&](int c) { const int gx = x0 - 1 + c; return gx < 0 ? 0 : (gx >= g.nnx ? g.nnx - 1 : gx); };
    auto stage_plane = [&](int p) {  // raw sources of node plane p, then combined into sx[p & 1]
      auto rowb = [&](int r) {
        int gy = y0 - 1 + r;
        gy = gy < 0 ? 0 : (gy >= g.nny ? g.nny - 1 : gy);
        return (p * g.nny + gy) * g.nnx;
      };
#pragma unroll
      for (int k = 0; k < NSRC; ++k)
#pragma unroll
        for (int c = 0; c < NC; ++c)
          fem_stage_2d(sraw + (k * NC + c) * NS, src[k] ? src[k] + c * nn : nullptr, SX, SY, rowb, colx);
      fem_stage_wait();
      double* dst = sx + (p & 1) * NC * NS;
      for (int s = threadIdx.x; s < NC * NS; s += blockDim.x) {
        double v[NSRC];
#pragma unroll
        for (int k = 0; k < NSRC; ++k) v[k] = sraw[k * NC * NS + s];
        dst[s] = comb(s, v);
      }
      __syncthreads();
    };
    if (threadIdx.x == 0) fem_c3_issue(g, fq, x0, y0, kfirst, sf, tma);
    stage_plane(kfirst);
    double pend[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) pend[c] = 0.0;
    const int x = x0 + tx, y = y0 + ty;
    const bool own = gather && x < g.nnx && y < g.nny;
    for (int ke = kfirst; ke <= klast; ++ke) {
      stage_plane(ke + 1);  // ends with __syncthreads (via fem_stage_wait) before the combine
      if (!fem_mbar_wait(tma.bar, *tma.phase)) {
        if (threadIdx.x == 0) atomicOr(tma.err, FEM_ERR_BARRIER_TIMEOUT);
        fem_mbar_wait(tma.bar, *tma.phase);  // the copies must land before the buffer is reused
      }
      __syncthreads();
      if (threadIdx.x == 0) *tma.phase ^= 1u;
      // element rows of layer ke
      const double* pl0 = sx + (ke & 1) * NC * NS;
      const double* pl1 = sx + ((ke + 1) & 1) * NC * NS;
      for (int w = threadIdx.x; w < NE * NC; w += blockDim.x) {
        const int el = w % NE, c = w / NE;
        const int ley = el / EX, lex = el - ley * EX;
        const int ie = x0 - 1 + lex, je = y0 - 1 + ley;
        double yv[8];
        if (ie >= 0 && ie < g.nex && je >= 0 && je < g.ney) {
          double xl[8];
          const int s00 = ley * SX + lex;
          xl[0] = pl0[c * NS + s00];
          xl[1] = pl0[c * NS + s00 + 1];
          xl[2] = pl0[c * NS + s00 + SX + 1];
          xl[3] = pl0[c * NS + s00 + SX];
          xl[4] = pl1[c * NS + s00];
          xl[5] = pl1[c * NS + s00 + 1];
          xl[6] = pl1[c * NS + s00 + SX + 1];
          xl[7] = pl1[c * NS + s00 + SX];
          fem_conv3_element(T, xl, sf + el * FEM_C3_NF, cc, alpha, Ash, yv);
        } else {
#pragma unroll
          for (int a = 0; a < 8; ++a) yv[a] = 0.0;
        }
#pragma unroll
        for (int a = 0; a < 8; ++a) er[(el * NC + c) * 8 + a] = yv[a];
      }
      __syncthreads();
      if (threadIdx.x == 0 && ke < klast) fem_c3_issue(g, fq, x0, y0, ke + 1, sf, tma);
      if (own) {
        // incident elements of the layer: (lex, ley) = (tx + 1 - di, ty + 1 - dj),
        // the node being their local (di, dj) corner, bottom face (plane ke) or
        // top face (plane ke + 1)
        double bot[NC], top[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) bot[c] = top[c] = 0.0;
#pragma unroll
        for (int dj = 0; dj < 2; ++dj)
#pragma unroll
          for (int di = 0; di < 2; ++di) {
            const int el = (ty + 1 - dj) * EX + (tx + 1 - di);
            const int a = (dj == 0) ? (di == 0 ? 0 : 1) : (di == 0 ? 3 : 2);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
              bot[c] += er[(el * NC + c) * 8 + a];
              top[c] += er[(el * NC + c) * 8 + a + 4];
            }
          }
        const int cen = (ty + 1) * SX + tx + 1;
        if (ke >= z0) {
          double v[NC], ctr[NC];
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            v[c] = pend[c] + bot[c];
            ctr[c] = pl0[c * NS + cen];
          }
          body((ke * g.nny + y) * g.nnx + x, v, ctr);
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) pend[c] = top[c];
        if (ke == g.nez - 1 && ke + 1 < z1) {  // the top plane: no layer above
          double ctr[NC];
#pragma unroll
          for (int c = 0; c < NC; ++c) ctr[c] = pl1[c * NS + cen];
          body(((ke + 1) * g.nny + y) * g.nnx + x, pend, ctr);
        }
      }
      __syncthreads();
    }
  }
}
