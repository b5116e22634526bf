// Mixed-precision momentum solve of the 2D step with on-the-fly convection:
// FP64 iterative refinement around a fixed number of FP32 BiCGSTAB iterations.
//
// The system is the momentum solve of solvers/standard.py:14-43, A U = b with
// A = Kd + cc Ce(U_n) (Kd = (rho/dt) Me + theta mu Le shared, cc = theta rho)
// and identity rows on gamma_d. Outer (FP64): r = b - A x with the FP64 tiled
// operator (k_conv_apply), its norm, x += d. Inner (FP32 vectors, FP32 Gauss
// factors, FP32 sums within an element row, FP64 dot products): `inner`
// iterations of the reference's BiCGSTAB (utils/jax_iterative_solvers.py:
// 123-167, no preconditioner) on A d = r from d = 0. The FP32 operator is
// applied one thread per node: the thread evaluates the rows of its incident
// elements from the element's factors and its nodes' values (no staging; the
// element rows are recomputed per node, which keeps the kernel a plain
// streaming loop). The whole refinement loop is one CUDA graph with a
// conditional WHILE node whose condition is set on the device.
#include <cstring>

#include "fem_b200.h"
#include "fem_args.cuh"
#include "fem_mg3.cuh"

#define MM_THREADS 256
#define MM_PARTS 4096
#define MM_WATCHDOG_NS 10000000000ull

struct MmScal {
  double tol;
  int max_cycles, cycles, status;
  double rr, bb, atol2;
  double rho, rho_next, alpha, omega;
  int out_iters, out_status;
  unsigned long long t0;
};

struct MmArgs {
  FemGrid g;
  FemQuadTab qt;
  const float* fq;       // FP32 Gauss-point factors, structure of arrays fq[k * ne + e]
  const double* Ash;     // the shared matrix Kd (nen x nen, device)
  float cc;              // coefficient of Ce
  const uint8_t* mask;   // ncomp * nn identity rows (or null)
  int ncomp;
};

// Row a of (Kd + cc Ce) x_e for element e (lattice (ex, ey)), component base x.
template <int KIND>
__device__ __forceinline__ float mm_row(const MmArgs& A, int ex, int ey, int a, const float* __restrict__ x) {
  constexpr int NEN = KI<KIND>::NEN, NQ = KQ<KIND>::NQ;
  const FemGrid& g = A.g;
  float xl[NEN];
#pragma unroll
  for (int b = 0; b < NEN; ++b) xl[b] = x[fem_elem_node(g, ex, ey, 0, b)];
  const size_t ne = g.ne, e = (size_t)ey * g.nex + ex;
  float sh = 0.0f;
#pragma unroll
  for (int b = 0; b < NEN; ++b) sh += (float)__ldg(A.Ash + a * NEN + b) * xl[b];
  float acc = 0.0f;
#pragma unroll 1
  for (int q = 0; q < NQ; ++q) {
    float xq = 0.0f, gx = 0.0f, gy = 0.0f;
#pragma unroll
    for (int b = 0; b < NEN; ++b) {
      xq += (float)A.qt.N[q][b] * xl[b];
      gx += (float)A.qt.dx[q][b] * xl[b];
      gy += (float)A.qt.dy[q][b] * xl[b];
    }
    const float s = (A.fq[(3 * q) * ne + e] * gx + A.fq[(3 * q + 1) * ne + e] * gy) + A.fq[(3 * q + 2) * ne + e] * xq;
    acc += (float)A.qt.N[q][a] * s;
  }
  return sh + A.cc * acc;
}

// y_c = A x_c (identity rows on the mask), per component; partials of <w1, y>
// (mode 1) or of <w1, y> and <y, y> (mode 2), over all components.
template <int KIND, int MODE>
__global__ void __launch_bounds__(MM_THREADS) k_mm_apply(const __grid_constant__ MmArgs A, const float* __restrict__ x,
                                                          float* __restrict__ y, const float* __restrict__ w1,
                                                          double* parts) {
  const FemGrid& g = A.g;
  const size_t N = g.nn;
  double acc[2] = {0.0, 0.0};
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < g.nn; n += gridDim.x * blockDim.x) {
    int ix, iy, iz;
    fem_ij(g, n, ix, iy, iz);
    for (int c = 0; c < A.ncomp; ++c) {
      const float* xc = x + c * N;
      float v = 0.0f;
      if (A.mask && A.mask[n + c * N]) {
        v = xc[n];
      } else {
        fem_incident_k<KIND>(g, ix, iy, 0, [&](int ie, int je, int, int, int a) { v += mm_row<KIND>(A, ie, je, a, xc); });
      }
      y[n + c * N] = v;
      acc[0] += (double)w1[n + c * N] * (double)v;
      if (MODE == 2) acc[1] += (double)v * (double)v;
    }
  }
  __shared__ double s[2][32];
#pragma unroll
  for (int k = 0; k < 2; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if ((threadIdx.x & 31) == 0) {
    s[0][threadIdx.x >> 5] = acc[0];
    s[1][threadIdx.x >> 5] = acc[1];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 0; k < MODE; ++k) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[k][w];
      parts[k * MM_PARTS + blockIdx.x] = t;
    }
  }
}

__device__ __forceinline__ double mm_sum(const double* __restrict__ part, int np) {
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
template <int NV>
__device__ __forceinline__ void mm_parts(double (&v)[NV], double* parts) {
  __shared__ double s[NV][32];
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) s[k][threadIdx.x >> 5] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[k][w];
      parts[k * MM_PARTS + blockIdx.x] = t;
    }
}

// p = r + beta (p - omega v), beta = (rho' / rho)(alpha / omega), rho' = sum of
// the r_hat . r partials (first iteration: p = v = 0, rho = alpha = omega = 1)
__global__ void k_mm_p(int n, const float* __restrict__ r, float* __restrict__ p, const float* __restrict__ v,
                       MmScal* sc, const double* __restrict__ prh, int np) {
  const double rhon = mm_sum(prh, np);
  double beta = (rhon / sc->rho) * (sc->alpha / sc->omega);
  if (!isfinite(beta)) beta = 0.0;
  const float b = (float)beta, om = (float)sc->omega;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = r[i] + b * (p[i] - om * v[i]);
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->rho_next = rhon;
}
// alpha = rho' / (r_hat . v); s = r - alpha v
__global__ void k_mm_s(int n, const float* __restrict__ r, const float* __restrict__ v, float* __restrict__ s,
                       MmScal* sc, const double* __restrict__ prv, int np) {
  const double rv = mm_sum(prv, np);
  double alpha = sc->rho_next / rv;
  if (!isfinite(alpha)) alpha = 0.0;
  const float a = (float)alpha;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s[i] = r[i] - a * v[i];
  if (blockIdx.x == 0 && threadIdx.x == 0) sc->alpha = alpha;
}
// omega = (t . s) / (t . t); d += alpha p + omega s; r = s - omega t; partials of r_hat . r
__global__ void k_mm_xr(int n, float* __restrict__ d, float* __restrict__ r, const float* __restrict__ p,
                        const float* __restrict__ s, const float* __restrict__ t, const float* __restrict__ rhat,
                        MmScal* sc, const double* __restrict__ pts, int np, double* parts) {
  const double ts = mm_sum(pts, np), tt = mm_sum(pts + MM_PARTS, np);
  double omega = ts / tt;
  if (!isfinite(omega)) omega = 0.0;
  const float a = (float)sc->alpha, om = (float)omega;
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    d[i] += a * p[i] + om * s[i];
    const float rn = s[i] - om * t[i];
    r[i] = rn;
    acc[0] += (double)rhat[i] * (double)rn;
  }
  mm_parts<1>(acc, parts);
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->omega = omega == 0.0 ? 1.0 : omega;  // a zero omega restarts the directions next time (beta = 0)
    sc->rho = sc->rho_next;
  }
}
// inner start: r_hat = r, p = v = d = 0, rho = alpha = omega = 1, partials of r_hat . r
__global__ void k_mm_init(int n, const float* __restrict__ r, float* __restrict__ rhat, float* __restrict__ p,
                          float* __restrict__ v, float* __restrict__ d, MmScal* sc, double* parts) {
  double acc[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    rhat[i] = r[i];
    p[i] = 0.0f;
    v[i] = 0.0f;
    d[i] = 0.0f;
    acc[0] += (double)r[i] * (double)r[i];
  }
  mm_parts<1>(acc, parts);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    sc->rho = 1.0;
    sc->alpha = 1.0;
    sc->omega = 1.0;
  }
}
// FP64 residual r = b - A x (identity rows on the mask; y = the FP64 operator
// applied to x) into FP32, partials of r . r and b . b
__global__ void k_mm_res(int n, const double* __restrict__ b, const double* __restrict__ x,
                         const double* __restrict__ y, const uint8_t* __restrict__ mask, float* __restrict__ r32,
                         double* parts) {
  double acc[2] = {0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double ri = b[i] - ((mask && mask[i]) ? x[i] : y[i]);
    r32[i] = (float)ri;
    acc[0] += ri * ri;
    acc[1] += b[i] * b[i];
  }
  mm_parts<2>(acc, parts);
}
__global__ void k_mm_add(int n, double* __restrict__ x, const float* __restrict__ d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += (double)d[i];
}
__global__ void k_mm_cvt(size_t n, const double* __restrict__ a, float* __restrict__ o) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    o[i] = (float)a[i];
}
__global__ void k_mm_set(MmScal* sc, double tol, int max_cycles) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sc->tol = tol;
  sc->max_cycles = max_cycles;
}
__device__ __forceinline__ unsigned long long mm_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// refinement control: first = prologue (cycles = 0), else one cycle done
__global__ void k_mm_ctl(MmScal* sc, int first, const double* __restrict__ prr, int np,
                         cudaGraphConditionalHandle h) {
  const double rr = mm_sum(prr, np);
  const double bb = first ? mm_sum(prr + MM_PARTS, np) : 0.0;
  if (threadIdx.x != 0) return;
  if (first) {
    sc->t0 = mm_now();
    sc->status = 0;
    sc->cycles = 0;
    sc->bb = bb;
    sc->atol2 = sc->tol * sc->tol * bb;
  } else {
    sc->cycles += 1;
  }
  sc->rr = rr;
  unsigned cond = (rr > sc->atol2 && sc->cycles < sc->max_cycles) ? 1u : 0u;
  if (!isfinite(rr) || !isfinite(sc->bb)) {
    sc->status |= FEM_STATUS_NONFINITE;
    cond = 0;
  }
  if (cond && mm_now() - sc->t0 > MM_WATCHDOG_NS) {
    sc->status |= FEM_STATUS_WATCHDOG;
    cond = 0;
  }
  cudaGraphSetConditional(h, cond);
}
__global__ void k_mm_finish(MmScal* sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int st = sc->status;
  if (!(sc->rr <= sc->atol2) && !(st & (FEM_STATUS_NONFINITE | FEM_STATUS_WATCHDOG))) st |= FEM_STATUS_MAXITER;
  sc->out_iters = sc->cycles;
  sc->out_status = st;
}

// ------------------------------------------------------------------ host ----

#define MM_TRY(...)             \
  do {                          \
    int _r = (__VA_ARGS__);     \
    if (_r) return _r;          \
  } while (0)
#define MM_CUDA(call)                                          \
  do {                                                         \
    cudaError_t _e = (call);                                   \
    if (_e != cudaSuccess) return fem_cuda_error(#call, _e);   \
  } while (0)

struct MixMom {
  FemGrid g;
  int ncomp = 2, nb = 0, cap = 1184, inner = 0;
  double cc = 0.0;                   // the graph's baked-in values
  const double *Kd = nullptr, *fq64 = nullptr;
  const uint8_t* mask = nullptr;
  float* f32 = nullptr;   // FP32 factors
  float* v32 = nullptr;   // r, rhat, p, v, s, t, d (ncomp * nn each)
  double* y64 = nullptr;  // the FP64 operator applied to x
  double *x64 = nullptr, *b64 = nullptr;
  double* parts = nullptr;
  MmScal* sc = nullptr;
  cudaStream_t s2 = nullptr;
  cudaGraphExec_t exec = nullptr;
};

void mixmom_destroy(MixMom* M) {
  if (!M) return;
  if (M->exec) cudaGraphExecDestroy(M->exec);
  void* ps[] = {M->f32, M->v32, M->y64, M->x64, M->b64, M->parts, M->sc};
  for (void* p : ps)
    if (p) cudaFree(p);
  if (M->s2) cudaStreamDestroy(M->s2);
  delete M;
}

int mixmom_create(MixMom** out, const FemGrid& g, int ncomp, int nq, int sms) {
  *out = nullptr;
  if (g.kind == FEM_HEX8) return FEM_E_ARG;
  MixMom* M = new MixMom();
  M->g = g;
  M->ncomp = ncomp;
  M->cap = sms * 8;
  const size_t n = (size_t)ncomp * g.nn;
  bool ok = cudaMalloc(&M->f32, sizeof(float) * 3 * nq * (size_t)g.ne) == cudaSuccess &&
            cudaMalloc(&M->v32, sizeof(float) * 7 * n) == cudaSuccess &&
            cudaMalloc(&M->y64, sizeof(double) * n) == cudaSuccess &&
            cudaMalloc(&M->x64, sizeof(double) * n) == cudaSuccess &&
            cudaMalloc(&M->b64, sizeof(double) * n) == cudaSuccess &&
            cudaMalloc(&M->parts, sizeof(double) * 3 * MM_PARTS) == cudaSuccess &&
            cudaMalloc(&M->sc, sizeof(MmScal)) == cudaSuccess &&
            cudaStreamCreateWithFlags(&M->s2, cudaStreamNonBlocking) == cudaSuccess;
  if (!ok) {
    mixmom_destroy(M);
    return fem_cuda_error("mixed momentum buffers", cudaGetLastError());
  }
  *out = M;
  return FEM_OK;
}

template <int KIND>
static int mm_inner_iter(const MixMom* M, const MmArgs& A, cudaStream_t s) {
  const int n = M->ncomp * M->g.nn, ge = fem_nblocks(n, MM_THREADS, M->cap), gn = fem_nblocks(M->g.nn, MM_THREADS, M->cap);
  const size_t N = n;
  float *r = M->v32, *rhat = r + N, *p = rhat + N, *v = p + N, *sv = v + N, *t = sv + N, *d = t + N;
  double *pa = M->parts, *pb = M->parts + MM_PARTS;  // pa: r_hat . r (and t . s / t . t), pb: r_hat . v
  k_mm_p<<<ge, MM_THREADS, 0, s>>>(n, r, p, v, M->sc, pa, ge);
  k_mm_apply<KIND, 1><<<gn, MM_THREADS, 0, s>>>(A, p, v, rhat, pb);
  k_mm_s<<<ge, MM_THREADS, 0, s>>>(n, r, v, sv, M->sc, pb, gn);
  k_mm_apply<KIND, 2><<<gn, MM_THREADS, 0, s>>>(A, sv, t, sv, pb);
  k_mm_xr<<<ge, MM_THREADS, 0, s>>>(n, d, r, p, sv, t, rhat, M->sc, pb, gn, pa);
  return fem_after_launch("k_mm_iter");
}

// The refinement graph: x64, b64 in M; the FP64 operator through
// fem_launch_conv_apply (Kd, cc, factors fq64); FP32 inner iterations.
template <int KIND>
static int mm_build(MixMom* M, const MmArgs& A, const FemQuadTab& qt, const double* fq64, const double* Kd,
                    double cc, int sms, cudaStream_t cs) {
  const int n = M->ncomp * M->g.nn, ge = fem_nblocks(n, MM_THREADS, M->cap);
  const size_t N = n;
  float *r = M->v32, *rhat = r + N, *p = rhat + N, *v = p + N, *d = v + 3 * N;
  double* prr = M->parts + MM_PARTS;  // the FP64 residual's r . r and b . b partials: slots 1, 2
  auto res64 = [&](cudaStream_t st) -> int {
    MM_TRY(fem_launch_conv_apply(M->ncomp, M->g, qt, fq64, cc, 1.0, Kd, M->x64, M->y64, sms, st));
    k_mm_res<<<ge, MM_THREADS, 0, st>>>(n, M->b64, M->x64, M->y64, A.mask, r, prr);
    return fem_after_launch("k_mm_res");
  };
  MM_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int rc = FEM_OK;
  cudaStreamCaptureStatus st;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  cudaGraphConditionalHandle h = 0;
  if (cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &ndeps) != cudaSuccess ||
      cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) != cudaSuccess)
    rc = fem_cuda_error("conditional handle", cudaGetLastError());
  if (rc == FEM_OK) {
    rc = res64(cs);
    if (rc == FEM_OK) {
      k_mm_ctl<<<1, 256, 0, cs>>>(M->sc, 1, prr, ge, h);
      rc = fem_after_launch("k_mm_ctl");
    }
  }
  if (rc == FEM_OK) {
    cudaGraphNode_t cnode = nullptr;
    if (cudaStreamGetCaptureInfo(cs, &st, nullptr, &g, &deps, &ndeps) != cudaSuccess) {
      rc = fem_cuda_error("cudaStreamGetCaptureInfo", cudaGetLastError());
    } else {
      cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      if (cudaGraphAddNode(&cnode, g, deps, ndeps, &cp) != cudaSuccess) {
        rc = fem_cuda_error("cudaGraphAddNode(conditional)", cudaGetLastError());
      } else if (cudaStreamUpdateCaptureDependencies(cs, &cnode, 1, cudaStreamSetCaptureDependencies) !=
                 cudaSuccess) {
        rc = fem_cuda_error("cudaStreamUpdateCaptureDependencies", cudaGetLastError());
      } else if (cudaStreamBeginCaptureToGraph(M->s2, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        rc = fem_cuda_error("cudaStreamBeginCaptureToGraph", cudaGetLastError());
      } else {
        cudaStream_t bs = M->s2;
        k_mm_init<<<ge, MM_THREADS, 0, bs>>>(n, r, rhat, p, v, d, M->sc, M->parts);
        rc = fem_after_launch("k_mm_init");
        for (int k = 0; k < M->inner && rc == FEM_OK; ++k) rc = mm_inner_iter<KIND>(M, A, bs);
        if (rc == FEM_OK) {
          k_mm_add<<<ge, MM_THREADS, 0, bs>>>(n, M->x64, d);
          rc = res64(bs);
        }
        if (rc == FEM_OK) {
          k_mm_ctl<<<1, 256, 0, bs>>>(M->sc, 0, prr, ge, h);
          rc = fem_after_launch("k_mm_ctl");
        }
        cudaGraph_t bout = nullptr;
        const cudaError_t e = cudaStreamEndCapture(bs, &bout);
        if (rc == FEM_OK && e != cudaSuccess) rc = fem_cuda_error("cudaStreamEndCapture(body)", e);
      }
    }
  }
  if (rc == FEM_OK) {
    k_mm_finish<<<1, 32, 0, cs>>>(M->sc);
    rc = fem_after_launch("k_mm_finish");
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(cs, &graph);
  if (rc == FEM_OK && e != cudaSuccess) rc = fem_cuda_error("cudaStreamEndCapture", e);
  if (rc == FEM_OK && cudaGraphInstantiate(&M->exec, graph, 0) != cudaSuccess) {
    rc = fem_cuda_error("cudaGraphInstantiate", cudaGetLastError());
    M->exec = nullptr;
  }
  if (graph) cudaGraphDestroy(graph);
  cudaGetLastError();
  return rc;
}

// Solve (Kd + cc Ce) x = b (identity rows on mask) to ||b - A x|| <= tol ||b||
// by FP64 refinement around `inner` FP32 BiCGSTAB iterations per cycle. Kd is
// the device shared matrix (FP64), fq64 the FP64 Gauss factors of Ce (already
// formed for the step). The graph bakes in the pointers, cc and `inner`, so a
// change of those rebuilds it; b and x go through M's own buffers.
int mixmom_solve(MixMom* M, const FemQuadTab& qt, const double* fq64, const double* Kd, double cc,
                 const uint8_t* mask, const double* b, double* x, double tol, int inner, int max_cycles,
                 int* cycles, int* status, int sms, cudaStream_t s, cudaStream_t cs) {
  const FemGrid& g = M->g;
  const int nq = g.kind == FEM_Q2_2D ? 9 : 4;
  const size_t n = (size_t)M->ncomp * g.nn;
  if (M->exec && (M->inner != inner || M->cc != cc || M->Kd != Kd || M->mask != mask || M->fq64 != fq64)) {
    cudaGraphExecDestroy(M->exec);
    M->exec = nullptr;
  }
  if (!M->exec) {
    MmArgs A;
    memset(&A, 0, sizeof(A));
    A.g = g;
    A.qt = qt;
    A.fq = M->f32;
    A.Ash = Kd;
    A.cc = (float)cc;
    A.mask = mask;
    A.ncomp = M->ncomp;
    M->inner = inner;
    M->cc = cc;
    M->Kd = Kd;
    M->mask = mask;
    M->fq64 = fq64;
    if (g.kind == FEM_Q1_2D)
      MM_TRY(mm_build<FEM_Q1_2D>(M, A, qt, fq64, Kd, cc, sms, cs));
    else
      MM_TRY(mm_build<FEM_Q2_2D>(M, A, qt, fq64, Kd, cc, sms, cs));
  }
  // the step's FP32 factors, the per-call scalars and the input vectors
  k_mm_cvt<<<fem_nblocks((long long)3 * nq * g.ne, MM_THREADS, M->cap), MM_THREADS, 0, s>>>(
      (size_t)3 * nq * g.ne, fq64, M->f32);
  k_mm_set<<<1, 32, 0, s>>>(M->sc, tol, max_cycles);
  MM_TRY(fem_after_launch("k_mm_set"));
  MM_CUDA(cudaMemcpyAsync(M->b64, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  MM_CUDA(cudaMemcpyAsync(M->x64, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  MM_CUDA(cudaGraphLaunch(M->exec, s));
  MM_CUDA(cudaMemcpyAsync(x, M->x64, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  if (cycles) MM_CUDA(cudaMemcpyAsync(cycles, &M->sc->out_iters, sizeof(int), cudaMemcpyDeviceToDevice, s));
  if (status) MM_CUDA(cudaMemcpyAsync(status, &M->sc->out_status, sizeof(int), cudaMemcpyDeviceToDevice, s));
  return FEM_OK;
}
