// Host side of libfemb200: contexts, workspace, cooperative launches and the
// extern "C" entry points declared in include/fem_b200.h.
#include <algorithm>
#include <climits>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include <nvtx3/nvToolsExt.h>

#include <vector>
#include "fem_b200.h"
#include "fem_args.cuh"
#include "fem_mg3.cuh"

// NVTX range over one host entry point (a no-op unless a profiler is attached)
struct FemRange {
  explicit FemRange(const char* name) { nvtxRangePushA(name); }
  ~FemRange() { nvtxRangePop(); }
};

static std::atomic<long long> g_launches{0};
static thread_local char g_err[256] = "";

static int set_err(const char* where, cudaError_t e) {
  snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
  return FEM_E_CUDA;
}
#define FEM_CHECK(call)                             \
  do {                                              \
    cudaError_t _e = (call);                        \
    if (_e != cudaSuccess) return set_err(#call, _e); \
  } while (0)
int fem_cuda_error(const char* where, cudaError_t e) { return set_err(where, e); }
char* fem_err_buf() { return g_err; }
int fem_after_launch(const char* what) {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(what, e);
  return FEM_OK;
}
#define FEM_TRY(call)      \
  do {                     \
    int _rc = (call);      \
    if (_rc) return _rc;   \
  } while (0)

static inline int nblocks(long long n, int threads, int cap = 148 * 16) { return fem_nblocks(n, threads, cap); }

static bool make_grid(int kind, int periodic, int nex, int ney, int nez, FemGrid& g) {
  if (nex < 1 || ney < 1) return false;
  memset(&g, 0, sizeof(g));
  g.kind = kind;
  g.periodic = periodic ? 1 : 0;
  g.nex = nex;
  g.ney = ney;
  g.nez = 1;
  if (kind == FEM_Q1_2D) {
    g.nnx = periodic ? nex : nex + 1;
    g.nny = periodic ? ney : ney + 1;
    g.nnz = 1;
    g.nen = 4;
  } else if (kind == FEM_Q2_2D) {
    g.nnx = periodic ? 2 * nex : 2 * nex + 1;
    g.nny = periodic ? 2 * ney : 2 * ney + 1;
    g.nnz = 1;
    g.nen = 9;
  } else if (kind == FEM_HEX8) {
    if (periodic || nez < 1) return false;
    g.nez = nez;
    g.nnx = nex + 1;
    g.nny = ney + 1;
    g.nnz = nez + 1;
    g.nen = 8;
  } else {
    return false;
  }
  const long long nn = (long long)g.nnx * g.nny * g.nnz, ne = (long long)nex * ney * g.nez;
  if (nn > (1LL << 31) - 1 || ne * g.nen > (1LL << 31) - 1) return false;
  g.nn = (int)nn;
  g.ne = (int)ne;
  return true;
}

static FemLattice lattice_of(const FemGrid& g) {
  FemLattice L;
  const int s = (g.kind == FEM_Q2_2D) ? 2 : 1;
  L.nx = s * g.nex + 1;
  L.ny = s * g.ney + 1;
  L.periodic = g.periodic;
  return L;
}


#define FEM_FLAG_BOUNDARY_SKIPPED 0
// FP32 BiCGSTAB iterations per refinement cycle of the mixed momentum solve
#define FEM_MIXED_MOMENTUM_INNER 3

struct CtxLevel {
  FemGrid g;
  double *Le = nullptr, *Leoff = nullptr, *diag = nullptr, *x = nullptr, *r = nullptr, *t = nullptr;
  double *tab = nullptr, *tab_off = nullptr, *invD = nullptr, *winvD = nullptr;
  uint8_t* pin = nullptr;
  double sum_invD = 0.0, sum_colw = 0.0, sum_rc = 0.0, sum_rcD = 0.0;
};

struct fem_ctx {
  int device = 0, sms = 148;
  FemGrid g;
  int ndim = 2, nq = 4;
  double lx = 1, ly = 1, lz = 1;
  // element data
  double *coords = nullptr, *wq = nullptr, *N = nullptr, *dN = nullptr;
  double *Me = nullptr, *Le = nullptr, *Leoff = nullptr, *Ge = nullptr, *M = nullptr, *Ldiag = nullptr;
  double* Kd = nullptr;  // combined shared matrix of a solve (nen*nen)
  // boundary sets
  uint8_t *dmask = nullptr, *pmask = nullptr, *aipin = nullptr;
  int has_dmask = 0, set_zeroP = 1;
  // multigrid
  int nlev = 0, block_from = 0;
  double coarse_tol = 1e-8;
  CtxLevel lv[FEM_MAX_LEVELS];
  double *cr = nullptr, *cp = nullptr, *cq = nullptr;  // coarse CG scratch
  // barrier / reduction state
  unsigned int* bar = nullptr;
  int* err = nullptr;
  double* partials = nullptr;
  int max_coop = 148;       // CTAs of the persistent cooperative launches
  int coop_capacity = 148;  // upper bound of max_coop (co-resident capacity)
  // vectors (nn or ndim*nn)
  double *pr = nullptr, *pz = nullptr, *pp0 = nullptr, *pp1 = nullptr, *pAp = nullptr, *pb = nullptr;  // CG
  double *br = nullptr, *brh = nullptr, *bp0 = nullptr, *bp1 = nullptr, *bq0 = nullptr, *bq1 = nullptr,
         *bt = nullptr;                                                                      // BiCGSTAB
  double *rhsU = nullptr, *Uhat = nullptr, *gPn = nullptr, *Ustar = nullptr, *rhsP = nullptr;  // step
  double *Ce = nullptr, *Ce2 = nullptr, *Ct = nullptr, *Mt = nullptr, *Ek = nullptr, *tau = nullptr;  // per element
  double *dotpart = nullptr, *Fe = nullptr;
  double* vcv = nullptr;   // (mu Le + rho Ce(U_n)) U_n of the on-the-fly step (ndim*nn)
  double* cvf = nullptr;   // Gauss-point factors of Ce(U_n) (3 nq per element, structure of arrays)
  double* ebe_tab = nullptr;  // stencil table of the shared matrix of fem_ebe_apply
  FemQuadTab qt{};         // Gauss table of the mesh (2D), for on-the-fly convection
  int conv_otf = 0;        // fem_step4 applies Ce without building it
  size_t Fe_cap = 0;       // face entries the boundary-flux scratch holds
  int *bs_cnt = nullptr, *bs_off = nullptr, *bs_list = nullptr;  // boundary scatter CSR (nn, nn + 1 + scan chunks, Fe_cap)
  int* flags = nullptr;  // device ints: [FEM_FLAG_BOUNDARY_SKIPPED] faces skipped by the last flux call,
                         // [1], [2] cycles and status of the last hex8 mixed solve
  // optional stage timing
  int timing = 0, nev = 0;
  cudaEvent_t ev[16] = {};
  unsigned long long* trace = nullptr;
  int trace_cap = 0;
  cudaStream_t cap_stream = nullptr;  // private stream for graph captures (fem_step4_graph)
  float* mx32 = nullptr;              // FP32 vectors of the mixed-precision solve (first use)
  double* mx64 = nullptr;             // its partial sums and scalars
  MxGraphCache mxg;                   // its captured inner solve
  double* step_tab = nullptr;         // hex8: stencil tables of Me, Ge_d, Ge_d^T (7 x FEM_TAB_MAX)
  Mg3* mg3 = nullptr;                 // hex8 multigrid hierarchy and its solve graphs
  Mg3* mg2 = nullptr;                 // 2D hierarchy of the graph-driven mixed-precision solve (first use)
  MixMom* mixmom = nullptr;           // the mixed-precision momentum solve of fem_step4 (2D, first use)
  double* vjp = nullptr;              // per-element scratch of fem_conv_vjp (first use)
  double* vjp2 = nullptr;             // per-element scratch of fem_transport_vjp (first use)
  int precision = FEM_PRECISION_FP64; // pressure solve of fem_step4
  int mx_inner = 6, mx_cycles = 10;   // its mixed-precision parameters
};

struct fem_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
};

static inline void stage_mark(fem_ctx* c, cudaStream_t s) {
  if (c->timing && c->nev < 16) cudaEventRecord(c->ev[c->nev++], s);
}

template <class T>
static int dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    set_err("cudaMalloc", e);
    return FEM_E_OOM;
  }
  return FEM_OK;
}
#define FEM_ALLOC(p, n)                 \
  do {                                  \
    int _r = dalloc(&(p), (size_t)(n)); \
    if (_r) return _r;                  \
  } while (0)

static int ctx_grid_for(const fem_ctx* c, long long work) {
  // enough CTAs for ~1 node per thread, capped by co-residency
  return nblocks(work, FEM_THREADS, c->max_coop);
}

// --------------------------------------------------------------- mesh ----

extern "C" int fem_mesh_counts(const fem_mesh_desc* m, int* nn, int* ne, int* nen) {
  if (!m) return FEM_E_ARG;
  FemGrid g;
  if (!make_grid(m->kind, m->periodic, m->nex, m->ney, m->nez, g)) return FEM_E_ARG;
  if (nn) *nn = g.nn;
  if (ne) *ne = g.ne;
  if (nen) *nen = g.nen;
  return FEM_OK;
}

static void spacings(const fem_mesh_desc* m, double& dx, double& dy, double& dz) {
  dx = m->lx / m->nex;
  dy = m->ly / m->ney;
  dz = (m->kind == FEM_HEX8) ? m->lz / m->nez : 0.0;
}

extern "C" int fem_mesh_generate(const fem_mesh_desc* m, double* coords, int64_t* nconn, cudaStream_t s) {
  if (!m || !coords) return FEM_E_ARG;
  FemGrid g;
  if (!make_grid(m->kind, m->periodic, m->nex, m->ney, m->nez, g)) return FEM_E_ARG;
  double dx, dy, dz;
  spacings(m, dx, dy, dz);
  FEM_TRY(fem_launch_mesh_generate(g, dx, dy, dz, coords, nconn, s));
  return FEM_OK;
}

extern "C" int fem_shape_functions(int family, const double* coords, double* wq, double* N, double* Nderiv,
                                   cudaStream_t s) {
  if (family < 0 || family > 4 || !coords || !wq || !N || !Nderiv) return FEM_E_ARG;
  return fem_launch_shape_functions(family, coords, wq, N, Nderiv, s);
}

// element-0 coordinates of a structured mesh (host computed, tiny)
static void elem0_coords(const FemGrid& g, double dx, double dy, double dz, double* out) {
  const int s = (g.kind == FEM_Q2_2D) ? 2 : 1;
  const int dim = (g.kind == FEM_HEX8) ? 3 : 2;
  static const int q2i[9] = {0, 1, 2, 2, 2, 1, 0, 0, 1}, q2j[9] = {0, 0, 0, 1, 2, 2, 2, 1, 1};
  static const int q1i[4] = {0, 1, 1, 0}, q1j[4] = {0, 0, 1, 1};
  for (int a = 0; a < g.nen; ++a) {
    int i, j, k;
    if (g.kind == FEM_Q2_2D) {
      i = q2i[a]; j = q2j[a]; k = 0;
    } else {
      i = q1i[a & 3]; j = q1j[a & 3]; k = a >> 2;
    }
    if (s == 2) {
      out[a * dim + 0] = i * dx / 2;
      out[a * dim + 1] = j * dy / 2;
    } else {
      out[a * dim + 0] = i * dx;
      out[a * dim + 1] = j * dy;
      if (dim == 3) out[a * 3 + 2] = k * dz;
    }
  }
}

// Element data of a grid: shape functions on element 0, Me, Le, Le_off, Ge, diag.
static int element_setup(const FemGrid& g, double dx, double dy, double dz, double* tmp_coords, double* wq,
                         double* N, double* dN, double* Me, double* Le, double* Leoff, double* Ge, double* M,
                         double* Ldiag, int ndim, cudaStream_t s) {
  double hc[27];
  elem0_coords(g, dx, dy, dz, hc);
  const int dim = (g.kind == FEM_HEX8) ? 3 : 2;
  FEM_CHECK(cudaMemcpyAsync(tmp_coords, hc, sizeof(double) * g.nen * dim, cudaMemcpyHostToDevice, s));
  const int family = g.kind == FEM_Q1_2D ? 0 : (g.kind == FEM_Q2_2D ? 1 : 2);
  FEM_TRY(fem_launch_shape_functions(family, tmp_coords, wq, N, dN, s));
  FEM_TRY(fem_launch_element_matrices(g.nen, g.nen, dim, wq, N, dN, Me, Le, Leoff, Ge, s));
  FEM_TRY(fem_launch_assemble_diag(g, ndim, Me, Le, M, Ldiag, s));
  // the copy source hc lives on this stack frame: finish before returning
  FEM_CHECK(cudaStreamSynchronize(s));
  return FEM_OK;
}

// ------------------------------------------------------------ context ----

extern "C" void fem_ctx_destroy(fem_ctx* c) {
  if (!c) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  for (int i = 0; i < 16; ++i)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  if (c->mxg.exec) cudaGraphExecDestroy(c->mxg.exec);
  if (c->mx32) cudaFree(c->mx32);
  if (c->mx64) cudaFree(c->mx64);
  mg3_destroy(c->mg3);
  mg3_destroy(c->mg2);
  mixmom_destroy(c->mixmom);
  void* ptrs[] = {c->coords, c->wq, c->N, c->dN, c->Me, c->Le, c->Leoff, c->Ge, c->M, c->Ldiag, c->Kd,
                  c->dmask, c->pmask, c->aipin, c->cr, c->cp, c->cq, c->bar, c->err, c->partials, c->pr,
                  c->pz, c->pp0, c->pp1, c->pAp, c->pb, c->br, c->brh, c->bp0, c->bp1, c->bq0, c->bq1, c->bt,
                  c->rhsU, c->Uhat, c->gPn, c->Ustar, c->rhsP, c->Ce, c->Ce2, c->Ct, c->Mt, c->Ek, c->tau,
                  c->dotpart, c->Fe, c->flags, c->vcv, c->cvf, c->ebe_tab, c->bs_cnt, c->bs_off, c->bs_list, c->vjp, c->vjp2,
                  c->step_tab};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int l = 0; l < FEM_MAX_LEVELS; ++l) {
    CtxLevel& L = c->lv[l];
    void* lp[] = {L.Le, L.Leoff, L.diag, L.x, L.t, L.pin, (l > 0) ? L.r : nullptr, L.tab, L.tab_off, L.invD, L.winvD};
    for (void* p : lp)
      if (p) cudaFree(p);
  }
  cudaSetDevice(prev);
  delete c;
}

// The 1D factors of a Q2 Gauss table (see FemQuadTab): by partition of unity,
// nx[q][i] = N[q][(i,1)] / sum_i' N[q][(i',1)] and ny[q][j] likewise along the
// middle column; the derivative factors divide dx / dy by the other direction's
// middle value. Gauss points are grouped into columns qx and rows qy by equal
// factors, and every entry of N, dx and dy is checked against the products
// (relative 1e-12). Returns false if the table does not factor.
static bool q2_tensor_factors(FemQuadTab& T) {
  int node[3][3];
  for (int b = 0; b < 9; ++b) node[(FEM_Q2_DI >> (2 * b)) & 3u][(FEM_Q2_DJ >> (2 * b)) & 3u] = b;  // [i][j]
  double fx[9][3], fy[9][3], gx[9][3], gy[9][3];
  for (int q = 0; q < 9; ++q) {
    double sx = 0.0, sy = 0.0;
    for (int k = 0; k < 3; ++k) {
      sx += T.N[q][node[k][1]];
      sy += T.N[q][node[1][k]];
    }
    if (std::fabs(sx) < 1e-6 || std::fabs(sy) < 1e-6) return false;
    const double mx = T.N[q][node[1][1]] / sy, my = T.N[q][node[1][1]] / sx;  // nx[q][1], ny[q][1]
    if (std::fabs(mx) < 1e-6 || std::fabs(my) < 1e-6) return false;
    for (int k = 0; k < 3; ++k) {
      fx[q][k] = T.N[q][node[k][1]] / sx;
      fy[q][k] = T.N[q][node[1][k]] / sy;
      gx[q][k] = T.dx[q][node[k][1]] / sx;
      gy[q][k] = T.dy[q][node[1][k]] / sy;
    }
  }
  auto same = [](const double* a, const double* b) {
    for (int k = 0; k < 3; ++k)
      if (std::fabs(a[k] - b[k]) > 1e-12 * (1.0 + std::fabs(a[k]))) return false;
    return true;
  };
  int colq[3], rowq[3], nc = 0, nr = 0, qxof[9], qyof[9];
  for (int q = 0; q < 9; ++q) {
    int cx = -1, cy = -1;
    for (int k = 0; k < nc; ++k)
      if (same(fx[q], fx[colq[k]])) cx = k;
    for (int k = 0; k < nr; ++k)
      if (same(fy[q], fy[rowq[k]])) cy = k;
    if (cx < 0) {
      if (nc == 3) return false;
      colq[nc] = q;
      cx = nc++;
    }
    if (cy < 0) {
      if (nr == 3) return false;
      rowq[nr] = q;
      cy = nr++;
    }
    qxof[q] = cx;
    qyof[q] = cy;
  }
  if (nc != 3 || nr != 3) return false;
  int seen[3][3] = {};
  for (int q = 0; q < 9; ++q) {
    if (seen[qyof[q]][qxof[q]]++) return false;
    T.qi[qyof[q]][qxof[q]] = q;
  }
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i) {
      T.nx[k][i] = fx[colq[k]][i];
      T.ddx[k][i] = gx[colq[k]][i];
      T.ny[k][i] = fy[rowq[k]][i];
      T.ddy[k][i] = gy[rowq[k]][i];
    }
  for (int q = 0; q < 9; ++q)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const int b = node[i][j], qx = qxof[q], qy = qyof[q];
        const double n = T.nx[qx][i] * T.ny[qy][j], ddx = T.ddx[qx][i] * T.ny[qy][j],
                     ddy = T.nx[qx][i] * T.ddy[qy][j];
        const double sc = 1.0 + std::fabs(T.dx[q][b]) + std::fabs(T.dy[q][b]);
        if (std::fabs(n - T.N[q][b]) > 1e-12 || std::fabs(ddx - T.dx[q][b]) > 1e-12 * sc ||
            std::fabs(ddy - T.dy[q][b]) > 1e-12 * sc)
          return false;
      }
  return true;
}

static int ctx_create_impl(const fem_mesh_desc* m, int device, fem_ctx* c) {
  if (!make_grid(m->kind, m->periodic, m->nex, m->ney, m->nez, c->g)) return FEM_E_ARG;
  c->device = device;
  FEM_CHECK(cudaSetDevice(device));
  cudaDeviceProp prop;
  FEM_CHECK(cudaGetDeviceProperties(&prop, device));
  c->sms = prop.multiProcessorCount;
  int occ_cg = 0, occ_bi = 0;
  if (fem_coop_occupancy_cg(&occ_cg) || fem_coop_occupancy_bi(&occ_bi)) return set_err("occupancy", cudaGetLastError());
  const int occ = std::max(1, std::min(occ_cg, occ_bi));
  c->max_coop = c->sms * occ;
  const char* ev = getenv("FEM_MAX_CTAS");
  if (ev && atoi(ev) > 0) c->max_coop = std::min(c->max_coop, atoi(ev));
  c->coop_capacity = c->max_coop;  // partials are sized for this many CTAs
  const FemGrid& g = c->g;
  c->ndim = (g.kind == FEM_HEX8) ? 3 : 2;
  c->nq = g.nen;
  c->lx = m->lx;
  c->ly = m->ly;
  c->lz = m->lz;
  const int nen = g.nen, nd = c->ndim;
  const size_t nn = g.nn, vn = (size_t)nd * nn, per = (size_t)nen * nen;
  FEM_ALLOC(c->coords, nn * nd);
  FEM_ALLOC(c->wq, c->nq);
  FEM_ALLOC(c->N, c->nq * nen);
  FEM_ALLOC(c->dN, c->nq * nd * nen);
  FEM_ALLOC(c->Me, per);
  FEM_ALLOC(c->Le, per);
  FEM_ALLOC(c->Leoff, per);
  FEM_ALLOC(c->Ge, nd * per);
  FEM_ALLOC(c->Kd, per);
  FEM_ALLOC(c->M, vn);
  FEM_ALLOC(c->Ldiag, nn);
  FEM_ALLOC(c->dmask, vn);
  FEM_ALLOC(c->pmask, nn);
  FEM_ALLOC(c->aipin, nn);
  FEM_ALLOC(c->bar, 2);
  FEM_ALLOC(c->err, 1);
  FEM_ALLOC(c->partials, (size_t)FEM_NSLOTS * c->max_coop);
  FEM_ALLOC(c->flags, 16);
  for (double** p : {&c->pr, &c->pz, &c->pp0, &c->pp1, &c->pAp, &c->pb, &c->rhsP}) FEM_ALLOC(*p, nn);
  for (double** p : {&c->br, &c->brh, &c->bp0, &c->bp1, &c->bq0, &c->bq1, &c->bt, &c->rhsU, &c->Uhat, &c->gPn,
                     &c->Ustar})
    FEM_ALLOC(*p, vn);
  FEM_ALLOC(c->Ce, (size_t)g.ne * per);
  FEM_ALLOC(c->vcv, vn);
  FEM_ALLOC(c->ebe_tab, FEM_TAB_MAX);
  FEM_ALLOC(c->cvf, g.kind == FEM_HEX8 ? (size_t)FEM_C3_NF * g.ne : (size_t)3 * c->nq * g.ne);
  FEM_ALLOC(c->dotpart, 4096);
  cudaStream_t s = 0;
  FEM_CHECK(cudaMemset(c->bar, 0, 2 * sizeof(unsigned int)));
  FEM_CHECK(cudaMemset(c->err, 0, sizeof(int)));
  FEM_CHECK(cudaMemset(c->flags, 0, 16 * sizeof(int)));
  FEM_CHECK(cudaMemset(c->dmask, 0, vn));
  FEM_CHECK(cudaMemset(c->pmask, 0, nn));
  FEM_CHECK(cudaMemset(c->aipin, 0, nn));
  FEM_CHECK(cudaMemset(c->pmask, 1, 1));  // default gamma_p = node 0 (setup/simulation.py:181)
  FEM_CHECK(cudaMemset(c->aipin, 1, 1));
  double dx, dy, dz;
  spacings(m, dx, dy, dz);
  FEM_TRY(fem_launch_mesh_generate(g, dx, dy, dz, c->coords, nullptr, s));
  double* tmp;
  FEM_ALLOC(tmp, 32);
  int rc = element_setup(g, dx, dy, dz, tmp, c->wq, c->N, c->dN, c->Me, c->Le, c->Leoff, c->Ge, c->M, c->Ldiag,
                         nd, s);
  cudaFree(tmp);
  if (rc) return rc;
  // level 0 of the hierarchy is the mesh itself (used by the plain CG path too)
  CtxLevel& L0 = c->lv[0];
  L0.g = g;
  L0.Le = nullptr;  // level 0 aliases the context matrices
  FEM_ALLOC(L0.x, nn);
  FEM_ALLOC(L0.t, nn);
  FEM_ALLOC(L0.tab, FEM_TAB_MAX);
  FEM_ALLOC(L0.tab_off, FEM_TAB_MAX);
  FEM_ALLOC(L0.invD, nn);
  FEM_ALLOC(L0.winvD, nn);
  L0.r = c->pr;
  FEM_TRY(fem_launch_stencil_build(g, c->Le, 0, 0, L0.tab, s));
  FEM_TRY(fem_launch_stencil_build(g, c->Le, 0, 1, L0.tab_off, s));
  FEM_TRY(fem_launch_invdiag(g.nn, c->Ldiag, c->pmask, L0.invD, L0.winvD, s));
  if (g.kind == FEM_HEX8) {
    // assembled stencils of the step's shared matrices: Me, Ge_d, Ge_d^T (StepArgs::tab3)
    FEM_ALLOC(c->step_tab, 7 * (size_t)FEM_TAB_MAX);
    FEM_TRY(fem_launch_stencil_build(g, c->Me, 0, 0, c->step_tab, s));
    for (int d = 0; d < 3; ++d) {
      FEM_TRY(fem_launch_stencil_build(g, c->Ge + d * 64, 0, 0, c->step_tab + (1 + d) * FEM_TAB_MAX, s));
      FEM_TRY(fem_launch_stencil_build(g, c->Ge + d * 64, 1, 0, c->step_tab + (4 + d) * FEM_TAB_MAX, s));
    }
  }
  c->nlev = 1;
  FEM_CHECK(cudaDeviceSynchronize());
  // Gauss table for the on-the-fly convection of fem_step4
  if (c->nq <= FEM_QT_MAX && nen <= FEM_QT_MAX) {
    double hw[FEM_QT_MAX], hN[FEM_QT_MAX * FEM_QT_MAX], hdN[3 * FEM_QT_MAX * FEM_QT_MAX];
    FEM_CHECK(cudaMemcpy(hw, c->wq, sizeof(double) * c->nq, cudaMemcpyDeviceToHost));
    FEM_CHECK(cudaMemcpy(hN, c->N, sizeof(double) * c->nq * nen, cudaMemcpyDeviceToHost));
    FEM_CHECK(cudaMemcpy(hdN, c->dN, sizeof(double) * c->nq * nd * nen, cudaMemcpyDeviceToHost));
    for (int q = 0; q < c->nq; ++q) {
      c->qt.w[q] = hw[q];
      for (int b = 0; b < nen; ++b) {
        c->qt.N[q][b] = hN[q * nen + b];
        c->qt.dx[q][b] = hdN[(q * nd + 0) * nen + b];
        c->qt.dy[q][b] = hdN[(q * nd + 1) * nen + b];
        c->qt.dz[q][b] = nd == 3 ? hdN[(q * nd + 2) * nen + b] : 0.0;
      }
    }
    // on the fly by default in 2D; hex8 keeps the explicit Ce unless asked
    // (FEM_CONV_OTF=1): on the 256 x 64 x 64 channel the explicit form ran
    // 96.2 steps/s against 83.4, its 64 coefficients per element costing less
    // than the on-the-fly element rows (~5x the FP64 work of a Ce row product)
    const char* ev = getenv("FEM_CONV_OTF");
    c->conv_otf = ev ? (atoi(ev) != 0) : (g.kind != FEM_HEX8);
    // Q2: the tensor factors of the on-the-fly operator; without them (a table
    // that does not factor) fem_step4 builds Ce explicitly
    if (g.kind == FEM_Q2_2D && !q2_tensor_factors(c->qt)) c->conv_otf = 0;
  }
  return FEM_OK;
}

extern "C" int fem_ctx_create(const fem_mesh_desc* m, int device, fem_ctx** out) {
  if (!m || !out) return FEM_E_ARG;
  fem_ctx* c = new (std::nothrow) fem_ctx();
  if (!c) return FEM_E_OOM;
  int rc = ctx_create_impl(m, device, c);
  if (rc) {
    fem_ctx_destroy(c);
    *out = nullptr;
    return rc;
  }
  *out = c;
  return FEM_OK;
}

extern "C" int fem_ctx_dims(const fem_ctx* c, int* nn, int* ne, int* nen, int* ndim, int* nq) {
  if (!c) return FEM_E_ARG;
  if (nn) *nn = c->g.nn;
  if (ne) *ne = c->g.ne;
  if (nen) *nen = c->g.nen;
  if (ndim) *ndim = c->ndim;
  if (nq) *nq = c->nq;
  return FEM_OK;
}

extern "C" int fem_ctx_element_data(const fem_ctx* c, double* wq, double* N, double* Nderiv, double* Me, double* Le,
                                    double* Ge, double* M, double* Ldiag, cudaStream_t s) {
  if (!c) return FEM_E_ARG;
  const size_t per = (size_t)c->g.nen * c->g.nen, d = sizeof(double);
  struct {
    double* dst;
    const double* src;
    size_t n;
  } cp[] = {{wq, c->wq, (size_t)c->nq},
            {N, c->N, (size_t)c->nq * c->g.nen},
            {Nderiv, c->dN, (size_t)c->nq * c->ndim * c->g.nen},
            {Me, c->Me, per},
            {Le, c->Le, per},
            {Ge, c->Ge, c->ndim * per},
            {M, c->M, (size_t)c->ndim * c->g.nn},
            {Ldiag, c->Ldiag, (size_t)c->g.nn}};
  for (auto& e : cp)
    if (e.dst) FEM_CHECK(cudaMemcpyAsync(e.dst, e.src, e.n * d, cudaMemcpyDeviceToDevice, s));
  return FEM_OK;
}

extern "C" int fem_ctx_set_bc(fem_ctx* c, const uint8_t* dmask, const uint8_t* pmask, int set_zeroP,
                              cudaStream_t s) {
  if (!c) return FEM_E_ARG;
  const size_t nn = c->g.nn;
  if (dmask) {
    FEM_CHECK(cudaMemcpyAsync(c->dmask, dmask, c->ndim * nn, cudaMemcpyDeviceToDevice, s));
    c->has_dmask = 1;
  } else {
    FEM_CHECK(cudaMemsetAsync(c->dmask, 0, c->ndim * nn, s));
    c->has_dmask = 0;
  }
  if (pmask) {
    FEM_CHECK(cudaMemcpyAsync(c->pmask, pmask, nn, cudaMemcpyDeviceToDevice, s));
    FEM_CHECK(cudaMemcpyAsync(c->aipin, pmask, nn, cudaMemcpyDeviceToDevice, s));
  }
  c->set_zeroP = set_zeroP ? 1 : 0;
  if (c->mg2) {  // its pins and mean-zero form follow the boundary sets
    FEM_CHECK(cudaStreamSynchronize(s));
    mg3_destroy(c->mg2);
    c->mg2 = nullptr;
  }
  FEM_TRY(fem_launch_invdiag(c->g.nn, c->Ldiag, c->pmask, c->lv[0].invD, c->lv[0].winvD, s));
  return FEM_OK;
}

extern "C" int fem_ctx_setup_multigrid(fem_ctx* c, int nlev, const uint8_t* level_pmasks, double coarse_tol,
                                       cudaStream_t s) {
  if (!c || nlev < 1 || nlev > FEM_MAX_LEVELS) return FEM_E_ARG;
  FEM_CHECK(cudaSetDevice(c->device));
  FEM_CHECK(cudaStreamSynchronize(s));
  if (c->g.kind == FEM_HEX8) {
    // hex8: the Chebyshev-smoothed hierarchy of k_mg3.cu (coarse_tol is unused:
    // its coarsest level is solved exactly)
    mg3_destroy(c->mg3);
    c->mg3 = nullptr;
    c->nlev = 1;
    FEM_TRY(mg3_setup(&c->mg3, c->g.nex, c->g.ney, c->g.nez, c->lx, c->ly, c->lz, nlev, level_pmasks, c->sms, s));
    c->nlev = nlev;
    c->coarse_tol = coarse_tol;
    return FEM_OK;
  }
  // a new hierarchy invalidates the mixed-precision solve's buffers and graph
  if (c->mxg.exec) {
    cudaGraphExecDestroy(c->mxg.exec);
    c->mxg.exec = nullptr;
  }
  if (c->mx32) {
    cudaFree(c->mx32);
    c->mx32 = nullptr;
  }
  if (c->mx64) {
    cudaFree(c->mx64);
    c->mx64 = nullptr;
  }
  mg3_destroy(c->mg2);
  c->mg2 = nullptr;
  const FemGrid& g0 = c->g;
  for (int l = 1; l < nlev; ++l)
    if ((g0.nex >> l) < 1 || (g0.ney >> l) < 1) return FEM_E_ARG;
  // release previous levels
  for (int l = 1; l < FEM_MAX_LEVELS; ++l) {
    CtxLevel& L = c->lv[l];
    void* lp[] = {L.Le, L.Leoff, L.diag, L.x, L.t, L.pin, L.r, L.tab, L.tab_off, L.invD, L.winvD};
    for (void* p : lp)
      if (p) cudaFree(p);
    L = CtxLevel();
  }
  if (c->lv[0].pin) cudaFree(c->lv[0].pin);
  c->lv[0].pin = nullptr;
  if (c->cr) cudaFree(c->cr), cudaFree(c->cp), cudaFree(c->cq);
  c->cr = c->cp = c->cq = nullptr;
  double* tmp;
  FEM_ALLOC(tmp, 64);
  double *wq, *N, *dN, *Me, *Ge, *Mtmp;
  FEM_ALLOC(wq, 9);
  FEM_ALLOC(N, 81);
  FEM_ALLOC(dN, 162);
  FEM_ALLOC(Me, 81);
  FEM_ALLOC(Ge, 162);
  size_t off = 0;
  int rc = FEM_OK;
  double* sums;
  FEM_ALLOC(sums, 4 * FEM_MAX_LEVELS);
  for (int l = 0; l < nlev && rc == FEM_OK; ++l) {
    CtxLevel& L = c->lv[l];
    if (l == 0) {
      L.g = g0;
    } else if (!make_grid(g0.kind, g0.periodic, g0.nex >> l, g0.ney >> l, 1, L.g)) {
      rc = FEM_E_ARG;
      break;
    }
    const size_t nn = L.g.nn;
    if (l > 0) {
      rc |= dalloc(&L.Le, 81);
      rc |= dalloc(&L.Leoff, 81);
      rc |= dalloc(&L.diag, nn);
      rc |= dalloc(&L.x, nn);
      rc |= dalloc(&L.r, nn);
      rc |= dalloc(&L.t, nn);
      if (rc) break;
      rc |= dalloc(&Mtmp, 2 * nn);
      if (rc) break;
      const double dx = c->lx / L.g.nex, dy = c->ly / L.g.ney;
      rc = element_setup(L.g, dx, dy, 0.0, tmp, wq, N, dN, Me, L.Le, L.Leoff, Ge, Mtmp, L.diag, 2, s);
      cudaFree(Mtmp);
      if (rc) break;
    }
    rc |= dalloc(&L.pin, nn);
    if (rc) break;
    if (level_pmasks) {
      FEM_CHECK(cudaMemcpyAsync(L.pin, level_pmasks + off, nn, cudaMemcpyDeviceToDevice, s));
    } else {
      FEM_CHECK(cudaMemsetAsync(L.pin, 0, nn, s));
      FEM_CHECK(cudaMemsetAsync(L.pin, 1, 1, s));
    }
    off += nn;
    const double* diag = (l == 0) ? c->Ldiag : L.diag;
    if (l > 0) {
      rc |= dalloc(&L.tab, FEM_TAB_MAX);
      rc |= dalloc(&L.tab_off, FEM_TAB_MAX);
      rc |= dalloc(&L.invD, nn);
      rc |= dalloc(&L.winvD, nn);
      if (rc) break;
      FEM_TRY(fem_launch_stencil_build(L.g, L.Le, 0, 0, L.tab, s));
      FEM_TRY(fem_launch_stencil_build(L.g, L.Le, 0, 1, L.tab_off, s));
    }
    FEM_TRY(fem_launch_invdiag(L.g.nn, diag, L.pin, L.invD, L.winvD, s));
    FEM_TRY(fem_launch_level_sums(L.g, lattice_of(L.g), diag, sums + 4 * l, s));
  }
  double hs[4 * FEM_MAX_LEVELS];
  if (rc == FEM_OK) {
    FEM_CHECK(cudaMemcpyAsync(hs, sums, sizeof(double) * 4 * nlev, cudaMemcpyDeviceToHost, s));
    FEM_CHECK(cudaStreamSynchronize(s));
  }
  cudaFree(tmp);
  cudaFree(wq);
  cudaFree(N);
  cudaFree(dN);
  cudaFree(Me);
  cudaFree(Ge);
  cudaFree(sums);
  if (rc) return rc;
  for (int l = 0; l < nlev; ++l) {
    c->lv[l].sum_invD = hs[4 * l];
    c->lv[l].sum_colw = hs[4 * l + 1];
    c->lv[l].sum_rc = hs[4 * l + 2];
    c->lv[l].sum_rcD = hs[4 * l + 3];
  }
  c->nlev = nlev;
  c->coarse_tol = coarse_tol;
  // coarse scratch for the in-CTA CG
  const size_t ncn = c->lv[nlev - 1].g.nn;
  FEM_ALLOC(c->cr, ncn);
  FEM_ALLOC(c->cp, ncn);
  FEM_ALLOC(c->cq, ncn);
  // First level handled by the coarse-level team: the coarsest levels of at
  // most FEM_MG_TEAM_NN nodes.
  int small = FEM_MG_TEAM_NN;
  if (const char* ev = getenv("FEM_MG_TEAM_NN")) small = atoi(ev);
  int bf = nlev - 1;
  for (int l = nlev - 2; l >= 0 && c->lv[l].g.nn <= small; --l) bf = l;
  c->block_from = bf;
  return FEM_OK;
}

extern "C" int fem_ctx_level_info(const fem_ctx* c, int level, int* nn, int* nnx, int* nny, int* nex, int* ney) {
  if (!c || level < 0 || level >= c->nlev) return FEM_E_ARG;
  if (c->g.kind == FEM_HEX8) {
    if (!c->mg3) return FEM_E_STATE;
    const Mg3Geo& G = c->mg3->geo[level];
    if (nn) *nn = c->mg3->nn[level];
    if (nnx) *nnx = G.nx;
    if (nny) *nny = G.ny;
    if (nex) *nex = G.nx - 1;
    if (ney) *ney = G.ny - 1;
    return FEM_OK;
  }
  const FemGrid& g = c->lv[level].g;
  FemLattice L = lattice_of(g);
  if (nn) *nn = g.nn;
  if (nnx) *nnx = L.nx;
  if (nny) *nny = L.ny;
  if (nex) *nex = g.nex;
  if (ney) *ney = g.ney;
  return FEM_OK;
}

// ------------------------------------------------------- element products ----

extern "C" int fem_ebe_apply(fem_ctx* c, int ncomp, const double* x, double* y, double alpha, const double* A,
                             double beta, const double* B, int transB, double gamma, const double* C,
                             cudaStream_t s) {
  if (!c || !x || !y || ncomp < 1 || ncomp > 3) return FEM_E_ARG;
  if (A && !B && !C) {
    // shared element matrix only: its assembled stencil (built on the device),
    // streamed in register strips, instead of the per-node element gather
    return fem_launch_shared_apply(ncomp, c->g, A, c->ebe_tab, alpha, x, y, c->sms, s);
  }
  const MatCombo m{A, alpha, B, beta, transB, C, gamma};
  return fem_launch_ebe(ncomp, c->g, m, x, y, s);
}

extern "C" int fem_grad_apply(fem_ctx* c, const double* P, const double* Ge, double* y, cudaStream_t s) {
  if (!c || !P || !y) return FEM_E_ARG;
  if (!Ge) Ge = c->Ge;
  return fem_launch_grad(c->ndim, c->g, Ge, P, y, s);
}

extern "C" int fem_div_apply(fem_ctx* c, const double* U, const double* Ge, double* y, cudaStream_t s) {
  if (!c || !U || !y) return FEM_E_ARG;
  if (!Ge) Ge = c->Ge;
  return fem_launch_div(c->ndim, c->g, Ge, U, y, s);
}

static FemQuad quad_of(const fem_ctx* c) { return FemQuad{c->wq, c->N, c->dN, c->nq, c->g.nen, c->ndim}; }
static FemQuad quad_with(const fem_ctx* c, const double* wq, const double* N, const double* dN) {
  FemQuad Q = quad_of(c);
  if (wq) Q.wq = wq;
  if (N) Q.N = N;
  if (dN) Q.dN = dN;
  return Q;
}

extern "C" int fem_convection_build(fem_ctx* c, const double* U, double beta, const double* wq, const double* N,
                                    const double* dN, double* Ce, cudaStream_t s) {
  if (!c || !U || !Ce) return FEM_E_ARG;
  return fem_launch_convection(c->g, quad_with(c, wq, N, dN), U, beta, 0, Ce, s);
}

extern "C" int fem_ctau_tilde_build(fem_ctx* c, const double* U, const double* wq, const double* N, const double* dN,
                                    double* Ct, cudaStream_t s) {
  if (!c || !U || !Ct) return FEM_E_ARG;
  return fem_launch_convection(c->g, quad_with(c, wq, N, dN), U, 0.0, 1, Ct, s);
}

extern "C" int fem_supg_tau(fem_ctx* c, const double* U, const double* Ce, const double* Ct, double D, double dt,
                            double r, const double* N, double* tau, cudaStream_t s) {
  if (!c || !U || !Ce || !Ct || !tau) return FEM_E_ARG;
  return fem_launch_supg_tau(c->g, quad_with(c, nullptr, N, nullptr), U, Ce, Ct, D, dt, r, tau, s);
}

extern "C" int fem_element_matrices(int nq, int nen, int dim, const double* wq, const double* N, const double* dN,
                                    double* Me, double* Le, double* Leoff, double* Ge, cudaStream_t s) {
  if (nq < 1 || nq > 27 || nen < 1 || nen > 9 || dim < 1 || dim > 3 || !wq || !N || !dN || !Me || !Le || !Leoff ||
      !Ge)
    return FEM_E_ARG;
  return fem_launch_element_matrices(nq, nen, dim, wq, N, dN, Me, Le, Leoff, Ge, s);
}

extern "C" int fem_assemble_diag(fem_ctx* c, const double* Me, const double* Le, int ndim, double* M, double* Ldiag,
                                 cudaStream_t s) {
  if (!c || ndim < 1 || ndim > 3 || (Me && !M) || (Le && !Ldiag) || (!Me && !Le)) return FEM_E_ARG;
  return fem_launch_assemble_diag(c->g, ndim, Me, Le, Me ? M : nullptr, Le ? Ldiag : nullptr, s);
}

// ------------------------------------------------------------ multigrid ----

static bool lattice_ok(int Hx, int Hy, int hx, int hy) {
  return Hx >= 2 && Hy >= 2 && hx == 2 * Hx - 1 && hy == 2 * Hy - 1;
}

extern "C" int fem_lattice_interpolate(int nHx, int nHy, int nhx, int nhy, int periodic, const double* xH, double* xh,
                                       cudaStream_t s) {
  if (!xH || !xh || !lattice_ok(nHx, nHy, nhx, nhy)) return FEM_E_ARG;
  return fem_launch_interp(FemLattice{nHx, nHy, periodic ? 1 : 0}, FemLattice{nhx, nhy, periodic ? 1 : 0}, xH, xh, s);
}

extern "C" int fem_lattice_restrict(int nhx, int nhy, int nHx, int nHy, int periodic, const double* xh, double* xH,
                                    cudaStream_t s) {
  if (!xH || !xh || !lattice_ok(nHx, nHy, nhx, nhy)) return FEM_E_ARG;
  return fem_launch_restrict(FemLattice{nhx, nhy, periodic ? 1 : 0}, FemLattice{nHx, nHy, periodic ? 1 : 0}, xh, xH, s);
}

// First multigrid level of the V-cycle run inside CTA 0 from shared memory
// (mg_block_levels): the coarsest levels, from the team's first level down,
// whose r and x plus one scratch of the finest of them fit the tile region
// after the warp CG's buffer and whose 1/D fit FEM_BLK_SMEM; pinned pressure
// also needs a coarsest level the warp CG takes. c->nlev: none. 2D only, and
// only with FEM_MG_BLOCK=1: on the Taylor-Green 256^2 Q2 solve the CTA-0
// levels took 36.6 us per V-cycle against ~40 us on the team, and the step
// ran 470 against 504 steps/s with them.
static int mg_block_from(const fem_ctx* c) {
  const int N = c->nlev;
  if (N < 2 || c->g.kind == FEM_HEX8) return N;
  const char* ev = getenv("FEM_MG_BLOCK");
  if (!ev || atoi(ev) != 1) return N;
  if (c->set_zeroP && c->lv[N - 1].g.nn > FEM_COARSE_WARP_NN) return N;
  int b = N;
  long long vec = 0, d = 0;
  for (int l = N - 1; l >= 1 && l >= c->block_from; --l) {
    const CtxLevel& L = c->lv[l];
    if (!L.invD || !L.winvD || !L.r || !L.t) break;
    vec += 2LL * L.g.nn;
    d += L.g.nn;
    if (FEM_COARSE_WARP_NN + vec + L.g.nn > FEM_TILE_SMEM || d > FEM_BLK_SMEM) break;
    b = l;
  }
  return b;
}

static void fill_cg_args(fem_ctx* c, CgArgs& A) {
  memset(&A, 0, sizeof(A));
  A.sync = FemSync{c->bar, c->bar + 1, c->err, c->partials, FEM_NSLOTS, c->trace, c->trace_cap};
  A.nlev = c->nlev;
  A.block_from = c->block_from;
  A.pinned = c->set_zeroP;
  A.coarse_maxiter = 1000;
  A.coarse_tol = c->coarse_tol;
  A.r = c->pr;
  A.z = c->pz;
  A.p0 = c->pp0;
  A.p1 = c->pp1;
  A.Ap = c->pAp;
  A.bwork = c->pb;
  A.ai_pin = c->aipin;
  for (int l = 0; l < c->nlev; ++l) {
    CtxLevel& L = c->lv[l];
    MgLevel& M = A.lv[l];
    M.g = L.g;
    M.lat = lattice_of(L.g);
    M.tab = L.tab;
    M.tab_off = L.tab_off;
    M.invD = L.invD;
    M.winvD = L.winvD;
    M.diag = (l == 0) ? c->Ldiag : L.diag;
    M.pin = (l == 0) ? (L.pin ? L.pin : c->pmask) : L.pin;
    M.sum_invD = L.sum_invD;
    M.sum_colw = L.sum_colw;
    M.sum_rc = L.sum_rc;
    M.sum_rcD = L.sum_rcD;
    M.inv_nn = 1.0 / (double)L.g.nn;
    M.x = L.x;
    M.r = (l == 0) ? c->pr : L.r;
    M.t = L.t;
  }
  // level 0 pins of the plain (non-multigrid) solve are the context gamma_p
  if (c->nlev == 1 || !c->lv[0].pin) A.lv[0].pin = c->pmask;
  A.block_smem_from = mg_block_from(c);
}

// CTAs of the coarse-level multigrid team for a launch of `grid` CTAs
static int team_size(int grid) {
  int t = FEM_MG_TEAM;
  if (const char* ev = getenv("FEM_MG_TEAM")) t = atoi(ev);
  if (t < 1) t = 1;
  return t < grid ? t : grid;
}

static int reset_sync(fem_ctx* c, cudaStream_t s) {
  FEM_CHECK(cudaMemsetAsync(c->bar, 0, 2 * sizeof(unsigned int), s));  // grid and team arrival counts
  FEM_CHECK(cudaMemsetAsync(c->err, 0, sizeof(int), s));
  return FEM_OK;
}

static int run_cg(fem_ctx* c, const double* b, double* x, double tol, double atol, int maxiter, int precond,
                  int center, int post, int* iters, int* status, cudaStream_t s) {
  CgArgs A;
  fill_cg_args(c, A);
  A.prec = precond;
  A.center_rhs = center;
  A.post = post;
  A.maxiter = maxiter;
  A.tol = tol;
  A.atol = atol;
  A.b = b;
  A.x = x;
  A.iters = iters;
  A.status = status;
  A.final_rr = nullptr;
  FEM_TRY(reset_sync(c, s));
  const int grid = ctx_grid_for(c, c->g.nn);
  A.team = team_size(grid);
  double* cr = c->cr ? c->cr : c->pz;
  double* cp = c->cp ? c->cp : c->pz;
  double* cq = c->cq ? c->cq : c->pz;
  return fem_launch_cg(A, grid, cr, cp, cq, s);
}

// hex8 multigrid-preconditioned CG (k_mg3.cu): pinned pressure only; one graph
// launch, so the stream must not be capturing
static int mg3_ready(fem_ctx* c, int center_rhs, cudaStream_t s) {
  if (!c->mg3 || !c->set_zeroP || center_rhs) {
    snprintf(g_err, sizeof(g_err), "hex8 multigrid needs a hierarchy and pinned pressure (set_zeroP)");
    return FEM_E_STATE;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  FEM_CHECK(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    snprintf(g_err, sizeof(g_err), "hex8 multigrid solves launch their own graph and cannot be captured");
    return FEM_E_STATE;
  }
  if (!c->cap_stream) FEM_CHECK(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
  return FEM_OK;
}

static int run_mg3(fem_ctx* c, const double* b, double* x, double tol, double atol, int maxiter, int center_rhs,
                   int* iters, int* status, cudaStream_t s) {
  FEM_TRY(mg3_ready(c, center_rhs, s));
  return mg3_pcg(c->mg3, b, x, tol, atol, maxiter, iters, status, s, c->cap_stream);
}

// 2D multigrid hierarchy of the graph-driven mixed-precision solve, built on
// first use from the context's multigrid levels (k_mg3.cu, mg2_setup)
static int mg2_ready(fem_ctx* c, cudaStream_t s) {
  if (c->nlev < 2 || c->g.kind == FEM_HEX8) return FEM_E_STATE;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  FEM_CHECK(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone) {
    snprintf(g_err, sizeof(g_err), "mixed-precision solves launch their own graph and cannot be captured");
    return FEM_E_STATE;
  }
  if (!c->cap_stream) FEM_CHECK(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
  if (c->mg2) return FEM_OK;
  FemGrid grids[FEM_MAX_LEVELS];
  const double* tabs[FEM_MAX_LEVELS];
  const double* diags[FEM_MAX_LEVELS];
  const uint8_t* pins[FEM_MAX_LEVELS];
  for (int l = 0; l < c->nlev; ++l) {
    const CtxLevel& L = c->lv[l];
    grids[l] = L.g;
    tabs[l] = L.tab;
    diags[l] = (l == 0) ? c->Ldiag : L.diag;
    pins[l] = (l == 0 && !L.pin) ? c->pmask : L.pin;
  }
  FEM_CHECK(cudaStreamSynchronize(s));
  return mg2_setup(&c->mg2, c->nlev, grids, tabs, diags, pins, c->set_zeroP ? 0 : 1, c->sms, s);
}

extern "C" int fem_pressure_solve(fem_ctx* c, const double* b, double* x, double tol, double atol, int maxiter,
                                  int precond, int center_rhs, int post, int* iters, int* status, cudaStream_t s) {
  const FemRange range("fem_pressure_solve");
  if (!c || !b || !x || !iters || !status || precond < 0 || precond > 4 || maxiter < 0) return FEM_E_ARG;
  if (precond == FEM_PREC_MG && c->nlev < 2) return FEM_E_STATE;
  if (precond == FEM_PREC_MG && c->g.kind == FEM_HEX8) return run_mg3(c, b, x, tol, atol, maxiter, center_rhs,
                                                                       iters, status, s);
  return run_cg(c, b, x, tol, atol, maxiter, precond, center_rhs, post, iters, status, s);
}

extern "C" int fem_mg_vcycle(fem_ctx* c, const double* r, double* z, cudaStream_t s) {
  if (!c || !r || !z || c->nlev < 2) return FEM_E_ARG;
  if (c->g.kind == FEM_HEX8) {
    if (!c->mg3) return FEM_E_STATE;
    return mg3_vcycle64(c->mg3, r, z, s);
  }
  CgArgs A;
  fill_cg_args(c, A);
  FEM_CHECK(cudaMemcpyAsync(c->pr, r, sizeof(double) * c->g.nn, cudaMemcpyDeviceToDevice, s));
  FEM_TRY(reset_sync(c, s));
  const int grid = ctx_grid_for(c, c->g.nn);
  A.team = team_size(grid);
  return fem_launch_vcycle(A, grid, c->cr, c->cp, c->cq, z, s);
}

static int run_bicgstab(fem_ctx* c, int ncomp, const MatCombo& op, const uint8_t* mask, const double* b, double* x,
                        double tol, double atol, int maxiter, int* iters, int* status, cudaStream_t s,
                        const double* cvf = nullptr, double cv_coef = 0.0) {
  if (ncomp < 1 || ncomp > c->ndim) return FEM_E_ARG;  // workspace holds ndim*nn per vector
  BiArgs A;
  memset(&A, 0, sizeof(A));
  A.sync = FemSync{c->bar, c->bar + 1, c->err, c->partials, FEM_NSLOTS, c->trace, c->trace_cap};
  A.g = c->g;
  A.op = op;
  A.mask = mask;
  A.b = b;
  A.x = x;
  A.r = c->br;
  A.rhat = c->brh;
  A.p0 = c->bp0;
  A.p1 = c->bp1;
  A.q0 = c->bq0;
  A.q1 = c->bq1;
  A.t = c->bt;
  A.tol = tol;
  A.atol = atol;
  A.maxiter = maxiter > 0 ? maxiter : 10 * ncomp * c->g.nn;  // utils/jax_iterative_solvers.py:181-183
  A.iters = iters;
  A.status = status;
  A.cvf = cvf;
  A.cv_coef = cv_coef;
  A.qt = c->qt;
  FEM_TRY(reset_sync(c, s));
  return fem_launch_bicgstab(ncomp, A, ctx_grid_for(c, c->g.nn), s);
}

extern "C" int fem_bicgstab_solve(fem_ctx* c, int ncomp, double alpha, const double* Ash, double beta,
                                  const double* B, double gamma, const double* C, const uint8_t* mask,
                                  const double* b, double* x, double tol, double atol, int maxiter, int* iters,
                                  int* status, cudaStream_t s) {
  const FemRange range("fem_bicgstab_solve");
  if (!c || !b || !x || !iters || !status) return FEM_E_ARG;
  const MatCombo op{Ash, alpha, B, beta, 0, C, gamma};
  return run_bicgstab(c, ncomp, op, mask, b, x, tol, atol, maxiter, iters, status, s);
}

extern "C" int fem_step4(fem_ctx* c, const double* Un, const double* Pn, double dt, double rho, double mu,
                         const double* Ud, const double* Fp, const double* F, double tol, int precond, double* Uo,
                         double* Po, int* iters, int* status, cudaStream_t s) {
  const FemRange range("fem_step4");
  if (!c || !Un || !Pn || !Uo || !Po || !iters || !status) return FEM_E_ARG;
  if (c->has_dmask && !Ud) return FEM_E_ARG;
  if (precond < 0 || precond > 4) return FEM_E_ARG;
  if (precond == FEM_PREC_MG && c->nlev < 2) return FEM_E_STATE;
  const FemGrid& g = c->g;
  const int nd = c->ndim, nen = g.nen;
  const double theta = 0.5;
  c->nev = 0;
  stage_mark(c, s);
  // 1. Ce(U_n), beta = 1/2 (solvers/standard.py:152). On the fly: Ce is never
  // built; its Gauss-point factors are, and (mu Le + rho Ce) U_n of the momentum
  // rhs is applied here.
  const bool otf = c->conv_otf && c->cvf;
  if (otf && g.kind == FEM_HEX8) {
    FEM_TRY(fem_launch_conv_factors3(g, c->qt, Un, 0.5, c->cvf, s));
    FEM_TRY(fem_launch_conv_apply3(g, c->qt, c->cvf, rho, mu, c->Le, Un, c->vcv, c->sms, c->err, s));
  } else if (otf) {
    FEM_TRY(fem_launch_conv_factors(g, c->qt, Un, 0.5, c->cvf, s));
    FEM_TRY(fem_launch_conv_apply(2, g, c->qt, c->cvf, rho, mu, c->Le, Un, c->vcv, c->sms, s));
  } else {
    FEM_TRY(fem_launch_convection(g, quad_of(c), Un, 0.5, 0, c->Ce, s));
  }
  // hex8 with the explicit Ce: (mu Le + rho Ce) U_n of the rhs by the element-centric product
  const bool vcv3 = !otf && g.kind == FEM_HEX8 && nd == 3;
  if (vcv3) FEM_TRY(fem_launch_ebe3e(g, MatCombo{c->Le, mu, c->Ce, rho, 0, nullptr, 0.0}, Un, c->vcv, c->sms, s));
  stage_mark(c, s);
  // 2. momentum rhs, x0 and G P_n (solvers/standard.py:31-37)
  StepArgs S;
  S.g = g;
  S.ndim = nd;
  S.dt = dt;
  S.rho = rho;
  S.mu = mu;
  S.theta = theta;
  S.Me = c->Me;
  S.Le = c->Le;
  S.Ge = c->Ge;
  S.M = c->M;
  S.Ce = otf ? nullptr : c->Ce;
  S.vcv = (otf || vcv3) ? c->vcv : nullptr;
  S.tab3 = c->step_tab;
  S.dmask = c->has_dmask ? c->dmask : nullptr;
  S.pmask = c->pmask;
  S.pinned = c->set_zeroP;
  FEM_TRY(fem_launch_mom_rhs(S, Un, Pn, Ud, F, c->rhsU, c->Uhat, c->gPn, s));
  // 3. BiCGSTAB on (rho/dt) Me + theta (rho Ce + mu Le), identity rows on gamma_d (:20-28, :41)
  FEM_TRY(fem_launch_lincomb(nen * nen, rho / dt, c->Me, theta * mu, c->Le, c->Kd, s));
  stage_mark(c, s);
  if (otf && c->precision == FEM_PRECISION_MIXED && g.kind != FEM_HEX8) {
    // FP64 refinement around FP32 BiCGSTAB iterations (k_mixmom.cu)
    FEM_TRY(mg2_ready(c, s));  // the same capture check and private stream as the mixed pressure solve
    if (!c->mixmom) FEM_TRY(mixmom_create(&c->mixmom, g, nd, c->nq, c->sms));
    FEM_TRY(mixmom_solve(c->mixmom, c->qt, c->cvf, c->Kd, theta * rho, S.dmask, c->rhsU, c->Uhat, tol,
                         FEM_MIXED_MOMENTUM_INNER, c->mx_cycles, iters, status, c->sms, s, c->cap_stream));
  } else if (otf) {
    const MatCombo op{c->Kd, 1.0, nullptr, 0.0, 0, nullptr, 0.0};
    FEM_TRY(run_bicgstab(c, nd, op, S.dmask, c->rhsU, c->Uhat, tol, 0.0, 0, iters, status, s, c->cvf, theta * rho));
  } else {
    const MatCombo op{c->Kd, 1.0, c->Ce, theta * rho, 0, nullptr, 0.0};
    FEM_TRY(run_bicgstab(c, nd, op, S.dmask, c->rhsU, c->Uhat, tol, 0.0, 0, iters, status, s));
  }
  stage_mark(c, s);
  // 4. U* = U_hat + (dt/rho) G P_n / M (:156)
  FEM_TRY(fem_launch_ustar(nd * g.nn, dt / rho, c->Uhat, c->gPn, c->M, c->Ustar, s));
  stage_mark(c, s);
  // 5. PPE rhs and x0 (:97-107)
  FEM_TRY(fem_launch_p_rhs(S, c->Ustar, Fp, Pn, c->rhsP, Po, s));
  stage_mark(c, s);
  // 6. pressure (P)CG, maxiter 1000 (:115-123); hex8 multigrid runs the k_mg3.cu
  // solve, in mixed precision when the context asks for it
  if (precond == FEM_PREC_MG && g.kind == FEM_HEX8) {
    FEM_TRY(mg3_ready(c, c->set_zeroP ? 0 : 1, s));
    if (c->precision == FEM_PRECISION_MIXED)
      FEM_TRY(mg3_mixed(c->mg3, c->rhsP, Po, tol, c->mx_inner, c->mx_cycles, iters + 1, status + 1, s,
                        c->cap_stream));
    else
      FEM_TRY(mg3_pcg(c->mg3, c->rhsP, Po, tol, 0.0, 1000, iters + 1, status + 1, s, c->cap_stream));
  } else if (precond == FEM_PREC_MG && c->precision == FEM_PRECISION_MIXED) {
    FEM_TRY(mg2_ready(c, s));
    FEM_TRY(mg3_mixed(c->mg2, c->rhsP, Po, tol, c->mx_inner, c->mx_cycles, iters + 1, status + 1, s,
                      c->cap_stream));
  } else {
    FEM_TRY(run_cg(c, c->rhsP, Po, tol, 0.0, 1000, precond, c->set_zeroP ? 0 : 1, 1, iters + 1, status + 1, s));
  }
  stage_mark(c, s);
  // 7. projection and Dirichlet values (:160-163)
  FEM_TRY(fem_launch_ufinal(S, c->Ustar, Po, Ud, Uo, s));
  stage_mark(c, s);
  return FEM_OK;
}

static int transport_mats(fem_ctx* c, const double* Un, const double* U, double dt, double D, int supg,
                          cudaStream_t s);

extern "C" int fem_transport_phi(fem_ctx* c, const double* Un, const double* U, const double* phin, double dt,
                                 double D, int supg, const uint8_t* phi_mask, const double* phid, double tol,
                                 double* phio, int* iters, int* status, cudaStream_t s) {
  if (!c || !Un || !U || !phin || !phio || !iters || !status) return FEM_E_ARG;
  if (phi_mask && !phid) return FEM_E_ARG;
  const FemGrid& g = c->g;
  const size_t ntot = (size_t)g.ne * g.nen * g.nen;
  FEM_TRY(transport_mats(c, Un, U, dt, D, supg, s));
  // rhs and x0 (solvers/passive_transport.py:26-33 / :50-57)
  FEM_TRY(fem_launch_phi_rhs(g, c->Me, c->Le, dt, D, c->Mt, c->Ce, c->Ct, phin, phi_mask, phid, c->rhsP, phio, s));
  // lhs: [(1/dt) Me + 0.5 D Le] + [(1/dt) Mtau + 0.5 (Ce + Ctau)]
  FEM_TRY(fem_launch_lincomb(g.nen * g.nen, 1.0 / dt, c->Me, 0.5 * D, c->Le, c->Kd, s));
  FEM_TRY(fem_launch_elem_combine(ntot, 1.0 / dt, c->Mt, 0.5, c->Ce2, c->Ct, c->Ek, 0, s));
  const MatCombo op{c->Kd, 1.0, c->Ek, 1.0, 0, nullptr, 0.0};
  return run_bicgstab(c, 1, op, phi_mask, c->rhsP, phio, tol, 0.0, 0, iters, status, s);
}

extern "C" int fem_transport_elements(fem_ctx* c, const double* Un, const double* U, double dt, double D, int supg,
                                      int transpose, double* Ek, double* Bk, cudaStream_t s) {
  if (!c || !Un || !U || !Ek || !Bk) return FEM_E_ARG;
  const size_t ntot = (size_t)c->g.ne * c->g.nen * c->g.nen;
  FEM_TRY(transport_mats(c, Un, U, dt, D, supg, s));
  FEM_TRY(fem_launch_elem_combine(ntot, 1.0 / dt, c->Mt, 0.5, c->Ce2, c->Ct, Ek, transpose ? c->g.nen : 0, s));
  return fem_launch_elem_combine(ntot, 1.0 / dt, c->Mt, -0.5, c->Ce, c->Ct, Bk, transpose ? c->g.nen : 0, s);
}

// Element matrices of the passive-scalar step into the context: Ce = Ce(U_n, 1),
// Ce2 = Ce(U, 1), and with SUPG Ct = tau Ct(U_n), Mt = tau Ce(U_n)^T (both zero
// without it).
static int transport_mats(fem_ctx* c, const double* Un, const double* U, double dt, double D, int supg,
                          cudaStream_t s) {
  const FemGrid& g = c->g;
  const size_t per = (size_t)g.nen * g.nen, ntot = (size_t)g.ne * per;
  if (!c->Ce2) {
    FEM_ALLOC(c->Ce2, ntot);
    FEM_ALLOC(c->Ct, ntot);
    FEM_ALLOC(c->Mt, ntot);
    FEM_ALLOC(c->Ek, ntot);
    FEM_ALLOC(c->tau, g.ne);
  }
  const FemQuad Q = quad_of(c);
  // Ce(U_n, 1) -> Ce, Ce(U, 1) -> Ce2 (solvers/passive_transport.py:80-81)
  FEM_TRY(fem_launch_convection(g, Q, Un, 1.0, 0, c->Ce, s));
  FEM_TRY(fem_launch_convection(g, Q, U, 1.0, 0, c->Ce2, s));
  if (supg) {
    // Ctau_tilde(U_n); tau(U_n, Ce(U), Ct); Ctau = tau Ct; Mtau = tau Ce_n^T (:84-88)
    FEM_TRY(fem_launch_convection(g, Q, Un, 0.0, 1, c->Ct, s));
    FEM_TRY(fem_launch_supg_tau(g, Q, Un, c->Ce2, c->Ct, D, dt, 2.0, c->tau, s));
    FEM_TRY(fem_launch_scale_elem(g.ne, g.nen, c->tau, c->Ct, 0, c->Ct, s));
    FEM_TRY(fem_launch_scale_elem(g.ne, g.nen, c->tau, c->Ce, 1, c->Mt, s));
  } else {
    FEM_CHECK(cudaMemsetAsync(c->Ct, 0, ntot * sizeof(double), s));
    FEM_CHECK(cudaMemsetAsync(c->Mt, 0, ntot * sizeof(double), s));
  }
  return FEM_OK;
}

extern "C" int fem_boundary_flux(fem_ctx* c, const int32_t* bconn, const double* nvec, int nb, int npf,
                                 const double* U, double* Fp, cudaStream_t s) {
  if (!c || !bconn || !nvec || !U || !Fp || nb < 0 || npf < 2 || npf > 4) return FEM_E_ARG;
  const long long need = (long long)nb * npf;
  if (need > INT_MAX) {
    snprintf(g_err, sizeof(g_err), "fem_boundary_flux: nb * nodes_per_face = %lld exceeds INT_MAX", need);
    return FEM_E_ARG;
  }
  if (need > (long long)c->Fe_cap) {
    FEM_CHECK(cudaStreamSynchronize(s));
    if (c->Fe) cudaFree(c->Fe);
    if (c->bs_list) cudaFree(c->bs_list);
    c->Fe = nullptr;
    c->bs_list = nullptr;
    c->Fe_cap = 0;
    FEM_ALLOC(c->Fe, (size_t)need);
    FEM_ALLOC(c->bs_list, (size_t)need);
    c->Fe_cap = (size_t)need;
  }
  if (!c->bs_cnt) {
    FEM_ALLOC(c->bs_cnt, (size_t)c->g.nn);
    // offsets, then the chunk sums of their scan (k_ops.cu, FEM_SCAN_CHUNK = 4096 nodes per chunk)
    FEM_ALLOC(c->bs_off, (size_t)c->g.nn + 1 + (c->g.nn + 4095) / 4096);
  }
  return fem_launch_boundary_csr(c->coords, c->ndim, bconn, nvec, nb, npf, U, c->g.nn, c->Fe, c->bs_cnt, c->bs_off,
                                 c->bs_list, c->flags + FEM_FLAG_BOUNDARY_SKIPPED, Fp, s);
}

extern "C" int fem_boundary_flux_skipped(fem_ctx* c, int* count, cudaStream_t s) {
  if (!c || !count) return FEM_E_ARG;
  FEM_CHECK(cudaMemcpyAsync(count, c->flags + FEM_FLAG_BOUNDARY_SKIPPED, sizeof(int), cudaMemcpyDeviceToHost, s));
  FEM_CHECK(cudaStreamSynchronize(s));
  return FEM_OK;
}

// Fixed scratch of fem_boundary_flux_noalloc: one copy per device in this
// library's device image, shared by every call on that device. The tables of
// the node-parallel assembly are sized by the face-entry limit alone (a hash
// table of 2 FEM_NOALLOC_FACE_VALUES node slots replaces the per-node table),
// 44 bytes per face entry, 2.9 MB in all. Each call clears the tables it
// counts in and writes every other value before reading it, on its stream.
#define FEM_NOALLOC_SLOTS (2 * FEM_NOALLOC_FACE_VALUES)
struct NoallocScratch {
  double fe[FEM_NOALLOC_FACE_VALUES];
  int keys[FEM_NOALLOC_SLOTS];
  int cnt[FEM_NOALLOC_SLOTS];
  int off[FEM_NOALLOC_SLOTS + 1];
  int slot[FEM_NOALLOC_FACE_VALUES];
  int list[FEM_NOALLOC_FACE_VALUES];
};
static __device__ __align__(256) NoallocScratch g_noalloc;

#define FEM_NOALLOC_MAX_DEVICES 64
static std::mutex g_noalloc_mu;
static NoallocScratch* g_noalloc_ptr[FEM_NOALLOC_MAX_DEVICES] = {};

// Device address of `device`'s copy of g_noalloc (host code cannot use the
// symbol itself). Looked up once per device on its first call, with that
// device current; later calls read the cached value.
static int noalloc_scratch(int device, NoallocScratch** out) {
  if (device < 0 || device >= FEM_NOALLOC_MAX_DEVICES) {
    snprintf(g_err, sizeof(g_err), "fem_boundary_flux_noalloc: device %d beyond the %d supported", device,
             FEM_NOALLOC_MAX_DEVICES);
    return FEM_E_ARG;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    NoallocScratch* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc);
    if (e != cudaSuccess) return set_err("cudaGetSymbolAddress(g_noalloc)", e);
    g_noalloc_ptr[device] = p;
  }
  *out = g_noalloc_ptr[device];
  return FEM_OK;
}

extern "C" int fem_boundary_flux_noalloc(fem_ctx* c, const int32_t* bconn, const double* nvec, int nb, int npf,
                                         const double* U, double* Fp, cudaStream_t s) {
  if (!c || !bconn || !nvec || !U || !Fp || nb < 0 || npf < 2 || npf > 4) return FEM_E_ARG;
  const long long need = (long long)nb * npf;
  if (need > FEM_NOALLOC_FACE_VALUES) {
    snprintf(g_err, sizeof(g_err),
             "fem_boundary_flux_noalloc: nb * nodes_per_face = %lld exceeds the fixed scratch of %d values "
             "(use fem_boundary_flux)",
             need, FEM_NOALLOC_FACE_VALUES);
    return FEM_E_ARG;
  }
  int cur = -1;
  FEM_CHECK(cudaGetDevice(&cur));
  if (cur != c->device) {
    snprintf(g_err, sizeof(g_err), "fem_boundary_flux_noalloc: current device %d is not the context's device %d",
             cur, c->device);
    return FEM_E_STATE;
  }
  NoallocScratch* sc = nullptr;
  FEM_TRY(noalloc_scratch(cur, &sc));
  const FemBoundaryHash H{FEM_NOALLOC_SLOTS, sc->fe,   sc->keys, sc->cnt,
                          sc->off,           sc->slot, sc->list, c->flags + FEM_FLAG_BOUNDARY_SKIPPED};
  return fem_launch_boundary_hash(c->coords, c->ndim, bconn, nvec, nb, npf, U, c->g.nn, H, Fp, s);
}

extern "C" int fem_conv_vjp(fem_ctx* c, int ncomp, const double* a, const double* b, double beta, double* y,
                            cudaStream_t s) {
  if (!c || !a || !b || !y || ncomp < 1 || ncomp > c->ndim) return FEM_E_ARG;
  if (!c->vjp) FEM_ALLOC(c->vjp, (size_t)c->g.ne * c->ndim * c->g.nen);
  return fem_launch_conv_vjp(c->g, c->qt, ncomp, a, b, beta, c->vjp, y, s);
}

extern "C" int fem_transport_vjp(fem_ctx* c, const double* Un, const double* U, const double* lam,
                                 const double* phin, const double* phi, double dt, double D, int supg, double* gUn,
                                 double* gU, cudaStream_t s) {
  if (!c || !Un || !U || !lam || !phin || !phi || !gUn || !gU) return FEM_E_ARG;
  if (c->g.kind == FEM_HEX8) return FEM_E_STATE;
  if (!c->vjp2) FEM_ALLOC(c->vjp2, (size_t)2 * c->g.ne * c->ndim * c->g.nen);
  const size_t half = (size_t)c->g.ne * c->ndim * c->g.nen;
  return fem_launch_transport_vjp(c->g, c->qt, Un, U, lam, phin, phi, dt, D, supg, c->vjp2, c->vjp2 + half, gUn, gU,
                                  s);
}

extern "C" int fem_scatter(const int64_t* idx, const double* vals, double value, int n, double* out,
                           cudaStream_t s) {
  if (n < 0 || (n > 0 && (!idx || !out))) return FEM_E_ARG;
  if (n == 0) return FEM_OK;
  return fem_launch_scatter(idx, vals, value, n, out, s);
}

extern "C" int fem_make_mask(const int64_t* idx, int n, int len, uint8_t* mask, cudaStream_t s) {
  if (n < 0 || len < 0 || !mask || (n > 0 && !idx)) return FEM_E_ARG;
  FEM_CHECK(cudaMemsetAsync(mask, 0, (size_t)len, s));
  if (n == 0) return FEM_OK;
  return fem_launch_make_mask(idx, n, len, mask, s);
}

extern "C" int fem_dot(fem_ctx* c, const double* x, const double* y, int n, double* out, cudaStream_t s) {
  if (!c || !x || !y || !out || n < 0) return FEM_E_ARG;
  return fem_launch_dot(x, y, n, c->dotpart, out, s);
}

extern "C" int fem_axpby(fem_ctx* c, double a, const double* x, double b, double* y, int n, cudaStream_t s) {
  if (!c || !x || !y || n < 0) return FEM_E_ARG;
  return fem_launch_axpby(a, x, b, y, n, s);
}

extern "C" int fem_ctx_enable_timing(fem_ctx* c, int enable) {
  if (!c) return FEM_E_ARG;
  if (enable && !c->ev[0])
    for (int i = 0; i < 16; ++i) FEM_CHECK(cudaEventCreate(&c->ev[i]));
  c->timing = enable ? 1 : 0;
  c->nev = 0;
  return FEM_OK;
}

extern "C" int fem_ctx_stage_times(fem_ctx* c, float* ms, int max_n) {
  if (!c || !ms || max_n < 0) return FEM_E_ARG;
  if (!c->timing || c->nev < 2) return 0;
  FEM_CHECK(cudaEventSynchronize(c->ev[c->nev - 1]));
  int n = 0;
  for (int i = 0; i + 1 < c->nev && n < max_n; ++i, ++n) FEM_CHECK(cudaEventElapsedTime(&ms[n], c->ev[i], c->ev[i + 1]));
  return n;
}

extern "C" int fem_ctx_set_trace(fem_ctx* c, unsigned long long* buf, int cap) {
  if (!c || cap < 0 || (cap > 0 && !buf)) return FEM_E_ARG;
  c->trace = cap > 0 ? buf : nullptr;
  c->trace_cap = cap;
  return FEM_OK;
}

// ------------------------------------------------------ captured steps ----

extern "C" int fem_step4_graph(fem_ctx* c, double* U0, double* P0, double* U1, double* P1, double dt, double rho,
                               double mu, const double* Ud, const double* Fp, const double* F, double tol, int precond,
                               int nsteps, int* iters, int* status, fem_graph** out) {
  if (!c || !out || !U0 || !P0 || !U1 || !P1 || nsteps < 2 || (nsteps & 1)) return FEM_E_ARG;
  if (c->timing) return FEM_E_STATE;  // stage events cannot be captured
  *out = nullptr;
  int prev = 0;
  cudaGetDevice(&prev);
  FEM_CHECK(cudaSetDevice(c->device));
  int rc = FEM_OK;
  if (!c->cap_stream) {
    const cudaError_t e = cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) rc = set_err("cudaStreamCreateWithFlags", e);
  }
  // thread-local capture: work that other host threads issue meanwhile is not captured
  if (rc == FEM_OK) {
    const cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) rc = set_err("cudaStreamBeginCapture", e);
  }
  if (rc != FEM_OK) {
    cudaSetDevice(prev);
    return rc;
  }
  for (int k = 0; k < nsteps && rc == FEM_OK; ++k) {
    const bool even = (k & 1) == 0;
    rc = fem_step4(c, even ? U0 : U1, even ? P0 : P1, dt, rho, mu, Ud, Fp, F, tol, precond, even ? U1 : U0,
                   even ? P1 : P0, iters, status, c->cap_stream);
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t e_end = cudaStreamEndCapture(c->cap_stream, &graph);
  if (rc == FEM_OK && e_end != cudaSuccess) rc = set_err("cudaStreamEndCapture", e_end);
  cudaGraphExec_t exec = nullptr;
  if (rc == FEM_OK) {
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) rc = set_err("cudaGraphInstantiate", e);
  }
  if (rc != FEM_OK) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();  // a failed capture leaves no sticky error behind
    cudaSetDevice(prev);
    return rc;
  }
  fem_graph* g = new fem_graph;
  g->graph = graph;
  g->exec = exec;
  g->device = c->device;
  *out = g;
  cudaSetDevice(prev);
  return FEM_OK;
}

extern "C" int fem_graph_launch(fem_graph* g, cudaStream_t s) {
  if (!g || !g->exec) return FEM_E_ARG;
  FEM_CHECK(cudaGraphLaunch(g->exec, s));
  return FEM_OK;
}

extern "C" int fem_graph_destroy(fem_graph* g) {
  if (!g) return FEM_OK;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return FEM_OK;
}

extern "C" int fem_pressure_solve_mixed(fem_ctx* c, const double* b, double* x, double tol, int inner,
                                        int max_cycles, int* cycles, double* relres, cudaStream_t s) {
  const FemRange range("fem_pressure_solve_mixed");
  if (!c || !b || !x || !(tol > 0.0) || inner < 1 || max_cycles < 1) return FEM_E_ARG;
  if (c->g.kind == FEM_HEX8) {
    if (c->nlev < 2) return FEM_E_STATE;
    FEM_TRY(mg3_ready(c, 0, s));
    int* dev = c->flags + 1;  // cycles, status
    FEM_TRY(mg3_mixed(c->mg3, b, x, tol, inner, max_cycles, dev, dev + 1, s, c->cap_stream));
    int h[2] = {0, 0};
    FEM_CHECK(cudaMemcpyAsync(h, dev, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    double rr = 0.0;
    FEM_TRY(mg3_last_relres(c->mg3, &rr, s));
    if (cycles) *cycles = h[0];
    if (relres) *relres = rr;
    return FEM_OK;
  }
  if (c->nlev < 2) return FEM_E_STATE;
  if (c->g.kind != FEM_Q1_2D || !c->set_zeroP) {
    // quad9 or mean-zero: the graph-driven solve over the 2D hierarchy
    FEM_TRY(mg2_ready(c, s));
    int* dev = c->flags + 1;  // cycles, status
    FEM_TRY(mg3_mixed(c->mg2, b, x, tol, inner, max_cycles, dev, dev + 1, s, c->cap_stream));
    int h[2] = {0, 0};
    FEM_CHECK(cudaMemcpyAsync(h, dev, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    double rr = 0.0;
    FEM_TRY(mg3_last_relres(c->mg2, &rr, s));
    if (cycles) *cycles = h[0];
    if (relres) *relres = rr;
    return FEM_OK;
  }
  if (c->lv[c->nlev - 1].g.nn > 128) return FEM_E_STATE;  // the one-warp coarse CG
  const int grid = c->sms * 8;
  if (!c->mx32) {
    size_t nf = 3 * (size_t)c->lv[0].g.nn;
    for (int l = 0; l < c->nlev; ++l) nf += 6 * (size_t)c->lv[l].g.nn;
    FEM_ALLOC(c->mx32, nf);
    FEM_ALLOC(c->mx64, (size_t)grid + 8);
  }
  if (!c->cap_stream) FEM_CHECK(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
  CgArgs A;
  fill_cg_args(c, A);
  return fem_mixed_poisson(A, grid, c->mx32, c->mx64, b, x, tol, inner, max_cycles, cycles, relres, s, &c->mxg,
                           c->cap_stream);
}

extern "C" int fem_selftest_barrier_timeout(fem_ctx* c, int* status, cudaStream_t s) {
  if (!c || !status) return FEM_E_ARG;
  FEM_TRY(reset_sync(c, s));
  const FemSync S{c->bar, c->bar + 1, c->err, c->partials, FEM_NSLOTS, nullptr, 0};
  return fem_launch_selftest_barrier(S, status, s);
}

extern "C" int fem_ctx_set_precision(fem_ctx* c, int precision, int inner, int max_cycles) {
  if (!c || (precision != FEM_PRECISION_FP64 && precision != FEM_PRECISION_MIXED) || inner < 1 || max_cycles < 1)
    return FEM_E_ARG;
  c->precision = precision;
  c->mx_inner = inner;
  c->mx_cycles = max_cycles;
  return FEM_OK;
}

extern "C" int fem_ctx_set_max_ctas(fem_ctx* c, int ctas, int* capacity) {
  if (!c || ctas < 0) return FEM_E_ARG;
  c->max_coop = (ctas > 0 && ctas < c->coop_capacity) ? ctas : c->coop_capacity;
  if (capacity) *capacity = c->coop_capacity;
  return FEM_OK;
}

// ------------------------------------------------------------ packed steps ----

struct fem_pack {
  int k = 0, ctas = 0, capacity = 0;
  int blk = 0;                   // the members' multigrid runs its coarsest levels inside CTA 0
  PackMember* dmem = nullptr;    // k members (device)
  unsigned int* sync = nullptr;  // [2m] grid and [2m + 1] team arrival counts, [2k + m] error word
};

extern "C" int fem_pack_create(fem_ctx* const* ctxs, int k, double* const* U0, double* const* P0,
                               double* const* U1, double* const* P1, const double* const* Ud, int* stat,
                               double tol, int precond, fem_pack** out) {
  if (!ctxs || !U0 || !P0 || !U1 || !P1 || !stat || !out || k < 1 || k > FEM_PACK_MAX) return FEM_E_ARG;
  if (precond < 0 || precond > 4) return FEM_E_ARG;
  *out = nullptr;
  const fem_ctx* c0 = ctxs[0];
  if (!c0) return FEM_E_ARG;
  const int ctas = ctx_grid_for(c0, c0->g.nn);
  for (int m = 0; m < k; ++m) {
    const fem_ctx* c = ctxs[m];
    if (!c || !U0[m] || !P0[m] || !U1[m] || !P1[m]) return FEM_E_ARG;
    if (c->has_dmask && (!Ud || !Ud[m])) return FEM_E_ARG;
    if (c->g.kind != FEM_Q1_2D || c->ndim != 2 || !c->set_zeroP || !c->conv_otf || !c->cvf ||
        c->precision != FEM_PRECISION_FP64 || (precond == FEM_PREC_MG && c->nlev < 2)) {
      snprintf(g_err, sizeof(g_err),
               "fem_pack_create: member %d is not a Q1 2D pinned-pressure FP64 context with on-the-fly convection",
               m);
      return FEM_E_STATE;
    }
    if (c->g.nnx != c0->g.nnx || c->g.nny != c0->g.nny || c->g.periodic != c0->g.periodic ||
        c->device != c0->device || ctx_grid_for(c, c->g.nn) != ctas) {
      snprintf(g_err, sizeof(g_err), "fem_pack_create: member %d differs in mesh, device or CTA count", m);
      return FEM_E_STATE;
    }
  }
  int per_sm = 0;
  if (fem_pack_occupancy(&per_sm) != 0 || per_sm < 1) return set_err("fem_pack_occupancy", cudaGetLastError());
  const int capacity = per_sm * c0->sms;
  if (ctas > capacity) {
    snprintf(g_err, sizeof(g_err), "fem_pack_create: %d CTAs per member exceed the %d co-resident CTAs", ctas,
             capacity);
    return FEM_E_STATE;
  }
  fem_pack* p = new fem_pack();
  p->k = k;
  p->ctas = ctas;
  p->capacity = capacity;
  std::vector<PackMember> hm(k);
  int rc = dalloc(&p->dmem, (size_t)k);
  if (!rc) rc = dalloc(&p->sync, (size_t)3 * k);
  const double theta = 0.5, rho = 1.0;
  for (int m = 0; m < k && !rc; ++m) {
    fem_ctx* c = ctxs[m];
    PackMember& M = hm[m];
    memset(&M, 0, sizeof(M));
    int* st = stat + 5 * m;
    const FemSync sync{p->sync + 2 * m, p->sync + 2 * m + 1, reinterpret_cast<int*>(p->sync + 2 * k + m),
                       c->partials, FEM_NSLOTS, nullptr, 0};
    // the fem_step4 stage arguments (dt, mu set per launch)
    StepArgs& S = M.S;
    S.g = c->g;
    S.ndim = 2;
    S.rho = rho;
    S.theta = theta;
    S.Me = c->Me;
    S.Le = c->Le;
    S.Ge = c->Ge;
    S.M = c->M;
    S.Ce = nullptr;
    S.vcv = c->vcv;
    S.dmask = c->has_dmask ? c->dmask : nullptr;
    S.pmask = c->pmask;
    S.pinned = c->set_zeroP;
    // the momentum BiCGSTAB of run_bicgstab (its shared matrix is built in the kernel)
    BiArgs& B = M.B;
    B.sync = sync;
    B.g = c->g;
    B.op = MatCombo{nullptr, 1.0, nullptr, 0.0, 0, nullptr, 0.0};
    B.mask = S.dmask;
    B.b = c->rhsU;
    B.x = c->Uhat;
    B.r = c->br;
    B.rhat = c->brh;
    B.p0 = c->bp0;
    B.p1 = c->bp1;
    B.q0 = c->bq0;
    B.q1 = c->bq1;
    B.t = c->bt;
    B.tol = tol;
    B.atol = 0.0;
    B.maxiter = 10 * 2 * c->g.nn;  // utils/jax_iterative_solvers.py:181-183
    B.iters = st;
    B.status = st + 2;
    B.cvf = c->cvf;
    B.cv_coef = theta * rho;
    B.qt = c->qt;
    // the pressure solve of run_cg (x is the step's output pressure)
    CgArgs& C = M.C;
    fill_cg_args(c, C);
    C.sync = sync;
    C.prec = precond;
    C.center_rhs = 0;
    C.post = 1;
    C.maxiter = 1000;
    C.tol = tol;
    C.atol = 0.0;
    C.b = c->rhsP;
    C.x = nullptr;
    C.iters = st + 1;
    C.status = st + 3;
    C.final_rr = nullptr;
    C.team = team_size(ctas);
    if (C.block_smem_from < C.nlev) p->blk = 1;
    M.U[0] = U0[m];
    M.U[1] = U1[m];
    M.P[0] = P0[m];
    M.P[1] = P1[m];
    M.Ud = c->has_dmask ? Ud[m] : nullptr;
    M.cvf = c->cvf;
    M.vcv = c->vcv;
    M.rhsU = c->rhsU;
    M.Uhat = c->Uhat;
    M.gPn = c->gPn;
    M.Ustar = c->Ustar;
    M.rhsP = c->rhsP;
    M.cr = c->cr ? c->cr : c->pz;
    M.cp = c->cp ? c->cp : c->pz;
    M.cq = c->cq ? c->cq : c->pz;
    M.stat = st;
  }
  if (!rc) {
    const cudaError_t e = cudaMemcpy(p->dmem, hm.data(), sizeof(PackMember) * k, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) rc = set_err("fem_pack_create", e);
  }
  if (rc) {
    fem_pack_destroy(p);
    return rc;
  }
  *out = p;
  return FEM_OK;
}

extern "C" int fem_pack_step(fem_pack* p, const double* dt, const double* mu, const int* steps, const int* cur,
                             cudaStream_t s) {
  if (!p || !dt || !mu || !steps || !cur) return FEM_E_ARG;
  PackParams P;
  memset(&P, 0, sizeof(P));
  int active = 0;
  for (int m = 0; m < p->k; ++m) {
    if (steps[m] < 0 || (cur[m] != 0 && cur[m] != 1)) return FEM_E_ARG;
    if (steps[m] > 0 && !(dt[m] > 0.0)) return FEM_E_ARG;
    P.m[m] = PackStep{dt[m], mu[m], steps[m], cur[m]};
    if (steps[m] > 0) P.idx[active++] = m;
  }
  if (!active) return FEM_OK;
  if (active * p->ctas > p->capacity) {
    snprintf(g_err, sizeof(g_err), "fem_pack_step: %d active members x %d CTAs exceed the %d co-resident CTAs",
             active, p->ctas, p->capacity);
    return FEM_E_STATE;
  }
  FEM_CHECK(cudaMemsetAsync(p->sync, 0, sizeof(unsigned int) * 3 * p->k, s));
  return fem_launch_step_pack(FEM_Q1_2D, p->dmem, P, active, p->ctas, p->blk, s);
}

extern "C" int fem_pack_info(const fem_pack* p, int* k, int* ctas, int* capacity) {
  if (!p) return FEM_E_ARG;
  if (k) *k = p->k;
  if (ctas) *ctas = p->ctas;
  if (capacity) *capacity = p->capacity;
  return FEM_OK;
}

extern "C" int fem_pack_destroy(fem_pack* p) {
  if (!p) return FEM_OK;
  if (p->dmem) cudaFree(p->dmem);
  if (p->sync) cudaFree(p->sync);
  delete p;
  return FEM_OK;
}

extern "C" long long fem_launch_count(void) { return g_launches.load(); }
extern "C" const char* fem_last_error(void) { return g_err; }
