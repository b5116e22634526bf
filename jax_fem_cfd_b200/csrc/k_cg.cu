// Persistent cooperative (P)CG kernel with the multigrid V-cycle preconditioner.
#include "fem_cg_body.cuh"


template <int KIND, bool PIN>
__global__ void __launch_bounds__(FEM_THREADS, 1) k_cg(CgArgs Aparam, double* cg_r, double* cg_p, double* cg_q) {
  // [0,128) reductions, [128, +FEM_TILE_SMEM) tiles, [.., +FEM_TAB_SMEM) stencil tables,
  // [.., +FEM_BLK_SMEM) 1/D of the levels run inside CTA 0
  extern __shared__ double smem[];
  __shared__ __align__(16) CgArgs sA;
  fem_stage_args(Aparam, &sA);
  fem_trace_init(sA.sync);
  fem_tables_to_smem<KIND>(sA, smem + 128 + FEM_TILE_SMEM);
  fem_block_levels_to_smem(sA, smem + 128 + FEM_TILE_SMEM + FEM_TAB_SMEM);
  __shared__ unsigned int s_round, s_team_round;
  if (threadIdx.x == 0) {
    s_round = 0u;
    s_team_round = 0u;
  }
  cg_solve<KIND, PIN>(sA, smem, &s_round, &s_team_round, cg_r, cg_p, cg_q);
}

template <int KIND, bool PIN>
__global__ void __launch_bounds__(FEM_THREADS, 1) k_vcycle(CgArgs Aparam, double* cg_r, double* cg_p, double* cg_q,
                                                            double* z) {
  // [0,128) reductions, [128, +FEM_TILE_SMEM) tiles, [.., +FEM_TAB_SMEM) stencil tables,
  // [.., +FEM_BLK_SMEM) 1/D of the levels run inside CTA 0
  extern __shared__ double smem[];
  __shared__ __align__(16) CgArgs sA;
  fem_stage_args(Aparam, &sA);
  fem_trace_init(sA.sync);
  fem_tables_to_smem<KIND>(sA, smem + 128 + FEM_TILE_SMEM);
  fem_block_levels_to_smem(sA, smem + 128 + FEM_TILE_SMEM + FEM_TAB_SMEM);
  const CgArgs& A = sA;
  __shared__ unsigned int s_round, s_team_round;
  if (threadIdx.x == 0) {
    s_round = 0u;
    s_team_round = 0u;
  }
  const GridTeam gt = GridTeam::grid(&A.sync, &s_round);
  const GridReducer gr{&A.sync};
  const MgLevel& L0 = A.lv[0];
  const int nn = L0.g.nn;
  fem_zero_partials(A.sync);
  if (!gt.sync()) return;
  double a[2] = {0.0, 0.0};
  for (int i = gt.rank(); i < nn; i += gt.size()) {
    a[0] += L0.r[i];
    a[1] += L0.r[i] * L0.invD[i];
  }
  gr.reduce<2>(a, SL_R(0), smem);
  if (!gt.sync()) return;
  if (!mg_vcycle<KIND, PIN>(gt, gr, A, smem, &s_team_round, cg_r, cg_p, cg_q)) return;
  double sx[2];
  gr.result<2>(sx, SL_X(0), smem);
  const double mz = PIN ? 0.0 : sx[0] * L0.inv_nn;
  for (int i = gt.rank(); i < nn; i += gt.size()) z[i] = L0.t[i] - mz;
}

static int coop_launch(const void* fn, int grid, void** args, cudaStream_t s, const char* what, size_t dyn = 0) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(FEM_THREADS);
  cfg.stream = s;
  cfg.dynamicSmemBytes = dyn;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelExC(&cfg, fn, args);
  return fem_after_launch(what);
}

// kernels by element kind and pressure mode (pinned gamma_p rows or mean-zero)
template <bool PIN>
static const void* cg_fn_p(int kind) {
  return kind == FEM_Q1_2D ? (const void*)k_cg<FEM_Q1_2D, PIN>
                           : (kind == FEM_Q2_2D ? (const void*)k_cg<FEM_Q2_2D, PIN> : (const void*)k_cg<FEM_HEX8, PIN>);
}
template <bool PIN>
static const void* vc_fn_p(int kind) {
  return kind == FEM_Q1_2D ? (const void*)k_vcycle<FEM_Q1_2D, PIN>
                           : (kind == FEM_Q2_2D ? (const void*)k_vcycle<FEM_Q2_2D, PIN>
                                                : (const void*)k_vcycle<FEM_HEX8, PIN>);
}
static const void* cg_fn(int kind, int pinned) { return pinned ? cg_fn_p<true>(kind) : cg_fn_p<false>(kind); }
static const void* vc_fn(int kind, int pinned) { return pinned ? vc_fn_p<true>(kind) : vc_fn_p<false>(kind); }
// dynamic smem of a launch: the region of the CTA-0 levels' 1/D only when they run
// (shared memory taken from the L1 carveout otherwise costs cache for nothing)
static size_t cg_dyn_smem(const CgArgs& A) {
  return (size_t)(128 + FEM_TILE_SMEM + FEM_TAB_SMEM + (A.block_smem_from < A.nlev ? FEM_BLK_SMEM : 0)) *
         sizeof(double);
}
int fem_launch_cg(const CgArgs& A, int grid, double* cr, double* cp, double* cq, cudaStream_t s) {
  CgArgs a = A;
  void* args[] = {&a, &cr, &cp, &cq};
  return coop_launch(cg_fn(A.lv[0].g.kind, A.pinned), grid, args, s, "k_cg", cg_dyn_smem(A));
}
int fem_launch_vcycle(const CgArgs& A, int grid, double* cr, double* cp, double* cq, double* z, cudaStream_t s) {
  CgArgs a = A;
  void* args[] = {&a, &cr, &cp, &cq, &z};
  return coop_launch(vc_fn(A.lv[0].g.kind, A.pinned), grid, args, s, "k_vcycle", cg_dyn_smem(A));
}
int fem_coop_occupancy_cg(int* occ) {
  int m = 1 << 30;
  for (int kind = 0; kind < 3; ++kind)
    for (int pin = 0; pin < 2; ++pin) {
      const void* fns[2] = {cg_fn(kind, pin), vc_fn(kind, pin)};
      for (const void* fn : fns) {
        // allow the dynamic smem of the tile buffer and the stencil tables
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, FEM_DYN_SMEM_MAX) != cudaSuccess)
          return -1;
        int a = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, fn, FEM_THREADS, FEM_DYN_SMEM_MAX) != cudaSuccess)
          return -1;
        m = a < m ? a : m;
      }
    }
  *occ = m;
  return 0;
}
