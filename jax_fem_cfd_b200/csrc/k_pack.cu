// Packed 4-step projection step for serving: one persistent cooperative launch
// advances every active request of one mesh size by `steps` steps.
//
// Grid (ctas, active members): blockIdx.y picks an active member (a request),
// its blockIdx.x < ctas CTAs are the group that runs the member's whole step,
// stage after stage, with the member's own barrier counters. Inside a group the stages are the stage bodies
// of the solo kernels (fem_step_body.cuh, the BiCGSTAB and MG-PCG solves), run
// on the same number of CTAs as the member's solo solves, so a packed request's
// results equal the solo fem_step4's bit for bit. Groups never wait on each other:
// a member with a slow solve holds only its own CTAs.
//
// The step (solvers/standard.py:148-165, theta = 1/2, rho = 1, Ce(U_n) with
// beta = 1/2 applied on the fly, pinned pressure with the multigrid V-cycle):
//   1. Gauss-point factors of Ce(U_n); (mu Le + Ce) U_n
//   2. momentum rhs and x0, G P_n
//   3. BiCGSTAB on (1/dt) Me + theta (Ce + mu Le), identity rows on gamma_d
//   4. U* = U_hat + dt G P_n / M
//   5. PPE rhs and x0
//   6. MG-PCG pressure solve
//   7. U = U* - dt G P / M, U_d on gamma_d
#include "fem_cg_body.cuh"
#include "fem_bicgstab_body.cuh"
#include "fem_step_body.cuh"

// dynamic smem (doubles): [0,128) reductions | tiles of the convection apply,
// the BiCGSTAB operator and the CG phases | CG stencil tables | 1/D of the
// multigrid levels run inside one CTA
#define FEM_PACK_SMEM (128 + FEM_CONV_SMEM + FEM_TAB_SMEM + FEM_BLK_SMEM)
static_assert(FEM_CONV_SMEM >= FEM_TILE_SMEM, "the tile region holds the CG tiles too");

template <int KIND>
__global__ void __launch_bounds__(FEM_THREADS, 1) k_step_pack(const PackMember* __restrict__ mem,
                                                              const __grid_constant__ PackParams P) {
  extern __shared__ __align__(128) double smem[];
  __shared__ __align__(16) CgArgs sC;
  __shared__ __align__(16) BiArgs sB;
  __shared__ __align__(16) StepArgs sS;
  __shared__ double sKd[81], sLe[81];
  __shared__ unsigned int s_round, s_team_round;
  constexpr int NEN = KI<KIND>::NEN;
  const int mi = P.idx[blockIdx.y];  // the member this group runs
  const PackStep ps = P.m[mi];
  if (ps.steps <= 0) return;  // (not launched by fem_pack_step; a group with nothing to do leaves)
  const PackMember& M = mem[mi];
  fem_stage_args(M.C, &sC);
  fem_stage_args(M.B, &sB);
  fem_stage_args(M.S, &sS);
  fem_tables_to_smem<KIND>(sC, smem + 128 + FEM_CONV_SMEM);
  fem_block_levels_to_smem(sC, smem + 128 + FEM_CONV_SMEM + FEM_TAB_SMEM);
  const double theta = 0.5, rho = 1.0, dt = ps.dt, mu = ps.mu;
  // the momentum operator's shared matrix (the solo step's k_lincomb expression)
  const double ka = rho / dt, kb = theta * mu;
  for (int t = threadIdx.x; t < NEN * NEN; t += blockDim.x) {
    sKd[t] = ka * sS.Me[t] + kb * sS.Le[t];
    sLe[t] = sS.Le[t];
  }
  if (threadIdx.x == 0) {
    s_round = 0u;
    s_team_round = 0u;
    sS.dt = dt;
    sS.mu = mu;
    sS.rho = rho;
    sS.theta = theta;
  }
  __syncthreads();
  const MatCombo op{sKd, 1.0, nullptr, 0.0, 0, nullptr, 0.0};
  const FemC3Tma tma{nullptr, nullptr, sC.sync.err};  // 2D: no TMA factor copies
  const GridTeam gt = GridTeam::grid(&sC.sync, &s_round);
  const size_t nn = sS.g.nn;
  int* stat = M.stat;
  fem_zero_partials(sC.sync);
  if (!gt.sync()) return;
  for (int j = 0; j < ps.steps; ++j) {
    const int cur = (ps.cur + j) & 1;
    double* Un = M.U[cur];
    double* Pn = M.P[cur];
    double* Uo = M.U[cur ^ 1];
    double* Po = M.P[cur ^ 1];
    // 1. Ce(U_n) factors (beta = 1/2), then (mu Le + rho Ce) U_n
    step_conv_factors<KIND>(sS.g, sB.qt, Un, 0.5, M.cvf);
    if (!gt.sync()) return;
    step_conv_apply<KIND, 2>(sS.g, sB.qt, M.cvf, rho, mu, sLe, Un, M.vcv, smem + 128);
    if (!gt.sync()) return;
    // 2. momentum rhs, x0 and G P_n
    step_mom_rhs<KIND>(sS, Un, Pn, M.Ud, nullptr, M.rhsU, M.Uhat, M.gPn);
    if (!gt.sync()) return;
    // 3. momentum BiCGSTAB (ends on a barrier)
    bicgstab_solve<KIND, 2, true>(sB, op, smem, smem + 128, tma, &s_round);
    // 4. U*
    step_ustar((int)(2 * nn), dt / rho, M.Uhat, M.gPn, sS.M, M.Ustar);
    if (!gt.sync()) return;
    // 5. PPE rhs, x0 into the output pressure
    step_p_rhs<KIND>(sS, M.Ustar, nullptr, Pn, M.rhsP, Po);
    if (threadIdx.x == 0) sC.x = Po;
    if (!gt.sync()) return;
    // 6. pressure MG-PCG (its pinned rows are zeroed after its last barrier)
    cg_solve<KIND, true>(sC, smem, &s_round, &s_team_round, M.cr, M.cp, M.cq);
    if (!gt.sync()) return;
    // 7. projection and Dirichlet values
    step_ufinal<KIND>(sS, M.Ustar, Po, M.Ud, Uo);
    if (blockIdx.x == 0 && threadIdx.x == 0) stat[4] |= stat[2] | stat[3];
    if (!gt.sync()) return;
  }
}

int fem_launch_step_pack(int kind, const PackMember* members, const PackParams& P, int k, int ctas, int blk,
                         cudaStream_t s) {
  if (kind != FEM_Q1_2D || k < 1 || k > FEM_PACK_MAX || ctas < 1) return FEM_E_ARG;
  const void* fn = (const void*)k_step_pack<FEM_Q1_2D>;
  // the region of the CTA-0 multigrid levels' 1/D only when they run
  const int dyn = (FEM_PACK_SMEM - (blk ? 0 : FEM_BLK_SMEM)) * (int)sizeof(double);
  cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, FEM_PACK_SMEM * (int)sizeof(double));
  const PackMember* m = members;
  PackParams p = P;
  void* args[] = {&m, &p};
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas, k);
  cfg.blockDim = dim3(FEM_THREADS);
  cfg.stream = s;
  cfg.dynamicSmemBytes = dyn;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelExC(&cfg, fn, args);
  return fem_after_launch("k_step_pack");
}

int fem_pack_occupancy(int* per_sm) {
  const void* fn = (const void*)k_step_pack<FEM_Q1_2D>;
  const int dyn = FEM_PACK_SMEM * (int)sizeof(double);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, FEM_THREADS, dyn) != cudaSuccess) return -1;
  return 0;
}
