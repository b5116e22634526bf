// Persistent cooperative BiCGSTAB kernel on element-by-element operators.
#include "fem_bicgstab_body.cuh"


template <int KIND, int NC, bool OTF>
__global__ void __launch_bounds__(FEM_THREADS, 1) k_bicgstab(const __grid_constant__ BiArgs A) {
  __shared__ double smem[128];
  __shared__ double sAsh[81];
  extern __shared__ __align__(128) double tsm[];  // staging of the tiled operator (dynamic)
  // hex8 on-the-fly convection: the mbarrier of its TMA factor copies
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ unsigned s_phase;
  if (OTF && KIND == FEM_HEX8 && threadIdx.x == 0) {
    fem_mbar_init(&s_bar, 1);
    s_phase = 0u;
  }
  const FemC3Tma tma{&s_bar, &s_phase, A.sync.err};
  MatCombo op = A.op;
  if (op.A) {
    for (int t = threadIdx.x; t < KI<KIND>::NEN * KI<KIND>::NEN; t += blockDim.x) sAsh[t] = op.A[t];
    op.A = sAsh;
  }
  __shared__ unsigned int s_round;
  if (threadIdx.x == 0) s_round = 0u;
  fem_trace_init(A.sync);
  __syncthreads();
  bicgstab_solve<KIND, NC, OTF>(A, op, smem, tsm, tma, &s_round);
}

static const void* bi_fn(int kind, int ncomp, bool otf) {
  if (otf && kind == FEM_HEX8) return (const void*)k_bicgstab<FEM_HEX8, 3, true>;
  if (otf) return kind == FEM_Q1_2D ? (const void*)k_bicgstab<FEM_Q1_2D, 2, true>
                                    : (const void*)k_bicgstab<FEM_Q2_2D, 2, true>;
  if (kind == FEM_Q1_2D)
    return ncomp == 1 ? (const void*)k_bicgstab<FEM_Q1_2D, 1, false> : (const void*)k_bicgstab<FEM_Q1_2D, 2, false>;
  if (kind == FEM_Q2_2D)
    return ncomp == 1 ? (const void*)k_bicgstab<FEM_Q2_2D, 1, false> : (const void*)k_bicgstab<FEM_Q2_2D, 2, false>;
  return ncomp == 1 ? (const void*)k_bicgstab<FEM_HEX8, 1, false> : (const void*)k_bicgstab<FEM_HEX8, 3, false>;
}
// dynamic smem (doubles) of the tiled operator: the EBE gather of fem_tiled_ebe
// needs NC (32+2R)(16+2R)(3 in 3D); hex8 per-element matrices the element-centric
// fem_tiled_ebe3e (fem_ebe3e_smem); the on-the-fly convection fem_conv_smem
static int bi_smem_doubles(int kind, int ncomp, bool otf) {
  if (otf && kind == FEM_HEX8) return FEM_C3_SMEM_MAX;
  if (otf) return FEM_CONV_SMEM;
  if (kind == FEM_HEX8) return fem_ebe3e_smem(3) > 3 * 1836 ? fem_ebe3e_smem(3) : 3 * 1836;
  return 3 * 1836;
}

int fem_launch_bicgstab(int ncomp, const BiArgs& A, int grid, cudaStream_t s) {
  BiArgs a = A;
  void* args[] = {&a};
  const bool otf = A.cvf != nullptr;
  if (otf && ncomp != (A.g.kind == FEM_HEX8 ? 3 : 2)) return FEM_E_ARG;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(FEM_THREADS);
  cfg.stream = s;
  cfg.dynamicSmemBytes = (size_t)bi_smem_doubles(A.g.kind, ncomp, otf) * sizeof(double);
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelExC(&cfg, bi_fn(A.g.kind, ncomp, otf), args);
  return fem_after_launch("k_bicgstab");
}
int fem_coop_occupancy_bi(int* occ) {
  int m = 1 << 30;
  for (int kind = 0; kind < 3; ++kind)
    for (int v = 0; v < 3; ++v) {
      const bool otf = (v == 2);
      const int nc = otf ? (kind == FEM_HEX8 ? 3 : 2) : v + 1;
      const void* fn = bi_fn(kind, nc, otf);
      const int dyn = bi_smem_doubles(kind, nc, otf) * (int)sizeof(double);
      if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) != cudaSuccess) return -1;
      int a = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, fn, FEM_THREADS, dyn) != cudaSuccess) return -1;
      m = a < m ? a : m;
    }
  *occ = m;
  return 0;
}
