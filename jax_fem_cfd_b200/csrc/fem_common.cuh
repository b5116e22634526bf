// Common device-side building blocks for the B200 matrix-free FEM path.
//
// Meshes are the structured lattices of jax_fem_cfd setup/regular_mesh.py
// (quad4 / quad9 2D, periodic or not, hex8 3D). Connectivity is never read
// from memory: a node's incident elements and its local index in each are
// computed from its lattice coordinates, and an element's nodes from the
// element's lattice coordinates. This reproduces nconn of regular_mesh.py
// exactly (local node order, periodic wrap) at zero connectivity bytes.
//
// Every assembled product y = sum_e P_e^T A_e P_e x is evaluated node-centrically:
// the thread that owns output node n sums the rows of its incident elements in a
// fixed order, so results are bitwise reproducible run to run without atomics or
// element colouring (the reference's segment_sum is an atomic scatter on GPU).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define FEM_Q1_2D 0
#define FEM_Q2_2D 1
#define FEM_HEX8 2

#define FEM_MAX_NEN 9

struct FemGrid {
  int kind;       // FEM_Q1_2D | FEM_Q2_2D | FEM_HEX8
  int periodic;   // 2D only
  int nex, ney, nez;
  int nnx, nny, nnz;  // unique-node lattice extents (periodic drops the duplicate row/column)
  int nn, ne, nen;
};

// local node a of an element sits at lattice offset (di[a], dj[a], dk[a]) from
// (s*ie, s*je, ke), s = 2 for quad9 (setup/regular_mesh.py:24-26, 68-73, 119-126).
// Tables are bit-packed constants (2 bits per entry) so they stay in registers.
//   quad9 di = 0,1,2,2,2,1,0,0,1   dj = 0,0,0,1,2,2,2,1,1
//   quad4 di = 0,1,1,0             dj = 0,0,1,1   (hex8: same, dk = a >> 2)
#define FEM_Q2_DI 0x106A4u  // entries a = 0..8 at bits 2a
#define FEM_Q2_DJ 0x16A40u
#define FEM_Q1_DI 0x14u
#define FEM_Q1_DJ 0x50u
__device__ __forceinline__ void fem_local_offset(int kind, int a, int& di, int& dj, int& dk) {
  if (kind == FEM_Q2_2D) {
    di = (FEM_Q2_DI >> (2 * a)) & 3;
    dj = (FEM_Q2_DJ >> (2 * a)) & 3;
    dk = 0;
  } else {
    di = (FEM_Q1_DI >> (2 * (a & 3))) & 3;
    dj = (FEM_Q1_DJ >> (2 * (a & 3))) & 3;
    dk = (kind == FEM_HEX8) ? (a >> 2) : 0;
  }
}

// Inverse tables, indexed [dj][di]: quad9 {0,1,2,7,8,3,6,5,4} (4 bits per
// entry), quad4 {0,1,3,2} (2 bits per entry).
#define FEM_Q2_INV 0x456387210ull
#define FEM_Q1_INV 0xB4u
__device__ __forceinline__ int fem_local_index(int kind, int di, int dj, int dk) {
  if (kind == FEM_Q2_2D) return (int)((FEM_Q2_INV >> (4 * (dj * 3 + di))) & 15ull);
  return (int)((FEM_Q1_INV >> (2 * (dj * 2 + di))) & 3u) + 4 * dk;
}

struct FemElem {
  int ie, je, ke;
  int e;
};

__device__ __forceinline__ int fem_node_at(const FemGrid& g, int i, int j, int k) {
  if (g.periodic) {
    if (i >= g.nnx) i -= g.nnx;
    if (j >= g.nny) j -= g.nny;
  }
  return (k * g.nny + j) * g.nnx + i;
}

// Global node index of local node b of element (ie, je, ke).
__device__ __forceinline__ int fem_elem_node(const FemGrid& g, int ie, int je, int ke, int b) {
  int di, dj, dk;
  fem_local_offset(g.kind, b, di, dj, dk);
  const int s = (g.kind == FEM_Q2_2D) ? 2 : 1;
  return fem_node_at(g, s * ie + di, s * je + dj, ke + dk);
}

__device__ __forceinline__ void fem_node_ijk(const FemGrid& g, int n, int& i, int& j, int& k) {
  i = n % g.nnx;
  int t = n / g.nnx;
  j = t % g.nny;
  k = t / g.nny;
}

// Candidate (element coordinate, local offset) pairs along one lattice axis for
// lattice coordinate c: (e0, d0) and, when the count is 2, (e1, d1). The
// element on the low side (node is its last node along the axis) comes first.
__device__ __forceinline__ int fem_axis_candidates(int kind, int periodic, int c, int nel, int& e0, int& d0,
                                                   int& e1, int& d1) {
  int h = c, dl = 1;
  if (kind == FEM_Q2_2D) {
    if (c & 1) {
      e0 = (c - 1) >> 1;
      d0 = 1;
      return 1;
    }
    h = c >> 1;
    dl = 2;
  }
  const bool has_lo = (h >= 1) || periodic;
  const int elo = (h >= 1) ? h - 1 : nel - 1;
  const bool has_hi = h < nel;
  if (has_lo && has_hi) {
    e0 = elo; d0 = dl; e1 = h; d1 = 0;
    return 2;
  }
  if (has_lo) {
    e0 = elo; d0 = dl;
    return 1;
  }
  e0 = h; d0 = 0;
  return 1;
}

// Iterate over (element, local index) pairs incident to node n and call
// f(ie, je, ke, e, a). Order: k-candidates outer, then j, then i.
template <class F>
__device__ __forceinline__ void fem_for_incident(const FemGrid& g, int n, F&& f) {
  int i, j, k;
  fem_node_ijk(g, n, i, j, k);
  int ei0, ei1 = 0, di0, di1 = 0, ej0, ej1 = 0, dj0, dj1 = 0, ek0 = 0, ek1 = 0, dk0 = 0, dk1 = 0;
  const int ni = fem_axis_candidates(g.kind, g.periodic, i, g.nex, ei0, di0, ei1, di1);
  const int nj = fem_axis_candidates(g.kind, g.periodic, j, g.ney, ej0, dj0, ej1, dj1);
  int nk = 1;
  if (g.kind == FEM_HEX8) nk = fem_axis_candidates(FEM_HEX8, 0, k, g.nez, ek0, dk0, ek1, dk1);
  const int cnt = ni * nj * nk;
#pragma unroll 1
  for (int z = 0; z < cnt; ++z) {
    const int zi = z % ni, zj = (z / ni) % nj, zk = z / (ni * nj);
    const int ei = zi ? ei1 : ei0, di = zi ? di1 : di0;
    const int ej = zj ? ej1 : ej0, dj = zj ? dj1 : dj0;
    const int ek = zk ? ek1 : ek0, dk = zk ? dk1 : dk0;
    const int e = (ek * g.ney + ej) * g.nex + ei;
    f(ei, ej, ek, e, fem_local_index(g.kind, di, dj, dk));
  }
}

// ---------------------------------------------------------------------------
// Teams: a set of threads that executes one solver phase, with its own barrier
// and deterministic reductions. GridTeam = every thread of a cooperative
// (co-resident) launch; BlockTeam = the threads of one CTA (coarse levels).
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned long long fem_globaltimer_early() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

#define FEM_ERR_BARRIER_TIMEOUT 1
#define FEM_ERR_NONFINITE 2
#define FEM_ERR_MAXITER 4
#define FEM_ERR_BREAKDOWN 8
#define FEM_ERR_BAD_ARG 16
#define FEM_ERR_WATCHDOG 32

// Wall-clock budget of one persistent solve. CTA 0 raises FEM_ERR_WATCHDOG
// before a barrier once it is exceeded; every CTA sees the flag after that
// barrier and leaves the loop at the same iteration.
#define FEM_WATCHDOG_NS 10000000000ull
__device__ __forceinline__ void fem_watchdog_arm(int* err, unsigned long long t0) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && fem_globaltimer_early() - t0 > FEM_WATCHDOG_NS) atomicOr(err, FEM_ERR_WATCHDOG);
}
__device__ __forceinline__ bool fem_watchdog_fired(const int* err) {
  return (*(volatile const int*)err & FEM_ERR_WATCHDOG) != 0;
}

struct FemSync {
  unsigned int* count;    // arrivals in the current barrier generation
  unsigned int* team_count;  // arrivals at the coarse-level team barrier (GridTeam::team)
  int* err;               // sticky error flags (FEM_ERR_*)
  double* partials;       // [slot][cta] partial sums
  int nslots;
  unsigned long long* trace;  // optional: globaltimer at each barrier exit (CTA 0), trace[0] = count
  int trace_cap;
};

__device__ __forceinline__ unsigned int fem_ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fem_st_release(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long fem_globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier wait limit: a wait that exceeds it sets FEM_ERR_BARRIER_TIMEOUT and
// every CTA leaves the kernel at its next barrier instead of hanging the GPU.
#define FEM_BARRIER_TIMEOUT_NS 2000000000ull

// Diagnostic trace (CTA 0, thread 0): appends %globaltimer | (tag << 56) to
// trace[1..], trace[0] = count. The running count lives in shared memory
// (fem_trace_init at kernel start), so a mark is two stores and no load.
__device__ __forceinline__ int* fem_trace_count() {
  __shared__ int n;
  return &n;
}
__device__ __forceinline__ void fem_trace_init(const FemSync& s) {
  if (s.trace && blockIdx.x == 0 && threadIdx.x == 0) *fem_trace_count() = (int)s.trace[0];
}
__device__ __forceinline__ void fem_trace_put(unsigned long long* tr, int cap, unsigned long long tag) {
  int* cnt = fem_trace_count();
  const int n = *cnt + 1;
  if (n < cap) {
    tr[n] = (fem_globaltimer() & 0x00FFFFFFFFFFFFFFull) | (tag << 56);
    tr[0] = (unsigned long long)n;
    *cnt = n;
  }
}
__device__ __forceinline__ void fem_trace_mark(const FemSync& s, unsigned long long tag) {
  if (s.trace && blockIdx.x == 0 && threadIdx.x == 0) fem_trace_put(s.trace, s.trace_cap, tag);
}

// Shared-memory staging from global memory. fem_stage issues dst[q] = src[idx(q)]
// for q < n by 8-byte cp.async (no register round trip, every copy of the
// thread in flight); fem_stage_wait completes all of them and makes them visible
// to the whole CTA. Sources are global-memory vectors (one code path keeps the
// persistent solvers' hot code small).
template <class Idx>
__device__ __forceinline__ void fem_stage(double* dst, const double* src, int n, const Idx& idx) {
  if (src == nullptr) return;  // unused source slot
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst + q);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(src + idx(q)) : "memory");
  }
}
// Row-wise staging of an SH x SW region: dst[r * SW + c] = src[rowbase(r) + colx(c)].
// Each thread owns one column (its wrapped / clamped x is computed once) and
// walks rows, so an element costs one multiply-add instead of a full 2D
// index decomposition.
template <class RowBase, class ColX>
__device__ __forceinline__ void fem_stage_2d(double* dst, const double* src, int SW, int SH, const RowBase& rowbase,
                                             const ColX& colx) {
  if (src == nullptr) return;
  const int tpr = blockDim.x / SW;  // rows in flight per pass
  const int c = threadIdx.x % SW, r0 = threadIdx.x / SW;
  if (r0 >= tpr) return;
  const int gx = colx(c);
  for (int r = r0; r < SH; r += tpr) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(dst + r * SW + c);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(src + rowbase(r) + gx) : "memory");
  }
}
__device__ __forceinline__ void fem_stage_wait() {
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
}
__device__ __forceinline__ int fem_floordiv2(int v) { return v >> 1; }  // arithmetic shift: floor for v < 0
// v mod n in [0, n) for any int v (periodic lattice coordinates of staged halos,
// which can lie more than one period away when a tile is wider than the level)
__device__ __forceinline__ int fem_wrap(int v, int n) {
  if ((unsigned)v < (unsigned)n) return v;
  if (v < 0 && v >= -n) return v + n;
  if (v >= n && v < 2 * n) return v - n;
  v %= n;
  return v < 0 ? v + n : v;
}

// Grid barrier on a monotonic arrival counter (reset to 0 before each launch):
// barrier number k of the launch completes when the counter reaches
// k * gridDim.x. One fire-and-forget release-add per CTA, then acquire polling.
// Bounded barrier on a monotonic arrival counter shared by `parties` CTAs
// (thread 0 of each; reset to 0 before each launch): barrier number k of the
// launch completes when the counter reaches k * parties. Ordering: the CTA's
// writes reach thread 0 through __syncthreads, its release-add publishes them
// at gpu scope, the pollers' acquire-load of the final count orders every later
// read after them, and the closing __syncthreads passes that on to the CTA's
// other threads. Returns false on timeout (or a timeout raised elsewhere).
struct FemNoPartials {
  __device__ __forceinline__ void warp_part(double*) const {}
  __device__ __forceinline__ void store(const FemSync*, const double*) const {}
};
// K per-thread values bound for K partial slots, summed as part of a barrier:
// warps reduce by a fixed shuffle tree, thread 0 adds the warp sums in warp
// order and writes this CTA's partials right before it arrives.
template <int K>
struct FemPartials {
  double* v;         // the thread's K values (summed in place)
  const int* slots;  // K slot numbers
  __device__ __forceinline__ void warp_part(double* smem) const {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    }
    if (lane == 0)
#pragma unroll
      for (int q = 0; q < K; ++q) smem[q * 16 + warp] = v[q];
  }
  __device__ __forceinline__ void store(const FemSync* s, const double* smem) const {
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double t = 0.0;
      for (int w = 0; w < nw; ++w) t += smem[q * 16 + w];
      s->partials[(size_t)slots[q] * gridDim.x + blockIdx.x] = t;
    }
  }
};

// A party whose wait times out also sets FEM_BAR_ABORT in the arrival counter:
// every other poller then sees a count at or above its target with that bit
// set and leaves at this barrier, with no separate load of the error word after
// each completed wait (counts stay far below the bit: k * parties).
#define FEM_BAR_ABORT 0x40000000u
template <class Parts = FemNoPartials>
__device__ __forceinline__ bool fem_counter_barrier(const FemSync* s, unsigned int* cnt, unsigned int* round,
                                                    int parties, unsigned long long tag, const Parts& parts = Parts(),
                                                    double* smem = nullptr) {
  __shared__ int s_ok;
  parts.warp_part(smem);
  __syncthreads();
  if (threadIdx.x == 0) {
    parts.store(s, smem);
    int ok = 1;
    const unsigned int target = (*round + 1u) * (unsigned)parties;
    *round = *round + 1u;
    int* err = s->err;
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(cnt), "r"(1u) : "memory");
    if (parties > 1) {
      const unsigned long long t0 = fem_globaltimer();
      unsigned int polls = 0, c;
      while ((c = fem_ld_acquire(cnt)) < target) {
        if (((++polls) & 63u) == 0u) {
          // a timeout raised by another party on another counter
          if (*(volatile int*)err & FEM_ERR_BARRIER_TIMEOUT) { ok = 0; break; }
          if (fem_globaltimer() - t0 > FEM_BARRIER_TIMEOUT_NS) {
            atomicOr(err, FEM_ERR_BARRIER_TIMEOUT);
            atomicOr(cnt, FEM_BAR_ABORT);
            ok = 0;
            break;
          }
        }
      }
      if (c & FEM_BAR_ABORT) ok = 0;
    }
    s_ok = ok;
    if (s->trace && blockIdx.x == 0) fem_trace_put(s->trace, s->trace_cap, tag);
  }
  __syncthreads();
  return s_ok != 0;
}

// A set of CTAs that synchronise on one arrival counter: every CTA of the
// launch (grid(): cooperative, all co-resident), or the first n CTAs (team():
// the coarse multigrid levels, with their own counter). One type for both, so
// the phase functions are compiled once.
struct GridTeam {
  const FemSync* s;     // the launch's barrier state (shared-memory copy of the kernel arguments)
  unsigned int* cnt;    // arrival counter (global)
  unsigned int* round;  // per-CTA count of completed barriers on cnt (shared memory, thread 0, starts at 0)
  int n;                // CTAs taking part: blockIdx.x < n
  unsigned int tag;     // trace tag of its barriers
  __device__ static GridTeam grid(const FemSync* s, unsigned int* round) {
    return GridTeam{s, s->count, round, (int)gridDim.x, 31u};
  }
  __device__ static GridTeam team(const FemSync* s, unsigned int* round, int n) {
    return GridTeam{s, s->team_count, round, n, 30u};
  }
  __device__ __forceinline__ int rank() const { return blockIdx.x * blockDim.x + threadIdx.x; }
  __device__ __forceinline__ int size() const { return n * blockDim.x; }
  __device__ __forceinline__ int cta() const { return blockIdx.x; }
  __device__ __forceinline__ int ncta() const { return n; }
  __device__ bool sync() const { return fem_counter_barrier(s, cnt, round, n, tag); }
  // reduce K values into K partial slots and sync, in one step (smem: 16*K doubles)
  template <int K>
  __device__ bool reduce_sync(double (&v)[K], const int (&slots)[K], double* smem) const {
    return fem_counter_barrier(s, cnt, round, n, tag, FemPartials<K>{v, slots}, smem);
  }
};

struct BlockTeam {
  __device__ __forceinline__ int rank() const { return threadIdx.x; }
  __device__ __forceinline__ int size() const { return blockDim.x; }
  __device__ __forceinline__ int cta() const { return 0; }
  __device__ __forceinline__ int ncta() const { return 1; }
  __device__ __forceinline__ bool sync() const {
    __syncthreads();
    return true;
  }
};

// Deterministic block-wide sum of K values (fixed shuffle tree + fixed warp order).
template <int K>
__device__ __forceinline__ void fem_block_sum(double (&v)[K], double* smem /* >= 16*K (32*K above 512 threads) */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  const int S = nw > 16 ? 32 : 16;
#pragma unroll
  for (int q = 0; q < K; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < K; ++q) smem[q * S + warp] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < K; ++q) {
    double t = (lane < nw) ? smem[q * S + lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    v[q] = t;
  }
}

// Reduction handles. reduce() is called by every thread of the team inside a
// phase; totals are read by result() after the team's next sync().
struct GridReducer {
  const FemSync* s;
  template <int K>
  __device__ __forceinline__ void reduce(double (&v)[K], int slot, double* smem) const {
    fem_block_sum<K>(v, smem);
    if (threadIdx.x == 0) {
      double* part = s->partials;
#pragma unroll
      for (int q = 0; q < K; ++q) part[(size_t)(slot + q) * gridDim.x + blockIdx.x] = v[q];
    }
  }
  // One block sum for K values bound for any K slots.
  template <int K>
  __device__ __forceinline__ void reduce_slots(double (&v)[K], const int (&slots)[K], double* smem) const {
    fem_block_sum<K>(v, smem);
    if (threadIdx.x == 0) {
      double* part = s->partials;
#pragma unroll
      for (int q = 0; q < K; ++q) part[(size_t)slots[q] * gridDim.x + blockIdx.x] = v[q];
    }
  }
  // Totals of K <= 8 slots (any slot numbers). Thread c loads CTA c's partial of
  // every slot (all loads of a thread in flight at once), warps combine theirs
  // by a fixed shuffle tree, and every thread adds the warp sums in warp order:
  // the same order, hence the same bits, in every CTA. Uses smem[0, 16*K).
  // Split in two so that other loads (a phase's staging copies) can be issued
  // between them: result_begin issues this thread's partial loads,
  // result_end combines them (both called by every thread of the CTA).
  template <int K>
  struct Pending {
    double acc[K];
  };
  __device__ __forceinline__ int data_warps() const {
    int nwd = (gridDim.x + 31) >> 5;
    if (nwd > 16) nwd = 16;
    if (nwd > (int)(blockDim.x >> 5)) nwd = blockDim.x >> 5;
    return nwd;
  }
  template <int K>
  __device__ __forceinline__ Pending<K> result_begin(const int (&slots)[K]) const {
    static_assert(K <= 8, "result_slots: at most 8 slots");
    Pending<K> p;
    const int G = gridDim.x, nwd = data_warps();
    const double* __restrict__ part = s->partials;
#pragma unroll
    for (int q = 0; q < K; ++q) p.acc[q] = 0.0;
    if ((int)(threadIdx.x >> 5) < nwd) {
      // first column: plain loads, not consumed here (result_end waits for them)
      if ((int)threadIdx.x < G)
#pragma unroll
        for (int q = 0; q < K; ++q) p.acc[q] = __ldcg(&part[(size_t)slots[q] * G + threadIdx.x]);
      for (int c = threadIdx.x + nwd * 32; c < G; c += nwd * 32) {
#pragma unroll
        for (int q = 0; q < K; ++q) p.acc[q] += __ldcg(&part[(size_t)slots[q] * G + c]);
      }
    }
    return p;
  }
  template <int K>
  __device__ __forceinline__ void result_end(Pending<K>& p, double (&out)[K], double* smem) const {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwd = data_warps();
    __syncthreads();
    if (warp < nwd) {
#pragma unroll
      for (int q = 0; q < K; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p.acc[q] += __shfl_xor_sync(0xffffffffu, p.acc[q], o);
      }
      if (lane == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) smem[q * 16 + warp] = p.acc[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double t = 0.0;
      for (int w = 0; w < nwd; ++w) t += smem[q * 16 + w];
      out[q] = t;
    }
    __syncthreads();
  }
  template <int K>
  __device__ __forceinline__ void result_slots(double (&out)[K], const int (&slots)[K], double* smem) const {
    Pending<K> p = result_begin<K>(slots);
    result_end<K>(p, out, smem);
  }
  template <int K>
  __device__ __forceinline__ void result(double (&out)[K], int slot, double* smem) const {
    int sl[K];
#pragma unroll
    for (int q = 0; q < K; ++q) sl[q] = slot + q;
    result_slots<K>(out, sl, smem);
  }
};

struct BlockReducer {
  double* store;  // shared memory, >= nslots doubles
  template <int K>
  __device__ __forceinline__ void reduce(double (&v)[K], int slot, double* smem) const {
    fem_block_sum<K>(v, smem);
    if (threadIdx.x == 0)
#pragma unroll
      for (int q = 0; q < K; ++q) store[slot + q] = v[q];
  }
  template <int K>
  __device__ __forceinline__ void reduce_slots(double (&v)[K], const int (&slots)[K], double* smem) const {
    fem_block_sum<K>(v, smem);
    if (threadIdx.x == 0)
#pragma unroll
      for (int q = 0; q < K; ++q) store[slots[q]] = v[q];
  }
  template <int K>
  __device__ __forceinline__ void result_slots(double (&out)[K], const int (&slots)[K], double*) const {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) out[q] = store[slots[q]];
  }
  template <int K>
  __device__ __forceinline__ void result(double (&out)[K], int slot, double*) const {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q) out[q] = store[slot + q];
  }
};

__device__ __forceinline__ bool fem_isfinite(double x) { return isfinite(x); }

// Node iteration in 2D tiles of 32 x (blockDim/32) lattice nodes, one tile per
// CTA at a time, so stencil neighbours in adjacent rows are read by the same
// CTA (L1 hits). f(n, x, y, z) with n the node index of lattice (x, y, z).
template <class Team, class F>
__device__ __forceinline__ void fem_tile_loop(const Team& tm, int nx, int ny, int nz, F&& f) {
  const int TY = blockDim.x >> 5;
  const int ntx = (nx + 31) >> 5, nty = (ny + TY - 1) / TY;
  const int nt2 = ntx * nty, ntile = nt2 * nz;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  for (int t = tm.cta(); t < ntile; t += tm.ncta()) {
    const int z = t / nt2, r = t - z * nt2, by = r / ntx, bx = r - by * ntx;
    const int x = bx * 32 + tx, y = by * TY + ty;
    if (x < nx && y < ny) f((z * ny + y) * nx + x, x, y, z);
  }
}
