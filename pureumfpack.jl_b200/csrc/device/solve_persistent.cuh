// solve_persistent.cuh -- one persistent launch per solve pass.
//
// The supernodal solve (src/solve.jl:10-39 restated by supernode, see
// solve_kernels.cuh) is a chain of dependent steps: per tree level the small
// supernodes, the gather of the large supernodes' right-hand-side blocks and
// their block products.  As separate launches many of these steps are a few
// microseconds of work behind a launch and a drain.
// Here one cooperative launch (every CTA resident) walks the whole step
// table: each step's work items (supernode x right-hand-side chunk, GEMM
// tile) are spread over the CTAs, and a grid barrier
// separates dependent steps.  The barrier is this library's own and is
// bounded in time: a CTA that waits longer than the handle's wait limit
// (GridBarrier::wait_ns, kBarrierWaitNs unless set) raises the error word and
// leaves, so a stuck launch turns into an error status, and every later
// barrier of the launch fails at once.
#pragma once

#include "gemm_kernels.cuh"
#include "solve_kernels.cuh"

namespace mfgpu {

constexpr uint64_t kBarrierWaitNs = 4000000000ull;   // 4 s

enum SolvePhaseKind : int32_t {
  kPhFwdSmall = 0, kPhFwdAssemble = 1, kPhGemm = 3, kPhBwdSmall = 4, kPhBwdGather = 5
};

struct SolvePhase {
  int32_t kind;
  int32_t rows;      // items of one task: right-hand-side chunks (or 1 for GEMM tiles)
  int64_t first;     // offset into ids / blocks / gemms
  int64_t count;     // tasks (GEMM: task count for the tile search)
  int64_t items;     // work items of the phase (count * rows, or tiles)
};

struct GridBarrier {
  unsigned int* count;   // arrivals of the current barrier
  unsigned int* gen;     // barrier generation
  int* err;              // err[0]: a barrier of this launch failed; err[1]: sticky over launches
  uint64_t wait_ns;      // bound on one CTA's wait at a barrier
  const int* stall;      // test hook (mfgpu_test_stall): CTA 0 never arrives, the others' waits expire
};

__device__ __forceinline__ uint64_t solve_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Bounded grid-wide barrier.  Block-uniform result: false when this CTA gave
// up waiting or another one already did.
__device__ __forceinline__ bool grid_barrier(const GridBarrier& b) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int good = 1;
    volatile unsigned int* vgen = b.gen;
    volatile int* verr = b.err;
    const unsigned int g = *vgen;
    __threadfence();
    if (*b.stall && blockIdx.x == 0) {
      good = -1;   // never arrives and leaves without a word: every other CTA's wait runs out by the clock
    } else if (atomicAdd(b.count, 1u) + 1u == gridDim.x) {
      atomicExch(b.count, 0u);
      __threadfence();
      atomicAdd(b.gen, 1u);
    } else {
      const uint64_t t0 = solve_ns();
      for (unsigned int i = 1; *vgen == g; ++i) {
        if ((i & 63u) == 0u && (*verr || solve_ns() - t0 > b.wait_ns)) {
          good = 0;
          break;
        }
      }
    }
    __threadfence();
    if (good == 0 || (good > 0 && *verr)) {
      atomicOr(b.err, 1);
      atomicOr(b.err + 1, 1);
      good = 0;
    }
    ok = good > 0;
  }
  __syncthreads();
  return ok != 0;
}

struct PersistentArgs {
  const SolvePhase* phases;
  int32_t nphases;
  const int32_t* ids;
  const GemmTask* gemms;
  GridBarrier bar;
  unsigned long long* stamps;   // nphases + 1 globaltimer stamps (profiling) or nullptr
};

template <typename T>
__device__ __forceinline__ void gemm_tile(const GemmTask* tasks, int ntasks, const T* pa, const T* pb, T* pc,
                                          int64_t tile, T* smem);
template <>
__device__ __forceinline__ void gemm_tile<double>(const GemmTask* tasks, int ntasks, const double* pa,
                                                  const double* pb, double* pc, int64_t tile, double* smem) {
  gemm_tile_f64(tasks, ntasks, pa, pb, pc, tile, smem);
}
template <>
__device__ __forceinline__ void gemm_tile<float>(const GemmTask* tasks, int ntasks, const float* pa,
                                                 const float* pb, float* pc, int64_t tile, float* smem) {
  gemm_tile_f32(tasks, ntasks, pa, pb, pc, tile, smem);
}

// Shared memory of the persistent kernel: the largest item's need.
template <typename T>
constexpr size_t persistent_smem_bytes() {
  constexpr size_t small = (size_t)2 * kSmallFront * kSolveCols * sizeof(T);
  constexpr size_t gemm = sizeof(T) == 8 ? (size_t)kGemmSmemF64 * 8 : (size_t)kGemmSmemF32 * 4;
  return small > gemm ? small : gemm;
}

template <typename T>
__global__ void __launch_bounds__(kSolveThreads) k_solve_persistent(DevPlan P, DevState S, SolveArgs A,
                                                                    PersistentArgs X, const T* __restrict__ pool,
                                                                    T* fsol, T* xw) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  if (X.stamps && blockIdx.x == 0 && threadIdx.x == 0) X.stamps[0] = solve_ns();
  for (int p = 0; p < X.nphases; ++p) {
    const SolvePhase ph = X.phases[p];
    for (int64_t it = blockIdx.x; it < ph.items; it += gridDim.x) {
      if (ph.kind == kPhGemm) {
        gemm_tile<T>(X.gemms + ph.first, (int)ph.count, pool, fsol, fsol, it, sm);
        continue;
      }
      const int bx = (int)(it % ph.count), by = (int)(it / ph.count);
      switch (ph.kind) {
        case kPhFwdSmall: fwd_small_item<T>(P, S, A, X.ids + ph.first, pool, fsol, bx, by, sm); break;
        case kPhFwdAssemble: fwd_assemble_item<T>(P, S, A, X.ids + ph.first, fsol, bx, by); break;
        case kPhBwdSmall: bwd_small_item<T>(P, A, X.ids + ph.first, pool, fsol, xw, bx, by, sm); break;
        case kPhBwdGather: bwd_gather_item<T>(P, A, X.ids + ph.first, fsol, xw, bx, by); break;
        default: break;
      }
      __syncwarp();
    }
    if (!grid_barrier(X.bar)) return;
    if (X.stamps && blockIdx.x == 0 && threadIdx.x == 0) X.stamps[p + 1] = solve_ns();
  }
}

}  // namespace mfgpu
