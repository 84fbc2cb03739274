// gemm_kernels.cuh -- batched C -= A * B over heterogeneous problems.
//
// The dense updates of the large fronts (the trailing updates of the blocked
// pivot-block LU and the Schur update F22 -= L21 * U12 of
// src/multifrontal.jl:267-268) and the block updates of the supernodal solves
// are all column-major C -= A * B on sub-blocks of resident buffers.  One
// launch covers every problem of a level/step: a CTA owns one 64x64 tile of
// one problem, located by binary search over the tile prefix.
//
// FP64: 8x8x4 DMMA tensor-core tiles (tcgen05 has no FP64 kind); operands are
// staged through shared memory with cp.async double buffering.
#pragma once

#include "common.cuh"

namespace mfgpu {

constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 16;
constexpr int kGemmThreads = 128;

__device__ __forceinline__ int find_task(const GemmTask* __restrict__ tasks, int ntasks, int64_t tile) {
  int lo = 0, hi = ntasks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tasks[mid].tile_base <= tile) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// pa / pb / pc: base pointers the task offsets refer to.
__global__ void __launch_bounds__(kGemmThreads) k_gemm_f64(const GemmTask* __restrict__ tasks, int ntasks,
                                                           const double* __restrict__ pa, const double* __restrict__ pb,
                                                           double* __restrict__ pc) {
  constexpr int BM = kGemmBM, BN = kGemmBN, BK = kGemmBK;
  constexpr int LDA_S = BM + 8;   // A tile stored k-major: As[k][m]
  constexpr int LDB_S = BK + 4;   // B tile stored n-major: Bs[n][k]
  __shared__ __align__(16) double smem[2 * BK * LDA_S + 2 * BN * LDB_S];
  double* As = smem;
  double* Bs = smem + 2 * BK * LDA_S;

  const GemmTask tk = tasks[find_task(tasks, ntasks, blockIdx.x)];
  const int64_t local = blockIdx.x - tk.tile_base;
  const int m0 = (int)(local % tk.tiles_m) * BM;
  const int n0 = (int)(local / tk.tiles_m) * BN;
  const double* A = pa + tk.a;
  const double* B = pb + tk.b;
  double* C = pc + tk.c;
  const int M = tk.m, N = tk.n, K = tk.k, lda = tk.lda, ldb = tk.ldb, ldc = tk.ldc;
  const int tid = threadIdx.x, lane = lane_id(), warp = warp_id();
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;

  auto load_stage = [&](int stage, int k0) {
    double* as = As + stage * BK * LDA_S;
    double* bs = Bs + stage * BN * LDB_S;
#pragma unroll
    for (int i = 0; i < (BM * BK) / kGemmThreads; ++i) {
      const int idx = tid + i * kGemmThreads;
      const int m = idx % BM, k = idx / BM;
      const bool ok = (m0 + m < M) && (k0 + k < K);
      const double* src = ok ? A + (int64_t)(m0 + m) + (int64_t)(k0 + k) * lda : A;
      cp_async8(as + k * LDA_S + m, src, ok);
    }
#pragma unroll
    for (int i = 0; i < (BN * BK) / kGemmThreads; ++i) {
      const int idx = tid + i * kGemmThreads;
      const int k = idx % BK, n = idx / BK;
      const bool ok = (n0 + n < N) && (k0 + k < K);
      const double* src = ok ? B + (int64_t)(k0 + k) + (int64_t)(n0 + n) * ldb : B;
      cp_async8(bs + n * LDB_S + k, src, ok);
    }
    cp_async_commit();
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int ktiles = (K + BK - 1) / BK;
  load_stage(0, 0);
  for (int kt = 0; kt < ktiles; ++kt) {
    if (kt + 1 < ktiles) {
      load_stage((kt + 1) & 1, (kt + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const double* as = As + (kt & 1) * BK * LDA_S;
    const double* bs = Bs + (kt & 1) * BN * LDB_S;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = as[(kk + (lane & 3)) * LDA_S + wm + i * 8 + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = bs[(wn + j * 8 + (lane >> 2)) * LDB_S + kk + (lane & 3)];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
    __syncthreads();
  }

  // epilogue through shared memory so the read-modify-write of C is coalesced
  constexpr int LDC_S = BM + 1;
  double* Cs = smem;   // BN x LDC_S doubles fit in the operand buffers
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int m = wm + i * 8 + (lane >> 2);
        const int n = wn + j * 8 + 2 * (lane & 3) + e;
        Cs[n * LDC_S + m] = acc[i][j][e];
      }
  __syncthreads();
  for (int idx = tid; idx < BM * BN; idx += kGemmThreads) {
    const int m = idx % BM, n = idx / BM;
    if (m0 + m < M && n0 + n < N) {
      double* cp = C + (int64_t)(m0 + m) + (int64_t)(n0 + n) * ldc;
      *cp -= Cs[n * LDC_S + m];
    }
  }
}

// FP32 variant (mixed-precision fronts), CUDA-core FFMA with 4x4 register
// micro-tiles; same task format.
__global__ void __launch_bounds__(256) k_gemm_f32(const GemmTask* __restrict__ tasks, int ntasks,
                                                  const float* __restrict__ pa, const float* __restrict__ pb,
                                                  float* __restrict__ pc) {
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ float As[2][BK][BM + 4];
  __shared__ float Bs[2][BK][BN + 4];
  const GemmTask tk = tasks[find_task(tasks, ntasks, blockIdx.x)];
  const int64_t local = blockIdx.x - tk.tile_base;
  const int m0 = (int)(local % tk.tiles_m) * BM;
  const int n0 = (int)(local / tk.tiles_m) * BN;
  const float* A = pa + tk.a;
  const float* B = pb + tk.b;
  float* C = pc + tk.c;
  const int M = tk.m, N = tk.n, K = tk.k, lda = tk.lda, ldb = tk.ldb, ldc = tk.ldc;
  const int tid = threadIdx.x;
  const int tm = (tid & 15) * 4, tn = (tid >> 4) * 4;
  float acc[4][4] = {};
  auto load = [&](int st, int k0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int idx = tid + i * 256;
      const int m = idx % BM, k = idx / BM;
      const bool ok = (m0 + m < M) && (k0 + k < K);
      cp_async4(&As[st][k][m], ok ? A + (int64_t)(m0 + m) + (int64_t)(k0 + k) * lda : A, ok);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int idx = tid + i * 256;
      const int k = idx % BK, n = idx / BK;
      const bool ok = (n0 + n < N) && (k0 + k < K);
      cp_async4(&Bs[st][k][n], ok ? B + (int64_t)(k0 + k) + (int64_t)(n0 + n) * ldb : B, ok);
    }
    cp_async_commit();
  };
  const int ktiles = (K + BK - 1) / BK;
  load(0, 0);
  for (int kt = 0; kt < ktiles; ++kt) {
    if (kt + 1 < ktiles) {
      load((kt + 1) & 1, (kt + 1) * BK);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const int st = kt & 1;
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[st][k][tm + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[st][k][tn + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int m = m0 + tm + i, n = n0 + tn + j;
      if (m < M && n < N) C[(int64_t)m + (int64_t)n * ldc] -= acc[i][j];
    }
}

}  // namespace mfgpu

namespace mfgpu {

// FP64 batched GEMM, C -= A * B, templated on the CTA tile (BM x BN), the warp
// tile (WM x WN, multiples of 8) and the cp.async pipeline depth.  Same task
// format as k_gemm_f64; the tasks' tiles_m / tiles_n must use BM / BN.
template <int BM, int BN, int WM, int WN, int STAGES>
struct GemmCfg {
  static constexpr int kWarps = (BM / WM) * (BN / WN);
  static constexpr int kThreads = kWarps * 32;
  static constexpr int BK = 16;
  static constexpr int kLdA = BM + 8;     // A stage: k-major [BK][BM + 8]
  static constexpr int kLdB = BK + 4;     // B stage: n-major [BN][BK + 4]
  static constexpr int kStageA = BK * kLdA;
  static constexpr int kStageB = BN * kLdB;
  static constexpr int kLdC = BM + 1;
  static constexpr size_t kSmemOps = (size_t)STAGES * (kStageA + kStageB);
  static constexpr size_t kSmemC = (size_t)BN * kLdC;
  static constexpr size_t kSmem = (kSmemOps > kSmemC ? kSmemOps : kSmemC) * sizeof(double);
};

template <int BM, int BN, int WM, int WN, int STAGES>
__global__ void __launch_bounds__(GemmCfg<BM, BN, WM, WN, STAGES>::kThreads)
    k_gemm_f64_t(const GemmTask* __restrict__ tasks, int ntasks, const double* __restrict__ pa,
                 const double* __restrict__ pb, double* __restrict__ pc) {
  using C = GemmCfg<BM, BN, WM, WN, STAGES>;
  constexpr int BK = C::BK, NT = C::kThreads;
  constexpr int FM = WM / 8, FN = WN / 8;           // 8x8 fragments per warp
  extern __shared__ __align__(16) double gsm[];
  double* As = gsm;
  double* Bs = gsm + STAGES * C::kStageA;

  const GemmTask tk = tasks[find_task(tasks, ntasks, blockIdx.x)];
  const int64_t local = blockIdx.x - tk.tile_base;
  const int m0 = (int)(local % tk.tiles_m) * BM;
  const int n0 = (int)(local / tk.tiles_m) * BN;
  const double* A = pa + tk.a;
  const double* B = pb + tk.b;
  double* Cg = pc + tk.c;
  const int M = tk.m, N = tk.n, K = tk.k, lda = tk.lda, ldb = tk.ldb, ldc = tk.ldc;
  const int tid = threadIdx.x, lane = lane_id(), warp = warp_id();
  const int wm = (warp % (BM / WM)) * WM, wn = (warp / (BM / WM)) * WN;

  auto load_stage = [&](int stage, int k0) {
    double* as = As + stage * C::kStageA;
    double* bs = Bs + stage * C::kStageB;
#pragma unroll
    for (int i = 0; i < (BM * BK) / NT; ++i) {
      const int idx = tid + i * NT;
      const int m = idx % BM, k = idx / BM;
      const bool ok = (m0 + m < M) && (k0 + k < K);
      cp_async8(as + k * C::kLdA + m, ok ? A + (int64_t)(m0 + m) + (int64_t)(k0 + k) * lda : A, ok);
    }
#pragma unroll
    for (int i = 0; i < (BN * BK) / NT; ++i) {
      const int idx = tid + i * NT;
      const int k = idx % BK, n = idx / BK;
      const bool ok = (n0 + n < N) && (k0 + k < K);
      cp_async8(bs + n * C::kLdB + k, ok ? B + (int64_t)(k0 + k) + (int64_t)(n0 + n) * ldb : B, ok);
    }
  };

  double acc[FM][FN][2];
#pragma unroll
  for (int i = 0; i < FM; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int ktiles = (K + BK - 1) / BK;
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) load_stage(s, s * BK);
    cp_async_commit();
  }
  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    const int pre = kt + STAGES - 1;
    if (pre < ktiles) load_stage(pre % STAGES, pre * BK);
    cp_async_commit();
    const double* as = As + (kt % STAGES) * C::kStageA;
    const double* bs = Bs + (kt % STAGES) * C::kStageB;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double af[FM], bf[FN];
#pragma unroll
      for (int i = 0; i < FM; ++i) af[i] = as[(kk + (lane & 3)) * C::kLdA + wm + i * 8 + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < FN; ++j) bf[j] = bs[(wn + j * 8 + (lane >> 2)) * C::kLdB + kk + (lane & 3)];
#pragma unroll
      for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  double* Cs = gsm;
#pragma unroll
  for (int i = 0; i < FM; ++i)
#pragma unroll
    for (int j = 0; j < FN; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e)
        Cs[(wn + j * 8 + 2 * (lane & 3) + e) * C::kLdC + wm + i * 8 + (lane >> 2)] = acc[i][j][e];
  __syncthreads();
  for (int idx = tid; idx < BM * BN; idx += NT) {
    const int m = idx % BM, n = idx / BM;
    if (m0 + m < M && n0 + n < N) Cg[(int64_t)(m0 + m) + (int64_t)(n0 + n) * ldc] -= Cs[n * C::kLdC + m];
  }
}

}  // namespace mfgpu
