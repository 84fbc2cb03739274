// gemm_kernels.cuh -- batched C = f(C, A * B) over heterogeneous problems.
//
// The dense updates of the large fronts (the trailing updates of the blocked
// pivot-block LU and the Schur update F22 -= L21 * U12 of
// src/multifrontal.jl:267-268) and the block updates of the supernodal solves
// are all column-major C -= A * B on sub-blocks of resident buffers; the
// inversion of the pivot blocks and the inverse-based solves also need
// C = A * B, C = -(A * B) and C = D - A * B (GemmTask::mode).  One launch
// covers every problem of a level/step: a CTA owns one 64x64 tile of one
// problem, located by binary search over the tile prefix.
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

constexpr int kGemmSmemF64 = 2 * kGemmBK * (kGemmBM + 4) + 2 * kGemmBN * (kGemmBK + 4);   // doubles

// One 64 x 64 tile (index `tile` of the launch) of C -= A * B, 128 threads.
// pa / pb / pc: base pointers the task offsets refer to; smem: kGemmSmemF64
// doubles, 16-byte aligned.  C and B may be written by other steps of the
// same persistent launch, so neither is read through the non-coherent path.
__device__ __forceinline__ void gemm_tile_f64(const GemmTask* __restrict__ tasks, int ntasks,
                                              const double* pa, const double* pb, double* pc, int64_t tile,
                                              double* smem) {
  constexpr int BM = kGemmBM, BN = kGemmBN, BK = kGemmBK;
  // A tile stored k-major: As[k][m].  A fragment load reads rows k..k+3 of
  // the tile at 8 consecutive m per row; a row stride of 68 doubles puts the
  // four rows of a half-warp on distinct banks (72 put rows k and k+2 on the
  // same ones: a 2-way conflict on every A fragment).
  constexpr int LDA_S = BM + 4;
  constexpr int LDB_S = BK + 4;   // B tile stored n-major: Bs[n][k]
  double* As = smem;
  double* Bs = smem + 2 * BK * LDA_S;

  const GemmTask tk = tasks[find_task(tasks, ntasks, tile)];
  const int64_t local = tile - tk.tile_base;
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
  // all loads of C before any store: the stores could alias later loads as
  // far as the compiler knows, which would serialise one round trip each
  constexpr int kPer = BM * BN / kGemmThreads / 2;   // two passes of 16 keep the register peak low
  const double* D = tk.mode == kGemmFrom ? pc + tk.d : C;
  const int ldD = tk.mode == kGemmFrom ? tk.ldd : ldc;
  const bool load = tk.mode == kGemmSub || tk.mode == kGemmFrom;
  const double sgn = tk.mode == kGemmSet ? -1.0 : 1.0;   // Set: C = +AB; Neg: C = -AB = 0 - AB
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    double cv[kPer];
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int idx = tid + (pass * kPer + i) * kGemmThreads, m = idx % BM, n = idx / BM;
      cv[i] = (load && m0 + m < M && n0 + n < N) ? D[(int64_t)(m0 + m) + (int64_t)(n0 + n) * ldD] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int idx = tid + (pass * kPer + i) * kGemmThreads, m = idx % BM, n = idx / BM;
      if (m0 + m < M && n0 + n < N)
        C[(int64_t)(m0 + m) + (int64_t)(n0 + n) * ldc] = cv[i] - sgn * Cs[n * LDC_S + m];
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kGemmThreads) k_gemm_f64(const GemmTask* __restrict__ tasks, int ntasks,
                                                           const double* __restrict__ pa, const double* __restrict__ pb,
                                                           double* __restrict__ pc) {
  __shared__ __align__(16) double smem[kGemmSmemF64];
  gemm_tile_f64(tasks, ntasks, pa, pb, pc, blockIdx.x, smem);
}

// FP32 64 x 64 tile for 128 threads (4 x 8 register micro-tiles), the same
// task format; smem: kGemmSmemF32 floats.
constexpr int kGemmSmemF32 = 2 * 16 * (64 + 4) * 2;
__device__ __forceinline__ void gemm_tile_f32(const GemmTask* __restrict__ tasks, int ntasks, const float* pa,
                                              const float* pb, float* pc, int64_t tile, float* smem) {
  constexpr int BM = 64, BN = 64, BK = 16, LD = 64 + 4;
  float* As = smem;                  // [2][BK][LD]
  float* Bs = smem + 2 * BK * LD;    // [2][BK][LD]
  const GemmTask tk = tasks[find_task(tasks, ntasks, tile)];
  const int64_t local = tile - tk.tile_base;
  const int m0 = (int)(local % tk.tiles_m) * BM;
  const int n0 = (int)(local / tk.tiles_m) * BN;
  const float* A = pa + tk.a;
  const float* B = pb + tk.b;
  float* C = pc + tk.c;
  const int M = tk.m, N = tk.n, K = tk.k, lda = tk.lda, ldb = tk.ldb, ldc = tk.ldc;
  const int tid = threadIdx.x;
  const int tm = (tid & 15) * 4, tn = (tid >> 4) * 8;
  float acc[4][8] = {};
  auto load = [&](int st, int k0) {
#pragma unroll
    for (int i = 0; i < (BM * BK) / 128; ++i) {
      const int idx = tid + i * 128;
      const int m = idx % BM, k = idx / BM;
      const bool ok = (m0 + m < M) && (k0 + k < K);
      cp_async4(As + (st * BK + k) * LD + m, ok ? A + (int64_t)(m0 + m) + (int64_t)(k0 + k) * lda : A, ok);
    }
#pragma unroll
    for (int i = 0; i < (BN * BK) / 128; ++i) {
      const int idx = tid + i * 128;
      const int k = idx % BK, n = idx / BK;
      const bool ok = (n0 + n < N) && (k0 + k < K);
      cp_async4(Bs + (st * BK + k) * LD + n, ok ? B + (int64_t)(k0 + k) + (int64_t)(n0 + n) * ldb : B, ok);
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
    const float* as = As + (kt & 1) * BK * LD;
    const float* bs = Bs + (kt & 1) * BK * LD;
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      float a[4], b[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = as[k * LD + tm + i];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = bs[k * LD + tn + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  const float* D = tk.mode == kGemmFrom ? pc + tk.d : C;
  const int ldD = tk.mode == kGemmFrom ? tk.ldd : ldc;
  const bool ld = tk.mode == kGemmSub || tk.mode == kGemmFrom;
  const float sgn = tk.mode == kGemmSet ? -1.0f : 1.0f;
  float cv[4][8];
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int m = m0 + tm + i, n = n0 + tn + j;
      cv[i][j] = (ld && m < M && n < N) ? D[(int64_t)m + (int64_t)n * ldD] : 0.0f;
    }
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int m = m0 + tm + i, n = n0 + tn + j;
      if (m < M && n < N) C[(int64_t)m + (int64_t)n * ldc] = cv[i][j] - sgn * acc[i][j];
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
  const float* D = tk.mode == kGemmFrom ? pc + tk.d : C;
  const int ldD = tk.mode == kGemmFrom ? tk.ldd : ldc;
  const bool ld = tk.mode == kGemmSub || tk.mode == kGemmFrom;
  const float sgn = tk.mode == kGemmSet ? -1.0f : 1.0f;
  float cv[4][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int m = m0 + tm + i, n = n0 + tn + j;
      cv[i][j] = (ld && m < M && n < N) ? D[(int64_t)m + (int64_t)n * ldD] : 0.0f;
    }
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int m = m0 + tm + i, n = n0 + tn + j;
      if (m < M && n < N) C[(int64_t)m + (int64_t)n * ldc] = cv[i][j] - sgn * acc[i][j];
    }
}

// Products with few rows (the solve products whose M is a supernode's pivot
// count, low in the tree: g = y - U12 x_u, x = inv(U11) g, y = inv(L11) f):
// a 64 x 64 tile would leave most of its rows idle and its CTAs would each
// re-stream the B operand.  BM x 128 tiles (BM = 16 or 32, tiles counted by
// tiles_m / tiles_n in that tiling), CUDA-core FMA, cp.async double buffer;
// thread (ty, tx) holds rows ty * BM/8 .. and columns tx + 32 j, so the B
// reads from shared memory are conflict-free and the A reads broadcast.
constexpr int kSkinnyMBN = 128;

template <typename T, int BM>
__global__ void __launch_bounds__(256) k_gemm_skinny_m(const GemmTask* __restrict__ tasks, int ntasks,
                                                       const T* __restrict__ pa, const T* pb, T* pc) {
  constexpr int BN = kSkinnyMBN, BK = 16, TM = BM / 8;
  __shared__ T As[2][BK][BM];
  __shared__ T Bs[2][BK][BN + 1];
  const GemmTask tk = tasks[find_task(tasks, ntasks, blockIdx.x)];
  const int64_t local = blockIdx.x - tk.tile_base;
  const int m0 = (int)(local % tk.tiles_m) * BM;
  const int n0 = (int)(local / tk.tiles_m) * BN;
  const T* A = pa + tk.a;
  const T* B = pb + tk.b;
  T* C = pc + tk.c;
  const int M = tk.m, N = tk.n, K = tk.k, lda = tk.lda, ldb = tk.ldb, ldc = tk.ldc;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  T acc[TM][4];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
  auto cp = [](T* dst, const T* src, bool ok) {
    if constexpr (sizeof(T) == 8) cp_async8(dst, src, ok);
    else cp_async4(dst, src, ok);
  };
  auto load = [&](int st, int k0) {
    for (int idx = tid; idx < BM * BK; idx += 256) {
      const int m = idx % BM, k = idx / BM;
      const bool ok = (m0 + m < M) && (k0 + k < K);
      cp(&As[st][k][m], ok ? A + (int64_t)(m0 + m) + (int64_t)(k0 + k) * lda : A, ok);
    }
#pragma unroll
    for (int i = 0; i < BK * BN / 256; ++i) {
      const int idx = tid + i * 256;
      const int k = idx % BK, n = idx / BK;
      const bool ok = (n0 + n < N) && (k0 + k < K);
      cp(&Bs[st][k][n], ok ? B + (int64_t)(k0 + k) + (int64_t)(n0 + n) * ldb : B, ok);
    }
    cp_async_commit();
  };
  const int ktiles = (K + BK - 1) / BK;
  if (ktiles > 0) load(0, 0);
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
      T a[TM], b[4];
#pragma unroll
      for (int i = 0; i < TM; ++i) a[i] = As[st][k][ty * TM + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[st][k][tx + 32 * j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
  const T* D = tk.mode == kGemmFrom ? pc + tk.d : C;
  const int ldD = tk.mode == kGemmFrom ? tk.ldd : ldc;
  const bool ld = tk.mode == kGemmSub || tk.mode == kGemmFrom;
  const T sgn = tk.mode == kGemmSet ? T(-1) : T(1);
  T cv[TM][4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int m = m0 + ty * TM + i, n = n0 + tx + 32 * j;
      cv[i][j] = (ld && m < M && n < N) ? D[(int64_t)m + (int64_t)n * ldD] : T(0);
    }
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int i = 0; i < TM; ++i) {
      const int m = m0 + ty * TM + i, n = n0 + tx + 32 * j;
      if (m < M && n < N) C[(int64_t)m + (int64_t)n * ldc] = cv[i][j] - sgn * acc[i][j];
    }
}

// ---------------------------------------------------------------------------
// Split-K products for few right-hand sides (N <= NMAX): the solve products
// g = y - U12 x_u have a handful of rows and thousands of K, which a 64 x 64
// tile would walk serially.  Stage 1: one CTA per (task, 128-row block,
// K chunk), one thread per row, partial sums of all N columns into a scratch
// array.  The chunk width (kc, at most kSkinnyKC) is chosen per step so that
// the step has enough CTAs to cover the GPU: one front's products are a
// latency-bound walk down K otherwise.  Stage 2: one CTA per (task, row
// block) sums the chunks in order (deterministic) and applies the task's
// mode.
constexpr int kSkinnyRows = 128;
constexpr int kSkinnyKC = 256;
constexpr int kSkinnyMaxN = 16;

struct SkinnyTask {
  int64_t a, b, c, d;
  int32_t m, n, k, lda, ldb, ldc, ldd, mode;
  int32_t rblocks, kchunks;
  int32_t kc, pad;       // K-chunk width (<= kSkinnyKC)
  int64_t part_base;     // prefix over tasks of rblocks * kchunks (stage-1 CTAs and scratch items)
  int64_t red_base;      // prefix over tasks of rblocks (stage-2 CTAs)
};

__device__ __forceinline__ int find_skinny(const SkinnyTask* __restrict__ t, int n, int64_t x, bool red) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if ((red ? t[mid].red_base : t[mid].part_base) <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <typename T, int NMAX>
__global__ void __launch_bounds__(kSkinnyRows) k_skinny_part(const SkinnyTask* __restrict__ tasks, int ntasks,
                                                             const T* pa, const T* pb, T* __restrict__ part) {
  __shared__ T bs[kSkinnyKC * NMAX];
  const SkinnyTask tk = tasks[find_skinny(tasks, ntasks, blockIdx.x, false)];
  const int64_t local = blockIdx.x - tk.part_base;
  const int rb = (int)(local % tk.rblocks), kc = (int)(local / tk.rblocks);
  const int k0 = kc * tk.kc, kn = min(tk.kc, tk.k - k0), N = tk.n;
  const T* A = pa + tk.a;
  const T* B = pb + tk.b;
  for (int e = threadIdx.x; e < kSkinnyKC * NMAX; e += blockDim.x) {
    const int k = e % kSkinnyKC, n = e / kSkinnyKC;
    bs[e] = (k < kn && n < N) ? B[(int64_t)(k0 + k) + (int64_t)n * tk.ldb] : T(0);
  }
  __syncthreads();
  const int row = rb * kSkinnyRows + threadIdx.x;
  T acc[NMAX];
#pragma unroll
  for (int n = 0; n < NMAX; ++n) acc[n] = T(0);
  if (row < tk.m) {
    const T* ar = A + row + (int64_t)k0 * tk.lda;
#pragma unroll 8
    for (int k = 0; k < kn; ++k) {
      const T a = ar[(int64_t)k * tk.lda];
#pragma unroll
      for (int n = 0; n < NMAX; ++n) acc[n] += a * bs[k + n * kSkinnyKC];
    }
  }
  T* out = part + (tk.part_base + local) * (int64_t)(kSkinnyRows * NMAX);
#pragma unroll
  for (int n = 0; n < NMAX; ++n) out[threadIdx.x + n * kSkinnyRows] = acc[n];
}

template <typename T, int NMAX>
__global__ void __launch_bounds__(kSkinnyRows) k_skinny_reduce(const SkinnyTask* __restrict__ tasks, int ntasks,
                                                               const T* __restrict__ part, T* pc) {
  const SkinnyTask tk = tasks[find_skinny(tasks, ntasks, blockIdx.x, true)];
  const int rb = (int)(blockIdx.x - tk.red_base);
  const int row = rb * kSkinnyRows + threadIdx.x;
  if (row >= tk.m) return;
  T* C = pc + tk.c;
  const T* D = tk.mode == kGemmFrom ? pc + tk.d : C;
  const int ldD = tk.mode == kGemmFrom ? tk.ldd : tk.ldc;
  for (int n = 0; n < tk.n; ++n) {
    T sum = T(0);
    for (int kc = 0; kc < tk.kchunks; ++kc)
      sum += part[(tk.part_base + rb + (int64_t)kc * tk.rblocks) * (int64_t)(kSkinnyRows * NMAX) + threadIdx.x +
                  n * kSkinnyRows];
    const T dv = (tk.mode == kGemmSub || tk.mode == kGemmFrom) ? D[(int64_t)row + (int64_t)n * ldD] : T(0);
    C[(int64_t)row + (int64_t)n * tk.ldc] = tk.mode == kGemmSet ? sum : dv - sum;
  }
}

// ---------------------------------------------------------------------------
// ComplexF64 C = f(C, A * B) (GemmTask::mode) for complex fronts, on the CUDA
// cores: 64 x 64 tiles located like k_gemm_f64's, 128 threads with a 4 x 8
// block of complex accumulators each, operands staged through shared memory
// kGemmZK values of K at a time.
// ---------------------------------------------------------------------------
constexpr int kGemmZK = 16;

__global__ void __launch_bounds__(kGemmThreads) k_gemm_z(const GemmTask* __restrict__ tasks, int ntasks,
                                                         const zc* pa, const zc* pb, zc* pc) {
  __shared__ zc As[kGemmZK][kGemmBM + 1];   // As[k][m]
  __shared__ zc Bs[kGemmBN][kGemmZK + 1];   // Bs[n][k]
  const GemmTask tk = tasks[find_task(tasks, ntasks, blockIdx.x)];
  const int64_t local = blockIdx.x - tk.tile_base;
  const int m0 = (int)(local % tk.tiles_m) * kGemmBM;
  const int n0 = (int)(local / tk.tiles_m) * kGemmBN;
  const zc* A = pa + tk.a;
  const zc* B = pb + tk.b;
  zc* C = pc + tk.c;
  const int M = tk.m, N = tk.n, K = tk.k;
  const int t = threadIdx.x;
  const int tm = (t & 15) * 4, tn = (t >> 4) * 8;
  zc acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = zc(0.0);
  for (int k0 = 0; k0 < K; k0 += kGemmZK) {
    for (int e = t; e < kGemmBM * kGemmZK; e += kGemmThreads) {
      const int m = e % kGemmBM, k = e / kGemmBM;
      As[k][m] = (m0 + m < M && k0 + k < K) ? A[(int64_t)(m0 + m) + (int64_t)(k0 + k) * tk.lda] : zc(0.0);
    }
    for (int e = t; e < kGemmBN * kGemmZK; e += kGemmThreads) {
      const int k = e % kGemmZK, n = e / kGemmZK;
      Bs[n][k] = (n0 + n < N && k0 + k < K) ? B[(int64_t)(k0 + k) + (int64_t)(n0 + n) * tk.ldb] : zc(0.0);
    }
    __syncthreads();
#pragma unroll 4
    for (int k = 0; k < kGemmZK; ++k) {
      zc a[4], b[8];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[k][tm + i];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = Bs[tn + j][k];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
  const zc* D = tk.mode == kGemmFrom ? pc + tk.d : C;
  const int ldD = tk.mode == kGemmFrom ? tk.ldd : tk.ldc;
  const bool ld = tk.mode == kGemmSub || tk.mode == kGemmFrom;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int r = m0 + tm + i, c = n0 + tn + j;
      if (r < M && c < N) {
        const zc dv = ld ? D[(int64_t)r + (int64_t)c * ldD] : zc(0.0);
        C[(int64_t)r + (int64_t)c * tk.ldc] = tk.mode == kGemmSet ? acc[i][j] : dv - acc[i][j];
      }
    }
}

}  // namespace mfgpu
