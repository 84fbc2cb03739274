// factor_kernels.cuh -- numeric multifrontal factorization kernels.
//
// Device restatement of the hot loop of src/multifrontal.jl:198-357:
//   * k_small_fronts     fronts with nf <= 64: zero-fill, original entries
//                        (multifrontal.jl:217-231), extend-add of the children
//                        in LIFO order (:235-243, :45-57), partial-pivot LU of
//                        the pivot block with the interchanges applied to the
//                        whole rows (:247-263), trsm/gemm Schur update folded
//                        into the right-looking elimination (:264-268); one
//                        CTA per front, the front lives in shared memory.
//   * k_assemble_columns larger fronts: one warp per front column.
//   * k_panel / k_panel_trsm + the batched GEMM: blocked LU of the first np
//                        columns (pivot search restricted to the np pivot
//                        rows), followed by the deferred Schur update
//                        F22 -= L21 * U12 with K = np.
//   * k_finalize_pivots  _pivot_rows (:363-375), prow and its inverse (:347).
//   * k_scatter_csc      direct CSC scatter of L and U (:278-317) with the
//                        relabelling of L's update rows (:347-350).
// Fronts stay resident in the front pool (column-major, leading dimension nf)
// after factorization: the parent reads each child's contribution block in
// place, the solves read L and U panels from it, and the CSC scatter runs
// once at the end.
#pragma once

#include "common.cuh"

namespace mfgpu {

constexpr int kSmallThreads = 128;

template <typename T>
__global__ void __launch_bounds__(kSmallThreads) k_small_fronts(DevPlan P, DevState S, const int32_t* __restrict__ tasks,
                                                                 T* __restrict__ pool, const Wide<T>* __restrict__ vx) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* F = reinterpret_cast<T*>(smem_raw);
  __shared__ int s_piv;
  const int s = tasks[blockIdx.x];
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  const int64_t fb = P.colbase[s];
  const int tid = threadIdx.x, nthr = blockDim.x;

  for (int e = tid; e < nf * nf; e += nthr) F[e] = T(0);
  __syncthreads();
  for (int c = warp_id(); c < nf; c += nthr >> 5) {
    const int b = P.fc_vbeg[fb + c], e = P.fc_vend[fb + c];
    for (int p = b + lane_id(); p < e; p += 32) F[P.v_frow[p] + c * nf] = to_front<T>(vx[p]);
  }
  __syncthreads();
  for (int ci = P.child_ptr[s + 1] - 1; ci >= P.child_ptr[s]; --ci) {
    const int k = P.child_idx[ci];
    const int m = P.nu[k], nfk = P.nf[k], npk = P.np[k];
    const T* cb = pool + P.front_off[k] + npk + (int64_t)npk * nfk;
    const int32_t* rl = P.rel + P.upd_off[k];
    if (m == 0) continue;
    const FastDiv dm((uint32_t)m);
    for (int e = tid; e < m * m; e += nthr) {
      const int t = (int)dm.div(e), r = e - t * m;
      F[rl[r] + rl[t] * nf] += cb[r + (int64_t)t * nfk];
    }
    __syncthreads();
  }

  int first_zero = INT32_MAX;
  for (int k = 0; k < np; ++k) {
    const int seg = P.seg_end[c1 + k];   // pivot rows of column k: k..seg-1
    if (warp_id() == 0) {
      ArgMax a{-1.0, k};
      for (int i = k + lane_id(); i < seg; i += 32) a = better(a, ArgMax{absd(F[i + k * nf]), i});
      a = warp_argmax(a);
      if (lane_id() == 0) s_piv = a.i;
    }
    __syncthreads();
    const int piv = s_piv;
    if (piv != k)
      for (int j = tid; j < nf; j += nthr) {
        const T t = F[k + j * nf];
        F[k + j * nf] = F[piv + j * nf];
        F[piv + j * nf] = t;
      }
    if (tid == 0) S.ipiv[c1 + k] = piv;
    __syncthreads();
    const T d = F[k + k * nf];
    if (d == T(0) && first_zero == INT32_MAX) first_zero = k;
    const T rcp = T(1) / d;
    for (int i = k + 1 + tid; i < nf; i += nthr)
      if (i >= seg || d != T(0)) F[i + k * nf] *= rcp;
    __syncthreads();
    const int rows = nf - k - 1;
    if (rows > 0) {
      const FastDiv drows((uint32_t)rows);
      for (int e = tid; e < rows * rows; e += nthr) {
        const int q = (int)drows.div(e), i = k + 1 + e - q * rows, j = k + 1 + q;
        F[i + j * nf] -= F[i + k * nf] * F[k + j * nf];
      }
    }
    __syncthreads();
  }
  T* G = pool + P.front_off[s];
  for (int e = tid; e < nf * nf; e += nthr) G[e] = F[e];
  if (tid == 0 && first_zero != INT32_MAX) S.info[s] = first_zero;
}

// One warp per front column of the large fronts of a level.
template <typename T>
__global__ void __launch_bounds__(256) k_assemble_columns(DevPlan P, int64_t fc0, int64_t count, T* __restrict__ pool,
                                                          const Wide<T>* __restrict__ vx) {
  const int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_id();
  if (w >= count) return;
  const int64_t fc = fc0 + w;
  const int s = P.fc_super[fc];
  const int c = (int)(fc - P.colbase[s]);
  const int nf = P.nf[s];
  const int lane = lane_id();
  T* col = pool + P.front_off[s] + (int64_t)c * nf;
  for (int r = lane; r < nf; r += 32) col[r] = T(0);
  __syncwarp();
  for (int p = P.fc_vbeg[fc] + lane; p < P.fc_vend[fc]; p += 32) col[P.v_frow[p]] = to_front<T>(vx[p]);
  __syncwarp();
  for (int e = P.fc_ch_ptr[fc]; e < P.fc_ch_ptr[fc + 1]; ++e) {
    const int k = P.fc_ch[2 * (int64_t)e], t = P.fc_ch[2 * (int64_t)e + 1];
    const int m = P.nu[k], nfk = P.nf[k], npk = P.np[k];
    const T* cb = pool + P.front_off[k] + npk + (int64_t)(npk + t) * nfk;
    const int32_t* rl = P.rel + P.upd_off[k];
    // kU rows per lane in flight (a child's rows map to distinct rows of
    // this column, so all loads may precede the stores); 4-byte fronts move
    // half the bytes per access, so they keep twice as many in flight
    constexpr int kU = sizeof(T) == 4 ? 8 : 4;
    int r = lane;
    for (; r + 32 * (kU - 1) < m; r += 32 * kU) {
      int pos[kU];
      T v[kU], o[kU];
#pragma unroll
      for (int q = 0; q < kU; ++q) {
        pos[q] = rl[r + 32 * q];
        v[q] = cb[r + 32 * q];
      }
#pragma unroll
      for (int q = 0; q < kU; ++q) o[q] = col[pos[q]];
#pragma unroll
      for (int q = 0; q < kU; ++q) col[pos[q]] = o[q] + v[q];
    }
    for (; r < m; r += 32) col[rl[r]] += cb[r];
    __syncwarp();
  }
}

// Partial-pivot LU of an R x kb panel A (leading dimension lda, shared or
// global memory); the pivot of column j is searched in rows j..seg[j]-1
// (seg[j] <= R: the pivot rows of the column's supernode) with idamax's
// first-maximum rule.  Records local pivots in piv[] (shared) and the first
// zero pivot (panel-relative) in *first_zero.
template <typename T>
__device__ void panel_lu_pivot(T* A, int lda, int R, int kb, const int* seg, int* piv, ArgMax* red,
                               int* first_zero) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int j = 0; j < kb; ++j) {
    ArgMax a{-1.0, j};
    for (int i = j + tid; i < seg[j]; i += nthr) a = better(a, ArgMax{absd(A[i + (int64_t)j * lda]), i});
    a = block_argmax(a, red);
    const int p = a.i;
    if (p != j)
      for (int c = tid; c < kb; c += nthr) {
        const T t = A[j + (int64_t)c * lda];
        A[j + (int64_t)c * lda] = A[p + (int64_t)c * lda];
        A[p + (int64_t)c * lda] = t;
      }
    if (tid == 0) piv[j] = p;
    __syncthreads();
    const T d = A[j + (int64_t)j * lda];
    if (d == T(0)) {
      if (tid == 0 && *first_zero == INT32_MAX) *first_zero = j;
    } else {
      const T rcp = T(1) / d;
      for (int i = j + 1 + tid; i < R; i += nthr) A[i + (int64_t)j * lda] *= rcp;
    }
    __syncthreads();
    const int rows = R - j - 1, cols = kb - j - 1;
    for (int e = tid; e < rows * cols; e += nthr) {
      const int i = j + 1 + e % rows, c = j + 1 + e / rows;
      A[i + (int64_t)c * lda] -= A[i + (int64_t)j * lda] * A[j + (int64_t)c * lda];
    }
    __syncthreads();
  }
}

constexpr int kPanelThreads = 256;
constexpr int kDinvElems = 2 * 64 * 64;   // inv(L_kk) then inv(U_kk), 64x64 col-major, zero padded

// Inverses of the unit-lower and the upper triangle of the factored kb x kb
// diagonal block D (shared, col-major, leading dimension ldd) into the 64x64
// zero-padded Linv / Uinv (shared, col-major ld 64).  Column c of each
// inverse is one thread's forward / backward substitution.
template <typename T>
__device__ void diag_block_inverses(const T* D, int ldd, int kb, T* Linv, T* Uinv) {
  for (int e = threadIdx.x; e < 2 * 64 * 64; e += blockDim.x) (e < 4096 ? Linv[e] : Uinv[e - 4096]) = T(0);
  __syncthreads();
  // one column per task; four partial sums break the FMA dependency chain
  for (int task = threadIdx.x; task < 2 * kb; task += blockDim.x) {
    if (task < kb) {
      const int c = task;
      T* x = Linv + c * 64;
      x[c] = T(1);
      for (int i = c + 1; i < kb; ++i) {
        T v0 = T(0), v1 = T(0), v2 = T(0), v3 = T(0);
        int k = c;
        for (; k + 3 < i; k += 4) {
          v0 += D[i + k * ldd] * x[k];
          v1 += D[i + (k + 1) * ldd] * x[k + 1];
          v2 += D[i + (k + 2) * ldd] * x[k + 2];
          v3 += D[i + (k + 3) * ldd] * x[k + 3];
        }
        for (; k < i; ++k) v0 += D[i + k * ldd] * x[k];
        x[i] = -((v0 + v1) + (v2 + v3));
      }
    } else {
      const int c = task - kb;
      T* x = Uinv + c * 64;
      x[c] = T(1) / D[c + c * ldd];
      for (int i = c - 1; i >= 0; --i) {
        T v0 = T(0), v1 = T(0), v2 = T(0), v3 = T(0);
        int k = i + 1;
        for (; k + 3 <= c; k += 4) {
          v0 += D[i + k * ldd] * x[k];
          v1 += D[i + (k + 1) * ldd] * x[k + 1];
          v2 += D[i + (k + 2) * ldd] * x[k + 2];
          v3 += D[i + (k + 3) * ldd] * x[k + 3];
        }
        for (; k <= c; ++k) v0 += D[i + k * ldd] * x[k];
        x[i] = -((v0 + v1) + (v2 + v3)) / D[i + i * ldd];
      }
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Register-tiled dense kernels for the panel.  A CTA of ROWS threads holds
// an (R <= ROWS) x (kb <= 64) panel in registers: thread t owns rows
// rb, rb+G, ..., rb+7G (rb = t % G, G = ROWS/8) of the 8 columns
// c0..c0+7 (c0 = 8 (t / G)).  The G owners of one 8-column block are
// consecutive lanes of one warp, and consecutive lanes own consecutive rows,
// so global and shared accesses are coalesced and conflict-free.  Every
// elimination step broadcasts one multiplier column and one pivot row through
// shared memory; a thread's 64 updates are then independent FMAs on
// registers (compile-time indices, predicated on the trailing region).
// ---------------------------------------------------------------------------
template <int G>
__device__ __forceinline__ ArgMax group_argmax(ArgMax a) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    ArgMax b;
    b.v = __shfl_xor_sync(0xffffffffu, a.v, o);
    b.i = __shfl_xor_sync(0xffffffffu, a.i, o);
    a = better(a, b);
  }
  return a;
}

// Value of row slot `slot` (runtime) of column q of a register tile.
template <typename T>
__device__ __forceinline__ T row_pick(const T (&a)[8][8], int slot, int q) {
  T v = a[0][q];
#pragma unroll
  for (int ii = 1; ii < 8; ++ii)
    if (ii == slot) v = a[ii][q];
  return v;
}
template <typename T>
__device__ __forceinline__ T col_pick(const T (&a)[8][8], int ii, int slot) {
  T v = a[ii][0];
#pragma unroll
  for (int q = 1; q < 8; ++q)
    if (q == slot) v = a[ii][q];
  return v;
}

__device__ __forceinline__ void named_barrier(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// LU of the register panel with the pivot search restricted to rows
// j..seg[j]-1 (PIVOT, LAPACK's first-maximum rule; seg[j] <= R ends the
// pivot rows of column j's supernode) or without interchanges and with the
// partial-pivoting order check on those rows (!PIVOT).  sm_urow, sm_buf: 64
// each; sm_lcol: ROWS.
template <typename T, int ROWS, bool PIVOT>
__device__ void tile_lu(T (&a)[8][8], int R, int kb, const int* seg, T* sm_urow, T* sm_buf, T* sm_lcol, int* sm_p,
                        int* piv, int* first_zero, bool* violated) {
  constexpr int G = ROWS / 8;
  const int t = threadIdx.x;
  const int rb = t % G, cb = t / G, c0 = cb * 8;
#pragma unroll 1
  for (int j = 0; j < kb; ++j) {
    const int jb = j >> 3, jo = j & 7;
    const int jr = j % G, js = j / G;         // owner lane and slot of row j
    int p = j;
    if (PIVOT) {
      // Every lane takes part in the shuffles (a warp holds 32/G column
      // groups); only the owner group of column j has real candidates.
      ArgMax m{-1.0, 0x7fffffff};
      if (cb == jb) {
        const int sj = seg[j];
#pragma unroll
        for (int ii = 0; ii < 8; ++ii) {
          const int i = rb + ii * G;
          if (i >= j && i < sj) m = better(m, ArgMax{absd(col_pick(a, ii, jo)), i});
        }
      }
      m = group_argmax<G>(m);
      if (cb == jb && rb == 0) *sm_p = m.i;
      __syncthreads();
      p = *sm_p;
      if (p != j) {                           // uniform: swap rows j and p
        const int pr = p % G, ps = p / G;
        if (rb == jr) {
#pragma unroll
          for (int q = 0; q < 8; ++q) sm_urow[c0 + q] = row_pick(a, js, q);
        }
        if (rb == pr) {
#pragma unroll
          for (int q = 0; q < 8; ++q) sm_buf[c0 + q] = row_pick(a, ps, q);
        }
        __syncthreads();
        if (rb == jr) {
#pragma unroll
          for (int ii = 0; ii < 8; ++ii)
            if (ii == js)
#pragma unroll
              for (int q = 0; q < 8; ++q) a[ii][q] = sm_buf[c0 + q];
        }
        if (rb == pr) {
#pragma unroll
          for (int ii = 0; ii < 8; ++ii)
            if (ii == ps)
#pragma unroll
              for (int q = 0; q < 8; ++q) a[ii][q] = sm_urow[c0 + q];
        }
        __syncthreads();
      }
    }
    if (rb == jr) {                           // broadcast the pivot row
#pragma unroll
      for (int q = 0; q < 8; ++q) sm_urow[c0 + q] = row_pick(a, js, q);
    }
    __syncthreads();
    const T d = sm_urow[j];
    if (t == 0) {
      piv[j] = p;
      if (d == T(0) && *first_zero == INT32_MAX) *first_zero = j;
    }
    if (cb == jb) {                           // multipliers of column j
      const T rcp = (d != T(0)) ? T(1) / d : T(1);
      const int sj = seg[j];
#pragma unroll
      for (int ii = 0; ii < 8; ++ii) {
        const int i = rb + ii * G;
        if (i > j && i < R) {
          const T aj = col_pick(a, ii, jo);
          if (!PIVOT && i < sj && absd(aj) > absd(d)) *violated = true;
          const T l = (d != T(0)) ? aj * rcp : aj;
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (q == jo) a[ii][q] = l;
          sm_lcol[i] = l;
        }
      }
    }
    __syncthreads();
    T u[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) u[q] = sm_urow[c0 + q];
#pragma unroll
    for (int ii = 0; ii < 8; ++ii) {
      const int i = rb + ii * G;
      if (i > j && i < R) {
        const T l = sm_lcol[i];
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (c0 + q > j) a[ii][q] -= l * u[q];
      }
    }
    __syncthreads();
  }
}

// inv(L_kk) (unit lower, !UPPER) or inv(U_kk) (UPPER) of the factored kb x kb
// block D (shared, col-major ld ldd) into dst (global 64 x 64 col-major, zero
// padded), by the 64 threads lane64 = 0..63 of one group synchronised on
// named barrier `bar`: X = I, then one broadcast row of X per step.
template <typename T, bool UPPER>
__device__ void tile_inverse(const T* D, int ldd, int kb, T* dst, T* sm_xrow, int lane64, int bar) {
  const int rb = lane64 % 8, c0 = (lane64 / 8) * 8;
  T x[8][8];
#pragma unroll
  for (int ii = 0; ii < 8; ++ii)
#pragma unroll
    for (int q = 0; q < 8; ++q) x[ii][q] = (rb + ii * 8 == c0 + q && c0 + q < kb) ? T(1) : T(0);
  for (int step = 0; step < kb; ++step) {
    const int k = UPPER ? kb - 1 - step : step;
    const int kr = k % 8, ks = k / 8;
    if (UPPER && rb == kr) {                  // row k is final once divided by U_kk
      const T rd = T(1) / D[k + k * ldd];
#pragma unroll
      for (int ii = 0; ii < 8; ++ii)
        if (ii == ks)
#pragma unroll
          for (int q = 0; q < 8; ++q) x[ii][q] *= rd;
    }
    if (rb == kr) {
#pragma unroll
      for (int q = 0; q < 8; ++q) sm_xrow[c0 + q] = row_pick(x, ks, q);
    }
    named_barrier(bar, 64);
    T xr[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) xr[q] = sm_xrow[c0 + q];
#pragma unroll
    for (int ii = 0; ii < 8; ++ii) {
      const int i = rb + ii * 8;
      if (UPPER ? (i < k) : (i > k && i < kb)) {
        const T f = D[i + k * ldd];
#pragma unroll
        for (int q = 0; q < 8; ++q) x[ii][q] -= f * xr[q];
      }
    }
    named_barrier(bar, 64);
  }
#pragma unroll
  for (int q = 0; q < 8; ++q)
#pragma unroll
    for (int ii = 0; ii < 8; ++ii) dst[(rb + ii * 8) + (c0 + q) * 64] = x[ii][q];
}

// Both inverses of the factored diagonal block into the 2 x 64 x 64 dinv slot.
template <typename T, int ROWS>
__device__ void block_inverses(const T* D, int ldd, int kb, T* dst, T* sm_xrow2) {
  const int t = threadIdx.x;
  if (ROWS >= 128) {
    if (t < 64) tile_inverse<T, false>(D, ldd, kb, dst, sm_xrow2, t, 1);
    else if (t < 128) tile_inverse<T, true>(D, ldd, kb, dst + 4096, sm_xrow2 + 64, t - 64, 2);
  } else {
    tile_inverse<T, false>(D, ldd, kb, dst, sm_xrow2, t, 1);
    tile_inverse<T, true>(D, ldd, kb, dst + 4096, sm_xrow2 + 64, t, 1);
  }
}

// ---------------------------------------------------------------------------
// Speculative panel: LU without interchanges of the 64 x 64 diagonal block of
// a panel step, and the inverses of its two triangles, by 8 x 8 blocks.  The
// block is padded to 64 x 64 with the identity (so L, U and both inverses are
// block diagonal with identity beyond kb).  Step s of 8: one warp factors the
// 8 x 8 diagonal block with shuffles and inverts its triangles; then the
// block column below (L_rs = A_rs inv(U_ss)) and the block row to the right
// (U_sc = inv(L_ss) A_sc) are formed, and the trailing blocks updated.  The
// off-diagonal blocks of inv(L) (by block rows) and inv(U) (by block
// columns) are built by block substitution one step behind, by warps 1-7
// while warp 0 factors the next diagonal block.
// Every multiplier is checked against the partial-pivoting order (|l| <= 1);
// a violation or a zero pivot raises flags[0] and the factorization is redone
// with pivoting panels.
// ---------------------------------------------------------------------------
constexpr int kSpecThreads = 256;
constexpr int kLdS = 65;   // shared leading dimension of the 64 x 64 blocks

// Off-diagonal blocks of block row i of inv(L) and block column i of inv(U)
// (8 x 8 blocks, i >= 1) of the speculative panel, from the finished blocks
// of L, U and of both inverses with smaller block index: thread u < 8i forms
// column b of Li(i, s) = -Li_ii (sum_{s<=k<i} L_ik Li_ks), thread
// 8i <= u < 16i row a of Ui(s, i) = -(sum_{s<=k<i} Ui_sk U_ki) Ui_ii.  No
// thread reads another's output, so block i can be formed while warp 0
// factors diagonal block i + 1.
template <typename T>
__device__ __forceinline__ void spec_inverse_blocks(const T* A, T* Li, T* Ui, int i, int u) {
  if (u < 8 * i) {
    const int s = u >> 3, b = u & 7;
    T col[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) col[a] = T(0);
    for (int k = 8 * s; k < 8 * i; ++k) {
      const T lk = Li[k + (8 * s + b) * kLdS];
#pragma unroll
      for (int a = 0; a < 8; ++a) col[a] += A[(8 * i + a) + k * kLdS] * lk;
    }
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      T v = T(0);
#pragma unroll
      for (int k = 0; k < 8; ++k) v -= Li[(8 * i + a) + (8 * i + k) * kLdS] * col[k];
      Li[(8 * i + a) + (8 * s + b) * kLdS] = v;
    }
  } else if (u < 16 * i) {
    const int s = (u - 8 * i) >> 3, a = (u - 8 * i) & 7;
    T row[8];
#pragma unroll
    for (int b = 0; b < 8; ++b) row[b] = T(0);
    for (int k = 8 * s; k < 8 * i; ++k) {
      const T uk = Ui[(8 * s + a) + k * kLdS];
#pragma unroll
      for (int b = 0; b < 8; ++b) row[b] += uk * A[k + (8 * i + b) * kLdS];
    }
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      T v = T(0);
#pragma unroll
      for (int k = 0; k < 8; ++k) v -= row[k] * Ui[(8 * i + k) + (8 * i + b) * kLdS];
      Ui[(8 * s + a) + (8 * i + b) * kLdS] = v;
    }
  }
}

// The triangles of factored diagonal block i inverted (into Li / Ui's
// diagonal block i) by one warp: lanes 0-7 a column of inv(L_ii) each,
// lanes 8-15 a column of inv(U_ii), the block and its pivots' reciprocals in
// every lane's registers so the dependent chains read no shared memory.
template <typename T>
__device__ __forceinline__ void spec_diag_inverses(const T* A, T* Li, T* Ui, int i, int lane) {
  const int s8 = 8 * i;
  T blk[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int q = 0; q < 8; ++q) blk[r][q] = A[(s8 + r) + (s8 + q) * kLdS];
  T rd[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) rd[r] = T(1) / blk[r][r];
  if (lane < 8) {          // column `lane` of inv(L_ii)
    const int c = lane;
    T x[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) x[r] = (r == c) ? T(1) : T(0);
#pragma unroll
    for (int r = 1; r < 8; ++r) {
      T v = x[r];
#pragma unroll
      for (int k = 0; k < r; ++k) v -= blk[r][k] * x[k];
      x[r] = (r > c) ? v : x[r];
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) Li[(s8 + r) + (s8 + c) * kLdS] = x[r];
  } else if (lane < 16) {  // column `lane - 8` of inv(U_ii)
    const int c = lane - 8;
    T x[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) x[r] = T(0);
#pragma unroll
    for (int r = 7; r >= 0; --r) {
      T v = (r == c) ? T(1) : T(0);
#pragma unroll
      for (int k = r + 1; k < 8; ++k) v -= blk[r][k] * x[k];
      x[r] = (r <= c) ? v * rd[r] : T(0);
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) Ui[(s8 + r) + (s8 + c) * kLdS] = x[r];
  }
}

template <typename T>
__global__ void __launch_bounds__(kSpecThreads) k_panel_spec(DevPlan P, DevState S, const PanelTask* __restrict__ tasks,
                                                             T* __restrict__ pool, T* __restrict__ dinv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);     // 64 x 64, ld kLdS: L\U
  T* Li = A + 64 * kLdS;                     // inv(L)
  T* Ui = Li + 64 * kLdS;                    // inv(U)
  __shared__ int bad;
  __shared__ int seg[64];                    // per block column: end of its pivot rows (block-relative)
  __shared__ T rdiag[64];                    // reciprocals of U's diagonal
  const PanelTask tk = tasks[blockIdx.x];
  const int s_ = tk.s, k0 = tk.k0;
  const int np = P.np[s_], nf = P.nf[s_], c1 = P.c1[s_];
  const int kb = min(kPanel, np - k0);
  const int t = threadIdx.x, lane = lane_id(), warp = warp_id();
  T* F = pool + P.front_off[s_];
  if (t == 0) bad = 0;
  if (t < 64) seg[t] = t < kb ? min(kb, P.seg_end[c1 + k0 + t] - k0) : 0;
  {
    // all 16 of this thread's block values in flight before any store
    T v[64 * 64 / kSpecThreads];
#pragma unroll
    for (int q = 0; q < 64 * 64 / kSpecThreads; ++q) {
      const int e = t + q * kSpecThreads, r = e & 63, c = e >> 6;
      v[q] = (r < kb && c < kb) ? F[(k0 + r) + (int64_t)(k0 + c) * nf] : (r == c ? T(1) : T(0));
    }
#pragma unroll
    for (int q = 0; q < 64 * 64 / kSpecThreads; ++q) {
      const int e = t + q * kSpecThreads, r = e & 63, c = e >> 6;
      A[r + c * kLdS] = v[q];
      Li[r + c * kLdS] = T(0);
      Ui[r + c * kLdS] = T(0);
    }
  }
  __syncthreads();
  bool violated = false;
  for (int sb = 0; sb < 8; ++sb) {
    const int s8 = sb * 8;
    // (A) warp 0 factors diagonal block sb; meanwhile warp 1 inverts the
    // triangles of block sb - 1, and warps 2-7 form the off-diagonal
    // inverse blocks of block row / column sb - 2 and apply step sb - 1's
    // update to the blocks beyond sb (its block row and column sb were
    // updated ahead, in (C) of step sb - 1).  All read final data only.
    if (warp == 0) {   // 8 x 8 diagonal block: lanes 0..7 hold its rows
      T a[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) a[q] = lane < 8 ? A[(s8 + lane) + (s8 + q) * kLdS] : T(0);
#pragma unroll
      for (int jj = 0; jj < 8; ++jj) {
        T u[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) u[q] = __shfl_sync(0xffffffffu, a[q], jj);
        const T d = u[jj];
        if (lane > jj && lane < 8) {
          if (d == T(0) || (s8 + lane < seg[s8 + jj] && absd(a[jj]) > absd(d))) violated = true;
          const T l = d != T(0) ? a[jj] * (T(1) / d) : a[jj];
          a[jj] = l;
#pragma unroll
          for (int q = jj + 1; q < 8; ++q) a[q] -= l * u[q];
        }
        if (lane == 0 && d == T(0)) violated = true;
      }
      if (lane < 8) {
#pragma unroll
        for (int q = 0; q < 8; ++q) A[(s8 + lane) + (s8 + q) * kLdS] = a[q];
        rdiag[s8 + lane] = T(1) / a[lane];   // the reciprocal of this row's pivot
      }
    } else if (warp == 1) {
      if (sb >= 1) spec_diag_inverses<T>(A, Li, Ui, sb - 1, lane);
    } else {
      const int u = t - 64;
      if (sb >= 2) spec_inverse_blocks<T>(A, Li, Ui, sb - 2, u);
      if (sb >= 1) {   // step sb - 1 on the blocks beyond sb
        const int p8 = s8 - 8, b0 = s8 + 8, nd = 64 - b0;
        if (nd > 0) {
          const FastDiv dnd((uint32_t)nd);
          for (int e = u; e < nd * nd; e += kSpecThreads - 64) {
            const int q = (int)dnd.div(e), r = b0 + e - q * nd, c = b0 + q;
            T v = A[r + c * kLdS];
#pragma unroll
            for (int k = 0; k < 8; ++k) v -= A[r + (p8 + k) * kLdS] * A[(p8 + k) + c * kLdS];
            A[r + c * kLdS] = v;
          }
        }
      }
    }
    __syncthreads();
    // (B) block column sb of L (X U_ss = A_rs, back substitution with the
    // pivots' reciprocals) and block row sb of U (L_ss Y = A_sc, forward
    // substitution with the unit lower triangle)
    const int rest = 56 - s8;   // rows / columns after this block
    if (t < rest) {
      const int r = s8 + 8 + t;
      T x[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        T v = A[r + (s8 + q) * kLdS];
#pragma unroll
        for (int k = 0; k < q; ++k) v -= x[k] * A[(s8 + k) + (s8 + q) * kLdS];
        x[q] = v * rdiag[s8 + q];
        if (r < seg[s8 + q] && absd(x[q]) > 1.0) violated = true;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) A[r + (s8 + q) * kLdS] = x[q];
    } else if (t >= 64 && t < 64 + rest) {
      const int c = s8 + 8 + (t - 64);
      T y[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        T v = A[(s8 + i) + c * kLdS];
#pragma unroll
        for (int k = 0; k < i; ++k) v -= A[(s8 + i) + (s8 + k) * kLdS] * y[k];
        y[i] = v;
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) A[(s8 + i) + c * kLdS] = y[i];
    }
    __syncthreads();
    // (C) this step's update of block column and block row sb + 1 only
    // (what the next diagonal block and its L column / U row read); the
    // rest of the update runs in (A) of the next step
    if (rest > 0) {
      const int b8 = s8 + 8, n1 = rest * 8, n2 = 8 * (rest - 8);
      const FastDiv drest((uint32_t)rest);
      for (int e = t; e < n1 + n2; e += kSpecThreads) {
        int r, c;
        if (e < n1) {
          const int q = (int)drest.div(e);
          r = b8 + e - q * rest;
          c = b8 + q;
        } else {
          const int e2 = e - n1;
          r = b8 + (e2 & 7);
          c = b8 + 8 + (e2 >> 3);
        }
        T v = A[r + c * kLdS];
#pragma unroll
        for (int k = 0; k < 8; ++k) v -= A[r + (s8 + k) * kLdS] * A[(s8 + k) + c * kLdS];
        A[r + c * kLdS] = v;
      }
    }
    __syncthreads();
  }
  // the inverses' remaining blocks: diagonal block 7 and block row / column
  // 6, then block row / column 7
  if (warp == 1) spec_diag_inverses<T>(A, Li, Ui, 7, lane);
  else if (warp >= 2) spec_inverse_blocks<T>(A, Li, Ui, 6, t - 64);
  __syncthreads();
  spec_inverse_blocks<T>(A, Li, Ui, 7, t);
  __syncthreads();
  if (violated) bad = 1;
  __syncthreads();
  if (t == 0 && bad) atomicOr(S.flags, 1);
  const FastDiv dkb((uint32_t)kb);
  for (int e = t; e < kb * kb; e += kSpecThreads) {
    const int c = (int)dkb.div(e), r = e - c * kb;
    F[(k0 + r) + (int64_t)(k0 + c) * nf] = A[r + c * kLdS];
  }
  T* dst = dinv + (P.dinv_off[s_] + k0 / kPanel) * (int64_t)kDinvElems;
  for (int e = t; e < 64 * 64; e += kSpecThreads) {
    const int r = e & 63, c = e >> 6;
    dst[e] = Li[r + c * kLdS];
    dst[4096 + e] = Ui[r + c * kLdS];
  }
  for (int j = t; j < kb; j += kSpecThreads) S.ipiv[c1 + k0 + j] = k0 + j;
}

// Panel factorization of one panel step (k0..k1-1) of one large front.
// The candidate rows of a column are the pivot rows of its supernode
// (seg_end; all np rows of the front unless fronts are merged).
//  * kPanelSmemPivot: the R <= 256 candidate rows are held one row
//    per thread in registers; the pivot of each column is a block-wide
//    argmax (warp shuffles, LAPACK's first-maximum rule), the pivot row is
//    broadcast through shared memory, and the interchanges are applied to
//    the whole rows of the front (LAPACK getrf + the R12 swap of
//    src/multifrontal.jl:247-263).
//  * kPanelSpeculative: only the kb x kb diagonal block, without
//    interchanges; any row that partial pivoting would have preferred raises
//    flags[0] and the factorization is redone with pivoting panels.
//  * kPanelGlobalPivot: R > 256 rows, partial pivoting on global memory.
// Every mode ends by inverting the diagonal block's two triangles into dinv,
// which turns the panel's triangular solves (and the solves' diagonal blocks)
// into tensor-core tile products.
// ROWS (= threads per CTA, 64 / 128 / 256) bounds the rows a launch holds in
// registers, so small pivot blocks do not pay for the largest panel's
// registers and shared memory.
template <typename T, int ROWS>
__global__ void __launch_bounds__(ROWS) k_panel(DevPlan P, DevState S, const PanelTask* __restrict__ tasks,
                                                T* __restrict__ pool, T* __restrict__ dinv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* stage = reinterpret_cast<T*>(smem_raw);            // panel copy, col-major ld ROWS (ROWS x 64)
  T* sm_urow = stage + ROWS * kPanel;                   // 64
  T* sm_buf = sm_urow + 64;                             // 64
  T* sm_xrow = sm_buf + 64;                             // 2 x 64
  T* sm_lcol = sm_xrow + 128;                           // ROWS
  __shared__ ArgMax red[ROWS / 32];
  __shared__ int piv[kPanel];
  __shared__ int first_zero;
  __shared__ int sm_p;
  __shared__ int any_violation;
  __shared__ int seg[kPanel];             // per panel column: end of its pivot rows (panel-relative)
  const PanelTask tk = tasks[blockIdx.x];
  const int s = tk.s, k0 = tk.k0, mode = tk.mode;
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  const int kb = min(kPanel, np - k0);
  const int t = threadIdx.x, nthr = blockDim.x;
  T* F = pool + P.front_off[s];
  T* dst = dinv + (P.dinv_off[s] + k0 / kPanel) * (int64_t)kDinvElems;
  // candidate rows: the diagonal block (speculative) or every pivot row of
  // the panel's columns (their supernodes' pivot rows, np - k0 unmerged)
  const int R = (mode == kPanelSpeculative) ? kb : P.seg_end[c1 + k0 + kb - 1] - k0;
  if (t == 0) {
    first_zero = INT32_MAX;
    any_violation = 0;
  }
  for (int c = t; c < kPanel; c += nthr) seg[c] = c < kb ? min(R, P.seg_end[c1 + k0 + c] - k0) : 0;
  __syncthreads();

  if (mode != kPanelGlobalPivot) {
    constexpr int G = ROWS / 8;
    const int rb = t % G, c0 = (t / G) * 8;
    T a[8][8];
#pragma unroll
    for (int ii = 0; ii < 8; ++ii)
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int i = rb + ii * G, c = c0 + q;
        a[ii][q] = (i < R && c < kb) ? F[(k0 + i) + (int64_t)(k0 + c) * nf] : T(0);
      }
    bool violated = false;
    if (mode == kPanelSmemPivot)
      tile_lu<T, ROWS, true>(a, R, kb, seg, sm_urow, sm_buf, sm_lcol, &sm_p, piv, &first_zero, &violated);
    else
      tile_lu<T, ROWS, false>(a, R, kb, seg, sm_urow, sm_buf, sm_lcol, &sm_p, piv, &first_zero, &violated);
    if (violated) any_violation = 1;
#pragma unroll
    for (int ii = 0; ii < 8; ++ii)
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int i = rb + ii * G, c = c0 + q;
        if (i < R && c < kb) {
          F[(k0 + i) + (int64_t)(k0 + c) * nf] = a[ii][q];
          stage[i + c * ROWS] = a[ii][q];
        }
      }
    __syncthreads();
    if (t == 0 && (any_violation || (mode == kPanelSpeculative && first_zero != INT32_MAX))) atomicOr(S.flags, 1);
    block_inverses<T, ROWS>(stage, ROWS, kb, dst, sm_xrow);
  } else {
    panel_lu_pivot(F + k0 + (int64_t)k0 * nf, nf, R, kb, seg, piv, red, &first_zero);
    for (int e = t; e < kb * kb; e += nthr) stage[(e % kb) + (e / kb) * ROWS] = F[(k0 + e % kb) + (int64_t)(k0 + e / kb) * nf];
    __syncthreads();
    block_inverses<T, ROWS>(stage, ROWS, kb, dst, sm_xrow);
  }
  __syncthreads();
  for (int j = t; j < kb; j += nthr) S.ipiv[c1 + k0 + j] = k0 + piv[j];
  if (t == 0 && first_zero != INT32_MAX) atomicMin(S.info + s, k0 + first_zero);
  if (mode == kPanelSpeculative) return;
  // interchanges on the columns outside the panel, in LAPACK order; only the
  // steps that actually swapped are replayed
  __shared__ int nswap;
  __shared__ int swaps[kPanel];
  if (t == 0) {
    int c = 0;
    for (int j = 0; j < kb; ++j)
      if (piv[j] != j) swaps[c++] = j;
    nswap = c;
  }
  __syncthreads();
  const int ns = nswap;
  if (ns == 0) return;
  for (int cc = t; cc < nf - kb; cc += nthr) {
    const int c = cc < k0 ? cc : cc + kb;
    T* col = F + (int64_t)c * nf;
    for (int q = 0; q < ns; ++q) {
      const int j = swaps[q], p = piv[j];
      const T tmp = col[k0 + j];
      col[k0 + j] = col[k0 + p];
      col[k0 + p] = tmp;
    }
  }
}

// Triangular solves of one panel step as tile products with the inverted
// diagonal block: L part (rows r0..nf-1 of the panel columns)
// X = A * inv(U_kk) (rdiv! with UpperTriangular, src/multifrontal.jl:265);
// U part (rows k0..k1-1 right of the panel) X = inv(L_kk) * A (ldiv! with
// UnitLowerTriangular, :266).  Each CTA owns one 64-row or 64-column tile,
// reads it whole before writing it back, so the update is in place.  In
// speculative panels an L entry with |l| > 1 on a pivot row (a row partial
// pivoting would have chosen) raises flags[0].
constexpr int kApplyThreads = 128;

template <typename T>
__global__ void __launch_bounds__(kApplyThreads) k_panel_apply(DevPlan P, DevState S, const TrsmTask* __restrict__ tasks,
                                                               int ntasks, T* __restrict__ pool,
                                                               const T* __restrict__ dinv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sP = reinterpret_cast<T*>(smem_raw);   // 64 x kLdP
  T* sQ = sP + 64 * kLdP;                    // kLdQ x 64
  const int64_t tile = blockIdx.x;
  int lo = 0, hi = ntasks - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tasks[mid].tile_base <= tile) lo = mid;
    else hi = mid - 1;
  }
  const TrsmTask tk = tasks[lo];
  const int local = (int)(tile - tk.tile_base);
  const int s = tk.s, k0 = tk.k0;
  const int np = P.np[s], nf = P.nf[s];
  const int kb = min(kPanel, np - k0), k1 = k0 + kb;
  const int t = threadIdx.x;
  T* F = pool + P.front_off[s];
  const T* W = dinv + (P.dinv_off[s] + k0 / kPanel) * (int64_t)kDinvElems;
  const int32_t* seg = P.seg_end + P.c1[s] + k0;   // per panel column: end of its pivot rows
  const int r = t & 63, cg = t >> 6;   // row of the tile, column parity
  if (local < tk.lrow_tiles) {
    const int i0 = tk.r0 + 64 * local;
    const int rows = min(64, nf - i0);
    const T* src = F + (i0 + r) + (int64_t)k0 * nf;
#pragma unroll 8
    for (int c = cg; c < 64; c += 2) {
      sP[r + c * kLdP] = (r < rows && c < kb) ? src[(int64_t)c * nf] : T(0);
      sQ[r + c * kLdQ] = W[4096 + r + c * 64];   // inv(U_kk)(r, c)
    }
    __syncthreads();
    mm64<T>(sP, sQ, sP, kLdP);
    bool violated = false;
    const FastDiv drows((uint32_t)(rows > 0 ? rows : 1));
    for (int e = t; e < rows * kb; e += blockDim.x) {
      const int c = (int)drows.div(e), r = e - c * rows;
      const T v = sP[r + c * kLdP];
      if (tk.check && i0 + r < seg[c] && absd(v) > 1.0) violated = true;
      F[(i0 + r) + (int64_t)(k0 + c) * nf] = v;
    }
    if (violated) atomicOr(S.flags, 1);
  } else {
    const int j0 = k1 + 64 * (local - tk.lrow_tiles);
    const int cols = min(64, nf - j0);
    const T* src = F + (k0 + r) + (int64_t)j0 * nf;
#pragma unroll 8
    for (int c = cg; c < 64; c += 2) {
      sP[r + c * kLdP] = W[r + c * 64];           // inv(L_kk)(r, c)
      sQ[r + c * kLdQ] = (r < kb && c < cols) ? src[(int64_t)c * nf] : T(0);
    }
    __syncthreads();
    mm64<T>(sP, sQ, sQ, kLdQ);
    const FastDiv dkb((uint32_t)kb);
    for (int e = t; e < kb * cols; e += blockDim.x) {
      const int c = (int)dkb.div(e), r = e - c * kb;
      F[(k0 + r) + (int64_t)(j0 + c) * nf] = sQ[r + c * kLdQ];
    }
  }
}

// _pivot_rows: prow[c1+a] = V-row at block position a after the block's
// sequential interchanges; rowfac = inverse of prow.
// One warp per supernode: the identity and the inverse in parallel; the
// interchanges in their sequential order, visiting only the positions that
// swap (found 32 at a time by ballot; none after speculative panels).
__global__ void k_finalize_pivots(DevPlan P, DevState S) {
  const int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (s >= P.ns) return;   // warp-uniform
  const int lane = lane_id();
  const int c1 = P.c1[s], np = P.np[s];
  int32_t* pr = S.prow + c1;
  for (int a = lane; a < np; a += 32) pr[a] = c1 + a;
  __syncwarp();
  for (int base = 0; base < np; base += 32) {
    const int a = base + lane;
    const int p = a < np ? S.ipiv[c1 + a] : a;
    unsigned mask = __ballot_sync(0xffffffffu, a < np && p != a);
    while (mask) {
      const int j = __ffs(mask) - 1;
      mask &= mask - 1;
      const int pj = __shfl_sync(0xffffffffu, p, j);
      if (lane == 0) {
        const int32_t t = pr[base + j];
        pr[base + j] = pr[pj];
        pr[pj] = t;
      }
      __syncwarp();
    }
  }
  __syncwarp();
  for (int a = lane; a < np; a += 32) S.rowfac[pr[a]] = c1 + a;
}

// Direct CSC scatter; row indices are written 1-based (Julia's convention).
template <typename T>
__global__ void __launch_bounds__(256) k_scatter_csc(DevPlan P, DevState S, const T* __restrict__ pool,
                                                     int64_t fc_total, int64_t* __restrict__ li,
                                                     Wide<T>* __restrict__ lx, int64_t* __restrict__ ui,
                                                     Wide<T>* __restrict__ ux) {
  const int64_t fc = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_id();
  if (fc >= fc_total) return;
  const int lane = lane_id();
  const int s = P.fc_super[fc];
  const int c = (int)(fc - P.colbase[s]);
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  const T* col = c < np ? pool + P.lpan_off[s] + (int64_t)c * nf
                        : pool + P.u12_off[s] + (int64_t)(c - np) * u12_ld(P, s);
  const int32_t* us = P.upd + P.upd_off[s];
  if (c < np) {
    const int a = c, j = c1 + a;
    const int64_t lb = P.lcolptr[j];
    for (int r = lane; r < nf - a; r += 32) {
      const int fr = a + r;
      lx[lb + r] = r == 0 ? Wide<T>(1.0) : (Wide<T>)col[fr];
      li[lb + r] = 1 + (fr < np ? (int64_t)(c1 + fr) : (int64_t)S.rowfac[us[fr - np]]);
    }
    const int64_t ub = P.ucolptr[j + 1] - (a + 1);
    for (int b = lane; b <= a; b += 32) {
      ux[ub + b] = (Wide<T>)col[b];
      ui[ub + b] = 1 + c1 + b;
    }
  } else {
    const int64_t ub = P.uoff[P.upd_off[s] + (c - np)];
    for (int a = lane; a < np; a += 32) {
      ux[ub + a] = (Wide<T>)col[a];
      ui[ub + a] = 1 + c1 + a;
    }
  }
}

// Direct CSC scatter of merged fronts, one warp per front column, in the
// original supernodes' structure: a pivot column writes its L column (the
// pivot rows of its supernode from the diagonal down, then the supernode's
// update rows, found through rowfac for rows that are pivot rows of the same
// front) and its own U triangle; every front column then writes the U blocks
// of the original supernodes whose update set holds it (fcu).
template <typename T>
__global__ void __launch_bounds__(256) k_scatter_csc_merged(DevPlan P, DevState S, const T* __restrict__ pool,
                                                            int64_t fc_total, int64_t* __restrict__ li,
                                                            Wide<T>* __restrict__ lx, int64_t* __restrict__ ui,
                                                            Wide<T>* __restrict__ ux) {
  const int64_t fc = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_id();
  if (fc >= fc_total) return;
  const int lane = lane_id();
  const int x = P.fc_super[fc];
  const int c = (int)(fc - P.colbase[x]);
  const int np = P.np[x], nf = P.nf[x], c1 = P.c1[x];
  const T* col = c < np ? pool + P.lpan_off[x] + (int64_t)c * nf
                        : pool + P.u12_off[x] + (int64_t)(c - np) * u12_ld(P, x);
  if (c < np) {
    const int j = c1 + c, s = P.col_orig[j];
    const int a0 = P.o_c1[s] - c1, a1 = a0 + P.o_np[s];
    const int64_t lb = P.lcolptr[j];
    for (int r = lane; r < a1 - c; r += 32) {
      lx[lb + r] = r == 0 ? Wide<T>(1.0) : (Wide<T>)col[c + r];
      li[lb + r] = 1 + (int64_t)(c1 + c + r);
    }
    const int64_t ob = P.o_upd_off[s], on = P.o_upd_off[s + 1] - ob;
    const int64_t lu = lb + (a1 - c);
    for (int64_t i = lane; i < on; i += 32) {
      const int u = P.o_upd[ob + i];
      const int rf = S.rowfac[u];
      const int pos = u < c1 + np ? rf - c1 : P.o_xpos[ob + i];
      lx[lu + i] = (Wide<T>)col[pos];
      li[lu + i] = 1 + (int64_t)rf;
    }
    const int64_t ub = P.ucolptr[j + 1] - (c - a0 + 1);
    for (int b = lane; b <= c - a0; b += 32) {
      ux[ub + b] = (Wide<T>)col[a0 + b];
      ui[ub + b] = 1 + (int64_t)(c1 + a0 + b);
    }
  }
  for (int64_t e = P.fcu_ptr[fc]; e < P.fcu_ptr[fc + 1]; ++e) {
    const UBlock blk = P.fcu[e];
    for (int b = lane; b < blk.rows; b += 32) {
      ux[blk.uoff + b] = (Wide<T>)col[blk.row0 + b];
      ui[blk.uoff + b] = 1 + (int64_t)(c1 + blk.row0 + b);
    }
  }
}

// Lean layout: copy the factored panel of every front of a level (one warp
// per front column: the whole column below the diagonal block's top for the
// first np columns, the np U12 rows for the rest) to the panel pool.
template <typename T>
__global__ void __launch_bounds__(256) k_copy_panels(DevPlan P, int64_t fc0, int64_t count, T* __restrict__ pool) {
  const int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_id();
  if (w >= count) return;
  const int64_t fc = fc0 + w;
  const int s = P.fc_super[fc];
  const int c = (int)(fc - P.colbase[s]);
  const int np = P.np[s], nf = P.nf[s];
  const T* src = pool + P.front_off[s] + (int64_t)c * nf;
  T* dst = c < np ? pool + P.lpan_off[s] + (int64_t)c * nf : pool + P.u12_off[s] + (int64_t)(c - np) * np;
  const int rows = c < np ? nf : np;
  for (int r = lane_id(); r < rows; r += 32) dst[r] = src[r];
}

// V = Diagonal(Rs) * A restricted to qf: vx[p] = Rs[row] * A.nzval[src]
// (apply_row_scaling, src/scaling.jl:118-126, fused with A[qf,qf]).
__global__ void k_build_values(int64_t nnz, const int32_t* __restrict__ src, const int32_t* __restrict__ srow,
                               const double* __restrict__ ax, const double* __restrict__ rs, double* __restrict__ vx) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nnz) return;
  const double v = ax[src[p]];
  vx[p] = rs ? rs[srow[p]] * v : v;
}

// The same for ComplexF64 values (interleaved re, im) and a real Rs.
__global__ void k_build_values_z(int64_t nnz, const int32_t* __restrict__ src, const int32_t* __restrict__ srow,
                                 const zc* __restrict__ ax, const double* __restrict__ rs, zc* __restrict__ vx) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nnz) return;
  const zc v = ax[src[p]];
  vx[p] = rs ? zc(rs[srow[p]] * v.re, rs[srow[p]] * v.im) : v;
}

// Panel step of a ComplexF64 front: partial-pivot LU of the panel's R
// candidate rows in global memory (panel_lu_pivot: the pivot of column j is
// the first of largest |re| + |im| among its supernode's pivot rows), the
// inverses of the diagonal block's two triangles into dinv by column
// substitution, then the interchanges on the columns outside the panel.
// Complex register tiles would not fit the register file, so the complex
// fronts take this global-memory variant for every panel (the pivoting
// launches of the plan; no speculative panels).
template <typename T>
__global__ void __launch_bounds__(kPanelThreads) k_panel_global(DevPlan P, DevState S,
                                                                const PanelTask* __restrict__ tasks,
                                                                T* __restrict__ pool, T* __restrict__ dinv) {
  __shared__ ArgMax red[kPanelThreads / 32];
  __shared__ int piv[kPanel];
  __shared__ int first_zero;
  __shared__ int seg[kPanel];
  __shared__ int nswap;
  __shared__ int swaps[kPanel];
  const PanelTask tk = tasks[blockIdx.x];
  const int s = tk.s, k0 = tk.k0;
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  const int kb = min(kPanel, np - k0);
  const int t = threadIdx.x, nthr = blockDim.x;
  T* F = pool + P.front_off[s];
  T* dst = dinv + (P.dinv_off[s] + k0 / kPanel) * (int64_t)kDinvElems;
  const int R = P.seg_end[c1 + k0 + kb - 1] - k0;
  if (t == 0) first_zero = INT32_MAX;
  for (int c = t; c < kPanel; c += nthr) seg[c] = c < kb ? min(R, P.seg_end[c1 + k0 + c] - k0) : 0;
  __syncthreads();
  T* D = F + k0 + (int64_t)k0 * nf;
  panel_lu_pivot(D, nf, R, kb, seg, piv, red, &first_zero);
  diag_block_inverses(D, nf, kb, dst, dst + 4096);
  for (int j = t; j < kb; j += nthr) S.ipiv[c1 + k0 + j] = k0 + piv[j];
  if (t == 0) {
    if (first_zero != INT32_MAX) atomicMin(S.info + s, k0 + first_zero);
    int c = 0;
    for (int j = 0; j < kb; ++j)
      if (piv[j] != j) swaps[c++] = j;
    nswap = c;
  }
  __syncthreads();
  const int ns = nswap;
  for (int cc = t; ns && cc < nf - kb; cc += nthr) {
    const int c = cc < k0 ? cc : cc + kb;
    T* col = F + (int64_t)c * nf;
    for (int q = 0; q < ns; ++q) {
      const int j = swaps[q], p = piv[j];
      const T tmp = col[k0 + j];
      col[k0 + j] = col[k0 + p];
      col[k0 + p] = tmp;
    }
  }
}

}  // namespace mfgpu

namespace mfgpu {

// Diagonal 64 x 64 blocks of the explicit pivot-block inverses, from the
// panel factorization's inverted diagonal blocks: inv(L11) gets the unit
// lower triangle, inv(U11) the upper one (the other triangles stay zero from
// the clear that precedes this kernel).  One CTA per (supernode, block) pair.
template <typename T>
__global__ void __launch_bounds__(256) k_inv_init(DevPlan P, const int32_t* __restrict__ pairs,
                                                  const T* __restrict__ dinv, T* __restrict__ pool) {
  const int s = pairs[2 * blockIdx.x], j = pairs[2 * blockIdx.x + 1];
  const int np = P.np[s], k0 = j * kPanel, kb = min(kPanel, np - k0);
  const T* W = dinv + (P.dinv_off[s] + j) * (int64_t)kDinvElems;
  T* li = pool + P.inv_off[s] + k0 + (int64_t)k0 * np;
  T* ui = li + (int64_t)np * np;
  for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
    const int r = e % kb, c = e / kb;
    li[r + (int64_t)c * np] = r > c ? W[r + c * 64] : (r == c ? T(1) : T(0));
    ui[r + (int64_t)c * np] = r <= c ? W[4096 + r + c * 64] : T(0);
  }
}

}  // namespace mfgpu
