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
                                                                 T* __restrict__ pool, const double* __restrict__ vx) {
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
    for (int p = b + lane_id(); p < e; p += 32) F[P.v_frow[p] + c * nf] = (T)vx[p];
  }
  __syncthreads();
  for (int ci = P.child_ptr[s + 1] - 1; ci >= P.child_ptr[s]; --ci) {
    const int k = P.child_idx[ci];
    const int m = P.nu[k], nfk = P.nf[k], npk = P.np[k];
    const T* cb = pool + P.front_off[k] + npk + (int64_t)npk * nfk;
    const int32_t* rl = P.rel + P.upd_off[k];
    for (int e = tid; e < m * m; e += nthr) {
      const int r = e % m, t = e / m;
      F[rl[r] + rl[t] * nf] += cb[r + (int64_t)t * nfk];
    }
    __syncthreads();
  }

  int first_zero = INT32_MAX;
  for (int k = 0; k < np; ++k) {
    if (warp_id() == 0) {
      ArgMax a{-1.0, k};
      for (int i = k + lane_id(); i < np; i += 32) a = better(a, ArgMax{absd(F[i + k * nf]), i});
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
      if (i >= np || d != T(0)) F[i + k * nf] *= rcp;
    __syncthreads();
    const int rows = nf - k - 1;
    for (int e = tid; e < rows * rows; e += nthr) {
      const int i = k + 1 + e % rows, j = k + 1 + e / rows;
      F[i + j * nf] -= F[i + k * nf] * F[k + j * nf];
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
                                                          const double* __restrict__ vx) {
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
  for (int p = P.fc_vbeg[fc] + lane; p < P.fc_vend[fc]; p += 32) col[P.v_frow[p]] = (T)vx[p];
  __syncwarp();
  for (int e = P.fc_ch_ptr[fc]; e < P.fc_ch_ptr[fc + 1]; ++e) {
    const int k = P.fc_ch[2 * (int64_t)e], t = P.fc_ch[2 * (int64_t)e + 1];
    const int m = P.nu[k], nfk = P.nf[k], npk = P.np[k];
    const T* cb = pool + P.front_off[k] + npk + (int64_t)(npk + t) * nfk;
    const int32_t* rl = P.rel + P.upd_off[k];
    for (int r = lane; r < m; r += 32) col[rl[r]] += cb[r];
    __syncwarp();
  }
}

// Partial-pivot LU of an R x kb panel A (leading dimension lda, shared or
// global memory); the pivot of column j is searched in rows j..R-1 with
// idamax's first-maximum rule.  Records local pivots in piv[] (shared) and the
// first zero pivot (panel-relative) in *first_zero.
template <typename T>
__device__ void panel_lu_pivot(T* A, int lda, int R, int kb, int* piv, ArgMax* red, int* first_zero) {
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int j = 0; j < kb; ++j) {
    ArgMax a{-1.0, j};
    for (int i = j + tid; i < R; i += nthr) a = better(a, ArgMax{absd(A[i + (int64_t)j * lda]), i});
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

template <typename T>
__global__ void __launch_bounds__(kPanelThreads) k_panel(DevPlan P, DevState S, const PanelTask* __restrict__ tasks,
                                                         T* __restrict__ pool) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  __shared__ ArgMax red[kPanelThreads / 32];
  __shared__ int piv[kPanel];
  __shared__ int first_zero;
  const PanelTask tk = tasks[blockIdx.x];
  const int s = tk.s, k0 = tk.k0;
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  const int kb = min(kPanel, np - k0), k1 = k0 + kb;
  const int tid = threadIdx.x, nthr = blockDim.x;
  T* F = pool + P.front_off[s];
  if (tid == 0) first_zero = INT32_MAX;

  if (tk.mode == kPanelSpeculative) {
    // diagonal block only, no interchanges; flag any row that partial
    // pivoting would have chosen instead of the diagonal.
    for (int e = tid; e < kb * kb; e += nthr) sm[e] = F[(k0 + e % kb) + (int64_t)(k0 + e / kb) * nf];
    __syncthreads();
    for (int j = 0; j < kb; ++j) {
      const T d = sm[j + j * kb];
      const double ad = absd(d);
      for (int i = j + 1 + tid; i < kb; i += nthr)
        if (absd(sm[i + j * kb]) > ad) atomicOr(S.flags, 1);
      if (d == T(0)) {
        if (tid == 0) atomicOr(S.flags, 1);
      } else {
        const T rcp = T(1) / d;
        for (int i = j + 1 + tid; i < kb; i += nthr) sm[i + j * kb] *= rcp;
      }
      __syncthreads();
      const int r = kb - j - 1;
      for (int e = tid; e < r * r; e += nthr) {
        const int i = j + 1 + e % r, c = j + 1 + e / r;
        sm[i + c * kb] -= sm[i + j * kb] * sm[j + c * kb];
      }
      __syncthreads();
    }
    for (int e = tid; e < kb * kb; e += nthr) F[(k0 + e % kb) + (int64_t)(k0 + e / kb) * nf] = sm[e];
    for (int j = tid; j < kb; j += nthr) S.ipiv[c1 + k0 + j] = k0 + j;
    return;
  }

  const int R = np - k0;
  if (tk.mode == kPanelSmemPivot) {
    for (int e = tid; e < R * kb; e += nthr) sm[e] = F[(k0 + e % R) + (int64_t)(k0 + e / R) * nf];
    __syncthreads();
    panel_lu_pivot(sm, R, R, kb, piv, red, &first_zero);
    for (int e = tid; e < R * kb; e += nthr) F[(k0 + e % R) + (int64_t)(k0 + e / R) * nf] = sm[e];
  } else {
    __syncthreads();
    panel_lu_pivot(F + k0 + (int64_t)k0 * nf, nf, R, kb, piv, red, &first_zero);
  }
  __syncthreads();
  for (int j = tid; j < kb; j += nthr) S.ipiv[c1 + k0 + j] = k0 + piv[j];
  if (tid == 0 && first_zero != INT32_MAX) atomicMin(S.info + s, k0 + first_zero);
  // interchanges on the columns outside the panel, in LAPACK order
  for (int cc = tid; cc < nf - kb; cc += nthr) {
    const int c = cc < k0 ? cc : cc + kb;
    T* col = F + (int64_t)c * nf;
    for (int j = 0; j < kb; ++j) {
      const int p = piv[j];
      if (p != j) {
        const T t = col[k0 + j];
        col[k0 + j] = col[k0 + p];
        col[k0 + p] = t;
      }
    }
  }
  (void)k1;
}

// Triangular solves of one panel step.  L part: rows r0..nf-1 of the panel
// columns, X * U_kk = A (rdiv! with UpperTriangular, multifrontal.jl:265);
// U part: rows k0..k1-1 of the columns right of the panel,
// L_kk * X = A (ldiv! with UnitLowerTriangular, multifrontal.jl:266).
constexpr int kTrsmThreads = 64;

template <typename T>
__global__ void __launch_bounds__(kTrsmThreads) k_panel_trsm(DevPlan P, DevState S, const TrsmTask* __restrict__ tasks,
                                                             int ntasks, T* __restrict__ pool) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sD = reinterpret_cast<T*>(smem_raw);
  T* sX = sD + 64 * 65;
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
  const int tid = threadIdx.x;
  T* F = pool + P.front_off[s];
  for (int e = tid; e < kb * kb; e += blockDim.x) sD[e % kb + (e / kb) * 65] = F[(k0 + e % kb) + (int64_t)(k0 + e / kb) * nf];
  if (local < tk.lrow_tiles) {
    const int i0 = tk.r0 + 64 * local;
    const int rows = min(64, nf - i0);
    for (int e = tid; e < rows * kb; e += blockDim.x)
      sX[e % rows + (e / rows) * 65] = F[(i0 + e % rows) + (int64_t)(k0 + e / rows) * nf];
    __syncthreads();
    if (tid < rows) {
      const bool chk = tk.check && (i0 + tid) < np;
      for (int j = 0; j < kb; ++j) {
        T num = sX[tid + j * 65];
        for (int i = 0; i < j; ++i) num -= sX[tid + i * 65] * sD[i + j * 65];
        const T d = sD[j + j * 65];
        if (chk && absd(num) > absd(d)) atomicOr(S.flags, 1);
        sX[tid + j * 65] = num * (T(1) / d);
      }
    }
    __syncthreads();
    for (int e = tid; e < rows * kb; e += blockDim.x)
      F[(i0 + e % rows) + (int64_t)(k0 + e / rows) * nf] = sX[e % rows + (e / rows) * 65];
  } else {
    const int j0 = k1 + 64 * (local - tk.lrow_tiles);
    const int cols = min(64, nf - j0);
    for (int e = tid; e < kb * cols; e += blockDim.x)
      sX[e % kb + (e / kb) * 65] = F[(k0 + e % kb) + (int64_t)(j0 + e / kb) * nf];
    __syncthreads();
    if (tid < cols) {
      T* x = sX + tid * 65;
      for (int i = 0; i < kb; ++i) {
        T v = x[i];
        for (int j = 0; j < i; ++j) v -= sD[i + j * 65] * x[j];
        x[i] = v;
      }
    }
    __syncthreads();
    for (int e = tid; e < kb * cols; e += blockDim.x)
      F[(k0 + e % kb) + (int64_t)(j0 + e / kb) * nf] = sX[e % kb + (e / kb) * 65];
  }
}

// _pivot_rows: prow[c1+a] = V-row at block position a after the block's
// sequential interchanges; rowfac = inverse of prow.
__global__ void k_finalize_pivots(DevPlan P, DevState S) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.ns) return;
  const int c1 = P.c1[s], np = P.np[s];
  int32_t* pr = S.prow + c1;
  for (int a = 0; a < np; ++a) pr[a] = c1 + a;
  for (int a = 0; a < np; ++a) {
    const int p = S.ipiv[c1 + a];
    if (p != a) {
      const int32_t t = pr[a];
      pr[a] = pr[p];
      pr[p] = t;
    }
  }
  for (int a = 0; a < np; ++a) S.rowfac[pr[a]] = c1 + a;
}

// Direct CSC scatter; row indices are written 1-based (Julia's convention).
template <typename T>
__global__ void __launch_bounds__(256) k_scatter_csc(DevPlan P, DevState S, const T* __restrict__ pool,
                                                     int64_t fc_total, int64_t* __restrict__ li,
                                                     double* __restrict__ lx, int64_t* __restrict__ ui,
                                                     double* __restrict__ ux) {
  const int64_t fc = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp_id();
  if (fc >= fc_total) return;
  const int lane = lane_id();
  const int s = P.fc_super[fc];
  const int c = (int)(fc - P.colbase[s]);
  const int np = P.np[s], nf = P.nf[s], c1 = P.c1[s];
  const T* col = pool + P.front_off[s] + (int64_t)c * nf;
  const int32_t* us = P.upd + P.upd_off[s];
  if (c < np) {
    const int a = c, j = c1 + a;
    const int64_t lb = P.lcolptr[j];
    for (int r = lane; r < nf - a; r += 32) {
      const int fr = a + r;
      lx[lb + r] = r == 0 ? 1.0 : (double)col[fr];
      li[lb + r] = 1 + (fr < np ? (int64_t)(c1 + fr) : (int64_t)S.rowfac[us[fr - np]]);
    }
    const int64_t ub = P.ucolptr[j + 1] - (a + 1);
    for (int b = lane; b <= a; b += 32) {
      ux[ub + b] = (double)col[b];
      ui[ub + b] = 1 + c1 + b;
    }
  } else {
    const int64_t ub = P.uoff[P.upd_off[s] + (c - np)];
    for (int a = lane; a < np; a += 32) {
      ux[ub + a] = (double)col[a];
      ui[ub + a] = 1 + c1 + a;
    }
  }
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

}  // namespace mfgpu
