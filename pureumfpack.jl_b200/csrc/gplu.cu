// gplu.cu -- C ABI of libmfgpu's Gilbert-Peierls LU on the GPU: gplu(A; q,
// tol, check, sort_factors) (src/gplu.jl:173-303), the method
// splu(A; method=:gplu, ordering) uses by default (src/interface.jl:93-120),
// and the solves over its factors, raw (src/solve.jl:66-77) or with the
// PureLU row scaling and refinement (src/interface.jl:123-177).
//
// One handle holds the factors of one or many independent systems; a system
// is factored by one warp (device/gplu_kernels.cuh), so a batch fills the GPU
// with systems side by side.  Each system's L and U live in a segment sized
// from the symbolic fill of (A + A^T)[q, q]; a system whose factors outgrow
// it (pivoting off the diagonal can add fill) stops, reports the overflow,
// and is factored again in a larger segment.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mfgpu.h"
#include "device/gplu_kernels.cuh"
#include "host/symbolic.h"

using namespace mfgpu;

namespace {

struct GpFail : std::runtime_error {
  int code;
  GpFail(int c, const std::string& w) : std::runtime_error(w), code(c) {}
};

#define GP_CK(x)                                                                                         \
  do {                                                                                                   \
    cudaError_t e_ = (x);                                                                                \
    if (e_ != cudaSuccess) throw GpFail(MFGPU_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct GBuf {
  void* p = nullptr;
  size_t bytes = 0;
  GBuf() = default;
  GBuf(const GBuf&) = delete;
  GBuf& operator=(const GBuf&) = delete;
  void swap(GBuf& o) {
    std::swap(p, o.p);
    std::swap(bytes, o.bytes);
  }
  void ensure(size_t need) {
    need = std::max<size_t>(need, 16);
    if (need <= bytes) return;
    release();
    if (cudaMalloc(&p, need) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      throw GpFail(MFGPU_ERR_NOMEM, "device allocation of " + std::to_string(need) + " bytes failed");
    }
    bytes = need;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
  ~GBuf() { release(); }
};

template <typename T>
void put(GBuf& b, const std::vector<T>& v, cudaStream_t st) {
  b.ensure(v.size() * sizeof(T));
  if (!v.empty()) GP_CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

// Room for one factor of an n x n system when the symbolic estimate is e.
int64_t clamp_cap(int64_t e, int64_t n) {
  const int64_t dense = n * (n + 1) / 2;   // no factor holds more
  return std::max<int64_t>(16, std::min<int64_t>(e, std::max<int64_t>(dense, 1)));
}

unsigned blocks_for(int64_t warps, int per_block) { return (unsigned)((warps + per_block - 1) / per_block); }

// Element types of a handle's factors: the reference's Tv.
enum GpType { kGpF64 = 0, kGpF32 = 1, kGpC64 = 2 };

// Value e of a system's input as the device type (ComplexF64 as interleaved
// re, im doubles).
inline double load_val(const double* p, int64_t e, double*) { return p[e]; }
inline float load_val(const float* p, int64_t e, float*) { return p[e]; }
inline GpComplex load_val(const double* p, int64_t e, GpComplex*) { return GpComplex{p[2 * e], p[2 * e + 1]}; }

}  // namespace

struct mfgpu_gplu {
  int device = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  std::string err;
  int64_t cap_first = 0;      // entries per factor for the first attempt (0: the symbolic estimate)
  // the factored batch
  int64_t nsys = 0, ncols = 0;
  std::vector<GpSys> sys;
  std::vector<int64_t> status;
  std::vector<int32_t> q;     // 0-based orders, every system
  bool factored = false, scaled = false;
  int vt = kGpF64;            // element type of the factors
  size_t esize = 8;           // bytes per value
  double t_factor_ms = 0, t_finish_ms = 0, t_solve_ms = 0;
  int64_t attempts = 0, reruns = 0;
  GBuf d_sys, d_sys_old, d_list, d_colsys, d_acp, d_ari, d_ax, d_rs, d_q, d_status;
  GBuf d_lp, d_up, d_li, d_lx, d_ui, d_ux, d_pinv, d_perm;   // factors being built
  GBuf d_lo_i, d_lo_x, d_uo_i, d_uo_x;                        // finished factors
  GBuf d_x, d_xi, d_stack, d_pstack, d_mark;                  // factor workspace
  GBuf d_b, d_xs, d_c, d_r;                                    // solves
};

namespace {

int fail(mfgpu_gplu* g, int code, const std::string& msg) {
  g->err = msg;
  return code;
}

template <typename F>
int guarded(mfgpu_gplu* g, F&& f) {
  try {
    if (cudaSetDevice(g->device) != cudaSuccess) return fail(g, MFGPU_ERR_CUDA, "cudaSetDevice failed");
    return f();
  } catch (const GpFail& e) {
    cudaGetLastError();
    return fail(g, e.code, e.what());
  } catch (const std::exception& e) {
    return fail(g, MFGPU_ERR_INTERNAL, e.what());
  }
}

// Symbolic fill estimate of every system (host threads over the systems).
void estimate_caps(mfgpu_gplu* g, const int64_t* n, const int64_t* const* colptr, const int64_t* const* rowval,
                   std::vector<int64_t>& cap) {
  const int64_t S = g->nsys;
  cap.assign(S, 16);
  auto one = [&](int64_t s) {
    const int64_t ns = n[s];
    if (ns == 0) return;
    const int64_t nnz = colptr[s][ns] - 1;
    if (g->cap_first > 0) {
      cap[s] = clamp_cap(g->cap_first, ns);
      return;
    }
    int64_t half = 0;
    try {
      std::vector<idx_t> cp(ns + 1), ri(nnz), qs(ns);
      for (int64_t j = 0; j <= ns; ++j) cp[j] = colptr[s][j] - 1;
      for (int64_t e = 0; e < nnz; ++e) ri[e] = rowval[s][e] - 1;
      for (int64_t k = 0; k < ns; ++k) qs[k] = g->q[g->sys[s].col0 + k];
      half = symbolic_mf(ns, cp.data(), ri.data(), qs.data()).predicted_fill() / 2;
    } catch (...) {
      half = 0;   // no estimate: the reference's first capacity, grown on overflow
    }
    cap[s] = clamp_cap(std::max<int64_t>(8 * nnz, half + half / 8 + ns), ns);
  };
  const int64_t nth = std::min<int64_t>(S, std::max(1u, std::thread::hardware_concurrency()));
  if (nth <= 1) {
    for (int64_t s = 0; s < S; ++s) one(s);
    return;
  }
  std::vector<std::thread> th;
  for (int64_t t = 0; t < nth; ++t)
    th.emplace_back([&, t] {
      for (int64_t s = t; s < S; s += nth) one(s);
    });
  for (auto& t : th) t.join();
}

// Segments of L and U for the capacities cap_l / cap_u.
void lay_out(std::vector<GpSys>& sys, const std::vector<int64_t>& cap_l, const std::vector<int64_t>& cap_u,
             int64_t& tot_l, int64_t& tot_u) {
  tot_l = tot_u = 0;
  for (size_t s = 0; s < sys.size(); ++s) {
    sys[s].l0 = tot_l;
    sys[s].lcap = cap_l[s];
    sys[s].u0 = tot_u;
    sys[s].ucap = cap_u[s];
    tot_l += cap_l[s];
    tot_u += cap_u[s];
  }
}

template <typename T>
GpFactors<T> working(mfgpu_gplu* g) {
  return GpFactors<T>{g->d_lp.as<int64_t>(), g->d_li.as<int32_t>(), g->d_lx.as<T>(), g->d_up.as<int64_t>(),
                      g->d_ui.as<int32_t>(), g->d_ux.as<T>(), g->d_pinv.as<int32_t>()};
}

template <typename T> constexpr int type_of();
template <> constexpr int type_of<double>() { return kGpF64; }
template <> constexpr int type_of<float>() { return kGpF32; }
template <> constexpr int type_of<GpComplex>() { return kGpC64; }

// T: the device value type; In: the caller's value array element (double
// pairs for ComplexF64); R: the real type of Rs and tol.
template <typename T, typename In>
int factor_impl(mfgpu_gplu* g, int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                const int64_t* const* rowval, const In* const* nzval, const int64_t* const* qin,
                const typename GpArith<T>::R* const* rs, typename GpArith<T>::R tol, int32_t check,
                int32_t sort_factors, int64_t* status_out) {
  using R = typename GpArith<T>::R;
  if (nsys < 0 || (nsys > 0 && (!n || !colptr))) return fail(g, MFGPU_ERR_ARGUMENT, "bad system arrays");
  g->factored = false;
  g->vt = type_of<T>();
  g->esize = sizeof(T);
  g->nsys = nsys;
  g->sys.assign(nsys, GpSys{});
  g->status.assign(nsys, kGpPending);
  // validate and lay out the inputs
  int64_t ncols = 0, ncp = 0, nnz_all = 0;
  bool any_rs = false;
  for (int64_t s = 0; s < nsys; ++s) {
    const int64_t ns = n[s];
    if (ns < 0 || ns >= INT32_MAX) return fail(g, MFGPU_ERR_ARGUMENT, "system order out of range");
    if (!colptr[s] || colptr[s][0] != 1) return fail(g, MFGPU_ERR_ARGUMENT, "colptr must start at 1");
    for (int64_t j = 0; j < ns; ++j)
      if (colptr[s][j + 1] < colptr[s][j]) return fail(g, MFGPU_ERR_ARGUMENT, "colptr must not decrease");
    const int64_t nnz = colptr[s][ns] - 1;
    if (nnz > 0 && (!rowval || !rowval[s] || !nzval || !nzval[s]))
      return fail(g, MFGPU_ERR_ARGUMENT, "missing rowval / nzval");
    for (int64_t j = 0; j < ns; ++j)
      for (int64_t e = colptr[s][j] - 1; e < colptr[s][j + 1] - 1; ++e) {
        const int64_t r = rowval[s][e];
        if (r < 1 || r > ns) return fail(g, MFGPU_ERR_ARGUMENT, "row index out of range");
        if (e > colptr[s][j] - 1 && r <= rowval[s][e - 1])
          return fail(g, MFGPU_ERR_ARGUMENT, "row indices must ascend within each column");
      }
    g->sys[s] = GpSys{ns, ncols, ncp, nnz_all, 0, 0, 0, 0};
    ncols += ns;
    ncp += ns + 1;
    nnz_all += nnz;
    any_rs |= rs && rs[s];
  }
  g->ncols = ncols;
  g->scaled = any_rs;
  // host arrays: 0-based pattern, values, orders, scaling
  std::vector<int64_t> acp(ncp);
  std::vector<int32_t> ari(nnz_all), colsys(ncols);
  std::vector<T> ax(nnz_all);
  std::vector<R> rsv(any_rs ? ncols : 0, R(1));
  g->q.assign(ncols, 0);
  for (int64_t s = 0; s < nsys; ++s) {
    const GpSys& d = g->sys[s];
    const int64_t ns = d.n, nnz = colptr[s][ns] - 1;
    for (int64_t j = 0; j <= ns; ++j) acp[d.cp0 + j] = colptr[s][j] - 1;
    for (int64_t e = 0; e < nnz; ++e) {
      ari[d.nz0 + e] = (int32_t)(rowval[s][e] - 1);
      ax[d.nz0 + e] = load_val(nzval[s], e, (T*)nullptr);
    }
    std::vector<char> seen(ns, 0);
    for (int64_t k = 0; k < ns; ++k) {
      const int64_t c = (qin && qin[s]) ? qin[s][k] - 1 : k;
      if (c < 0 || c >= ns || seen[c]) return fail(g, MFGPU_ERR_ARGUMENT, "q is not a permutation");
      seen[c] = 1;
      g->q[d.col0 + k] = (int32_t)c;
    }
    for (int64_t j = 0; j < ns; ++j) colsys[d.col0 + j] = (int32_t)s;
    if (any_rs && rs[s])
      for (int64_t i = 0; i < ns; ++i) rsv[d.col0 + i] = rs[s][i];
  }
  std::vector<int64_t> cap_l, cap_u;
  estimate_caps(g, n, colptr, rowval, cap_l);
  cap_u = cap_l;
  int64_t tot_l = 0, tot_u = 0;
  lay_out(g->sys, cap_l, cap_u, tot_l, tot_u);
  cudaStream_t st = g->st;
  put(g->d_acp, acp, st);
  put(g->d_ari, ari, st);
  put(g->d_ax, ax, st);
  put(g->d_q, g->q, st);
  put(g->d_colsys, colsys, st);
  if (any_rs) put(g->d_rs, rsv, st);
  put(g->d_sys, g->sys, st);
  put(g->d_status, g->status, st);
  g->d_lp.ensure(ncp * 8);
  g->d_up.ensure(ncp * 8);
  g->d_pinv.ensure(ncols * 4);
  g->d_perm.ensure(ncols * 4);
  g->d_li.ensure(tot_l * 4);
  g->d_lx.ensure(tot_l * sizeof(T));
  g->d_ui.ensure(tot_u * 4);
  g->d_ux.ensure(tot_u * sizeof(T));
  g->d_x.ensure(ncols * sizeof(T));
  g->d_xi.ensure(ncols * 4);
  g->d_stack.ensure(ncols * 4);
  g->d_pstack.ensure(ncols * 8);
  g->d_mark.ensure(ncols * 4);
  std::vector<int32_t> list(nsys);
  for (int64_t s = 0; s < nsys; ++s) list[s] = (int32_t)s;
  g->attempts = g->reruns = 0;
  g->t_factor_ms = g->t_finish_ms = 0;
  const GpWork<T> W{g->d_x.as<T>(), g->d_xi.as<int32_t>(), g->d_stack.as<int32_t>(), g->d_pstack.as<int64_t>(),
                    g->d_mark.as<int32_t>()};
  while (!list.empty()) {
    put(g->d_list, list, st);
    GP_CK(cudaEventRecord(g->ev[0], st));
    k_gplu_factor<T><<<blocks_for((int64_t)list.size(), kGpWarps), 32 * kGpWarps, 0, st>>>(
        g->d_sys.as<GpSys>(), g->d_list.as<int32_t>(), (int64_t)list.size(), g->d_acp.as<int64_t>(),
        g->d_ari.as<int32_t>(), g->d_ax.as<T>(), any_rs ? g->d_rs.as<R>() : nullptr, g->d_q.as<int32_t>(), tol,
        check ? 1 : 0, working<T>(g), W, g->d_status.as<int64_t>());
    GP_CK(cudaGetLastError());
    GP_CK(cudaEventRecord(g->ev[1], st));
    GP_CK(cudaMemcpyAsync(g->status.data(), g->d_status.p, nsys * 8, cudaMemcpyDeviceToHost, st));
    GP_CK(cudaStreamSynchronize(st));
    float ms = 0;
    GP_CK(cudaEventElapsedTime(&ms, g->ev[0], g->ev[1]));
    g->t_factor_ms += ms;
    ++g->attempts;
    // systems that outgrew their segments: more room, the finished ones
    // moved to their new segments, then factored again
    std::vector<int32_t> again, done;
    for (int64_t s = 0; s < nsys; ++s) {
      const int64_t c = g->status[s];
      if (c == kGpOverflowL || c == kGpOverflowU) {
        again.push_back((int32_t)s);
        const int64_t ns = g->sys[s].n;
        if (c == kGpOverflowL) cap_l[s] = clamp_cap(cap_l[s] * 3, ns);
        if (c == kGpOverflowU) cap_u[s] = clamp_cap(cap_u[s] * 3, ns);
      } else if (c == 0) {
        done.push_back((int32_t)s);
      }
    }
    if (again.empty()) break;
    if (g->attempts > 64) throw GpFail(MFGPU_ERR_INTERNAL, "gplu: factor segments kept overflowing");
    g->reruns += (int64_t)again.size();
    std::vector<GpSys> old = g->sys;
    lay_out(g->sys, cap_l, cap_u, tot_l, tot_u);
    GBuf nli, nlx, nui, nux;
    nli.ensure(tot_l * 4);
    nlx.ensure(tot_l * sizeof(T));
    nui.ensure(tot_u * 4);
    nux.ensure(tot_u * sizeof(T));
    put(g->d_sys_old, old, st);
    put(g->d_sys, g->sys, st);
    if (!done.empty()) {
      put(g->d_list, done, st);
      k_gplu_move<T><<<blocks_for((int64_t)done.size(), 4), 128, 0, st>>>(
          g->d_sys_old.as<GpSys>(), g->d_sys.as<GpSys>(), g->d_list.as<int32_t>(), (int64_t)done.size(),
          g->d_lp.as<int64_t>(), g->d_up.as<int64_t>(), g->d_li.as<int32_t>(), g->d_lx.as<T>(),
          g->d_ui.as<int32_t>(), g->d_ux.as<T>(), nli.as<int32_t>(), nlx.as<T>(), nui.as<int32_t>(), nux.as<T>());
      GP_CK(cudaGetLastError());
    }
    GP_CK(cudaStreamSynchronize(st));
    g->d_li.swap(nli);
    g->d_lx.swap(nlx);
    g->d_ui.swap(nui);
    g->d_ux.swap(nux);
    list = again;
  }
  // relabel and sort (gplu.jl:292-302)
  g->d_lo_i.ensure(tot_l * 4);
  g->d_lo_x.ensure(tot_l * sizeof(T));
  g->d_uo_i.ensure(tot_u * 4);
  g->d_uo_x.ensure(tot_u * sizeof(T));
  GP_CK(cudaEventRecord(g->ev[2], st));
  if (ncols > 0) {
    k_gplu_finish<T><<<blocks_for(ncols, kGpWarps), 32 * kGpWarps, 0, st>>>(
        g->d_sys.as<GpSys>(), g->d_colsys.as<int32_t>(), ncols, g->d_status.as<int64_t>(), working<T>(g),
        sort_factors ? 1 : 0, g->d_lo_i.as<int32_t>(), g->d_lo_x.as<T>(), g->d_uo_i.as<int32_t>(),
        g->d_uo_x.as<T>(), g->d_perm.as<int32_t>());
    GP_CK(cudaGetLastError());
  }
  GP_CK(cudaEventRecord(g->ev[3], st));
  GP_CK(cudaStreamSynchronize(st));
  float ms = 0;
  GP_CK(cudaEventElapsedTime(&ms, g->ev[2], g->ev[3]));
  g->t_finish_ms = ms;
  if (status_out) std::copy(g->status.begin(), g->status.end(), status_out);
  int64_t singular = 0;
  for (int64_t s = 0; s < nsys; ++s) {
    if (g->status[s] == kGpNotPermutation)
      return fail(g, MFGPU_ERR_ARGUMENT,
                  "system " + std::to_string(s) + ": the pivot rows are not a permutation (singular, check = false)");
    if (g->status[s] < 0)
      return fail(g, MFGPU_ERR_INTERNAL, "system " + std::to_string(s) + ": factorization stopped with status " +
                                             std::to_string(g->status[s]));
    singular += g->status[s] > 0;
  }
  g->factored = singular == 0;
  return check ? (int)std::min<int64_t>(singular, INT32_MAX) : MFGPU_OK;
}

}  // namespace

extern "C" {

int mfgpu_gplu_create(int32_t device, mfgpu_gplu** out) {
  if (!out) return MFGPU_ERR_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return MFGPU_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major < 10) return MFGPU_ERR_NO_DEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return MFGPU_ERR_CUDA;
  auto* g = new mfgpu_gplu();
  g->device = device;
  if (cudaStreamCreateWithFlags(&g->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete g;
    return MFGPU_ERR_CUDA;
  }
  for (auto& e : g->ev)
    if (cudaEventCreate(&e) != cudaSuccess) {
      delete g;
      return MFGPU_ERR_CUDA;
    }
  *out = g;
  return MFGPU_OK;
}

void mfgpu_gplu_destroy(mfgpu_gplu* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->st) cudaStreamSynchronize(g->st);
  for (auto& e : g->ev)
    if (e) cudaEventDestroy(e);
  if (g->st) cudaStreamDestroy(g->st);
  delete g;
}

const char* mfgpu_gplu_last_error(const mfgpu_gplu* g) { return g ? g->err.c_str() : "null handle"; }

int mfgpu_gplu_set_initial_capacity(mfgpu_gplu* g, int64_t entries) {
  if (!g || entries < 0) return MFGPU_ERR_ARGUMENT;
  g->cap_first = entries;
  return MFGPU_OK;
}

int mfgpu_gplu_factor(mfgpu_gplu* g, int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                      const int64_t* const* rowval, const double* const* nzval, const int64_t* const* q,
                      const double* const* rs, double tol, int32_t check, int32_t sort_factors, int64_t* status) {
  if (!g) return MFGPU_ERR_ARGUMENT;
  return guarded(g, [&] {
    return factor_impl<double, double>(g, nsys, n, colptr, rowval, nzval, q, rs, tol, check, sort_factors, status);
  });
}

int mfgpu_gplu_factor_f32(mfgpu_gplu* g, int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                          const int64_t* const* rowval, const float* const* nzval, const int64_t* const* q,
                          const float* const* rs, double tol, int32_t check, int32_t sort_factors, int64_t* status) {
  if (!g) return MFGPU_ERR_ARGUMENT;
  return guarded(g, [&] {
    return factor_impl<float, float>(g, nsys, n, colptr, rowval, nzval, q, rs, (float)tol, check, sort_factors,
                                     status);
  });
}

int mfgpu_gplu_factor_c64(mfgpu_gplu* g, int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                          const int64_t* const* rowval, const double* const* nzval_ri, const int64_t* const* q,
                          const double* const* rs, double tol, int32_t check, int32_t sort_factors,
                          int64_t* status) {
  if (!g) return MFGPU_ERR_ARGUMENT;
  return guarded(g, [&] {
    return factor_impl<GpComplex, double>(g, nsys, n, colptr, rowval, nzval_ri, q, rs, tol, check, sort_factors,
                                          status);
  });
}

int mfgpu_gplu_sizes(mfgpu_gplu* g, int64_t sys, int64_t* out3) {
  if (!g || !out3) return MFGPU_ERR_ARGUMENT;
  if (!g->factored) return fail(g, MFGPU_ERR_STATE, "no completed factorization");
  if (sys < 0 || sys >= g->nsys) return fail(g, MFGPU_ERR_ARGUMENT, "system index out of range");
  return guarded(g, [&] {
    const GpSys& d = g->sys[sys];
    int64_t nl = 0, nu = 0;
    GP_CK(cudaMemcpy(&nl, g->d_lp.as<int64_t>() + d.cp0 + d.n, 8, cudaMemcpyDeviceToHost));
    GP_CK(cudaMemcpy(&nu, g->d_up.as<int64_t>() + d.cp0 + d.n, 8, cudaMemcpyDeviceToHost));
    out3[0] = d.n;
    out3[1] = nl;
    out3[2] = nu;
    return MFGPU_OK;
  });
}

}  // extern "C"

namespace {

// One system's factors (values of the handle's element type, copied as
// bytes: ComplexF64 as interleaved re, im doubles).
int get_factors_impl(mfgpu_gplu* g, int vt, int64_t sys, int64_t* lcolptr, int64_t* lrowval, void* lnzval,
                     int64_t* ucolptr, int64_t* urowval, void* unzval, int64_t* p, int64_t* q, int64_t* pinv) {
  if (!g) return MFGPU_ERR_ARGUMENT;
  if (!g->factored) return fail(g, MFGPU_ERR_STATE, "no completed factorization");
  if (g->vt != vt) return fail(g, MFGPU_ERR_STATE, "the factors hold another element type");
  if (sys < 0 || sys >= g->nsys) return fail(g, MFGPU_ERR_ARGUMENT, "system index out of range");
  return guarded(g, [&] {
    const GpSys& d = g->sys[sys];
    const int64_t n = d.n;
    const size_t es = g->esize;
    std::vector<int64_t> lp(n + 1), up(n + 1);
    GP_CK(cudaMemcpy(lp.data(), g->d_lp.as<int64_t>() + d.cp0, (n + 1) * 8, cudaMemcpyDeviceToHost));
    GP_CK(cudaMemcpy(up.data(), g->d_up.as<int64_t>() + d.cp0, (n + 1) * 8, cudaMemcpyDeviceToHost));
    const int64_t nl = lp[n], nu = up[n];
    std::vector<int32_t> li(nl), ui(nu), pm(n), pv(n);
    GP_CK(cudaMemcpy(li.data(), g->d_lo_i.as<int32_t>() + d.l0, nl * 4, cudaMemcpyDeviceToHost));
    GP_CK(cudaMemcpy(ui.data(), g->d_uo_i.as<int32_t>() + d.u0, nu * 4, cudaMemcpyDeviceToHost));
    GP_CK(cudaMemcpy(pm.data(), g->d_perm.as<int32_t>() + d.col0, n * 4, cudaMemcpyDeviceToHost));
    GP_CK(cudaMemcpy(pv.data(), g->d_pinv.as<int32_t>() + d.col0, n * 4, cudaMemcpyDeviceToHost));
    if (lnzval) GP_CK(cudaMemcpy(lnzval, g->d_lo_x.as<char>() + d.l0 * es, nl * es, cudaMemcpyDeviceToHost));
    if (unzval) GP_CK(cudaMemcpy(unzval, g->d_uo_x.as<char>() + d.u0 * es, nu * es, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k <= n; ++k) {
      if (lcolptr) lcolptr[k] = lp[k] + 1;
      if (ucolptr) ucolptr[k] = up[k] + 1;
    }
    if (lrowval)
      for (int64_t e = 0; e < nl; ++e) lrowval[e] = li[e] + 1;
    if (urowval)
      for (int64_t e = 0; e < nu; ++e) urowval[e] = ui[e] + 1;
    for (int64_t k = 0; k < n; ++k) {
      if (p) p[k] = pm[k] + 1;
      if (q) q[k] = g->q[d.col0 + k] + 1;
      if (pinv) pinv[k] = pv[k] + 1;
    }
    return MFGPU_OK;
  });
}

template <typename T>
int solve_impl(mfgpu_gplu* g, int64_t nrhs, const void* const* b, void* const* x, int32_t refine) {
  using R = typename GpArith<T>::R;
  if (!g || nrhs < 0 || refine < 0) return MFGPU_ERR_ARGUMENT;
  if (!g->factored) return fail(g, MFGPU_ERR_STATE, "solve before a completed factorization");
  if (g->vt != type_of<T>()) return fail(g, MFGPU_ERR_STATE, "the factors hold another element type");
  if (nrhs == 0 || g->ncols == 0) return MFGPU_OK;
  if (!b || !x) return fail(g, MFGPU_ERR_ARGUMENT, "missing right-hand sides");
  return guarded(g, [&] {
    cudaStream_t st = g->st;
    const size_t bytes = (size_t)g->ncols * nrhs * sizeof(T);
    g->d_b.ensure(bytes);
    g->d_xs.ensure(bytes);
    g->d_c.ensure(bytes);
    g->d_r.ensure(bytes);
    for (int64_t s = 0; s < g->nsys; ++s) {
      const GpSys& d = g->sys[s];
      if (d.n == 0) continue;
      if (!b[s] || !x[s]) throw GpFail(MFGPU_ERR_ARGUMENT, "missing right-hand side of a system");
      GP_CK(cudaMemcpyAsync(g->d_b.as<T>() + d.col0 * nrhs, b[s], d.n * nrhs * sizeof(T), cudaMemcpyHostToDevice,
                            st));
    }
    const GpSolveArgs<T> A{g->d_sys.as<GpSys>(), g->d_lp.as<int64_t>(),    g->d_lo_i.as<int32_t>(),
                           g->d_lo_x.as<T>(),    g->d_up.as<int64_t>(),    g->d_uo_i.as<int32_t>(),
                           g->d_uo_x.as<T>(),    g->d_perm.as<int32_t>(),  g->d_q.as<int32_t>(),
                           g->scaled ? g->d_rs.as<R>() : nullptr,          g->d_acp.as<int64_t>(),
                           g->d_ari.as<int32_t>(), g->d_ax.as<T>()};
    GP_CK(cudaEventRecord(g->ev[0], st));
    k_gplu_solve<T><<<blocks_for(g->nsys * nrhs, 4), 128, 0, st>>>(A, g->nsys, nrhs, g->d_b.as<T>(), g->d_xs.as<T>(),
                                                                    g->d_c.as<T>(), g->d_r.as<T>(), refine);
    GP_CK(cudaGetLastError());
    GP_CK(cudaEventRecord(g->ev[1], st));
    for (int64_t s = 0; s < g->nsys; ++s) {
      const GpSys& d = g->sys[s];
      if (d.n == 0) continue;
      GP_CK(cudaMemcpyAsync(x[s], g->d_xs.as<T>() + d.col0 * nrhs, d.n * nrhs * sizeof(T), cudaMemcpyDeviceToHost,
                            st));
    }
    GP_CK(cudaStreamSynchronize(st));
    float ms = 0;
    GP_CK(cudaEventElapsedTime(&ms, g->ev[0], g->ev[1]));
    g->t_solve_ms = ms;
    return MFGPU_OK;
  });
}

}  // namespace

extern "C" {

int mfgpu_gplu_get_factors(mfgpu_gplu* g, int64_t sys, int64_t* lcolptr, int64_t* lrowval, double* lnzval,
                           int64_t* ucolptr, int64_t* urowval, double* unzval, int64_t* p, int64_t* q,
                           int64_t* pinv) {
  return get_factors_impl(g, kGpF64, sys, lcolptr, lrowval, lnzval, ucolptr, urowval, unzval, p, q, pinv);
}

int mfgpu_gplu_get_factors_f32(mfgpu_gplu* g, int64_t sys, int64_t* lcolptr, int64_t* lrowval, float* lnzval,
                               int64_t* ucolptr, int64_t* urowval, float* unzval, int64_t* p, int64_t* q,
                               int64_t* pinv) {
  return get_factors_impl(g, kGpF32, sys, lcolptr, lrowval, lnzval, ucolptr, urowval, unzval, p, q, pinv);
}

int mfgpu_gplu_get_factors_c64(mfgpu_gplu* g, int64_t sys, int64_t* lcolptr, int64_t* lrowval, double* lnzval_ri,
                               int64_t* ucolptr, int64_t* urowval, double* unzval_ri, int64_t* p, int64_t* q,
                               int64_t* pinv) {
  return get_factors_impl(g, kGpC64, sys, lcolptr, lrowval, lnzval_ri, ucolptr, urowval, unzval_ri, p, q, pinv);
}

int mfgpu_gplu_solve(mfgpu_gplu* g, int64_t nrhs, const double* const* b, double* const* x, int32_t refine) {
  return solve_impl<double>(g, nrhs, (const void* const*)b, (void* const*)x, refine);
}

int mfgpu_gplu_solve_f32(mfgpu_gplu* g, int64_t nrhs, const float* const* b, float* const* x, int32_t refine) {
  return solve_impl<float>(g, nrhs, (const void* const*)b, (void* const*)x, refine);
}

int mfgpu_gplu_solve_c64(mfgpu_gplu* g, int64_t nrhs, const double* const* b_ri, double* const* x_ri,
                         int32_t refine) {
  return solve_impl<GpComplex>(g, nrhs, (const void* const*)b_ri, (void* const*)x_ri, refine);
}

int mfgpu_gplu_timings(mfgpu_gplu* g, double* out5) {
  if (!g || !out5) return MFGPU_ERR_ARGUMENT;
  out5[0] = g->t_factor_ms;
  out5[1] = g->t_finish_ms;
  out5[2] = g->t_solve_ms;
  out5[3] = (double)g->attempts;
  out5[4] = (double)g->reruns;
  return MFGPU_OK;
}

}  // extern "C"
