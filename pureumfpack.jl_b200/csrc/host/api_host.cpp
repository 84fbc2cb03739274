// api_host.cpp -- C ABI of libmfgpu's host-side ordering and symbolic code.
// Index arrays crossing the ABI are 1-based int64 (SparseMatrixCSC{Float64,Int64}).

#include <atomic>
#include <cmath>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/mfgpu.h"
#include "symbolic.h"

using mfgpu::idx_t;

namespace {
thread_local std::string g_host_error;

void to_zero_based(idx_t n, const int64_t* colptr, const int64_t* rowval, std::vector<idx_t>& cp,
                   std::vector<idx_t>& ri) {
  cp.resize(n + 1);
  for (idx_t j = 0; j <= n; ++j) cp[j] = colptr[j] - 1;
  ri.resize(cp[n]);
  for (idx_t p = 0; p < cp[n]; ++p) ri[p] = rowval[p] - 1;
}

bool valid_csc(int64_t m, int64_t n, const int64_t* colptr, const int64_t* rowval) {
  if (n < 0 || m < 0 || !colptr || (colptr[n] > 1 && !rowval) || colptr[0] != 1) return false;
  for (int64_t j = 0; j < n; ++j)
    if (colptr[j + 1] < colptr[j]) return false;
  for (int64_t p = 0; p < colptr[n] - 1; ++p)
    if (rowval[p] < 1 || rowval[p] > m) return false;
  return true;
}
}  // namespace

struct mfgpu_symbolic {
  mfgpu::SymbolicMF s;
};

extern "C" {

const char* mfgpu_host_last_error(void) { return g_host_error.c_str(); }

int mfgpu_row_scaling(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval, int32_t kind,
                      double* rs) {
  if (!valid_csc(n, n, colptr, rowval) || !rs || kind < 0 || kind > 2) return MFGPU_ERR_ARGUMENT;
  const int64_t nz = colptr[n] - 1;
  std::vector<idx_t> ri(nz);
  for (int64_t p = 0; p < nz; ++p) ri[p] = rowval[p] - 1;
  mfgpu::row_scaling(n, nz, ri.data(), nzval, kind, rs);
  return MFGPU_OK;
}

int mfgpu_row_scaling_f32(int64_t n, const int64_t* colptr, const int64_t* rowval, const float* nzval,
                          int32_t kind, float* rs) {
  if (!valid_csc(n, n, colptr, rowval) || !rs || kind < 0 || kind > 2) return MFGPU_ERR_ARGUMENT;
  const int64_t nz = colptr[n] - 1;
  std::vector<idx_t> ri(nz);
  for (int64_t p = 0; p < nz; ++p) ri[p] = rowval[p] - 1;
  mfgpu::row_scaling(n, nz, ri.data(), nzval, kind, rs);
  return MFGPU_OK;
}

int mfgpu_row_scaling_c64(int64_t n, const int64_t* colptr, const int64_t* rowval, const double* nzval_ri,
                          int32_t kind, double* rs) {
  if (!valid_csc(n, n, colptr, rowval) || !rs || kind < 0 || kind > 2 || (colptr[n] > 1 && !nzval_ri))
    return MFGPU_ERR_ARGUMENT;
  const int64_t nz = colptr[n] - 1;
  std::vector<idx_t> ri(nz);
  std::vector<double> mag(nz);
  for (int64_t p = 0; p < nz; ++p) {
    ri[p] = rowval[p] - 1;
    mag[p] = std::hypot(nzval_ri[2 * p], nzval_ri[2 * p + 1]);   // abs(::ComplexF64)
  }
  mfgpu::row_scaling(n, nz, ri.data(), mag.data(), kind, rs);
  return MFGPU_OK;
}

int mfgpu_amd_order(int64_t n, const int64_t* colptr, const int64_t* rowval, double dense, int64_t* perm) {
  if (!valid_csc(n, n, colptr, rowval) || !perm) return MFGPU_ERR_ARGUMENT;
  try {
    std::vector<idx_t> cp, ri;
    to_zero_based(n, colptr, rowval, cp, ri);
    std::vector<idx_t> p = mfgpu::amd_order_sym(n, cp.data(), ri.data(), dense);
    for (int64_t k = 0; k < n; ++k) perm[k] = p[k] + 1;
  } catch (const std::exception& e) {
    g_host_error = e.what();
    return MFGPU_ERR_INTERNAL;
  }
  return MFGPU_OK;
}

int mfgpu_colamd_order(int64_t m, int64_t n, const int64_t* colptr, const int64_t* rowval, double dense,
                       int64_t* perm) {
  if (!valid_csc(m, n, colptr, rowval) || !perm) return MFGPU_ERR_ARGUMENT;
  try {
    std::vector<idx_t> cp, ri;
    to_zero_based(n, colptr, rowval, cp, ri);
    std::vector<idx_t> p = mfgpu::colamd_order(m, n, cp.data(), ri.data(), dense);
    for (int64_t k = 0; k < n; ++k) perm[k] = p[k] + 1;
  } catch (const std::exception& e) {
    g_host_error = e.what();
    return MFGPU_ERR_INTERNAL;
  }
  return MFGPU_OK;
}

int mfgpu_symbolic_create(int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* q,
                          mfgpu_symbolic** out) {
  if (!out) return MFGPU_ERR_ARGUMENT;
  *out = nullptr;
  if (!valid_csc(n, n, colptr, rowval)) return MFGPU_ERR_ARGUMENT;
  try {
    std::vector<idx_t> cp, ri, q0;
    to_zero_based(n, colptr, rowval, cp, ri);
    if (q) {
      q0.resize(n);
      std::vector<char> seen(n, 0);
      for (int64_t k = 0; k < n; ++k) {
        q0[k] = q[k] - 1;
        if (q0[k] < 0 || q0[k] >= n || seen[q0[k]]) return MFGPU_ERR_ARGUMENT;
        seen[q0[k]] = 1;
      }
    }
    auto* h = new mfgpu_symbolic();
    h->s = mfgpu::symbolic_mf(n, cp.data(), ri.data(), q ? q0.data() : nullptr);
    *out = h;
  } catch (const std::exception& e) {
    g_host_error = e.what();
    return MFGPU_ERR_INTERNAL;
  }
  return MFGPU_OK;
}

int mfgpu_symbolic_create_batch(int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                                const int64_t* const* rowval, int32_t ordering, mfgpu_symbolic** out) {
  if (!out) return MFGPU_ERR_ARGUMENT;
  *out = nullptr;
  if (nsys < 1 || !n || !colptr || !rowval || (ordering != MFGPU_ORDER_AMD && ordering != MFGPU_ORDER_COLAMD))
    return MFGPU_ERR_ARGUMENT;
  for (int64_t i = 0; i < nsys; ++i)
    if (n[i] < 1 || !valid_csc(n[i], n[i], colptr[i], rowval[i])) return MFGPU_ERR_ARGUMENT;
  std::vector<mfgpu::SymbolicMF> parts(nsys);
  std::vector<std::string> errs(nsys);
  // one task per system, handed out dynamically (the systems' sizes vary)
  std::atomic<int64_t> next{0};
  auto work = [&] {
    for (int64_t i; (i = next.fetch_add(1)) < nsys;) {
      try {
        std::vector<idx_t> cp, ri;
        to_zero_based(n[i], colptr[i], rowval[i], cp, ri);
        const std::vector<idx_t> q = ordering == MFGPU_ORDER_AMD
                                         ? mfgpu::amd_order_sym(n[i], cp.data(), ri.data(), 10.0)
                                         : mfgpu::colamd_order(n[i], n[i], cp.data(), ri.data(), 10.0);
        parts[i] = mfgpu::symbolic_mf(n[i], cp.data(), ri.data(), q.data());
      } catch (const std::exception& e) {
        errs[i] = e.what();
      }
    }
  };
  const int64_t nt = std::min<int64_t>(nsys, std::max(1u, std::thread::hardware_concurrency()));
  std::vector<std::thread> pool;
  for (int64_t t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  for (int64_t i = 0; i < nsys; ++i)
    if (!errs[i].empty()) {
      g_host_error = "system " + std::to_string(i + 1) + ": " + errs[i];
      return MFGPU_ERR_INTERNAL;
    }
  try {
    auto* h = new mfgpu_symbolic();
    h->s = mfgpu::concat_symbolic(parts);
    *out = h;
  } catch (const std::exception& e) {
    g_host_error = e.what();
    return MFGPU_ERR_INTERNAL;
  }
  return MFGPU_OK;
}

void mfgpu_symbolic_destroy(mfgpu_symbolic* sym) { delete sym; }

int mfgpu_symbolic_relax(mfgpu_symbolic* sym) {
  if (!sym) return MFGPU_ERR_ARGUMENT;
  try {
    mfgpu::relax_supernodes(sym->s);
  } catch (const std::exception& e) {
    g_host_error = e.what();
    return MFGPU_ERR_INTERNAL;
  }
  return MFGPU_OK;
}

int mfgpu_symbolic_sizes(const mfgpu_symbolic* sym, int64_t* out4) {
  if (!sym || !out4) return MFGPU_ERR_ARGUMENT;
  const auto& s = sym->s;
  out4[0] = s.n;
  out4[1] = s.nsuper();
  out4[2] = (int64_t)s.upd_idx.size();
  out4[3] = (int64_t)s.child_idx.size();
  return MFGPU_OK;
}

int mfgpu_symbolic_get(const mfgpu_symbolic* sym, int64_t* qf, int64_t* parent, int64_t* colcount, int64_t* sstart,
                       int64_t* upd_ptr, int64_t* upd_idx, int64_t* child_ptr, int64_t* child_idx) {
  if (!sym) return MFGPU_ERR_ARGUMENT;
  const auto& s = sym->s;
  const int64_t n = s.n, ns = s.nsuper();
  for (int64_t k = 0; k < n; ++k) {
    if (qf) qf[k] = s.qf[k] + 1;
    if (parent) parent[k] = s.parent[k] + 1;       // 0 marks a root, as in the reference
    if (colcount) colcount[k] = s.colcount[k];
  }
  for (int64_t k = 0; k <= ns; ++k) {
    if (sstart) sstart[k] = s.sstart[k] + 1;
    if (upd_ptr) upd_ptr[k] = s.upd_ptr[k] + 1;
    if (child_ptr) child_ptr[k] = s.child_ptr[k] + 1;
  }
  if (upd_idx)
    for (size_t k = 0; k < s.upd_idx.size(); ++k) upd_idx[k] = s.upd_idx[k] + 1;
  if (child_idx)
    for (size_t k = 0; k < s.child_idx.size(); ++k) child_idx[k] = s.child_idx[k] + 1;
  return MFGPU_OK;
}

int64_t mfgpu_symbolic_predicted_fill(const mfgpu_symbolic* sym) { return sym ? sym->s.predicted_fill() : -1; }

int mfgpu_factor_colptrs(const mfgpu_symbolic* sym, int64_t* lcolptr, int64_t* ucolptr) {
  if (!sym || !lcolptr || !ucolptr) return MFGPU_ERR_ARGUMENT;
  std::vector<idx_t> lp, up;
  mfgpu::factor_colptrs(sym->s, lp, up);
  for (size_t k = 0; k < lp.size(); ++k) {
    lcolptr[k] = lp[k] + 1;
    ucolptr[k] = up[k] + 1;
  }
  return MFGPU_OK;
}

}  // extern "C"
