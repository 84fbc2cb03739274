// plan.cpp -- pattern analysis for the device factorization (see plan.h).

#include "plan.h"

#include "host/symbolic.h"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <exception>
#include <map>
#include <numeric>
#include <stdexcept>
#include <thread>

namespace mfgpu {

namespace {
inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Host threads for the plan's parallel loops: the hardware's, capped by the
// environment variable MFGPU_HOST_THREADS when it holds a positive number.
int64_t host_threads() {
  int64_t nt = std::max(1u, std::thread::hardware_concurrency());
  if (const char* e = std::getenv("MFGPU_HOST_THREADS")) {
    const long v = std::strtol(e, nullptr, 10);
    if (v > 0) nt = std::min<int64_t>(nt, v);
  }
  return nt;
}

// body(i) for i in [0, n) on the host's cores (independent iterations, each
// writing its own outputs), handed out `grain` at a time; the first exception
// is rethrown after the join.
template <typename F>
void parallel_range(int64_t n, F&& body, int64_t grain = 4096) {
  const int64_t nt = std::min<int64_t>(std::max<int64_t>(1, n / grain), host_threads());
  if (nt <= 1) {
    for (int64_t i = 0; i < n; ++i) body(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::exception_ptr err;
  std::atomic<bool> failed{false};
  auto work = [&] {
    try {
      for (int64_t b; !failed && (b = next.fetch_add(grain)) < n;)
        for (int64_t i = b; i < std::min(n, b + grain); ++i) body(i);
    } catch (...) {
      if (!failed.exchange(true)) err = std::current_exception();
    }
  };
  std::vector<std::thread> pool;
  for (int64_t t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  if (err) std::rethrow_exception(err);
}

// Boundaries [b[c], b[c+1]) of consecutive supernode ranges that are closed
// under the parent relation (a cut after x only where no supernode <= x has
// a parent > x), grouped to about 16 ranges per host thread of similar work
// (1 + update rows per supernode).  Every update row of a supernode is a
// column of one of its ancestors, so the ranges own disjoint columns, fronts
// and front columns: loops that fill per-column arrays in ascending supernode
// order can run range by range in parallel and give the sequential result.
// A single tree is a single range.
std::vector<int64_t> tree_chunks(const std::vector<int32_t>& parent, const std::vector<int32_t>& nu) {
  const int64_t ns = (int64_t)parent.size();
  int64_t total = ns;
  for (int32_t u : nu) total += u;
  const int64_t nt = host_threads();
  const int64_t target = std::max<int64_t>(1, total / (16 * nt));
  std::vector<int64_t> b{0};
  int64_t acc = 0, reach = -1;
  for (int64_t x = 0; x < ns; ++x) {
    acc += 1 + nu[x];
    reach = std::max<int64_t>(reach, parent[x]);
    if (reach <= x && acc >= target) {
      b.push_back(x + 1);
      acc = 0;
    }
  }
  if (b.back() != ns) b.push_back(ns);
  return b;
}
}  // namespace

namespace {
// Record C = f(C, A * B) in both tilings (see push_gemm) into the inverse lists.
void push_inv(Plan& P, InvStep& st, GemmTask g) {
  g.tiles_m = (int32_t)ceil_div(g.m, 64);
  g.tiles_n = (int32_t)ceil_div(g.n, 64);
  g.tile_base = st.tiles;
  st.tiles += (int64_t)g.tiles_m * g.tiles_n;
  P.inv_tasks.push_back(g);
  g.tiles_m = (int32_t)ceil_div(g.m, kTcTile);
  g.tiles_n = (int32_t)ceil_div(g.n, kTcTile);
  g.tile_base = st.tiles_tc;
  st.tiles_tc += (int64_t)g.tiles_m * g.tiles_n;
  P.inv_tasks_tc.push_back(g);
  ++st.count;
  st.max_k = std::max(st.max_k, g.k);
  st.flops += 2.0 * g.m * g.n * g.k;
  st.elems += (double)g.m * g.n * (g.mode == kGemmSub || g.mode == kGemmFrom ? 2 : 1) + (double)g.m * g.k +
              (double)g.k * g.n;
}

// Blocked inversion of every large pivot block.  With the pivot block split
// into consecutive blocks of s rows, a merge of [A 0; B C] (unit lower) is
//   inv = [inv(A) 0; -inv(C) B inv(A)  inv(C)]
// and of [A B; 0 C] (upper)
//   inv = [inv(A) -inv(A) B inv(C); 0 inv(C)];
// merge level s = 64, 128, ... pairs blocks (i, i + s) of size s and
// min(s, np - i - s): first T = B inv(A) (L) and T' = B inv(C) (U) into the
// scratch, then the off-diagonal block of the inverse = -(inv(C) T) and
// -(inv(A) T').
void build_inverse_steps(Plan& P) {
  int32_t max_np = 0;
  for (int64_t s = 0; s < P.ns; ++s)
    if (P.inv_off[s] >= 0) max_np = std::max(max_np, P.np[s]);
  for (int64_t bs = kPanel; bs < max_np; bs *= 2) {
    InvStep t1{(int64_t)P.inv_tasks.size(), 0, 0, 0, 0, 0};
    std::vector<GemmTask> second;
    int64_t scratch = 0;
    for (int64_t s = 0; s < P.ns; ++s) {
      if (P.inv_off[s] < 0 || P.np[s] <= bs) continue;
      const int32_t npv = P.np[s], nf = P.nf[s];
      const int64_t fo = P.lpan_off[s], li = P.inv_off[s], ui = li + (int64_t)npv * npv;
      for (int64_t i = 0; i + bs < npv; i += 2 * bs) {
        const int32_t n1 = (int32_t)bs, n2 = (int32_t)std::min<int64_t>(bs, npv - i - bs);
        const int64_t i2 = i + bs;
        const int64_t tl = P.inv_scratch + scratch, tu = tl + (int64_t)n2 * n1;
        scratch += 2 * (int64_t)n1 * n2;
        GemmTask g{};
        // L: T = L[i2:, i:i2] * inv(A)   (n2 x n1)
        g.a = fo + i2 + i * nf; g.lda = nf;
        g.b = li + i + i * npv; g.ldb = npv;
        g.c = tl; g.ldc = n2;
        g.m = n2; g.n = n1; g.k = n1; g.mode = kGemmSet;
        push_inv(P, t1, g);
        // L: inv[i2:, i:i2] = -(inv(C) * T)
        g = GemmTask{};
        g.a = li + i2 + i2 * npv; g.lda = npv;
        g.b = tl; g.ldb = n2;
        g.c = li + i2 + i * npv; g.ldc = npv;
        g.m = n2; g.n = n1; g.k = n2; g.mode = kGemmNeg;
        second.push_back(g);
        // U: T' = U[i:i2, i2:] * inv(C)   (n1 x n2)
        g = GemmTask{};
        g.a = fo + i + i2 * nf; g.lda = nf;
        g.b = ui + i2 + i2 * npv; g.ldb = npv;
        g.c = tu; g.ldc = n1;
        g.m = n1; g.n = n2; g.k = n2; g.mode = kGemmSet;
        push_inv(P, t1, g);
        // U: inv[i:i2, i2:] = -(inv(A) * T')
        g = GemmTask{};
        g.a = ui + i + i * npv; g.lda = npv;
        g.b = tu; g.ldb = n1;
        g.c = ui + i + i2 * npv; g.ldc = npv;
        g.m = n1; g.n = n2; g.k = n1; g.mode = kGemmNeg;
        second.push_back(g);
      }
    }
    P.inv_scratch_elems = std::max(P.inv_scratch_elems, scratch);
    P.inv_steps.push_back(t1);
    InvStep t2{(int64_t)P.inv_tasks.size(), 0, 0, 0, 0, 0};
    for (const GemmTask& g : second) push_inv(P, t2, g);
    P.inv_steps.push_back(t2);
    P.flops_inverse += t1.flops + t2.flops;
  }
}
}  // namespace

namespace {
// csc: lay out the factor's CSC for this partition (merged plans lay it out
// for the original supernodes instead, in attach_original).
void build_plan_core(int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf, const int64_t* parent,
                int64_t ns, const int64_t* sstart, const int64_t* upd_ptr, const int64_t* upd_idx, Plan& P,
                bool csc) {
  P = Plan();
  P.n = n;
  P.ns = ns;
  P.nnz_a = colptr[n];
  if (P.nnz_a >= (int64_t(1) << 31)) throw std::invalid_argument("nnz(A) exceeds the 32-bit entry maps");
  if (ns < 0 || (n > 0 && ns == 0) || sstart[0] != 0 || sstart[ns] != n)
    throw std::invalid_argument("supernode partition does not cover 1:n");

  // ---- supernodes -----------------------------------------------------------
  std::vector<int32_t> super_of(n);
  P.c1.resize(ns); P.np.resize(ns); P.nu.resize(ns); P.nf.resize(ns);
  P.upd_off.resize(ns + 1);
  for (int64_t s = 0; s < ns; ++s) {
    if (sstart[s + 1] <= sstart[s]) throw std::invalid_argument("empty supernode");
    P.c1[s] = (int32_t)sstart[s];
    P.np[s] = (int32_t)(sstart[s + 1] - sstart[s]);
    P.nu[s] = (int32_t)(upd_ptr[s + 1] - upd_ptr[s]);
    P.nf[s] = P.np[s] + P.nu[s];
    P.upd_off[s] = upd_ptr[s];
    for (int64_t j = sstart[s]; j < sstart[s + 1]; ++j) super_of[j] = (int32_t)s;
    P.max_nf = std::max(P.max_nf, P.nf[s]);
    P.max_np = std::max(P.max_np, P.np[s]);
  }
  P.upd_off[ns] = upd_ptr[ns];
  P.upd.resize(upd_ptr[ns]);
  for (int64_t s = 0; s < ns; ++s) {
    const int64_t c2 = sstart[s + 1] - 1;
    for (int64_t p = upd_ptr[s]; p < upd_ptr[s + 1]; ++p) {
      if (upd_idx[p] <= c2 || upd_idx[p] >= n || (p > upd_ptr[s] && upd_idx[p] <= upd_idx[p - 1]))
        throw std::invalid_argument("update set must be sorted rows below the supernode");
      P.upd[p] = (int32_t)upd_idx[p];
    }
  }

  // children (ascending) and tree heights
  P.parent_super.assign(ns, -1);
  std::vector<int32_t> nkid(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s) {
    const int64_t pc = parent[sstart[s + 1] - 1];
    if (pc >= 0) {
      const int32_t ps = super_of[pc];
      if (ps <= s) throw std::invalid_argument("supernodes are not in postorder");
      if (P.nu[s] == 0 || P.upd[P.upd_off[s]] != pc) throw std::invalid_argument("parent is not the first update row");
      P.parent_super[s] = ps;
      ++nkid[ps + 1];
    } else if (P.nu[s] != 0) {
      throw std::invalid_argument("root supernode with a nonempty update set");
    }
  }
  P.child_ptr.assign(ns + 1, 0);
  for (int64_t s = 0; s < ns; ++s) P.child_ptr[s + 1] = P.child_ptr[s] + nkid[s + 1];
  P.child_idx.resize(P.child_ptr[ns]);
  {
    std::vector<int32_t> cur(P.child_ptr.begin(), P.child_ptr.end() - 1);
    for (int64_t s = 0; s < ns; ++s)
      if (P.parent_super[s] >= 0) P.child_idx[cur[P.parent_super[s]]++] = (int32_t)s;
  }
  P.height.assign(ns, 0);
  for (int64_t s = 0; s < ns; ++s)
    if (P.parent_super[s] >= 0) P.height[P.parent_super[s]] = std::max(P.height[P.parent_super[s]], P.height[s] + 1);
  P.nlevels = ns ? 1 + *std::max_element(P.height.begin(), P.height.end()) : 0;

  // relative maps: position of each child update row in the parent front
  P.rel.assign(P.upd.size(), -1);
  parallel_range(ns, [&](int64_t k) {
    const int32_t ps = P.parent_super[k];
    if (ps < 0) return;
    const int32_t pc1 = P.c1[ps], pc2 = P.c1[ps] + P.np[ps] - 1;
    const int32_t* pu = P.upd.data() + P.upd_off[ps];
    for (int64_t p = P.upd_off[k]; p < P.upd_off[k + 1]; ++p) {
      const int32_t g = P.upd[p];
      if (g < pc1) throw std::invalid_argument("child update row below its parent");
      if (g <= pc2) {
        P.rel[p] = g - pc1;
      } else {
        const int32_t* it = std::lower_bound(pu, pu + P.nu[ps], g);
        if (it == pu + P.nu[ps] || *it != g) throw std::invalid_argument("child update row missing from parent front");
        P.rel[p] = P.np[ps] + (int32_t)(it - pu);
      }
    }
  });

  // ---- slots: supernodes ordered by (height, small before large, id) -------
  // (a stable counting sort of the ids on the key 2 * height + large)
  {
    auto key = [&](int64_t s) { return 2 * (int64_t)P.height[s] + (P.nf[s] > kSmallFront ? 1 : 0); };
    std::vector<int64_t> start(2 * (int64_t)P.nlevels + 1, 0);
    for (int64_t s = 0; s < ns; ++s) ++start[key(s) + 1];
    for (size_t k = 1; k < start.size(); ++k) start[k] += start[k - 1];
    P.slot_super.resize(ns);
    for (int64_t s = 0; s < ns; ++s) P.slot_super[start[key(s)]++] = (int32_t)s;
  }
  P.slot.resize(ns);
  P.level_slot.assign(P.nlevels + 1, 0);
  P.level_large.assign(P.nlevels, 0);
  for (int64_t i = 0; i < ns; ++i) P.slot[P.slot_super[i]] = (int32_t)i;
  for (int64_t i = 0; i < ns; ++i) P.level_slot[P.height[P.slot_super[i]] + 1] = (int32_t)(i + 1);
  for (int32_t L = 0; L < P.nlevels; ++L) {
    P.level_slot[L + 1] = std::max(P.level_slot[L + 1], P.level_slot[L]);
    int32_t i = P.level_slot[L];
    while (i < P.level_slot[L + 1] && P.nf[P.slot_super[i]] <= kSmallFront) ++i;
    P.level_large[L] = i;
  }
  P.front_off.resize(ns);
  P.colbase.resize(ns + 1);
  int64_t fo = 0, cb = 0;
  for (int64_t i = 0; i < ns; ++i) {
    const int32_t s = P.slot_super[i];
    P.front_off[s] = fo;
    P.colbase[s] = cb;
    fo += (int64_t)P.nf[s] * P.nf[s];
    cb += P.nf[s];
  }
  P.colbase[ns] = cb;   // sentinel: total front columns (not indexed by supernode)
  P.front_elems = fo;
  P.fc_total = cb;
  P.fc_super.resize(cb);
  for (int64_t s = 0; s < ns; ++s)
    for (int32_t c = 0; c < P.nf[s]; ++c) P.fc_super[P.colbase[s] + c] = (int32_t)s;

  // ---- V = A[qf, qf] and the assembly map of its entries --------------------
  P.qf.resize(n);
  std::vector<int64_t> pinv(n, -1);
  for (int64_t k = 0; k < n; ++k) {
    if (qf[k] < 0 || qf[k] >= n || pinv[qf[k]] != -1) throw std::invalid_argument("qf is not a permutation");
    pinv[qf[k]] = k;
    P.qf[k] = (int32_t)qf[k];
  }
  const int64_t nz = P.nnz_a;
  std::vector<int64_t> vcol(n + 1, 0);
  for (int64_t g = 0; g < n; ++g) vcol[g + 1] = vcol[g] + (colptr[qf[g] + 1] - colptr[qf[g]]);
  P.v_src.resize(nz);
  P.v_srow.resize(nz);
  P.v_frow.assign(nz, -1);
  std::vector<int32_t> vrow(nz);
  parallel_range(n, [&](int64_t g) {
    thread_local std::vector<std::pair<int64_t, int64_t>> tmp;
    tmp.clear();
    for (int64_t p = colptr[qf[g]]; p < colptr[qf[g] + 1]; ++p) tmp.push_back({pinv[rowval[p]], p});
    std::sort(tmp.begin(), tmp.end());
    for (size_t t = 0; t < tmp.size(); ++t) {
      if (t && tmp[t].first == tmp[t - 1].first) throw std::invalid_argument("duplicate entries in A");
      const int64_t q = vcol[g] + (int64_t)t;
      vrow[q] = (int32_t)tmp[t].first;
      P.v_src[q] = (int32_t)tmp[t].second;
      P.v_srow[q] = (int32_t)rowval[tmp[t].second];
    }
  });
  P.fc_vbeg.assign(cb, 0);
  P.fc_vend.assign(cb, 0);
  parallel_range(ns, [&](int64_t s) {
    const int32_t c1 = P.c1[s], c2 = c1 + P.np[s] - 1, npv = P.np[s];
    const int32_t* us = P.upd.data() + P.upd_off[s];
    auto front_row = [&](int32_t i) -> int32_t {
      if (i <= c2) return i - c1;
      const int32_t* it = std::lower_bound(us, us + P.nu[s], i);
      if (it == us + P.nu[s] || *it != i) throw std::invalid_argument("entry of A outside the symbolic structure");
      return npv + (int32_t)(it - us);
    };
    for (int32_t c = 0; c < P.nf[s]; ++c) {
      const int32_t g = c < npv ? c1 + c : us[c - npv];
      const int32_t* rb = vrow.data() + vcol[g];
      const int32_t* re = vrow.data() + vcol[g + 1];
      const int32_t* lo = std::lower_bound(rb, re, c1);
      const int32_t* hi = c < npv ? re : std::upper_bound(lo, re, c2);
      const int64_t fc = P.colbase[s] + c;
      P.fc_vbeg[fc] = (int32_t)(vcol[g] + (lo - rb));
      P.fc_vend[fc] = (int32_t)(vcol[g] + (hi - rb));
      for (const int32_t* r = lo; r < hi; ++r) {
        const int64_t q = vcol[g] + (r - rb);
        if (P.v_frow[q] != -1) throw std::logic_error("V entry assembled twice");
        P.v_frow[q] = front_row(*r);
      }
    }
  });
  if (std::count(P.v_frow.begin(), P.v_frow.end(), -1) != 0)
    throw std::invalid_argument("pattern of A is not covered by the symbolic structure");

  // ---- children contributions per parent front column ------------------------
  // (tree ranges in parallel: a child and its parent share a range)
  const std::vector<int64_t> chunks = tree_chunks(P.parent_super, P.nu);
  const int64_t nchunks = (int64_t)chunks.size() - 1;
  P.fc_ch_ptr.assign(cb + 1, 0);
  parallel_range(nchunks, [&](int64_t c) {
    for (int64_t k = chunks[c]; k < chunks[c + 1]; ++k) {
      const int32_t ps = P.parent_super[k];
      if (ps < 0) continue;
      for (int64_t p = P.upd_off[k]; p < P.upd_off[k + 1]; ++p) ++P.fc_ch_ptr[P.colbase[ps] + P.rel[p] + 1];
    }
  }, 1);
  for (int64_t f = 0; f < cb; ++f) P.fc_ch_ptr[f + 1] += P.fc_ch_ptr[f];
  P.fc_ch.resize(2 * (size_t)P.fc_ch_ptr[cb]);
  // fc_ch_ptr[f] serves as column f's cursor, then shifts back by one
  parallel_range(nchunks, [&](int64_t c) {
    for (int64_t ps = chunks[c]; ps < chunks[c + 1]; ++ps) {
      for (int32_t ci = P.child_ptr[ps + 1] - 1; ci >= P.child_ptr[ps]; --ci) {   // last child first
        const int32_t k = P.child_idx[ci];
        for (int32_t t = 0; t < P.nu[k]; ++t) {
          const int64_t f = P.colbase[ps] + P.rel[P.upd_off[k] + t];
          const int32_t at = P.fc_ch_ptr[f]++;
          P.fc_ch[2 * (size_t)at] = k;
          P.fc_ch[2 * (size_t)at + 1] = t;
        }
      }
    }
  }, 1);
  for (int64_t f = cb; f > 0; --f) P.fc_ch_ptr[f] = P.fc_ch_ptr[f - 1];
  P.fc_ch_ptr[0] = 0;

  // ---- factor CSC layout -------------------------------------------------
  if (csc) {
  P.lcolptr.assign(n + 1, 0);
  P.ucolptr.assign(n + 1, 0);
  parallel_range(nchunks, [&](int64_t c) {
    for (int64_t s = chunks[c]; s < chunks[c + 1]; ++s) {
      const int32_t c1 = P.c1[s], c2 = c1 + P.np[s] - 1;
      for (int32_t j = c1; j <= c2; ++j) {
        P.lcolptr[j + 1] = 1 + (c2 - j) + P.nu[s];
        P.ucolptr[j + 1] += j - c1 + 1;
      }
      for (int64_t p = P.upd_off[s]; p < P.upd_off[s + 1]; ++p) P.ucolptr[P.upd[p] + 1] += P.np[s];
    }
  }, 1);
  for (int64_t j = 0; j < n; ++j) {
    P.lcolptr[j + 1] += P.lcolptr[j];
    P.ucolptr[j + 1] += P.ucolptr[j];
  }
  P.nnz_l = P.lcolptr[n];
  P.nnz_u = P.ucolptr[n];
  P.uoff.resize(P.upd.size());
  {
    std::vector<int64_t> cur(P.ucolptr.begin(), P.ucolptr.end() - 1);
    parallel_range(nchunks, [&](int64_t c) {
      for (int64_t s = chunks[c]; s < chunks[c + 1]; ++s)
        for (int64_t p = P.upd_off[s]; p < P.upd_off[s + 1]; ++p) {
          P.uoff[p] = cur[P.upd[p]];
          cur[P.upd[p]] += P.np[s];
        }
    }, 1);
  }
  }

  // ---- A in CSR (residual r = b - A x) ------------------------------------
  P.csr_ptr.assign(n + 1, 0);
  for (int64_t p = 0; p < nz; ++p) ++P.csr_ptr[rowval[p] + 1];
  for (int64_t i = 0; i < n; ++i) P.csr_ptr[i + 1] += P.csr_ptr[i];
  P.csr_col.resize(nz);
  P.csr_src.resize(nz);
  {
    std::vector<int32_t> cur(P.csr_ptr.begin(), P.csr_ptr.end() - 1);
    for (int64_t j = 0; j < n; ++j)
      for (int64_t p = colptr[j]; p < colptr[j + 1]; ++p) {
        const int32_t at = cur[rowval[p]]++;
        P.csr_col[at] = (int32_t)j;
        P.csr_src[at] = (int32_t)p;
      }
  }

  // ---- inverted diagonal blocks of large fronts ------------------------------
  P.dinv_off.assign(ns, -1);
  for (int64_t s = 0; s < ns; ++s)
    if (P.nf[s] > kSmallFront) {
      P.dinv_off[s] = P.dinv_blocks;
      P.dinv_blocks += ceil_div(P.np[s], kPanel);
    }

  // ---- statistics ------------------------------------------------------------
  for (int64_t s = 0; s < ns; ++s) {
    const double a = P.np[s], u = P.nu[s];
    P.flops_getrf += 2.0 / 3.0 * a * a * a;
    P.flops_trsm += 2.0 * a * a * u;
    P.flops_gemm += 2.0 * a * u * u;
    double moves = (double)P.nf[s] * P.nf[s] + u * u;   // front write + CB handed on
    for (int32_t ci = P.child_ptr[s]; ci < P.child_ptr[s + 1]; ++ci) {
      const double m = P.nu[P.child_idx[ci]];
      moves += 3.0 * m * m;                             // CB read + parent read-modify-write
    }
    P.assembly_bytes_per_elem += moves;
  }
  P.flops = P.flops_getrf + P.flops_trsm + P.flops_gemm;
  P.flops_orig = P.flops;
  P.front_elems_full = P.front_elems;
  P.seg_end.resize(n);
  for (int64_t s = 0; s < ns; ++s)
    for (int32_t a = 0; a < P.np[s]; ++a) P.seg_end[P.c1[s] + a] = P.np[s];
  // original entries assembled into each front (launch traffic accounting)
  P.front_nv.assign(ns, 0);
  for (int64_t s = 0; s < ns; ++s)
    for (int32_t c = 0; c < P.nf[s]; ++c) P.front_nv[s] += P.fc_vend[P.colbase[s] + c] - P.fc_vbeg[P.colbase[s] + c];
}
}  // namespace

void check_symbolic(int64_t n, const int64_t* qf, const int64_t* parent, int64_t ns, const int64_t* sstart,
                    const int64_t* upd_ptr, const int64_t* upd_idx) {
  auto bad = [](const char* what) { throw std::invalid_argument(what); };
  if (n < 0 || ns < 0 || (n > 0) != (ns > 0)) bad("supernode count does not match n");
  if (n >= (int64_t(1) << 31)) bad("n exceeds the 32-bit index maps");
  if (!sstart || !upd_ptr || (n > 0 && (!qf || !parent))) bad("null symbolic array");
  if (sstart[0] != 0 || sstart[ns] != n) bad("supernode partition does not cover 1:n");
  for (int64_t s = 0; s < ns; ++s)
    if (sstart[s + 1] <= sstart[s]) bad("empty supernode");
  if (upd_ptr[0] != 0) bad("update pointers do not start at 1");
  for (int64_t s = 0; s < ns; ++s)
    if (upd_ptr[s + 1] < upd_ptr[s]) bad("update pointers decrease");
  if (upd_ptr[ns] >= (int64_t(1) << 31)) bad("update sets exceed the 32-bit index maps");
  if (upd_ptr[ns] > 0 && !upd_idx) bad("null symbolic array");
  for (int64_t s = 0; s < ns; ++s) {
    const int64_t c2 = sstart[s + 1] - 1;
    for (int64_t p = upd_ptr[s]; p < upd_ptr[s + 1]; ++p)
      if (upd_idx[p] <= c2 || upd_idx[p] >= n || (p > upd_ptr[s] && upd_idx[p] <= upd_idx[p - 1]))
        bad("update set must be sorted rows below the supernode");
  }
  // an elimination tree of the permuted matrix: every parent comes later
  for (int64_t j = 0; j < n; ++j)
    if (parent[j] < -1 || parent[j] >= n || (parent[j] >= 0 && parent[j] <= j)) bad("parent is not an elimination tree");
  std::vector<char> seen(n, 0);
  for (int64_t k = 0; k < n; ++k) {
    if (qf[k] < 0 || qf[k] >= n || seen[qf[k]]) bad("qf is not a permutation");
    seen[qf[k]] = 1;
  }
}

void build_plan(int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf, const int64_t* parent,
                int64_t ns, const int64_t* sstart, const int64_t* upd_ptr, const int64_t* upd_idx, Plan& P) {
  check_symbolic(n, qf, parent, ns, sstart, upd_ptr, upd_idx);
  build_plan_core(n, colptr, rowval, qf, parent, ns, sstart, upd_ptr, upd_idx, P, true);
  set_layout(P, false);
}

namespace {
// Original supernodes inside the merged fronts of P: pivot segments, the
// factor's CSC layout, and where each original block sits in its front.
void attach_original(Plan& P, int64_t ns, const int64_t* sstart, const int64_t* upd_ptr, const int64_t* upd_idx) {
  const int64_t n = P.n;
  P.merged = true;
  P.ns_orig = ns;
  std::vector<int32_t> front_of(n);
  for (int64_t x = 0; x < P.ns; ++x)
    for (int32_t a = 0; a < P.np[x]; ++a) front_of[P.c1[x] + a] = (int32_t)x;
  P.o_c1.resize(ns);
  P.o_np.resize(ns);
  P.o_upd_off.assign(upd_ptr, upd_ptr + ns + 1);
  P.o_upd.assign(upd_idx, upd_idx + upd_ptr[ns]);
  P.o_xpos.resize(upd_ptr[ns]);
  P.col_orig.resize(n);
  parallel_range(ns, [&](int64_t s) {
    const int32_t c1 = (int32_t)sstart[s], npv = (int32_t)(sstart[s + 1] - sstart[s]);
    const int32_t x = front_of[c1], xc1 = P.c1[x], xnp = P.np[x];
    if (front_of[c1 + npv - 1] != x) throw std::logic_error("original supernode split across fronts");
    P.o_c1[s] = c1;
    P.o_np[s] = npv;
    for (int32_t a = 0; a < npv; ++a) {
      P.col_orig[c1 + a] = (int32_t)s;
      P.seg_end[c1 + a] = c1 + npv - xc1;
    }
    const int32_t* xu = P.upd.data() + P.upd_off[x];
    for (int64_t p = upd_ptr[s]; p < upd_ptr[s + 1]; ++p) {
      const int32_t u = (int32_t)upd_idx[p];
      if (u < c1 + npv) throw std::logic_error("update row inside its supernode");
      if (u < xc1 + xnp) {
        P.o_xpos[p] = u - xc1;
      } else {
        const int32_t* it = std::lower_bound(xu, xu + P.nu[x], u);
        if (it == xu + P.nu[x] || *it != u) throw std::logic_error("update row missing from the merged front");
        P.o_xpos[p] = xnp + (int32_t)(it - xu);
      }
    }
  });
  double fl = 0;
  for (int64_t s = 0; s < ns; ++s) {
    const double a = P.o_np[s], u = (double)(upd_ptr[s + 1] - upd_ptr[s]);
    fl += 2.0 / 3.0 * a * a * a + 2.0 * a * a * u + 2.0 * a * u * u;
  }
  P.flops_orig = fl;
  // factor CSC layout of the original structure (as build_plan's) and the U
  // blocks per front column in the order of the original supernodes, by the
  // fronts' tree ranges (every update row of an original supernode lies in
  // its front, checked above), mapped to the original supernodes they hold
  const std::vector<int64_t> fch = tree_chunks(P.parent_super, P.nu);
  const int64_t nchunks = (int64_t)fch.size() - 1;
  std::vector<int64_t> och(nchunks + 1, ns);
  for (int64_t c = 0; c < nchunks; ++c) och[c] = P.col_orig[P.c1[fch[c]]];
  P.lcolptr.assign(n + 1, 0);
  P.ucolptr.assign(n + 1, 0);
  parallel_range(nchunks, [&](int64_t c) {
    for (int64_t s = och[c]; s < och[c + 1]; ++s) {
      const int32_t c1 = P.o_c1[s], c2 = c1 + P.o_np[s] - 1;
      const int64_t nu = upd_ptr[s + 1] - upd_ptr[s];
      for (int32_t j = c1; j <= c2; ++j) {
        P.lcolptr[j + 1] = 1 + (c2 - j) + nu;
        P.ucolptr[j + 1] += j - c1 + 1;
      }
      for (int64_t p = upd_ptr[s]; p < upd_ptr[s + 1]; ++p) P.ucolptr[upd_idx[p] + 1] += P.o_np[s];
    }
  }, 1);
  for (int64_t j = 0; j < n; ++j) {
    P.lcolptr[j + 1] += P.lcolptr[j];
    P.ucolptr[j + 1] += P.ucolptr[j];
  }
  P.nnz_l = P.lcolptr[n];
  P.nnz_u = P.ucolptr[n];
  P.fcu_ptr.assign(P.fc_total + 1, 0);
  auto fcol = [&](int64_t s, int64_t p) { return P.colbase[front_of[P.o_c1[s]]] + P.o_xpos[p]; };
  parallel_range(nchunks, [&](int64_t c) {
    for (int64_t s = och[c]; s < och[c + 1]; ++s)
      for (int64_t p = upd_ptr[s]; p < upd_ptr[s + 1]; ++p) ++P.fcu_ptr[fcol(s, p) + 1];
  }, 1);
  for (int64_t f = 0; f < P.fc_total; ++f) P.fcu_ptr[f + 1] += P.fcu_ptr[f];
  P.fcu.resize(P.fcu_ptr[P.fc_total]);
  // fcu_ptr[f] serves as front column f's cursor, then shifts back by one
  std::vector<int64_t> ucur(P.ucolptr.begin(), P.ucolptr.end() - 1);
  parallel_range(nchunks, [&](int64_t c) {
    for (int64_t s = och[c]; s < och[c + 1]; ++s) {
      const int32_t row0 = P.o_c1[s] - P.c1[front_of[P.o_c1[s]]];
      for (int64_t p = upd_ptr[s]; p < upd_ptr[s + 1]; ++p) {
        const int64_t u = upd_idx[p];
        P.fcu[P.fcu_ptr[fcol(s, p)]++] = UBlock{row0, P.o_np[s], ucur[u]};
        ucur[u] += P.o_np[s];
      }
    }
  }, 1);
  for (int64_t f = P.fc_total; f > 0; --f) P.fcu_ptr[f] = P.fcu_ptr[f - 1];
  P.fcu_ptr[0] = 0;
}
}  // namespace

void build_plan_merged(int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf,
                       const int64_t* parent, int64_t ns, const int64_t* sstart, const int64_t* upd_ptr,
                       const int64_t* upd_idx, Plan& P, int64_t max_pivots) {
  check_symbolic(n, qf, parent, ns, sstart, upd_ptr, upd_idx);
  const std::vector<char> marks = amalgamation_marks(n, parent, ns, sstart, upd_ptr, max_pivots);
  if (std::find(marks.begin(), marks.end(), 1) == marks.end()) {
    build_plan_core(n, colptr, rowval, qf, parent, ns, sstart, upd_ptr, upd_idx, P, true);
    set_layout(P, false);
    return;
  }
  // merged partition: a group ends at a supernode that is not merged, and
  // keeps that supernode's update set
  std::vector<int64_t> ends, ms, mup{0};
  int64_t first = 0;
  for (int64_t s = 0; s < ns; ++s) {
    if (marks[s]) continue;
    ends.push_back(s);
    ms.push_back(sstart[first]);
    mup.push_back(mup.back() + (upd_ptr[s + 1] - upd_ptr[s]));
    first = s + 1;
  }
  ms.push_back(n);
  std::vector<int64_t> mui(mup.back());
  parallel_range((int64_t)ends.size(), [&](int64_t g) {
    std::copy(upd_idx + upd_ptr[ends[g]], upd_idx + upd_ptr[ends[g] + 1], mui.begin() + mup[g]);
  }, 256);
  build_plan_core(n, colptr, rowval, qf, parent, (int64_t)ms.size() - 1, ms.data(), mup.data(), mui.data(), P,
                  false);
  attach_original(P, ns, sstart, upd_ptr, upd_idx);
  set_layout(P, false);
}

void set_layout(Plan& P, bool lean) {
  const int64_t ns = P.ns;
  P.lean = lean;
  // ---- working fronts ---------------------------------------------------------
  if (!lean) {
    int64_t fo = 0;
    for (int64_t i = 0; i < ns; ++i) {
      const int32_t s = P.slot_super[i];
      P.front_off[s] = fo;
      fo += (int64_t)P.nf[s] * P.nf[s];
    }
    P.front_elems = fo;
  } else {
    // A front lives from its own level until the end of its parent's level
    // (where the parent assembles its contribution block); roots until the
    // end of their own level.  First fit over a free list, by level.
    std::map<int64_t, int64_t> freel;   // offset -> size
    int64_t end = 0;
    std::vector<std::vector<int32_t>> dies(P.nlevels + 1);
    for (int64_t s = 0; s < ns; ++s) {
      const int32_t last = P.parent_super[s] >= 0 ? P.height[P.parent_super[s]] : P.height[s];
      dies[last + 1].push_back((int32_t)s);
    }
    auto release = [&](int64_t off, int64_t sz) {
      auto it = freel.emplace(off, sz).first;
      auto nx = std::next(it);
      if (nx != freel.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        freel.erase(nx);
      }
      if (it != freel.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
          pv->second += it->second;
          freel.erase(it);
        }
      }
    };
    for (int32_t L = 0; L < P.nlevels; ++L) {
      for (int32_t s : dies[L]) release(P.front_off[s], (int64_t)P.nf[s] * P.nf[s]);
      for (int32_t i = P.level_slot[L]; i < P.level_slot[L + 1]; ++i) {
        const int32_t s = P.slot_super[i];
        const int64_t need = (int64_t)P.nf[s] * P.nf[s];
        auto it = freel.begin();
        while (it != freel.end() && it->second < need) ++it;
        if (it == freel.end()) {
          P.front_off[s] = end;
          end += need;
        } else {
          P.front_off[s] = it->first;
          const int64_t off = it->first + need, left = it->second - need;
          freel.erase(it);
          if (left > 0) freel.emplace(off, left);
        }
      }
    }
    P.front_elems = end;
  }
  // ---- panels -------------------------------------------------------------------
  P.lpan_off.assign(ns, 0);
  P.u12_off.assign(ns, 0);
  P.panel_base = P.front_elems;
  P.panel_elems = 0;
  for (int64_t i = 0; i < ns; ++i) {
    const int32_t s = P.slot_super[i];
    const int64_t npv = P.np[s], nf = P.nf[s];
    if (!lean) {
      P.lpan_off[s] = P.front_off[s];
      P.u12_off[s] = P.front_off[s] + npv * nf;
    } else {
      P.lpan_off[s] = P.panel_base + P.panel_elems;
      P.u12_off[s] = P.lpan_off[s] + nf * npv;
      P.panel_elems += nf * npv + npv * (nf - npv);
    }
  }
  // ---- explicit pivot-block inverses (blocked triangular inversion) -------------
  P.inv_off.assign(ns, -1);
  P.inv_blocks.clear();
  P.inv_tasks.clear();
  P.inv_tasks_tc.clear();
  P.inv_steps.clear();
  P.flops_inverse = 0;
  P.inv_elems = 0;
  P.inv_scratch_elems = 0;
  P.inv_base = P.panel_base + P.panel_elems;
  for (int64_t s = 0; s < ns; ++s)
    if (P.nf[s] > kSmallFront) {
      P.inv_off[s] = P.inv_base + P.inv_elems;
      P.inv_elems += 2 * (int64_t)P.np[s] * P.np[s];
      for (int32_t j = 0; j * kPanel < P.np[s]; ++j) {
        P.inv_blocks.push_back((int32_t)s);
        P.inv_blocks.push_back(j);
      }
    }
  P.inv_scratch = P.inv_base + P.inv_elems;
  build_inverse_steps(P);
  P.pool_elems = P.inv_scratch + P.inv_scratch_elems;
  build_launches(P, false);
}

namespace {
// Algorithmic traffic of assembling front s: the zero-filled front written
// once, each child's contribution block read once and added into the parent
// (read-modify-write), and the original entries (value + 4-byte row).
void assembly_work(const Plan& P, int32_t s, Launch& l) {
  double e = (double)P.nf[s] * P.nf[s];
  for (int32_t ci = P.child_ptr[s]; ci < P.child_ptr[s + 1]; ++ci) {
    const double m = P.nu[P.child_idx[ci]];
    e += 3.0 * m * m;
  }
  l.elems += e;
  l.extra_bytes += 12.0 * P.front_nv[s];
}
// Small fronts: assembly plus the dense factorization in shared memory.
void front_work(const Plan& P, int32_t s, Launch& l) {
  assembly_work(P, s, l);
  const double a = P.np[s], u = P.nu[s];
  l.flops += 2.0 / 3.0 * a * a * a + 2.0 * a * a * u + 2.0 * a * u * u;
}
}  // namespace

// Record C -= A * B in both tilings: 64 x 64 (FP64 and SIMT FP32 kernels)
// and 128 x 128 (tensor-core FP32 kernel).
void push_gemm(Plan& P, Launch& lg, const GemmTask& g0) {
  GemmTask g = g0;
  g.tiles_m = (int32_t)ceil_div(g.m, 64);
  g.tiles_n = (int32_t)ceil_div(g.n, 64);
  g.tile_base = lg.tiles;
  lg.tiles += (int64_t)g.tiles_m * g.tiles_n;
  P.gemm_tasks.push_back(g);
  g.tiles_m = (int32_t)ceil_div(g.m, kTcTile);
  g.tiles_n = (int32_t)ceil_div(g.n, kTcTile);
  g.tile_base = lg.tiles_tc;
  lg.tiles_tc += (int64_t)g.tiles_m * g.tiles_n;
  P.gemm_tasks_tc.push_back(g);
  ++lg.count;
  lg.max_k = std::max(lg.max_k, g.k);
}

void build_launches_core(Plan& P, bool safe) {
  P.small_tasks.clear();
  P.panel_tasks.clear();
  P.trsm_tasks.clear();
  P.gemm_tasks.clear();
  P.gemm_tasks_tc.clear();
  P.plane_tasks.clear();
  P.planes_bytes = 0;
  P.launches.clear();
  P.has_speculative = false;
  std::vector<int32_t> large;
  std::vector<PanelTask> cls[4];   // pivoting panels by row class, then speculative (reused per step)
  for (int32_t L = 0; L < P.nlevels; ++L) {
    // fused small fronts
    if (P.level_large[L] > P.level_slot[L]) {
      Launch l{kLaunchSmall, L, (int64_t)P.small_tasks.size(), P.level_large[L] - P.level_slot[L], 0};
      for (int32_t i = P.level_slot[L]; i < P.level_large[L]; ++i) {
        const int32_t s = P.slot_super[i];
        P.small_tasks.push_back(s);
        front_work(P, s, l);
      }
      l.tiles = l.count;
      P.launches.push_back(l);
    }
    if (P.level_slot[L + 1] == P.level_large[L]) continue;
    large.assign(P.slot_super.begin() + P.level_large[L], P.slot_super.begin() + P.level_slot[L + 1]);
    const int64_t fc0 = P.colbase[large.front()];
    const int64_t fc1 = P.colbase[large.back()] + P.nf[large.back()];
    {
      Launch la{kLaunchAssemble, L, fc0, fc1 - fc0, fc1 - fc0};
      for (int32_t s : large) assembly_work(P, s, la);
      P.launches.push_back(la);
    }
    int32_t maxnp = 0;
    for (int32_t s : large) maxnp = std::max(maxnp, P.np[s]);
    // Blocked right-looking LU of each pivot block: 64-column panels grouped
    // into blocks of kUpdateBlock columns.  Inside a block the updates stay
    // on the block's own columns (K = 64); the rows of the next panel get the
    // block's earlier panels applied to the columns right of the block just
    // before their triangular solve (K <= kUpdateBlock - 64); the rest of the
    // pivot block and the U12 rows receive the whole block at once
    // (K = kUpdateBlock) when its last panel is done.
    std::vector<GemmTask> g_left, g_step;
    for (int32_t k0 = 0; k0 < maxnp; k0 += kPanel) {
      Launch lt{kLaunchTrsm, L, (int64_t)P.trsm_tasks.size(), 0, 0};
      // panel tasks of this step, one launch per row class (64 / 128 / 256)
      for (auto& c : cls) c.clear();
      g_left.clear();
      g_step.clear();
      for (int32_t s : large) {
        const int32_t npv = P.np[s], nf = P.nf[s];
        if (npv <= k0) continue;
        const int32_t kb = std::min(kPanel, npv - k0), k1 = k0 + kb;
        const int32_t b0 = k0 - k0 % kUpdateBlock, b1 = std::min(b0 + kUpdateBlock, npv);
        // Speculative panels everywhere; the pivoting variants only run in
        // the safe rerun after a speculative panel met a larger candidate.
        // pivot rows of the panel's columns: up to the end of the last
        // column's segment (npv unless fronts are merged)
        const int32_t seg = P.seg_end[P.c1[s] + k1 - 1];
        int32_t mode = !safe ? kPanelSpeculative : (seg - k0 <= kPivRowsSmem ? kPanelSmemPivot : kPanelGlobalPivot);
        if (mode == kPanelSpeculative) P.has_speculative = true;
        const int32_t R = (mode == kPanelSpeculative) ? kb : seg - k0;
        const int c = mode == kPanelSpeculative ? 3 : ((mode == kPanelGlobalPivot || R > 128) ? 2 : (R > 64 ? 1 : 0));
        cls[c].push_back(PanelTask{s, k0, mode, 0});
        TrsmTask tt{};
        tt.s = s;
        tt.k0 = k0;
        tt.r0 = (mode == kPanelSpeculative) ? k1 : seg;
        tt.lrow_tiles = (int32_t)ceil_div(nf - tt.r0, 64);
        tt.ucol_tiles = (int32_t)ceil_div(nf - k1, 64);
        tt.check = (mode == kPanelSpeculative) ? 1 : 0;
        if (tt.lrow_tiles + tt.ucol_tiles > 0) {
          lt.flops += 2.0 * ((double)(nf - tt.r0) * kb * kb + (double)(nf - k1) * kb * kb);
          lt.elems += 2.0 * ((double)(nf - tt.r0) * kb + (double)(nf - k1) * kb) + 2.0 * 64 * 64;
          tt.tile_base = lt.tiles;
          lt.tiles += tt.lrow_tiles + tt.ucol_tiles;
          P.trsm_tasks.push_back(tt);
          ++lt.count;
        }
        const int64_t base = P.front_off[s];
        // C(r, c) -= A(r, kk) * B(kk, c) on front entries (row, column)
        auto upd = [&](std::vector<GemmTask>& into, int32_t r, int32_t cc, int32_t kk, int32_t m, int32_t n,
                       int32_t k) {
          if (m <= 0 || n <= 0 || k <= 0) return;
          GemmTask g{};
          g.a = base + r + (int64_t)kk * nf;
          g.b = base + kk + (int64_t)cc * nf;
          g.c = base + r + (int64_t)cc * nf;
          g.m = m; g.n = n; g.k = k;
          g.lda = g.ldb = g.ldc = nf;
          into.push_back(g);
        };
        // the rows of this panel, right of the block: the block's earlier
        // panels (after this panel's interchanges, so its own launch in the
        // pivoting rerun; speculative panels do not interchange, so the
        // previous step's update launch carries it)
        if (safe && k0 > b0) upd(g_left, k0, b1, b0, kb, nf - b1, k0 - b0);
        // this panel on the block's remaining columns, every row below
        upd(g_step, k1, k1, k0, nf - k1, b1 - k1, kb);
        if (!safe && k1 < b1) {
          const int32_t kbn = std::min(kPanel, npv - k1);
          upd(g_step, k1, b1, b0, kbn, nf - b1, k1 - b0);   // the next panel's rows, right of the block
        }
        if (k1 == b1) {   // block done: the rest of the pivot block and the U12 rows
          upd(g_step, b1, b1, b0, nf - b1, npv - b1, b1 - b0);
          upd(g_step, b1, npv, b0, npv - b1, nf - npv, b1 - b0);
        }
      }
      auto emit_gemms = [&](const std::vector<GemmTask>& tasks) {
        if (tasks.empty()) return;
        Launch lg{kLaunchGemm, L, (int64_t)P.gemm_tasks.size(), 0, 0};
        for (const GemmTask& g : tasks) {
          lg.flops += 2.0 * g.m * g.n * g.k;
          lg.elems += 2.0 * g.m * g.n + (double)g.m * g.k + (double)g.k * g.n;
          push_gemm(P, lg, g);
        }
        P.launches.push_back(lg);
      };
      for (int c = 0; c < 4; ++c) {
        if (cls[c].empty()) continue;
        Launch lp{kLaunchPanel, L, (int64_t)P.panel_tasks.size(), (int64_t)cls[c].size(), (int64_t)cls[c].size()};
        lp.rows = c < 3 ? 64 << c : 0;   // 0: speculative kernel
        for (const PanelTask& pt : cls[c]) {
          const int32_t kb = std::min(kPanel, P.np[pt.s] - pt.k0);
          const double R = (pt.mode == kPanelSpeculative) ? kb : (P.seg_end[P.c1[pt.s] + pt.k0 + kb - 1] - pt.k0);
          lp.flops += 2.0 * (R * kb * kb - (double)kb * kb * kb / 3.0) + 4.0 / 3.0 * kb * kb * kb;
          lp.elems += 2.0 * R * kb + 2.0 * 64 * 64;
          P.panel_tasks.push_back(pt);
        }
        P.launches.push_back(lp);
      }
      emit_gemms(g_left);
      if (lt.count) P.launches.push_back(lt);
      emit_gemms(g_step);
    }
    // deferred Schur update of every large front: F22 -= L21 * U12
    Launch lg{kLaunchGemm, L, (int64_t)P.gemm_tasks.size(), 0, 0};
    for (int32_t s : large) {
      const int32_t npv = P.np[s], nu = P.nu[s], nf = P.nf[s];
      if (nu == 0) continue;
      const int64_t base = P.front_off[s];
      GemmTask g{};
      g.a = base + npv;
      g.b = base + (int64_t)npv * nf;
      g.c = base + npv + (int64_t)npv * nf;
      g.m = nu; g.n = nu; g.k = npv;
      g.lda = g.ldb = g.ldc = nf;
      lg.flops += 2.0 * nu * nu * npv;
      lg.elems += 2.0 * nu * nu + 2.0 * nu * npv;
      push_gemm(P, lg, g);
    }
    if (lg.count) P.launches.push_back(lg);
  }
  // every GEMM launch's operand tiles as bf16 parts (the tensor-core form
  // that splits its operands once; the planes buffer is reused launch by
  // launch, the launches run in order on one stream)
  P.plane_tasks.assign(P.gemm_tasks_tc.size(), PlaneTask{});
  for (Launch& L : P.launches) {
    if (L.kind != kLaunchGemm) continue;
    int64_t off = 0, units = 0;
    for (int64_t i = L.first; i < L.first + L.count; ++i) {
      const GemmTask& g = P.gemm_tasks_tc[i];
      PlaneTask pt{};
      pt.kt = (int32_t)ceil_div(g.k, 64);
      pt.a_off = off;
      off += (int64_t)g.tiles_m * pt.kt * 3 * kPlaneTileBytes;
      pt.b_off = off;
      off += (int64_t)g.tiles_n * pt.kt * 3 * kPlaneTileBytes;
      pt.unit_base = units;
      units += (int64_t)(g.tiles_m + g.tiles_n) * pt.kt;
      P.plane_tasks[i] = pt;
    }
    L.split_units = units;
    L.planes_bytes = off;
    P.planes_bytes = std::max(P.planes_bytes, off);
  }
}

void add_copy_launches(Plan& P);

void build_launches(Plan& P, bool safe) {
  build_launches_core(P, safe);
  add_copy_launches(P);
}

// Lean layout: after each level, its fronts' panels go to the panel pool.
void add_copy_launches(Plan& P) {
  if (!P.lean) return;
  std::vector<Launch> out;
  int32_t cur = -1;
  auto flush = [&](int32_t L) {
    const int32_t a = P.level_slot[L], e = P.level_slot[L + 1];
    if (e <= a) return;
    const int64_t fc0 = P.colbase[P.slot_super[a]];
    const int64_t fc1 = P.colbase[P.slot_super[e - 1]] + P.nf[P.slot_super[e - 1]];
    Launch c{kLaunchCopyPanels, L, fc0, fc1 - fc0, fc1 - fc0};
    for (int32_t i = a; i < e; ++i) {
      const int32_t s = P.slot_super[i];
      c.elems += 2.0 * ((double)P.nf[s] * P.np[s] + (double)P.np[s] * P.nu[s]);
    }
    out.push_back(c);
  };
  for (const Launch& l : P.launches) {
    if (cur >= 0 && l.level != cur) flush(cur);
    cur = l.level;
    out.push_back(l);
  }
  if (cur >= 0) flush(cur);
  P.launches.swap(out);
}

}  // namespace mfgpu
