// mfgpu.cu -- C ABI of libmfgpu's GPU numeric factorization and solves.
//
// One context per handle: a plan (pattern analysis), its device copy, the
// front pool and the factors resident in HBM, one CUDA stream.  The numeric
// factorization replaces the hot loop of src/multifrontal.jl:198-357 and the
// solves replace src/interface.jl:123-177 / src/solve.jl:10-79; see the
// kernel headers for the step-by-step correspondence.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/mfgpu.h"
#include "device/factor_kernels.cuh"
#include "device/gemm_kernels.cuh"
#include "device/tc_gemm.cuh"
#include "device/solve_kernels.cuh"
#include "device/solve_persistent.cuh"
#include "host/symbolic.h"
#include "plan.h"

using namespace mfgpu;

struct mfgpu_symbolic {
  mfgpu::SymbolicMF s;
};

namespace {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const char* what) : std::runtime_error(what), code(c) {}
};

#define CK(x)                                                                                     \
  do {                                                                                            \
    cudaError_t e_ = (x);                                                                         \
    if (e_ != cudaSuccess)                                                                        \
      throw CudaError(e_, (std::string(#x) + ": " + cudaGetErrorString(e_)).c_str());            \
  } while (0)

// Grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  void ensure(size_t need) {
    if (need <= bytes) return;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    if (need == 0) return;
    cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw CudaError(e, ("device allocation of " + std::to_string(need) + " bytes failed").c_str());
    }
    bytes = need;
  }
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
};

template <typename T>
void upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
  b.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
  if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

inline unsigned grid1(int64_t work, int per) { return (unsigned)((work + per - 1) / per); }

enum KernelClass {
  KC_BUILD_VALUES, KC_SMALL, KC_ASSEMBLE, KC_PANEL, KC_TRSM, KC_GEMM_FACTOR, KC_PIVOTS, KC_SCATTER,
  KC_FWD_SMALL, KC_FWD_ASSEMBLE, KC_GEMM_SOLVE, KC_BWD_SMALL, KC_BWD_GATHER,
  KC_SOLVE_FINISH, KC_RESIDUAL, KC_INVERSE, KC_COPY_PANELS, KC_FWD_THIN, KC_COUNT
};
const char* const kKernelClassName[KC_COUNT] = {
    "build_values", "small_fronts", "assemble_columns", "panel", "panel_trsm", "gemm_factor", "finalize_pivots",
    "scatter_csc", "fwd_small", "fwd_assemble", "gemm_solve", "bwd_small", "bwd_gather",
    "solve_finish", "residual", "gemm_inverse", "copy_panels", "fwd_thin"};

struct KStat {
  double ms = 0, flops = 0, bytes = 0;
  int64_t launches = 0;
};

struct SolveSchedule {
  int64_t nrhs = -1;
  struct Step {
    int kind;        // 0 fwd_small, 1 fwd_assemble, 3 gemm (A: pool; B, C, D: solve arena), 4 bwd_small,
                     // 5 bwd_gather, 6 fwd_tiny, 7 bwd_tiny (nf <= kTinyFront, one warp per supernode),
                     // 8 fwd_thin (thin large supernodes; step launches only),
                     // 10 fwd_leaf (leaves with nf <= kLeafFront; step launches only)
    int64_t first, count, tiles;
    double flops = 0, elems = 0;
    int64_t tiles_tc = 0;   // GEMM steps: grid in 128 x 128 tensor-core tiles (gemms_tc)
    int64_t sk_first = 0, sk_count = 0, sk_parts = 0, sk_reds = 0;   // split-K form (few rhs)
    int32_t level = -1;     // tree level (small-supernode steps run beside the level's large ones)
    int32_t max_k = 0;      // GEMM steps: largest K of their tasks
    int64_t rt_first = 0, rt_count = 0;   // assemble / gather steps: their row tasks
    // GEMM steps with few tiles and a long K: the K-chunked form (tasks in
    // sgemms / sgemms_tc, then the reductions sreds[rd_first ..])
    int64_t sp_first = 0, sp_count = 0, sp_tiles = 0, sp_tiles_tc = 0;
    int32_t sp_max_k = 0;
    int64_t rd_first = 0, rd_count = 0, rd_elems = 0;
    // GEMM steps whose tasks have few rows: the same tasks in BM x 128 tiles
    int64_t sm_first = 0, sm_count = 0, sm_tiles = 0;
    int32_t sm_bm = 0;
  };
  std::vector<Step> steps;
  std::vector<int32_t> ids;
  std::vector<GemmTask> gemms, gemms_tc;   // 64 x 64 tiles; 128 x 128 tiles (FP32 on tensor cores)
  std::vector<SkinnyTask> skinny;          // split-K form of every GEMM step when nrhs <= kSkinnyMaxN
  int64_t skinny_scratch = 0;              // partial sums, elements
  std::vector<SolvePhase> phases;   // the steps as work-item phases of the persistent solve
  // one-launch-per-step solve only: row tasks of the assemble / gather
  // steps, the forward pull map, the K-chunked GEMM steps
  std::vector<RowTask> rows;
  std::vector<int64_t> aptr;
  std::vector<int2> asrc;
  std::vector<GemmTask> sgemms, sgemms_tc;
  std::vector<SplitRed> sreds;
  std::vector<GemmTask> gemms_sm;
  int64_t split_scratch = 0;        // partial products, elements (after x in the solve arena)
  int elem = 0;                     // front element size the K chunks were chosen for
  bool thin = false;                // thin supernodes have their own steps (not in the persistent solve)
  DevBuf d_ids, d_gemms, d_gemms_tc, d_phases, d_skinny, d_rows, d_aptr, d_asrc, d_sgemms, d_sgemms_tc, d_sreds,
      d_gemms_sm;
};

}  // namespace

// Run body(i) for i in [0, n) on up to 16 host threads (contiguous ranges).
template <typename F>
void parallel_for(int64_t n, F&& body) {
  const int64_t nt = std::min<int64_t>(n, std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
  if (nt <= 1) {
    for (int64_t i = 0; i < n; ++i) body(i);
    return;
  }
  std::vector<std::thread> pool;
  for (int64_t t = 0; t < nt; ++t)
    pool.emplace_back([&, t] {
      for (int64_t i = n * t / nt; i < n * (t + 1) / nt; ++i) body(i);
    });
  for (auto& th : pool) th.join();
}

// Page-locked host staging buffer (grows, never shrinks).
struct PinnedBuf {
  void* p = nullptr;
  size_t cap = 0;
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  PinnedBuf& operator=(PinnedBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      cap = o.cap;
      o.p = nullptr;
      o.cap = 0;
    }
    return *this;
  }
  void ensure(size_t bytes) {
    if (bytes <= cap) return;
    release();
    CK(cudaHostAlloc(&p, std::max<size_t>(bytes, 64), cudaHostAllocDefault));
    cap = std::max<size_t>(bytes, 64);
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
  double* d() const { return static_cast<double*>(p); }
  ~PinnedBuf() { release(); }
};

struct mfgpu_ctx {
  int device = 0;
  int precision = MFGPU_PRECISION_FP64;
  cudaStream_t own_stream = nullptr;
  cudaStream_t side_stream = nullptr;     // a level's small supernodes, beside its large ones
  cudaStream_t copy_stream = nullptr;     // right-hand sides in flight during a factorization
  cudaEvent_t ev_copy = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaStream_t stream = nullptr;
  std::string err;
  bool analyzed = false, factored = false, csc_ready = false;
  Plan plan;
  DevPlan dp{};
  // plan arrays
  DevBuf b_c1, b_np, b_nu, b_nf, b_upd_off, b_front_off, b_colbase, b_child_ptr, b_child_idx, b_upd, b_rel, b_uoff,
      b_v_src, b_v_srow, b_v_frow, b_fc_super, b_fc_vbeg, b_fc_vend, b_fc_ch_ptr, b_fc_ch, b_lcolptr, b_ucolptr, b_qf,
      b_csr_ptr, b_csr_col, b_csr_src;
  DevBuf b_small, b_panel, b_trsm, b_gemm, b_gemm_tc, b_plane_tasks;
  DevBuf b_planes;   // bf16 parts of one level's Schur-update operand tiles (FP32 fronts)
  bool use_tc = true;      // FP32 fronts: GEMMs on tensor cores
  uint64_t wait_ns = kTcWaitNs;   // bound on every device-side wait (mbarriers, grid barriers)
  bool tc_bf16x3 = true;   // tensor-core split: BF16x3 (FP32 accuracy) or 3xTF32
  bool launches_safe = false;
  // numeric state
  DevBuf b_pool, b_vx, b_ax, b_rs, b_ipiv, b_info, b_prow, b_rowfac, b_flags, b_dinv, b_dinv_off;
  DevBuf b_inv_off, b_inv_blocks, b_inv_tasks, b_inv_tasks_tc;   // pivot-block inversion
  DevBuf b_lpan_off, b_u12_off;                                   // factored panels
  DevBuf b_seg_end, b_col_orig, b_o_c1, b_o_np, b_o_upd_off, b_o_upd, b_o_xpos, b_fcu_ptr, b_fcu;   // merged fronts
  DevBuf b_skinny;                                                // split-K partial sums
  bool have_rs = false;
  int factor_precision = MFGPU_PRECISION_FP64;
  DevBuf b_li, b_lx, b_ui, b_ux;
  // solve state
  SolveSchedule sched;
  DevBuf b_fsol, b_b, b_x, b_r, b_d, b_err, b_norm;   // b_fsol: solve arena (blocks, then x)
  DevBuf b_f32;                                       // Float32 right-hand sides / solutions in transit
  // persistent solve: one cooperative launch per pass instead of one launch
  // per step, when the options ask for it (slower than per-step launches on
  // every measured case, many or few right-hand sides)
  int persistent_mode = 0;     // 0 default (per step), 1 persistent, 2 per step
  int lean_mode = 0;           // front layout: 0 by size, 1 always lean
  bool merge_fronts = true;    // factor supernode chains as merged fronts (factor structure unchanged)
  int num_sms = 148;           // SMs of the device (split-K chunk choice)
  bool f32_values = false;     // the last factorization is of a Float32 matrix (mfgpu_factor_f32)
  bool c64_values = false;     // the values given are ComplexF64 (mfgpu_factor_c64)
  bool c64_factors = false;    // the last completed factorization has ComplexF64 fronts
  bool persistent = false;     // the mode resolved for the current solve
  int persist_grid[2] = {0, 0};          // CTAs of the persistent kernel, FP32 / FP64
  DevBuf b_bar, b_stamps;                // barrier words {count, gen, err, sticky err}; profiling stamps
  struct PhaseProfile {                  // one profiled persistent launch
    size_t stamp0;
    int nphases;
    int elem_bytes;
  };
  std::vector<PhaseProfile> pending_phases;
  size_t stamp_next = 0;
  // stats
  double t_analyze_ms = 0, t_factor_ms = 0, t_solve_ms = 0, t_csc_ms = 0;
  int factor_reruns = 0;
  double growth = 0.0, growth_limit = 1e4;   // mixed form: element growth and the FP64 refactor limit
  bool refactored_fp64 = false;
  int32_t last_status = 0;
  std::vector<int32_t> last_info;   // per supernode: first zero pivot (block position) or INT32_MAX
  // batched systems analyzed as one block-diagonal matrix
  struct Batch {
    int64_t nsys = 0;
    std::vector<int64_t> off, nz_off;      // column and value offsets of every system (nsys + 1)
    std::vector<int64_t> colptr, rowval;   // the block-diagonal pattern, 1-based
    std::vector<int32_t> super_sys;        // system of every front
    PinnedBuf nz, b, x;                    // pinned host staging of the concatenated arrays
    bool have_factors = false;             // global factors fetched for per-system slicing
    std::vector<int64_t> lcolptr, lrowval, ucolptr, urowval, p, q;
    std::vector<double> lnzval, unzval;
  } batch;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // per-kernel-class profile (CUDA events around each launch when enabled)
  bool profiling = false;
  int64_t launch_count = 0;
  KStat kstat[KC_COUNT];
  struct Pending {
    int kc;
    cudaEvent_t a, b;
    double flops, bytes;
    int32_t level;
    int64_t tasks;
    int32_t tune;
  };
  std::vector<Pending> pending;
  struct Record {   // one profiled launch
    int kc;
    int32_t level;
    int64_t tasks;
    float ms;
    double flops, bytes;
    int32_t tune;     // index among the tunable GEMM launches, -1 otherwise
  };
  // autotuner: kernel variant of every tunable GEMM launch (factor GEMMs,
  // inversion GEMMs, solve GEMMs for the current right-hand-side count, in
  // issue order): 0 = built-in rule, 1 = tcgen05 3xTF32, 2 = CUDA-core FP32.
  std::vector<int8_t> gemm_choice;
  int64_t choice_version = 0;
  int32_t cur_tune = -1;      // tunable id of the launch being issued
  std::vector<Record> records;
  std::vector<cudaEvent_t> evpool;
  size_t evnext = 0;
  // CUDA graphs of the static launch sequences (keyed by everything a replay
  // bakes in: sizes, flags and buffer addresses)
  bool use_graphs = true;
  bool solve_graphs = true;   // false once a capture of the persistent solve failed
  std::vector<uintptr_t> factor_key, solve_key;
  cudaGraphExec_t factor_exec = nullptr, solve_exec = nullptr;
  int64_t factor_nodes = 0, solve_nodes = 0;   // kernel launches inside each graph
  int64_t graph_replays = 0, graph_captures = 0;
};

namespace {

constexpr int kTuneFeatures = 11;

int fail(mfgpu_ctx* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

template <typename F>
int guarded(mfgpu_ctx* h, F&& body) {
  try {
    return body();
  } catch (const CudaError& e) {
    return fail(h, e.code == cudaErrorMemoryAllocation ? MFGPU_ERR_NOMEM : MFGPU_ERR_CUDA, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(h, MFGPU_ERR_ARGUMENT, e.what());
  } catch (const std::exception& e) {
    return fail(h, MFGPU_ERR_INTERNAL, e.what());
  }
}

void upload_plan(mfgpu_ctx* h) {
  const Plan& P = h->plan;
  cudaStream_t st = h->stream;
  upload(h->b_c1, P.c1, st);
  upload(h->b_np, P.np, st);
  upload(h->b_nu, P.nu, st);
  upload(h->b_nf, P.nf, st);
  upload(h->b_upd_off, P.upd_off, st);
  upload(h->b_front_off, P.front_off, st);
  upload(h->b_colbase, P.colbase, st);
  upload(h->b_child_ptr, P.child_ptr, st);
  upload(h->b_child_idx, P.child_idx, st);
  upload(h->b_upd, P.upd, st);
  upload(h->b_rel, P.rel, st);
  upload(h->b_uoff, P.uoff, st);
  upload(h->b_v_src, P.v_src, st);
  upload(h->b_v_srow, P.v_srow, st);
  upload(h->b_v_frow, P.v_frow, st);
  upload(h->b_fc_super, P.fc_super, st);
  upload(h->b_fc_vbeg, P.fc_vbeg, st);
  upload(h->b_fc_vend, P.fc_vend, st);
  upload(h->b_fc_ch_ptr, P.fc_ch_ptr, st);
  upload(h->b_fc_ch, P.fc_ch, st);
  upload(h->b_lcolptr, P.lcolptr, st);
  upload(h->b_ucolptr, P.ucolptr, st);
  upload(h->b_qf, P.qf, st);
  upload(h->b_csr_ptr, P.csr_ptr, st);
  upload(h->b_csr_col, P.csr_col, st);
  upload(h->b_csr_src, P.csr_src, st);
  upload(h->b_dinv_off, P.dinv_off, st);
  upload(h->b_inv_off, P.inv_off, st);
  upload(h->b_lpan_off, P.lpan_off, st);
  upload(h->b_u12_off, P.u12_off, st);
  upload(h->b_inv_blocks, P.inv_blocks, st);
  upload(h->b_inv_tasks, P.inv_tasks, st);
  upload(h->b_inv_tasks_tc, P.inv_tasks_tc, st);
  upload(h->b_seg_end, P.seg_end, st);
  upload(h->b_col_orig, P.col_orig, st);
  upload(h->b_o_c1, P.o_c1, st);
  upload(h->b_o_np, P.o_np, st);
  upload(h->b_o_upd_off, P.o_upd_off, st);
  upload(h->b_o_upd, P.o_upd, st);
  upload(h->b_o_xpos, P.o_xpos, st);
  upload(h->b_fcu_ptr, P.fcu_ptr, st);
  upload(h->b_fcu, P.fcu, st);
  DevPlan& d = h->dp;
  d.n = P.n;
  d.ns = P.ns;
  d.c1 = h->b_c1.as<int32_t>();
  d.np = h->b_np.as<int32_t>();
  d.nu = h->b_nu.as<int32_t>();
  d.nf = h->b_nf.as<int32_t>();
  d.upd_off = h->b_upd_off.as<int64_t>();
  d.front_off = h->b_front_off.as<int64_t>();
  d.colbase = h->b_colbase.as<int64_t>();
  d.child_ptr = h->b_child_ptr.as<int32_t>();
  d.child_idx = h->b_child_idx.as<int32_t>();
  d.upd = h->b_upd.as<int32_t>();
  d.rel = h->b_rel.as<int32_t>();
  d.uoff = h->b_uoff.as<int64_t>();
  d.v_src = h->b_v_src.as<int32_t>();
  d.v_srow = h->b_v_srow.as<int32_t>();
  d.v_frow = h->b_v_frow.as<int32_t>();
  d.fc_super = h->b_fc_super.as<int32_t>();
  d.fc_vbeg = h->b_fc_vbeg.as<int32_t>();
  d.fc_vend = h->b_fc_vend.as<int32_t>();
  d.fc_ch_ptr = h->b_fc_ch_ptr.as<int32_t>();
  d.fc_ch = h->b_fc_ch.as<int32_t>();
  d.lcolptr = h->b_lcolptr.as<int64_t>();
  d.ucolptr = h->b_ucolptr.as<int64_t>();
  d.qf = h->b_qf.as<int32_t>();
  d.csr_ptr = h->b_csr_ptr.as<int32_t>();
  d.csr_col = h->b_csr_col.as<int32_t>();
  d.csr_src = h->b_csr_src.as<int32_t>();
  d.dinv_off = h->b_dinv_off.as<int64_t>();
  d.inv_off = h->b_inv_off.as<int64_t>();
  d.lpan_off = h->b_lpan_off.as<int64_t>();
  d.u12_off = h->b_u12_off.as<int64_t>();
  d.lean = P.lean ? 1 : 0;
  d.merged = P.merged ? 1 : 0;
  d.seg_end = h->b_seg_end.as<int32_t>();
  d.col_orig = h->b_col_orig.as<int32_t>();
  d.o_c1 = h->b_o_c1.as<int32_t>();
  d.o_np = h->b_o_np.as<int32_t>();
  d.o_upd_off = h->b_o_upd_off.as<int64_t>();
  d.o_upd = h->b_o_upd.as<int32_t>();
  d.o_xpos = h->b_o_xpos.as<int32_t>();
  d.fcu_ptr = h->b_fcu_ptr.as<int64_t>();
  d.fcu = h->b_fcu.as<UBlock>();
}

void upload_launches(mfgpu_ctx* h) {
  const Plan& P = h->plan;
  upload(h->b_small, P.small_tasks, h->stream);
  upload(h->b_panel, P.panel_tasks, h->stream);
  upload(h->b_trsm, P.trsm_tasks, h->stream);
  upload(h->b_gemm, P.gemm_tasks, h->stream);
  upload(h->b_gemm_tc, P.gemm_tasks_tc, h->stream);
  upload(h->b_plane_tasks, P.plane_tasks, h->stream);
}

DevState dev_state(mfgpu_ctx* h) {
  DevState s;
  s.ipiv = h->b_ipiv.as<int32_t>();
  s.info = h->b_info.as<int32_t>();
  s.prow = h->b_prow.as<int32_t>();
  s.rowfac = h->b_rowfac.as<int32_t>();
  s.flags = h->b_flags.as<int32_t>();
  return s;
}

cudaEvent_t next_event(mfgpu_ctx* h) {
  if (h->evnext == h->evpool.size()) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    h->evpool.push_back(e);
  }
  return h->evpool[h->evnext++];
}

// Every kernel launch of the library goes through here: it counts launches
// and, when profiling is on, brackets the launch with CUDA events on the
// launching stream and books its algorithmic work to its kernel class.
template <typename F>
void klaunch(mfgpu_ctx* h, int kc, double flops, double bytes, F&& f, int32_t level = -1, int64_t tasks = 0) {
  ++h->launch_count;
  if (!h->profiling) {
    f();
    return;
  }
  cudaEvent_t a = next_event(h), b = next_event(h);
  CK(cudaEventRecord(a, h->stream));
  f();
  CK(cudaEventRecord(b, h->stream));
  h->pending.push_back({kc, a, b, flops, bytes, level, tasks, h->cur_tune});
}

void prof_flush(mfgpu_ctx* h);

// Kernel class of a solve step / persistent phase kind.
int phase_class(int kind) {
  static const int kc[8] = {KC_FWD_SMALL, KC_FWD_ASSEMBLE, KC_FWD_SMALL, KC_GEMM_SOLVE, KC_BWD_SMALL,
                            KC_BWD_GATHER, KC_FWD_SMALL, KC_BWD_SMALL};
  return kc[kind];
}

void prof_book(mfgpu_ctx* h, int kc, float ms, double flops, double bytes, int32_t level, int64_t tasks) {
  KStat& k = h->kstat[kc];
  k.ms += ms;
  k.flops += flops;
  k.bytes += bytes;
  ++k.launches;
  if (h->records.size() < 200000) h->records.push_back({kc, level, tasks, ms, flops, bytes, -1});
}

void prof_flush(mfgpu_ctx* h) {
  if (!h->pending_phases.empty()) {
    // persistent solves: phase p ran between stamps p and p + 1 (block 0, after each grid barrier)
    std::vector<unsigned long long> stamps(h->stamp_next);
    CK(cudaMemcpy(stamps.data(), h->b_stamps.p, h->stamp_next * 8, cudaMemcpyDeviceToHost));
    const auto& S = h->sched;
    for (const auto& pp : h->pending_phases)
      for (int p = 0; p < pp.nphases && p < (int)S.steps.size(); ++p) {
        const auto& st = S.steps[p];
        const float ms = (float)((double)(stamps[pp.stamp0 + p + 1] - stamps[pp.stamp0 + p]) * 1e-6);
        const bool work = st.kind != kPhFwdAssemble && st.kind != kPhBwdGather;
        prof_book(h, phase_class(st.kind), ms, work ? st.flops : 0.0, work ? st.elems * pp.elem_bytes : 0.0, -2,
                  S.phases[p].items);
      }
    h->pending_phases.clear();
    h->stamp_next = 0;
  }
  for (auto& p : h->pending) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, p.a, p.b));
    KStat& k = h->kstat[p.kc];
    k.ms += ms;
    k.flops += p.flops;
    k.bytes += p.bytes;
    ++k.launches;
    if (h->records.size() < 200000) h->records.push_back({p.kc, p.level, p.tasks, ms, p.flops, p.bytes, p.tune});
  }
  h->pending.clear();
  h->evnext = 0;
}

template <typename T>
size_t panel_smem_bytes(int rows) {
  return ((size_t)rows * kPanel + 4 * 64 + rows) * sizeof(T);
}

template <typename T>
size_t spec_smem_bytes() {
  return (size_t)3 * 64 * kLdS * sizeof(T);
}

template <typename T>
size_t apply_smem_bytes() {
  return (size_t)64 * (kLdP + kLdQ) * sizeof(T);
}

template <typename T>
void configure_kernels() {
  static bool done = false;
  if (done) return;
  if constexpr (is_complex_v<T>) {   // complex fronts: no speculative, register-tiled or tensor-core kernels
    CK(cudaFuncSetAttribute(k_small_fronts<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(kSmallFront * kSmallFront * sizeof(T))));
    CK(cudaFuncSetAttribute(k_panel_apply<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)apply_smem_bytes<T>()));
    done = true;
    return;
  } else {
  CK(cudaFuncSetAttribute(k_panel_spec<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)spec_smem_bytes<T>()));
  CK(cudaFuncSetAttribute(k_panel<T, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)panel_smem_bytes<T>(64)));
  CK(cudaFuncSetAttribute(k_panel<T, 128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)panel_smem_bytes<T>(128)));
  CK(cudaFuncSetAttribute(k_panel<T, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)panel_smem_bytes<T>(256)));
  CK(cudaFuncSetAttribute(k_panel_apply<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)apply_smem_bytes<T>()));
  CK(cudaFuncSetAttribute(k_gemm_tc<128, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)TcCfg<128, 3>::kSmem));
  CK(cudaFuncSetAttribute(k_gemm_bx3<128, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)BxCfg<128, 2>::kSmem));
  CK(cudaFuncSetAttribute(k_gemm_bx3<128, 1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)BxCfg<128, 1, 1>::kSmem));
  CK(cudaFuncSetAttribute(k_gemm_bx3p<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)BxCfg<128, 2>::kSmem));
  CK(cudaFuncSetAttribute(k_solve_persistent<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)persistent_smem_bytes<T>()));
  done = true;
  }
}

// dst[i] = (To)src[i] (Float32 right-hand sides in, Float32 solutions out).
template <typename Ti, typename To>
__global__ void k_convert(int64_t n, const Ti* __restrict__ src, To* __restrict__ dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (To)src[i];
}

__global__ void k_fill_i32(int32_t* p, int64_t n, int32_t v) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

template <typename T>
void launch_gemm(const GemmTask* tasks, int64_t count, int64_t tiles, const T* pa, const T* pb, T* pc,
                 cudaStream_t st);
template <>
void launch_gemm<double>(const GemmTask* tasks, int64_t count, int64_t tiles, const double* pa, const double* pb,
                         double* pc, cudaStream_t st) {
  k_gemm_f64<<<(unsigned)tiles, kGemmThreads, 0, st>>>(tasks, (int)count, pa, pb, pc);
}
template <>
void launch_gemm<float>(const GemmTask* tasks, int64_t count, int64_t tiles, const float* pa, const float* pb,
                        float* pc, cudaStream_t st) {
  k_gemm_f32<<<(unsigned)tiles, 256, 0, st>>>(tasks, (int)count, pa, pb, pc);
}

template <>
void launch_gemm<zc>(const GemmTask* tasks, int64_t count, int64_t tiles, const zc* pa, const zc* pb, zc* pc,
                     cudaStream_t st) {
  k_gemm_z<<<(unsigned)tiles, kGemmThreads, 0, st>>>(tasks, (int)count, pa, pb, pc);
}

// Built-in rule for a batched FP32 GEMM launch: the tcgen05 kernel (one CTA
// of 288 threads per SM, 128 x 128 tiles) when its mean work per tile is at
// least that of a full tile over K = 64; launches of many small tasks (a few
// rows in each tile) run on the CUDA-core kernel, which keeps several CTAs
// per SM.
bool tc_worthwhile(double flops, int64_t tiles_tc) {
  return tiles_tc > 0 && flops >= 2.0 * kTcTile * kTcTile * 64.0 * (double)tiles_tc;
}

// A factor GEMM launch (FP32 fronts) takes the split-once form when its
// tiles walk K of at least kSplitPlanesMinK on average: a tile's epilogue
// and set-up are then small beside its K loop, and the split is shared by
// the tiles of a row (column).  Shorter K stays on k_gemm_bx3.
constexpr double kSplitPlanesMinK = 128;
bool split_worthwhile(const Launch& L) {
  return L.tiles_tc > 0 && L.flops >= 2.0 * kTcTile * kTcTile * kSplitPlanesMinK * (double)L.tiles_tc;
}

// Kernel variant of tunable GEMM launch `id` with FP32 operands: the
// autotuner's choice when it made one, else the built-in rule `dflt`.
bool gemm_use_tc(const mfgpu_ctx* h, int64_t id, bool dflt) {
  if (!h->use_tc) return false;
  if (id >= 0 && id < (int64_t)h->gemm_choice.size() && h->gemm_choice[id]) return h->gemm_choice[id] == 1;
  return dflt;
}

// One tensor-core GEMM launch over 128 x 128-tiled tasks: BF16x3 (default)
// or 3xTF32 (MFGPU_FLAG_TF32_SPLIT); BF16x3 launches whose tasks all have
// K <= 64 (max_k) take the one-stage, one-accumulator form, two CTAs per SM.
void launch_tc(const mfgpu_ctx* h, const GemmTask* tasks, int64_t count, int64_t tiles, const float* pa,
               const float* pb, float* pc, cudaStream_t st, int32_t max_k) {
  if (h->tc_bf16x3 && max_k <= BxCfg<128, 1, 1>::BK)
    k_gemm_bx3<128, 1, 1><<<(unsigned)tiles, BxCfg<128, 1, 1>::kThreads, BxCfg<128, 1, 1>::kSmem, st>>>(
        tasks, (int)count, pa, pb, pc, h->b_flags.as<int>(), h->wait_ns);
  else if (h->tc_bf16x3)
    k_gemm_bx3<128, 2><<<(unsigned)tiles, BxCfg<128, 2>::kThreads, BxCfg<128, 2>::kSmem, st>>>(tasks, (int)count, pa, pb, pc,
                                                                                  h->b_flags.as<int>(), h->wait_ns);
  else
    k_gemm_tc<128, 3><<<(unsigned)tiles, kTcThreads, TcCfg<128, 3>::kSmem, st>>>(tasks, (int)count, pa, pb, pc,
                                                                                h->b_flags.as<int>(), h->wait_ns);
}

// Tunable-launch ids: factor GEMM launches first, then the inversion steps,
// then the solve GEMM steps.
int64_t tune_factor_count(const Plan& P) {
  int64_t c = 0;
  for (const Launch& L : P.launches) c += L.kind == kLaunchGemm;
  return c;
}

// The small and the large supernodes of one tree level touch disjoint
// fronts and read only lower levels (factor, forward solve) or higher ones
// (backward solve), so a level's small-supernode launch runs on a second
// stream beside the level's large-supernode launches; the two streams join
// at every level change (and in a CUDA graph this is a fork / join of
// branches).  Off when profiling, whose per-launch events sit on one stream.
struct LevelFork {
  mfgpu_ctx* h;
  bool on;
  int level = -1;
  bool open = false;
  LevelFork(mfgpu_ctx* hh) : h(hh), on(!hh->profiling && hh->side_stream) {}
  void at(int L) {
    if (L != level) {
      join();
      level = L;
    }
  }
  cudaStream_t side() {   // the stream for this level's small supernodes
    if (!on) return h->stream;
    if (!open) {
      CK(cudaEventRecord(h->ev_fork, h->stream));
      CK(cudaStreamWaitEvent(h->side_stream, h->ev_fork, 0));
      open = true;
    }
    return h->side_stream;
  }
  void join() {
    if (!open) return;
    CK(cudaEventRecord(h->ev_join, h->side_stream));
    CK(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
    open = false;
  }
};

template <typename T>
void run_factor_launches(mfgpu_ctx* h) {
  const Plan& P = h->plan;
  cudaStream_t st = h->stream;
  T* pool = h->b_pool.as<T>();
  const Wide<T>* vx = h->b_vx.as<Wide<T>>();
  DevState S = dev_state(h);
  int64_t tune_id = 0;
  LevelFork fork(h);
  for (const Launch& L : P.launches) {
    const double bytes = L.elems * sizeof(T) + L.extra_bytes;
    fork.at(L.level);
    switch (L.kind) {
      case kLaunchSmall: {
        cudaStream_t ss = fork.side();
        klaunch(h, KC_SMALL, L.flops, bytes, [&] {
          k_small_fronts<T><<<(unsigned)L.count, kSmallThreads, kSmallFront * kSmallFront * sizeof(T), ss>>>(
              h->dp, S, h->b_small.as<int32_t>() + L.first, pool, vx);
        }, L.level, L.count);
        break;
      }
      case kLaunchAssemble:
        klaunch(h, KC_ASSEMBLE, 0, bytes, [&] {
          k_assemble_columns<T><<<grid1(L.count, 8), 256, 0, st>>>(h->dp, L.first, L.count, pool, vx);
        }, L.level, L.count);
        break;
      case kLaunchPanel:
        klaunch(h, KC_PANEL, L.flops, bytes, [&] {
          const PanelTask* pt = h->b_panel.as<PanelTask>() + L.first;
          T* dinv = h->b_dinv.as<T>();
          if constexpr (is_complex_v<T>)
            k_panel_global<T><<<(unsigned)L.count, kPanelThreads, 0, st>>>(h->dp, S, pt, pool, dinv);
          else if (L.rows == 0)
            k_panel_spec<T><<<(unsigned)L.count, kSpecThreads, spec_smem_bytes<T>(), st>>>(h->dp, S, pt, pool, dinv);
          else if (L.rows <= 64)
            k_panel<T, 64><<<(unsigned)L.count, 64, panel_smem_bytes<T>(64), st>>>(h->dp, S, pt, pool, dinv);
          else if (L.rows <= 128)
            k_panel<T, 128><<<(unsigned)L.count, 128, panel_smem_bytes<T>(128), st>>>(h->dp, S, pt, pool, dinv);
          else
            k_panel<T, 256><<<(unsigned)L.count, 256, panel_smem_bytes<T>(256), st>>>(h->dp, S, pt, pool, dinv);
        }, L.level * 1000 + L.rows, L.count);
        break;
      case kLaunchTrsm:
        klaunch(h, KC_TRSM, L.flops, bytes, [&] {
          k_panel_apply<T><<<(unsigned)L.tiles, kApplyThreads, apply_smem_bytes<T>(), st>>>(
              h->dp, S, h->b_trsm.as<TrsmTask>() + L.first, (int)L.count, pool, h->b_dinv.as<T>());
        }, L.level, L.tiles);
        break;
      case kLaunchCopyPanels:
        fork.join();   // the level's panels, small fronts' included
        klaunch(h, KC_COPY_PANELS, 0, bytes, [&] {
          k_copy_panels<T><<<grid1(L.count, 8), 256, 0, st>>>(h->dp, L.first, L.count, pool);
        }, L.level, L.count);
        break;
      case kLaunchGemm:
        h->cur_tune = (int32_t)tune_id;
        if (sizeof(T) == 4 && h->tc_bf16x3 && h->b_planes.p && split_worthwhile(L) &&
            gemm_use_tc(h, tune_id, tc_worthwhile(L.flops, L.tiles_tc)))
          // long-K updates: operand tiles split once, then moved by bulk copies
          klaunch(h, KC_GEMM_FACTOR, L.flops, bytes, [&] {
            const GemmTask* tk = h->b_gemm_tc.as<GemmTask>() + L.first;
            const PlaneTask* pk = h->b_plane_tasks.as<PlaneTask>() + L.first;
            uint8_t* planes = h->b_planes.as<uint8_t>();
            k_split_planes<<<(unsigned)L.split_units, 256, 0, st>>>(tk, pk, (int)L.count, (const float*)pool,
                                                                    (const float*)pool, planes);
            k_gemm_bx3p<2><<<(unsigned)L.tiles_tc, kBxpThreads, BxCfg<128, 2>::kSmem, st>>>(
                tk, pk, (int)L.count, planes, (float*)pool, h->b_flags.as<int>(), h->wait_ns);
          }, L.level, L.tiles_tc);
        else if (sizeof(T) == 4 && gemm_use_tc(h, tune_id, tc_worthwhile(L.flops, L.tiles_tc)))
          klaunch(h, KC_GEMM_FACTOR, L.flops, bytes, [&] {
            launch_tc(h, h->b_gemm_tc.as<GemmTask>() + L.first, L.count, L.tiles_tc, (const float*)pool,
                      (const float*)pool, (float*)pool, st, L.max_k);
          }, L.level, L.tiles_tc);
        else
          klaunch(h, KC_GEMM_FACTOR, L.flops, bytes, [&] {
            launch_gemm<T>(h->b_gemm.as<GemmTask>() + L.first, L.count, L.tiles, pool, pool, pool, st);
          }, L.level, L.tiles);
        h->cur_tune = -1;
        ++tune_id;
        break;
    }
  }
  fork.join();
  CK(cudaGetLastError());
}

// Run `issue` on the handle's stream: replayed from a CUDA graph when the
// key matches the cached one, captured first otherwise; eager when profiling
// (per-launch events) or when graphs are disabled.
template <typename F>
void run_sequence(mfgpu_ctx* h, std::vector<uintptr_t>& cached_key, cudaGraphExec_t& exec, int64_t& nodes,
                  const std::vector<uintptr_t>& key, F&& issue) {
  if (h->profiling || !h->use_graphs) {
    issue();
    return;
  }
  if (!exec || cached_key != key) {
    const int64_t before = h->launch_count;
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    try {
      issue();
    } catch (...) {
      cudaStreamEndCapture(h->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CK(cudaStreamEndCapture(h->stream, &g));
    cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    CK(e);
    cached_key = key;
    nodes = h->launch_count - before;
    h->launch_count = before;
    ++h->graph_captures;
  }
  CK(cudaGraphLaunch(exec, h->stream));
  h->launch_count += nodes;   // the kernels of the replayed graph
  ++h->graph_replays;
}

// Explicit inverses of the large pivot blocks for the solves: clear, copy
// the inverted 64 x 64 diagonal blocks, then the merge levels (plan.cpp:
// build_inverse_steps), each a batched GEMM launch.
template <typename T>
void issue_inverses(mfgpu_ctx* h) {
  const Plan& P = h->plan;
  cudaStream_t st = h->stream;
  if (!P.inv_elems) return;
  T* pool = h->b_pool.as<T>();
  CK(cudaMemsetAsync(pool + P.inv_base, 0, P.inv_elems * sizeof(T), st));
  const int64_t nblk = (int64_t)P.inv_blocks.size() / 2;
  klaunch(h, KC_INVERSE, 0, (double)nblk * 2 * 64 * 64 * sizeof(T) * 2, [&] {
    k_inv_init<T><<<(unsigned)nblk, 256, 0, st>>>(h->dp, h->b_inv_blocks.as<int32_t>(), h->b_dinv.as<T>(), pool);
  });
  int64_t tune_id = tune_factor_count(P) - 1;
  for (const InvStep& is : P.inv_steps) {
    ++tune_id;
    if (!is.count) continue;
    h->cur_tune = (int32_t)tune_id;
    if (sizeof(T) == 4 && gemm_use_tc(h, tune_id, tc_worthwhile(is.flops, is.tiles_tc)))
      klaunch(h, KC_INVERSE, is.flops, is.elems * sizeof(T), [&] {
        launch_tc(h, h->b_inv_tasks_tc.as<GemmTask>() + is.first, is.count, is.tiles_tc, (const float*)pool,
                  (const float*)pool, (float*)pool, st, is.max_k);
      }, -3, is.tiles_tc);
    else
      klaunch(h, KC_INVERSE, is.flops, is.elems * sizeof(T), [&] {
        launch_gemm<T>(h->b_inv_tasks.as<GemmTask>() + is.first, is.count, is.tiles, pool, pool, pool, st);
      }, -3, is.tiles);
    h->cur_tune = -1;
  }
}

template <typename T>
void issue_factor(mfgpu_ctx* h) {
  const Plan& P = h->plan;
  cudaStream_t st = h->stream;
  klaunch(h, KC_BUILD_VALUES, P.nnz_a, 32.0 * P.nnz_a, [&] {
    if constexpr (is_complex_v<T>)
      k_build_values_z<<<grid1(P.nnz_a, 256), 256, 0, st>>>(P.nnz_a, h->b_v_src.as<int32_t>(),
                                                              h->b_v_srow.as<int32_t>(), h->b_ax.as<zc>(),
                                                              h->have_rs ? h->b_rs.as<double>() : nullptr,
                                                              h->b_vx.as<zc>());
    else
      k_build_values<<<grid1(P.nnz_a, 256), 256, 0, st>>>(P.nnz_a, h->b_v_src.as<int32_t>(),
                                                            h->b_v_srow.as<int32_t>(), h->b_ax.as<double>(),
                                                            h->have_rs ? h->b_rs.as<double>() : nullptr,
                                                            h->b_vx.as<double>());
  });
  if (P.ns) k_fill_i32<<<grid1(P.ns, 256), 256, 0, st>>>(h->b_info.as<int32_t>(), P.ns, INT32_MAX);
  CK(cudaMemsetAsync(h->b_flags.p, 0, 8, st));   // flags[2] is the test hook's stall request
  run_factor_launches<T>(h);
  issue_inverses<T>(h);
  if (P.ns)
    klaunch(h, KC_PIVOTS, 0, 16.0 * P.n, [&] { k_finalize_pivots<<<grid1(P.ns * 32, 128), 128, 0, st>>>(h->dp, dev_state(h)); });
  if (P.fc_total)
    klaunch(h, KC_SCATTER, 0, (double)(P.nnz_l + P.nnz_u) * (8.0 + sizeof(Wide<T>) + sizeof(T)), [&] {
      if (P.merged)
        k_scatter_csc_merged<T><<<grid1(P.fc_total, 8), 256, 0, st>>>(
            h->dp, dev_state(h), h->b_pool.as<T>(), P.fc_total, h->b_li.as<int64_t>(), h->b_lx.as<Wide<T>>(),
            h->b_ui.as<int64_t>(), h->b_ux.as<Wide<T>>());
      else
        k_scatter_csc<T><<<grid1(P.fc_total, 8), 256, 0, st>>>(h->dp, dev_state(h), h->b_pool.as<T>(), P.fc_total,
                                                               h->b_li.as<int64_t>(), h->b_lx.as<Wide<T>>(),
                                                               h->b_ui.as<int64_t>(), h->b_ux.as<Wide<T>>());
    });
  CK(cudaGetLastError());
}

template <typename T>
int factor_impl(mfgpu_ctx* h, int32_t check) {
  Plan& P = h->plan;
  cudaStream_t st = h->stream;
  h->factored = h->csc_ready = false;   // until this factorization completes
  configure_kernels<T>();
  h->b_pool.ensure(std::max<size_t>(P.pool_elems * sizeof(T), 16));
  h->b_ipiv.ensure(std::max<int64_t>(P.n, 1) * 4);
  h->b_prow.ensure(std::max<int64_t>(P.n, 1) * 4);
  h->b_rowfac.ensure(std::max<int64_t>(P.n, 1) * 4);
  h->b_info.ensure(std::max<int64_t>(P.ns, 1) * 4);
  if (!h->b_flags.p) {
    h->b_flags.ensure(16);
    CK(cudaMemsetAsync(h->b_flags.p, 0, 16, st));
  }
  h->b_vx.ensure(std::max<int64_t>(P.nnz_a, 1) * sizeof(Wide<T>));
  h->b_dinv.ensure(std::max<size_t>((size_t)P.dinv_blocks * kDinvElems * sizeof(T), 16));
  h->b_li.ensure(std::max<int64_t>(P.nnz_l, 1) * 8);
  h->b_lx.ensure(std::max<int64_t>(P.nnz_l, 1) * sizeof(Wide<T>));
  h->b_ui.ensure(std::max<int64_t>(P.nnz_u, 1) * 8);
  h->b_ux.ensure(std::max<int64_t>(P.nnz_u, 1) * sizeof(Wide<T>));
  if constexpr (is_complex_v<T>) {
    // complex fronts factor every panel with partial pivoting (no speculative
    // panels): the plan's pivoting launch list
    if (!h->launches_safe) {
      build_launches(P, true);
      upload_launches(h);
      h->launches_safe = true;
    }
  }
  CK(cudaEventRecord(h->ev0, st));
  for (int attempt = 0; attempt < 2; ++attempt) {
    // the planes buffer of the long-K updates' split operands (FP32 fronts;
    // the pivoting launch list may need a different size)
    if constexpr (std::is_same_v<T, float>)
      if (P.planes_bytes > 0 && h->use_tc && h->tc_bf16x3) h->b_planes.ensure((size_t)P.planes_bytes);
    const std::vector<uintptr_t> key = {
        sizeof(T), (uintptr_t)h->launches_safe, (uintptr_t)h->have_rs, (uintptr_t)h->b_pool.p, (uintptr_t)h->b_vx.p,
        (uintptr_t)h->b_ax.p, (uintptr_t)h->b_rs.p, (uintptr_t)h->b_dinv.p, (uintptr_t)h->b_li.p,
        (uintptr_t)h->b_lx.p, (uintptr_t)h->b_ui.p, (uintptr_t)h->b_ux.p, (uintptr_t)h->b_small.p,
        (uintptr_t)h->b_panel.p, (uintptr_t)h->b_trsm.p, (uintptr_t)h->b_gemm.p, (uintptr_t)h->b_ipiv.p,
        (uintptr_t)h->b_gemm_tc.p, (uintptr_t)h->use_tc, (uintptr_t)h->tc_bf16x3, (uintptr_t)h->choice_version,
        (uintptr_t)h->wait_ns, (uintptr_t)h->b_planes.p, (uintptr_t)h->b_plane_tasks.p,
        (uintptr_t)h->b_info.p, (uintptr_t)h->b_flags.p, (uintptr_t)st};
    run_sequence(h, h->factor_key, h->factor_exec, h->factor_nodes, key, [&] { issue_factor<T>(h); });
    if (!P.has_speculative) break;
    int32_t flag[2] = {0, 0};
    CK(cudaMemcpyAsync(flag, h->b_flags.p, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (!flag[0] || flag[1]) break;   // no pivoting needed, or a bounded wait ran out (reported below)
    // a speculative panel met a row that partial pivoting would have chosen:
    // redo the factorization with pivoting panels everywhere.
    prof_flush(h);
    build_launches(P, true);
    upload_launches(h);
    h->launches_safe = true;
    ++h->factor_reruns;
  }
  CK(cudaEventRecord(h->ev1, st));
  // status: first supernode (postorder) with a zero pivot
  std::vector<int32_t> info(P.ns);
  int32_t flags[2] = {0, 0};
  if (P.ns) CK(cudaMemcpyAsync(info.data(), h->b_info.p, P.ns * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(flags, h->b_flags.p, 8, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (flags[1]) {
    prof_flush(h);
    h->factored = false;
    return fail(h, MFGPU_ERR_TIMEOUT, "a tensor-core GEMM gave up a bounded wait; the factorization is incomplete");
  }
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
  h->t_factor_ms = ms;
  prof_flush(h);
  h->factored = true;
  h->csc_ready = true;
  h->factor_precision = (sizeof(T) == 4) ? MFGPU_PRECISION_MIXED : MFGPU_PRECISION_FP64;
  h->c64_factors = is_complex_v<T>;
  int32_t status = 0;
  if (check)
    for (int64_t s = 0; s < P.ns; ++s)
      if (info[s] != INT32_MAX) {
        status = P.c1[s] + info[s] + 1;
        break;
      }
  h->last_status = status;
  h->last_info = std::move(info);
  h->batch.have_factors = false;
  return status;
}

// Element growth max|U| / max|Rs .* A| of the last factorization (FP64 on
// the GPU over the CSC values of U and the scaled values of V = A[qf, qf]).
double element_growth(mfgpu_ctx* h) {
  const Plan& P = h->plan;
  cudaStream_t st = h->stream;
  h->b_norm.ensure(16);
  unsigned long long* m = h->b_norm.as<unsigned long long>();
  CK(cudaMemsetAsync(m, 0, 16, st));
  k_abs_max<<<4 * 148, 256, 0, st>>>(h->b_ux.as<double>(), P.nnz_u, m);
  k_abs_max<<<4 * 148, 256, 0, st>>>(h->b_vx.as<double>(), P.nnz_a, m + 1);
  CK(cudaGetLastError());
  unsigned long long bits[2];
  CK(cudaMemcpyAsync(bits, m, 16, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  double u, a;
  std::memcpy(&u, &bits[0], 8);
  std::memcpy(&a, &bits[1], 8);
  return a > 0 ? u / a : 0.0;
}

// The mixed form factors in FP32, then checks the element growth: when it
// exceeds the limit (FP32 rounding amplified by the growth would keep the FP64
// refinement from converging), the matrix is refactored in FP64 and the
// solves use the FP64 factors.
int factor_dispatch(mfgpu_ctx* h, int32_t check) {
  h->refactored_fp64 = false;
  h->growth = 0.0;
  if (h->plan.n == 0) {   // a 0 x 0 matrix: empty factors, nothing to launch
    h->factored = h->csc_ready = true;
    h->c64_factors = h->c64_values;
    h->factor_precision = !h->c64_values && (h->f32_values || h->precision == MFGPU_PRECISION_MIXED)
                              ? MFGPU_PRECISION_MIXED : MFGPU_PRECISION_FP64;
    h->last_status = 0;
    h->last_info.clear();
    h->t_factor_ms = 0;
    return MFGPU_OK;
  }
  if (h->c64_values) return factor_impl<zc>(h, check);     // ComplexF64 matrix: complex FP64 fronts
  if (h->f32_values) return factor_impl<float>(h, check);   // Float32 matrix: FP32 factors, no refactor
  if (h->precision != MFGPU_PRECISION_MIXED) return factor_impl<double>(h, check);
  const int rc = factor_impl<float>(h, check);
  if (rc != MFGPU_OK) return rc;
  h->growth = element_growth(h);
  if (!(h->growth <= h->growth_limit)) {
    const double g = h->growth;
    const int rc64 = factor_impl<double>(h, check);
    h->growth = g;
    h->refactored_fp64 = true;
    return rc64;
  }
  return rc;
}

// ---- solves ---------------------------------------------------------------
// Product steps of the one-launch-per-step solve with fewer output tiles
// than SMs and a K of at least kSplitMinK run K-chunked: chunks of at least
// kSplitMinKC (a multiple of 64), as many as give about two tiles per SM.
constexpr int32_t kSplitMinK = 384;
constexpr int32_t kSplitMinKC = 128;

void build_solve_schedule(mfgpu_ctx* h, int64_t R, int elem) {
  SolveSchedule& S = h->sched;
  const bool thin = !h->persistent;
  if (S.nrhs == R && S.elem == elem && S.thin == thin) return;
  const Plan& P = h->plan;
  S = SolveSchedule{};
  S.nrhs = R;
  S.elem = elem;
  S.thin = thin;
  auto is_thin = [&](int32_t s) { return thin && P.np[s] <= kThinNp && P.nu[s] <= kThinNu; };
  auto ceil_div = [](int64_t a, int64_t b) { return (a + b - 1) / b; };
  // offsets: A operands in the front pool (fronts and pivot-block inverses);
  // B, C and D in the solve arena: the per-supernode blocks (nf x R each,
  // at colbase * R), then x in factor order (n x R) at xw0
  const int64_t xw0 = P.fc_total * R;
  const int n = (int)P.n;
  auto add_gemm = [&](SolveSchedule::Step& st, int32_t mode, int64_t a, int lda, int64_t b, int ldb, int64_t c,
                      int ldc, int m, int nn, int k, int64_t d = 0, int ldd = 0) {
    if (m <= 0 || nn <= 0 || k < 0 || (k == 0 && mode == kGemmSub)) return;
    GemmTask g{};
    g.a = a; g.b = b; g.c = c; g.d = d;
    g.m = m; g.n = nn; g.k = k;
    g.lda = lda; g.ldb = ldb; g.ldc = ldc; g.ldd = ldd;
    g.mode = mode;
    g.tiles_m = (int)ceil_div(m, 64);
    g.tiles_n = (int)ceil_div(nn, 64);
    g.tile_base = st.tiles;
    st.tiles += (int64_t)g.tiles_m * g.tiles_n;
    S.gemms.push_back(g);
    g.tiles_m = (int)ceil_div(m, kTcTile);
    g.tiles_n = (int)ceil_div(nn, kTcTile);
    g.tile_base = st.tiles_tc;
    st.tiles_tc += (int64_t)g.tiles_m * g.tiles_n;
    S.gemms_tc.push_back(g);
    ++st.count;
    st.max_k = std::max(st.max_k, k);
    st.flops += 2.0 * m * nn * k;
    st.elems += (double)m * nn * (mode == kGemmSet ? 1 : 2) + (double)m * k + (double)k * nn;
  };
  int32_t cur_level = -1;   // level of the steps being built
  auto gemm_step = [&]() {
    SolveSchedule::Step st{3, (int64_t)S.gemms.size(), 0, 0};
    st.level = cur_level;
    return st;
  };
  auto push = [&](const SolveSchedule::Step& st) {
    if (st.count) S.steps.push_back(st);
  };
  // small-supernode kernels: L or U panel read once, the rhs block read and written
  auto small_work = [&](SolveSchedule::Step& st, int32_t s) {
    const double a = P.np[s], u = P.nu[s];
    st.flops += (a * a + 2.0 * a * u) * R;
    st.elems += (a * a / 2 + a * u) + 2.0 * (a + u) * R;
  };
  // the small supernodes of slots [a, m): the tiny ones (one warp each) and
  // the rest (one CTA each), as two independent steps
  // class of a small supernode: 0 leaf (forward only: no children, nf <=
  // kLeafFront; step launches only), 1 tiny, 2 the rest
  auto small_class = [&](int32_t s, bool fwd) {
    if (fwd && thin && P.child_ptr[s + 1] == P.child_ptr[s] && P.nf[s] <= kLeafFront) return 0;
    return P.nf[s] <= kTinyFront ? 1 : 2;
  };
  auto small_steps = [&](int32_t a, int32_t m, int tiny_kind, int small_kind, int32_t level) {
    const bool fwd = tiny_kind == 6;
    for (int pass = fwd ? 0 : 1; pass < 3; ++pass) {
      const int kind = pass == 0 ? 10 : (pass == 1 ? tiny_kind : small_kind);
      SolveSchedule::Step st{kind, (int64_t)S.ids.size(), 0, 0};
      st.level = level;
      for (int32_t i = a; i < m; ++i) {
        const int32_t s = P.slot_super[i];
        if (small_class(s, fwd) != pass) continue;
        S.ids.push_back(s);
        small_work(st, s);
        ++st.count;
      }
      if (st.count) S.steps.push_back(st);
    }
  };
  // the thin large supernodes of slots [m, e): one CTA per (supernode,
  // kThinCols right-hand sides), forward (kind 8)
  auto thin_step = [&](int32_t m, int32_t e, int kind, int32_t level) {
    SolveSchedule::Step st{kind, (int64_t)S.ids.size(), 0, 0};
    st.level = level;
    for (int32_t i = m; i < e; ++i) {
      const int32_t s = P.slot_super[i];
      if (!is_thin(s)) continue;
      S.ids.push_back(s);
      const double a = P.np[s], u = P.nu[s];
      st.flops += 2.0 * (a * a + a * u) * R;
      st.elems += a * a + a * u + 2.0 * (a + u) * R;
      ++st.count;
    }
    if (st.count) S.steps.push_back(st);
  };
  // forward, leaves to root
  for (int32_t L = 0; L < P.nlevels; ++L) {
    const int32_t a = P.level_slot[L], m = P.level_large[L], e = P.level_slot[L + 1];
    cur_level = L;
    if (m > a) small_steps(a, m, 6, 0, L);
    if (e > m) {
      const int64_t first = (int64_t)S.ids.size();
      for (int32_t i = m; i < e; ++i) S.ids.push_back(P.slot_super[i]);
      S.steps.push_back({1, first, e - m, 0});
      S.steps.back().level = L;
      thin_step(m, e, 8, L);
      // y = inv(L11) f[0:np], into x's rows c1.. ; then w = f[np:] - L21 y
      SolveSchedule::Step gy = gemm_step();
      for (int32_t i = m; i < e; ++i) {
        const int32_t s = P.slot_super[i];
        if (is_thin(s)) continue;
        const int nf = P.nf[s], np = P.np[s];
        add_gemm(gy, kGemmSet, P.inv_off[s], np, P.colbase[s] * R, nf, xw0 + P.c1[s], n, np, (int)R, np);
      }
      push(gy);
      SolveSchedule::Step gw = gemm_step();
      for (int32_t i = m; i < e; ++i) {
        const int32_t s = P.slot_super[i];
        if (is_thin(s)) continue;
        const int nf = P.nf[s], np = P.np[s];
        add_gemm(gw, kGemmSub, P.lpan_off[s] + np, nf, xw0 + P.c1[s], n, P.colbase[s] * R + np, nf, P.nu[s],
                 (int)R, np);
      }
      push(gw);
    }
  }
  // backward, root to leaves
  for (int32_t L = P.nlevels - 1; L >= 0; --L) {
    const int32_t a = P.level_slot[L], m = P.level_large[L], e = P.level_slot[L + 1];
    cur_level = L;
    // the level's small supernodes read x of higher levels only: independent
    // of the level's large ones
    if (m > a) small_steps(a, m, 7, 4, L);
    if (e > m) {
      const int64_t first = (int64_t)S.ids.size();
      for (int32_t i = m; i < e; ++i) S.ids.push_back(P.slot_super[i]);
      S.steps.push_back({5, first, e - m, 0});
      S.steps.back().level = L;
      // g = y - U12 x[upd] into f[0:np]; then x = inv(U11) g into x's rows c1..
      SolveSchedule::Step gg = gemm_step();
      for (int32_t i = m; i < e; ++i) {
        const int32_t s = P.slot_super[i];
        const int nf = P.nf[s], np = P.np[s];
        add_gemm(gg, kGemmFrom, P.u12_off[s], u12_ld(P, s), P.colbase[s] * R + np, nf, P.colbase[s] * R, nf, np,
                 (int)R, P.nu[s], xw0 + P.c1[s], n);
      }
      push(gg);
      SolveSchedule::Step gx = gemm_step();
      for (int32_t i = m; i < e; ++i) {
        const int32_t s = P.slot_super[i];
        const int nf = P.nf[s], np = P.np[s];
        add_gemm(gx, kGemmSet, P.inv_off[s] + (int64_t)np * np, np, P.colbase[s] * R, nf, xw0 + P.c1[s], n, np,
                 (int)R, np);
      }
      push(gx);
    }

  }
  // split-K form of the GEMM steps for few right-hand sides
  constexpr int32_t kSkinnyMinK = 512;
  if (R <= kSkinnyMaxN) {
    const int nmax = R <= 1 ? 1 : (R <= 4 ? 4 : kSkinnyMaxN);
    for (auto& st : S.steps) {
      if (st.kind != 3) continue;
      // split-K pays only when some task walks a long K
      int32_t maxk = 0;
      for (int64_t i = st.first; i < st.first + st.count; ++i) maxk = std::max(maxk, S.gemms[i].k);
      if (maxk < kSkinnyMinK) continue;
      // the widest K chunk that still gives two CTAs per SM (down to 32)
      int32_t kc = kSkinnyKC;
      auto parts = [&](int32_t w) {
        int64_t c = 0;
        for (int64_t i = st.first; i < st.first + st.count; ++i)
          c += ceil_div(S.gemms[i].m, kSkinnyRows) * std::max<int64_t>(1, ceil_div(S.gemms[i].k, w));
        return c;
      };
      while (kc > 32 && parts(kc) < 2 * (int64_t)h->num_sms) kc /= 2;
      st.sk_first = (int64_t)S.skinny.size();
      for (int64_t i = st.first; i < st.first + st.count; ++i) {
        const GemmTask& g = S.gemms[i];
        SkinnyTask t{};
        t.a = g.a; t.b = g.b; t.c = g.c; t.d = g.d;
        t.m = g.m; t.n = g.n; t.k = g.k; t.lda = g.lda; t.ldb = g.ldb; t.ldc = g.ldc; t.ldd = g.ldd; t.mode = g.mode;
        t.rblocks = (int32_t)ceil_div(g.m, kSkinnyRows);
        t.kc = kc;
        t.kchunks = (int32_t)std::max<int64_t>(1, ceil_div(g.k, kc));
        t.part_base = st.sk_parts;
        t.red_base = st.sk_reds;
        st.sk_parts += (int64_t)t.rblocks * t.kchunks;
        st.sk_reds += t.rblocks;
        S.skinny.push_back(t);
      }
      st.sk_count = (int64_t)S.skinny.size() - st.sk_first;
      S.skinny_scratch = std::max<int64_t>(S.skinny_scratch, st.sk_parts * kSkinnyRows * nmax);
    }
  }
  // row tasks of the assemble / gather steps, and the forward pull map: for
  // each V-row position v of a large front, the (child, update row) pairs
  // that the extend-add adds at v, children in LIFO order
  for (auto& st : S.steps) {
    if (st.kind != 1 && st.kind != 5) continue;
    st.rt_first = (int64_t)S.rows.size();
    for (int64_t i = st.first; i < st.first + st.count; ++i) {
      const int32_t s = S.ids[i];
      const int nf = P.nf[s];
      int64_t pbase = 0;
      if (st.kind == 1) {
        pbase = (int64_t)S.aptr.size();
        std::vector<int64_t> pos(nf + 1, 0);
        for (int32_t ci = P.child_ptr[s]; ci < P.child_ptr[s + 1]; ++ci) {
          const int32_t k = P.child_idx[ci];
          for (int32_t r = 0; r < P.nu[k]; ++r) ++pos[P.rel[P.upd_off[k] + r] + 1];
        }
        const int64_t e0 = (int64_t)S.asrc.size();
        for (int v = 0; v < nf; ++v) {
          pos[v + 1] += pos[v];
          S.aptr.push_back(e0 + pos[v]);
        }
        S.asrc.resize(e0 + pos[nf]);
        for (int32_t ci = P.child_ptr[s + 1] - 1; ci >= P.child_ptr[s]; --ci) {
          const int32_t k = P.child_idx[ci];
          for (int32_t r = 0; r < P.nu[k]; ++r) S.asrc[e0 + pos[P.rel[P.upd_off[k] + r]]++] = make_int2(k, r);
          st.elems += (double)P.nu[k] * R;
        }
        st.elems += ((double)nf + P.np[s]) * R;
      } else {
        st.elems += 2.0 * P.nu[s] * R;
      }
      const int rows = st.kind == 1 ? nf : P.nu[s];
      for (int r0 = 0; r0 < rows; r0 += kAsmRows) S.rows.push_back({s, r0, pbase});
    }
    st.rt_count = (int64_t)S.rows.size() - st.rt_first;
  }
  S.aptr.push_back((int64_t)S.asrc.size());
  // K-chunked form of the product steps with few tiles (many right-hand
  // sides; the split-K form above serves few): tiles counted in the tiling
  // the element type runs on (128 x 128 for FP32 fronts, else 64 x 64)
  if (R > kSkinnyMaxN) {
    const int64_t scratch_base = xw0 + P.n * R;
    for (auto& st : S.steps) {
      if (st.kind != 3 || st.max_k < kSplitMinK) continue;
      const int64_t tiles = elem == 4 ? st.tiles_tc : st.tiles;
      if (tiles >= h->num_sms) continue;
      const int64_t parts = ceil_div(2 * (int64_t)h->num_sms, std::max<int64_t>(1, tiles));
      const int32_t kc = std::max<int32_t>(kSplitMinKC, (int32_t)(ceil_div(ceil_div(st.max_k, parts), 64) * 64));
      if (kc >= st.max_k) continue;
      st.sp_first = (int64_t)S.sgemms.size();
      st.rd_first = (int64_t)S.sreds.size();
      int64_t scratch = 0;
      auto push_tiled = [&](GemmTask t) {
        t.tiles_m = (int)ceil_div(t.m, 64);
        t.tiles_n = (int)ceil_div(t.n, 64);
        t.tile_base = st.sp_tiles;
        st.sp_tiles += (int64_t)t.tiles_m * t.tiles_n;
        S.sgemms.push_back(t);
        t.tiles_m = (int)ceil_div(t.m, kTcTile);
        t.tiles_n = (int)ceil_div(t.n, kTcTile);
        t.tile_base = st.sp_tiles_tc;
        st.sp_tiles_tc += (int64_t)t.tiles_m * t.tiles_n;
        S.sgemms_tc.push_back(t);
        st.sp_max_k = std::max(st.sp_max_k, t.k);
      };
      for (int64_t i = st.first; i < st.first + st.count; ++i) {
        const GemmTask g = S.gemms[i];
        const int32_t nch = (int32_t)std::max<int64_t>(1, ceil_div(g.k, kc));
        const int64_t mn = (int64_t)g.m * g.n;
        for (int32_t q = 0; q < nch; ++q) {
          GemmTask t = g;
          const int32_t k0 = q * kc;
          t.k = std::min(kc, g.k - k0);
          t.a = g.a + (int64_t)k0 * g.lda;
          t.b = g.b + k0;
          if (q > 0) {   // a plain product into the scratch area
            t.mode = kGemmSet;
            t.c = scratch_base + scratch + (q - 1) * mn;
            t.ldc = g.m;
            t.d = 0;
            t.ldd = 0;
          }
          push_tiled(t);
        }
        if (nch > 1) {
          SplitRed rd{};
          rd.c = g.c;
          rd.p = scratch_base + scratch;
          rd.m = g.m;
          rd.n = g.n;
          rd.ldc = g.ldc;
          rd.parts = nch - 1;
          rd.sign = g.mode == kGemmSet ? 1 : -1;
          rd.elem_base = st.rd_elems;
          st.rd_elems += mn;
          S.sreds.push_back(rd);
          scratch += (nch - 1) * mn;
        }
      }
      st.sp_count = (int64_t)S.sgemms.size() - st.sp_first;
      st.rd_count = (int64_t)S.sreds.size() - st.rd_first;
      S.split_scratch = std::max(S.split_scratch, scratch);
    }
  }
  // few-row products (M = a pivot count, low in the tree): BM x 128 tiles
  // when they waste at most half the work of 64 x 64 tiles on idle rows
  if (R > kSkinnyMaxN) {
    for (auto& st : S.steps) {
      if (st.kind != 3 || st.sp_count) continue;
      int32_t maxm = 0;
      for (int64_t i = st.first; i < st.first + st.count; ++i) maxm = std::max(maxm, S.gemms[i].m);
      const int bm = maxm <= 16 ? 16 : 32;
      double w64 = 0, wsm = 0;
      for (int64_t i = st.first; i < st.first + st.count; ++i) {
        const GemmTask& g = S.gemms[i];
        w64 += (double)ceil_div(g.m, 64) * 64 * ceil_div(g.n, 64) * 64 * g.k;
        wsm += (double)ceil_div(g.m, bm) * bm * ceil_div(g.n, kSkinnyMBN) * kSkinnyMBN * g.k;
      }
      if (!(wsm <= 0.5 * w64)) continue;
      st.sm_bm = bm;
      st.sm_first = (int64_t)S.gemms_sm.size();
      for (int64_t i = st.first; i < st.first + st.count; ++i) {
        GemmTask t = S.gemms[i];
        t.tiles_m = (int)ceil_div(t.m, bm);
        t.tiles_n = (int)ceil_div(t.n, kSkinnyMBN);
        t.tile_base = st.sm_tiles;
        st.sm_tiles += (int64_t)t.tiles_m * t.tiles_n;
        S.gemms_sm.push_back(t);
      }
      st.sm_count = st.count;
    }
  }
  // the same steps as phases of the persistent kernel (kSolveThreads per CTA:
  // kSolveThreads / 32 right-hand sides per gather item)
  const int64_t ych = ceil_div(R, kSolveCols), wch = ceil_div(R, kSolveThreads / 32);
  for (const auto& st : S.steps) {
    if (thin) break;   // the persistent solve runs the schedule without thin steps
    // tiny steps run as the small-supernode phases (the item handles any nf <= 64)
    const int pk = st.kind == 6 ? kPhFwdSmall : (st.kind == 7 ? kPhBwdSmall : st.kind);
    SolvePhase ph{pk, 1, st.first, st.count, 0};
    switch (pk) {
      case kPhFwdSmall: case kPhBwdSmall: ph.rows = (int32_t)ych; break;
      case kPhFwdAssemble: case kPhBwdGather: ph.rows = (int32_t)wch; break;
      default: break;
    }
    ph.items = pk == kPhGemm ? st.tiles : st.count * ph.rows;
    S.phases.push_back(ph);
  }
  upload(S.d_ids, S.ids, h->stream);
  upload(S.d_gemms, S.gemms, h->stream);
  upload(S.d_gemms_tc, S.gemms_tc, h->stream);
  upload(S.d_skinny, S.skinny, h->stream);
  upload(S.d_phases, S.phases, h->stream);
  upload(S.d_rows, S.rows, h->stream);
  upload(S.d_aptr, S.aptr, h->stream);
  upload(S.d_asrc, S.asrc, h->stream);
  upload(S.d_sgemms, S.sgemms, h->stream);
  upload(S.d_sgemms_tc, S.sgemms_tc, h->stream);
  upload(S.d_sreds, S.sreds, h->stream);
  upload(S.d_gemms_sm, S.gemms_sm, h->stream);
}

// One solve A x = b for device b (ldb) into device x (ldx) (x overwritten, or
// accumulated when `accumulate`).
template <typename T>
void prepare_solve(mfgpu_ctx* h, int64_t R, int refine) {
  const Plan& P = h->plan;
  h->persistent = h->persistent_mode == 1 && !is_complex_v<T>;   // complex fronts: per-step launches
  build_solve_schedule(h, R, (int)sizeof(T));
  // solve arena: the per-supernode blocks, then x in factor order, then the
  // partial products of the K-chunked steps
  h->b_fsol.ensure(std::max<size_t>(((size_t)(P.fc_total + P.n) * R + h->sched.split_scratch) * sizeof(T), 16));
  if (h->sched.skinny_scratch) h->b_skinny.ensure((size_t)h->sched.skinny_scratch * sizeof(T));
  if (refine > 0) h->b_r.ensure(std::max<size_t>((size_t)P.n * R * sizeof(Wide<T>), 16));
  configure_kernels<T>();
  if constexpr (!is_complex_v<T>)
  if (h->persistent) {
    h->b_bar.ensure(16);
    if (h->profiling) h->b_stamps.ensure((h->sched.phases.size() + 1) * (size_t)(refine + 1) * 8);
    int& grid = h->persist_grid[sizeof(T) == 8];
    if (!grid) {
      int per_sm = 0, sms = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_solve_persistent<T>, kSolveThreads,
                                                       persistent_smem_bytes<T>()));
      CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
      grid = std::max(1, per_sm) * sms;
    }
  }
}

template <typename T>
void solve_once(mfgpu_ctx* h, int64_t R, const Wide<T>* d_b, int64_t ldb, Wide<T>* d_x, int64_t ldx, bool use_rs,
                int accumulate) {
  const Plan& P = h->plan;
  cudaStream_t st = h->stream;
  SolveSchedule& S = h->sched;
  T* pool = h->b_pool.as<T>();
  T* fsol = h->b_fsol.as<T>();
  T* xw = fsol + P.fc_total * R;
  DevState DS = dev_state(h);
  SolveArgs A{R, reinterpret_cast<const double*>(d_b), ldb, (use_rs && h->have_rs) ? h->b_rs.as<double>() : nullptr,
              P.n, xw};
  klaunch(h, KC_FWD_ASSEMBLE, 0, (double)P.n * R * (16.0 + sizeof(T)), [&] {
    k_rhs_factor_order<T><<<grid_rows_groups(P.n, R), 256, 0, st>>>(P.n, R, d_b, ldb, A.rs, h->b_qf.as<int32_t>(),
                                                              h->b_prow.as<int32_t>(), xw, P.n);
  });
  const unsigned ychunks = (unsigned)((R + solve_cols<T>() - 1) / solve_cols<T>());
  const unsigned acols = (unsigned)((R + kAsmCols - 1) / kAsmCols);
  const unsigned tchunks = (unsigned)((R + kThinCols - 1) / kThinCols);
  const RowTask* rows = S.d_rows.as<RowTask>();
  const int32_t* ids = S.d_ids.as<int32_t>();
  const GemmTask* gemms = S.d_gemms.as<GemmTask>();
  int64_t tune_id = tune_factor_count(P) + (int64_t)P.inv_steps.size();
  if constexpr (is_complex_v<T>) {
  } else if (h->persistent && !S.phases.empty()) {
    unsigned int* bar = h->b_bar.as<unsigned int>();
    PersistentArgs X{S.d_phases.as<SolvePhase>(), (int32_t)S.phases.size(), ids, gemms,
                     GridBarrier{bar, bar + 1, reinterpret_cast<int*>(bar + 2), h->wait_ns, h->b_flags.as<int>() + 2},
                     nullptr};
    if (h->profiling) {
      X.stamps = h->b_stamps.as<unsigned long long>() + h->stamp_next;
      h->pending_phases.push_back({h->stamp_next, (int)S.phases.size(), (int)sizeof(T)});
      h->stamp_next += S.phases.size() + 1;
    }
    CK(cudaMemsetAsync(bar, 0, 3 * sizeof(unsigned int), st));
    ++h->launch_count;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)h->persist_grid[sizeof(T) == 8]);
    cfg.blockDim = dim3(kSolveThreads);
    cfg.dynamicSmemBytes = persistent_smem_bytes<T>();
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CK(cudaLaunchKernelEx(&cfg, k_solve_persistent<T>, h->dp, DS, A, X, (const T*)pool, fsol, xw));
  }
  if (is_complex_v<T> || !(h->persistent && !S.phases.empty())) {
  LevelFork fork(h);
  for (const auto& s : S.steps) {
    const double bytes = s.elems * sizeof(T);
    fork.at(s.level);
    const bool side = s.kind == 0 || s.kind == 4 || s.kind == 6 || s.kind == 7 || s.kind == 10;
    const cudaStream_t ss = side ? fork.side() : st;
    switch (s.kind) {
      case 0:
        klaunch(h, KC_FWD_SMALL, s.flops, bytes, [&] {
          k_fwd_small<T><<<dim3((unsigned)s.count, ychunks), kSolveThreads, 0, ss>>>(h->dp, DS, A, ids + s.first,
                                                                                     pool, fsol);
        }, s.level, s.count);
        break;
      case 1:
        if (!s.rt_count) break;
        klaunch(h, KC_FWD_ASSEMBLE, 0, bytes, [&] {
          k_fwd_assemble_rows<T><<<dim3((unsigned)((s.rt_count + 3) / 4), acols), 256, 0, st>>>(
              h->dp, DS, A, rows + s.rt_first, (int)s.rt_count, S.d_aptr.as<int64_t>(), S.d_asrc.as<int2>(), fsol);
        }, s.level, s.count);
        break;
      case 3: {
        h->cur_tune = (int32_t)tune_id;
        // the K-chunked form when the step has one, its partial products
        // folded into C right after the chunks
        const bool split = s.sp_count > 0;
        const GemmTask* g64 = split ? S.d_sgemms.as<GemmTask>() + s.sp_first : gemms + s.first;
        const GemmTask* gtc = split ? S.d_sgemms_tc.as<GemmTask>() + s.sp_first
                                    : S.d_gemms_tc.as<GemmTask>() + s.first;
        const int64_t gcount = split ? s.sp_count : s.count;
        const int64_t t64 = split ? s.sp_tiles : s.tiles, ttc = split ? s.sp_tiles_tc : s.tiles_tc;
        const int32_t gmaxk = split ? s.sp_max_k : s.max_k;
        auto fold = [&] {
          if (split)
            k_split_reduce<T><<<grid1(s.rd_elems, 256), 256, 0, st>>>(S.d_sreds.as<SplitRed>() + s.rd_first,
                                                                      (int)s.rd_count, s.rd_elems, fsol);
        };
        if constexpr (is_complex_v<T>)
          klaunch(h, KC_GEMM_SOLVE, s.flops, bytes, [&] {
            launch_gemm<T>(g64, gcount, t64, pool, fsol, fsol, st);
            fold();
          }, s.level, t64);
        else if (s.sk_count && !(sizeof(T) == 4 && gemm_use_tc(h, tune_id, false)))
          klaunch(h, KC_GEMM_SOLVE, s.flops, bytes, [&] {
            const SkinnyTask* sk = S.d_skinny.as<SkinnyTask>() + s.sk_first;
            T* part = h->b_skinny.as<T>();
            if (R <= 1) {
              k_skinny_part<T, 1><<<(unsigned)s.sk_parts, kSkinnyRows, 0, st>>>(sk, (int)s.sk_count, pool, fsol, part);
              k_skinny_reduce<T, 1><<<(unsigned)s.sk_reds, kSkinnyRows, 0, st>>>(sk, (int)s.sk_count, part, fsol);
            } else if (R <= 4) {
              k_skinny_part<T, 4><<<(unsigned)s.sk_parts, kSkinnyRows, 0, st>>>(sk, (int)s.sk_count, pool, fsol, part);
              k_skinny_reduce<T, 4><<<(unsigned)s.sk_reds, kSkinnyRows, 0, st>>>(sk, (int)s.sk_count, part, fsol);
            } else {
              k_skinny_part<T, kSkinnyMaxN><<<(unsigned)s.sk_parts, kSkinnyRows, 0, st>>>(sk, (int)s.sk_count, pool,
                                                                                         fsol, part);
              k_skinny_reduce<T, kSkinnyMaxN><<<(unsigned)s.sk_reds, kSkinnyRows, 0, st>>>(sk, (int)s.sk_count, part,
                                                                                           fsol);
            }
          }, s.level, s.sk_parts);
        else if (sizeof(T) == 4 && gemm_use_tc(h, tune_id, R >= 64 && tc_worthwhile(s.flops, ttc)))
          klaunch(h, KC_GEMM_SOLVE, s.flops, bytes, [&] {
            launch_tc(h, gtc, gcount, ttc, (const float*)pool, (const float*)fsol, (float*)fsol, st, gmaxk);
            fold();
          }, s.level, ttc);
        else if (s.sm_count)
          klaunch(h, KC_GEMM_SOLVE, s.flops, bytes, [&] {
            const GemmTask* gs = S.d_gemms_sm.as<GemmTask>() + s.sm_first;
            if (s.sm_bm == 16)
              k_gemm_skinny_m<T, 16><<<(unsigned)s.sm_tiles, 256, 0, st>>>(gs, (int)s.sm_count, pool, fsol, fsol);
            else
              k_gemm_skinny_m<T, 32><<<(unsigned)s.sm_tiles, 256, 0, st>>>(gs, (int)s.sm_count, pool, fsol, fsol);
          }, s.level, s.sm_tiles);
        else
          klaunch(h, KC_GEMM_SOLVE, s.flops, bytes, [&] {
            launch_gemm<T>(g64, gcount, t64, pool, fsol, fsol, st);
            fold();
          }, s.level, t64);
        h->cur_tune = -1;
        ++tune_id;
        break;
      }
      case 6:
        klaunch(h, KC_FWD_SMALL, s.flops, bytes, [&] {
          k_fwd_tiny<T><<<dim3((unsigned)((s.count + tiny_warps<T>() - 1) / tiny_warps<T>()), (unsigned)((R + 31) / 32)),
                          32 * tiny_warps<T>(), 0, ss>>>(h->dp, DS, A, ids + s.first, (int)s.count, pool, fsol);
        }, s.level, s.count);
        break;
      case 10:
        klaunch(h, KC_FWD_SMALL, s.flops, bytes, [&] {
          k_fwd_leaf<T><<<dim3((unsigned)((s.count + kLeafWarps - 1) / kLeafWarps), (unsigned)((R + 31) / 32)),
                          32 * kLeafWarps, 0, ss>>>(h->dp, A, ids + s.first, (int)s.count, pool, fsol);
        }, s.level, s.count);
        break;
      case 7:
        klaunch(h, KC_BWD_SMALL, s.flops, bytes, [&] {
          k_bwd_tiny<T><<<dim3((unsigned)((s.count + tiny_warps<T>() - 1) / tiny_warps<T>()), (unsigned)((R + 31) / 32)),
                          32 * tiny_warps<T>(), 0, ss>>>(h->dp, A, ids + s.first, (int)s.count, pool, fsol, xw);
        }, s.level, s.count);
        break;
      case 4:
        klaunch(h, KC_BWD_SMALL, s.flops, bytes, [&] {
          k_bwd_small<T><<<dim3((unsigned)s.count, ychunks), kSolveThreads, 0, ss>>>(h->dp, A, ids + s.first, pool,
                                                                                     fsol, xw);
        }, s.level, s.count);
        break;
      case 8:
        klaunch(h, KC_FWD_THIN, s.flops, bytes, [&] {
          k_fwd_thin<T><<<dim3((unsigned)s.count, tchunks), 256, 0, st>>>(h->dp, A, ids + s.first, pool, fsol, xw);
        }, s.level, s.count);
        break;
      case 5:
        if (!s.rt_count) break;   // roots only: no update rows to gather
        klaunch(h, KC_BWD_GATHER, 0, bytes, [&] {
          k_bwd_gather_rows<T><<<dim3((unsigned)((s.rt_count + 3) / 4), acols), 256, 0, st>>>(
              h->dp, A, rows + s.rt_first, (int)s.rt_count, fsol, xw);
        }, s.level, s.count);
        break;
    }
  }
  fork.join();
  }
  klaunch(h, KC_SOLVE_FINISH, 0, (double)P.n * R * (sizeof(T) + sizeof(Wide<T>) * (1.0 + accumulate)), [&] {
    k_solve_finish<T><<<grid_rows_groups(P.n, R), 256, 0, st>>>(P.n, R, h->b_qf.as<int32_t>(), xw, P.n, d_x, ldx,
                                                           accumulate);
  });
  CK(cudaGetLastError());
}

template <typename T>
void solve_refine(mfgpu_ctx* h, int64_t R, const Wide<T>* d_b, int64_t ldb, Wide<T>* d_x, int64_t ldx, int refine,
                  bool use_rs) {
  const Plan& P = h->plan;
  cudaStream_t st = h->stream;
  if (h->persistent) CK(cudaMemsetAsync(h->b_bar.as<unsigned int>() + 3, 0, sizeof(unsigned int), st));
  CK(cudaMemsetAsync(h->b_flags.as<int>() + 1, 0, sizeof(int), st));   // this solve's timeout flag
  solve_once<T>(h, R, d_b, ldb, d_x, ldx, use_rs, 0);
  if (refine > 0) {
    Wide<T>* r = h->b_r.as<Wide<T>>();
    for (int it = 0; it < refine; ++it) {
      klaunch(h, KC_RESIDUAL, 2.0 * P.nnz_a * R, (8.0 + sizeof(Wide<T>)) * P.nnz_a + 3.0 * sizeof(Wide<T>) * P.n * R,
              [&] {
        if constexpr (is_complex_v<T>)
          k_residual_z<<<grid_rows_cols(P.n, R), 256, 0, st>>>(P.n, R, h->b_csr_ptr.as<int32_t>(),
                                                            h->b_csr_col.as<int32_t>(), h->b_csr_src.as<int32_t>(),
                                                            h->b_ax.as<zc>(), d_b, ldb, d_x, ldx, r, P.n);
        else
          k_residual<<<grid_residual(P.n, R), 256, 0, st>>>(P.n, R, h->b_csr_ptr.as<int32_t>(),
                                                          h->b_csr_col.as<int32_t>(), h->b_csr_src.as<int32_t>(),
                                                          h->b_ax.as<double>(), d_b, ldb, d_x, ldx, r, P.n);
      });
      solve_once<T>(h, R, r, P.n, d_x, ldx, use_rs, 1);
    }
  }
  CK(cudaGetLastError());
}

template <typename T>
void solve_graph(mfgpu_ctx* h, int64_t R, const Wide<T>* d_b, int64_t ldb, Wide<T>* d_x, int64_t ldx, int refine) {
  prepare_solve<T>(h, R, refine);
  const SolveSchedule& S = h->sched;
  const std::vector<uintptr_t> key = {
      sizeof(T), (uintptr_t)R, (uintptr_t)d_b, (uintptr_t)ldb, (uintptr_t)d_x, (uintptr_t)ldx, (uintptr_t)refine,
      (uintptr_t)h->have_rs, (uintptr_t)h->b_rs.p, (uintptr_t)h->b_pool.p, (uintptr_t)h->b_dinv.p,
      (uintptr_t)h->b_fsol.p, (uintptr_t)h->b_inv_tasks.p, (uintptr_t)h->b_r.p, (uintptr_t)h->b_ax.p,
      (uintptr_t)S.d_ids.p, (uintptr_t)S.d_gemms.p, (uintptr_t)S.d_phases.p, (uintptr_t)h->b_prow.p,
      (uintptr_t)S.d_gemms_tc.p, (uintptr_t)S.d_skinny.p, (uintptr_t)h->b_skinny.p, (uintptr_t)h->use_tc,
      (uintptr_t)S.d_rows.p, (uintptr_t)S.d_aptr.p, (uintptr_t)S.d_asrc.p, (uintptr_t)S.d_sgemms.p,
      (uintptr_t)S.d_sgemms_tc.p, (uintptr_t)S.d_sreds.p, (uintptr_t)S.d_gemms_sm.p,
      (uintptr_t)h->tc_bf16x3, (uintptr_t)h->choice_version, (uintptr_t)h->wait_ns,
      (uintptr_t)h->persistent, (uintptr_t)h->b_bar.p,
      (uintptr_t)h->b_rowfac.p, (uintptr_t)h->stream};
  if (!h->solve_graphs) {
    solve_refine<T>(h, R, d_b, ldb, d_x, ldx, refine, true);
    return;
  }
  try {
    run_sequence(h, h->solve_key, h->solve_exec, h->solve_nodes, key,
                 [&] { solve_refine<T>(h, R, d_b, ldb, d_x, ldx, refine, true); });
  } catch (const CudaError&) {
    if (!h->persistent || h->solve_exec) throw;
    // the capture of the cooperative launch failed: solve without a graph
    cudaGetLastError();
    h->solve_graphs = false;
    solve_refine<T>(h, R, d_b, ldb, d_x, ldx, refine, true);
  }
}

// After a synchronised solve: MFGPU_ERR_TIMEOUT when a grid barrier of a
// persistent pass gave up (the solution is then incomplete).
int solve_status(mfgpu_ctx* h) {
  int flags[2] = {0, 0};
  if (h->b_flags.p) CK(cudaMemcpy(flags, h->b_flags.p, sizeof flags, cudaMemcpyDeviceToHost));
  if (flags[1]) return fail(h, MFGPU_ERR_TIMEOUT, "a tensor-core GEMM gave up a bounded wait");
  if (!h->persistent || !h->b_bar.p) return MFGPU_OK;
  int sticky = 0;
  CK(cudaMemcpy(&sticky, h->b_bar.as<unsigned int>() + 3, sizeof sticky, cudaMemcpyDeviceToHost));
  if (sticky) return fail(h, MFGPU_ERR_TIMEOUT, "a grid barrier of the persistent solve gave up a bounded wait");
  return MFGPU_OK;
}

void solve_dispatch(mfgpu_ctx* h, int64_t R, const double* d_b, int64_t ldb, double* d_x, int64_t ldx, int refine) {
  if (h->c64_factors) throw std::invalid_argument("the factorization is complex: use mfgpu_solve_c64");
  if (h->factor_precision == MFGPU_PRECISION_MIXED) solve_graph<float>(h, R, d_b, ldb, d_x, ldx, refine);
  else solve_graph<double>(h, R, d_b, ldb, d_x, ldx, refine);
}

int analyze_common(mfgpu_ctx* h, int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf,
                   const int64_t* parent, int64_t ns, const int64_t* sstart, const int64_t* upd_ptr,
                   const int64_t* upd_idx) {
  auto t0 = std::chrono::steady_clock::now();
  // until this analysis has completed, the handle holds no usable plan: a
  // failure below (an inconsistent symbolic analysis, an allocation) leaves
  // it unanalyzed rather than with a host plan that its device maps do not
  // match; a batch analysis sets its own state after this returns
  h->analyzed = h->factored = h->csc_ready = false;
  h->batch.nsys = 0;
  Plan plan;
  if (h->merge_fronts)
    build_plan_merged(n, colptr, rowval, qf, parent, ns, sstart, upd_ptr, upd_idx, plan, kMergeMaxPivots);
  else
    build_plan(n, colptr, rowval, qf, parent, ns, sstart, upd_ptr, upd_idx, plan);
  // all fronts resident when they fit comfortably (FP64 worst case), else
  // working fronts placed by lifetime and a compact panel pool
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  if (h->lean_mode == 1 || (h->lean_mode == 0 && (double)plan.front_elems_full * 8.0 > 0.45 * (double)total_b))
    set_layout(plan, true);
  h->plan = std::move(plan);
  upload_plan(h);
  upload_launches(h);
  h->launches_safe = false;
  if (h->factor_exec) cudaGraphExecDestroy(h->factor_exec);
  if (h->solve_exec) cudaGraphExecDestroy(h->solve_exec);
  h->factor_exec = h->solve_exec = nullptr;
  h->factor_key.clear();
  h->solve_key.clear();
  h->analyzed = true;
  h->factored = false;
  h->csc_ready = false;
  h->sched = SolveSchedule{};
  CK(cudaStreamSynchronize(h->stream));
  h->t_analyze_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return MFGPU_OK;
}

// One right-hand side's backward error r / den folded into the running
// maximum.  A non-finite residual or denominator (a NaN or Inf in x, b or A,
// or an overflow) gives NaN, and a NaN stays the maximum: an accuracy check
// can never pass on a broken solution.  den = 0 means b = 0 and A x = 0.
__host__ __device__ inline double worst_eta(double worst, double r, double den) {
  const bool finite = r - r == 0.0 && den - den == 0.0;   // false for NaN and +-Inf
  const double eta = finite ? (den > 0 ? r / den : 0.0) : nan("");
  if (worst != worst) return worst;
  return (eta != eta || eta > worst) ? eta : worst;
}

bool valid_csc(int64_t n, const int64_t* colptr, const int64_t* rowval) {
  if (n < 0 || !colptr || colptr[0] != 1) return false;
  for (int64_t j = 0; j < n; ++j)
    if (colptr[j + 1] < colptr[j]) return false;
  if (colptr[n] > 1 && !rowval) return false;
  for (int64_t p = 0; p < colptr[n] - 1; ++p)
    if (rowval[p] < 1 || rowval[p] > n) return false;
  return true;
}

}  // namespace

extern "C" {

int mfgpu_create(const mfgpu_options* opts, mfgpu_ctx** out) {
  if (!out) return MFGPU_ERR_ARGUMENT;
  *out = nullptr;
  auto* h = new mfgpu_ctx();
  if (opts) {
    h->device = opts->device;
    h->precision = opts->precision;
    h->use_tc = !(opts->flags & MFGPU_FLAG_NO_TENSOR_CORES);
    h->persistent_mode = (opts->flags & MFGPU_FLAG_PERSISTENT_SOLVE) ? 1 : (opts->flags & MFGPU_FLAG_STEP_SOLVE) ? 2 : 0;
    h->tc_bf16x3 = !(opts->flags & MFGPU_FLAG_TF32_SPLIT);
    h->lean_mode = (opts->flags & MFGPU_FLAG_LEAN_FRONTS) ? 1 : 0;
    h->merge_fronts = !(opts->flags & MFGPU_FLAG_NO_FRONT_MERGE);
  }
  int rc = guarded(h, [&]() -> int {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= h->device) {
      cudaGetLastError();
      return fail(h, MFGPU_ERR_NO_DEVICE, "no CUDA device");
    }
    CK(cudaSetDevice(h->device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, h->device));
    if (prop.major != 10) return fail(h, MFGPU_ERR_NO_DEVICE, "libmfgpu is built for sm_100a (B200)");
    h->num_sms = prop.multiProcessorCount;
    CK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->ev_copy, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
    h->stream = h->own_stream;
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    return MFGPU_OK;
  });
  if (rc != MFGPU_OK) {
    mfgpu_destroy(h);
    return rc;
  }
  *out = h;
  return MFGPU_OK;
}

void mfgpu_destroy(mfgpu_ctx* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  DevBuf* bufs[] = {&h->b_c1, &h->b_np, &h->b_nu, &h->b_nf, &h->b_upd_off, &h->b_front_off, &h->b_colbase,
                    &h->b_child_ptr, &h->b_child_idx, &h->b_upd, &h->b_rel, &h->b_uoff, &h->b_v_src, &h->b_v_srow,
                    &h->b_v_frow, &h->b_fc_super, &h->b_fc_vbeg, &h->b_fc_vend, &h->b_fc_ch_ptr, &h->b_fc_ch,
                    &h->b_lcolptr, &h->b_ucolptr, &h->b_qf, &h->b_csr_ptr, &h->b_csr_col, &h->b_csr_src,
                    &h->b_small, &h->b_panel, &h->b_trsm, &h->b_gemm, &h->b_gemm_tc, &h->b_plane_tasks, &h->b_planes, &h->b_pool, &h->b_vx, &h->b_ax, &h->b_rs,
                    &h->b_ipiv, &h->b_info, &h->b_prow, &h->b_rowfac, &h->b_flags, &h->b_dinv, &h->b_dinv_off,
                    &h->b_inv_off, &h->b_inv_blocks, &h->b_inv_tasks, &h->b_inv_tasks_tc, &h->b_lpan_off,
                    &h->b_u12_off, &h->b_skinny, &h->sched.d_skinny, &h->b_seg_end, &h->b_col_orig, &h->b_o_c1,
                    &h->b_o_np, &h->b_o_upd_off, &h->b_o_upd, &h->b_o_xpos, &h->b_fcu_ptr, &h->b_fcu,
                    &h->b_li, &h->b_lx, &h->b_ui,
                    &h->b_ux, &h->b_fsol, &h->b_b, &h->b_x, &h->b_f32, &h->b_r, &h->b_d, &h->b_err, &h->b_norm,
                    &h->sched.d_ids, &h->sched.d_gemms, &h->sched.d_gemms_tc, &h->sched.d_phases,
                    &h->sched.d_rows, &h->sched.d_aptr, &h->sched.d_asrc, &h->sched.d_sgemms, &h->sched.d_sgemms_tc,
                    &h->sched.d_sreds, &h->sched.d_gemms_sm, &h->b_bar,
                    &h->b_stamps};
  for (DevBuf* b : bufs) b->release();
  if (h->factor_exec) cudaGraphExecDestroy(h->factor_exec);
  if (h->solve_exec) cudaGraphExecDestroy(h->solve_exec);
  for (cudaEvent_t e : h->evpool) cudaEventDestroy(e);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  if (h->side_stream) cudaStreamDestroy(h->side_stream);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->ev_copy) cudaEventDestroy(h->ev_copy);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  delete h;
}

const char* mfgpu_last_error(const mfgpu_ctx* h) { return h ? h->err.c_str() : "null handle"; }

int mfgpu_set_stream(mfgpu_ctx* h, void* s) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  h->stream = s ? (cudaStream_t)s : h->own_stream;
  return MFGPU_OK;
}

int mfgpu_set_growth_limit(mfgpu_ctx* h, double limit) {
  if (!h || !(limit > 0)) return MFGPU_ERR_ARGUMENT;
  h->growth_limit = limit;
  return MFGPU_OK;
}

int mfgpu_set_wait_limit(mfgpu_ctx* h, double seconds) {
  if (!h || !(seconds > 0) || !(seconds <= 3600)) return MFGPU_ERR_ARGUMENT;
  h->wait_ns = std::max<uint64_t>(1, (uint64_t)(seconds * 1e9));   // part of the graph keys
  return MFGPU_OK;
}

int mfgpu_test_stall(mfgpu_ctx* h, int32_t on) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    if (!h->b_flags.p) {
      h->b_flags.ensure(16);
      CK(cudaMemsetAsync(h->b_flags.p, 0, 16, h->stream));
    }
    const int v = on ? 1 : 0;
    CK(cudaMemcpyAsync(h->b_flags.as<int>() + 2, &v, sizeof v, cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MFGPU_OK;
  });
}

int mfgpu_set_precision(mfgpu_ctx* h, int32_t p) {
  if (!h || (p != MFGPU_PRECISION_FP64 && p != MFGPU_PRECISION_MIXED)) return MFGPU_ERR_ARGUMENT;
  h->precision = p;
  return MFGPU_OK;
}

int mfgpu_analyze(mfgpu_ctx* h, int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf,
                  const int64_t* parent, int64_t nsuper, const int64_t* sstart, const int64_t* upd_ptr,
                  const int64_t* upd_idx) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    if (!valid_csc(n, colptr, rowval) || !qf || !parent || !sstart || !upd_ptr || nsuper < 0 || upd_ptr[0] != 1 ||
        upd_ptr[nsuper] < 1 || (upd_ptr[nsuper] > 1 && !upd_idx))
      return fail(h, MFGPU_ERR_ARGUMENT, "invalid analyze arguments");
    std::vector<int64_t> cp(n + 1), ri(colptr[n] - 1), q(n), par(n), ss(nsuper + 1), up(nsuper + 1),
        ui(upd_ptr[nsuper] - 1);
    for (int64_t j = 0; j <= n; ++j) cp[j] = colptr[j] - 1;
    for (size_t p = 0; p < ri.size(); ++p) ri[p] = rowval[p] - 1;
    for (int64_t k = 0; k < n; ++k) {
      q[k] = qf[k] - 1;
      par[k] = parent[k] - 1;
    }
    for (int64_t s = 0; s <= nsuper; ++s) {
      ss[s] = sstart[s] - 1;
      up[s] = upd_ptr[s] - 1;
    }
    for (size_t p = 0; p < ui.size(); ++p) ui[p] = upd_idx[p] - 1;
    return analyze_common(h, n, cp.data(), ri.data(), q.data(), par.data(), nsuper, ss.data(), up.data(), ui.data());
  });
}

int mfgpu_analyze_symbolic(mfgpu_ctx* h, int64_t n, const int64_t* colptr, const int64_t* rowval,
                           const mfgpu_symbolic* sym) {
  if (!h || !sym || sym->s.n != n) return MFGPU_ERR_ARGUMENT;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    if (!valid_csc(n, colptr, rowval)) return fail(h, MFGPU_ERR_ARGUMENT, "invalid CSC");
    std::vector<int64_t> cp(n + 1), ri(colptr[n] - 1);
    for (int64_t j = 0; j <= n; ++j) cp[j] = colptr[j] - 1;
    for (size_t p = 0; p < ri.size(); ++p) ri[p] = rowval[p] - 1;
    const auto& s = sym->s;
    return analyze_common(h, n, cp.data(), ri.data(), s.qf.data(), s.parent.data(), s.nsuper(), s.sstart.data(),
                          s.upd_ptr.data(), s.upd_idx.data());
  });
}

int mfgpu_factor_device(mfgpu_ctx* h, const double* d_nzval, const double* d_rs, int32_t check) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->analyzed) return fail(h, MFGPU_ERR_STATE, "factor before analyze");
  if (h->plan.nnz_a && !d_nzval) return fail(h, MFGPU_ERR_ARGUMENT, "null values");
  h->factored = h->csc_ready = false;
  h->f32_values = h->c64_values = false;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    const Plan& P = h->plan;
    h->b_ax.ensure(std::max<int64_t>(P.nnz_a, 1) * 8);
    if (P.nnz_a) CK(cudaMemcpyAsync(h->b_ax.p, d_nzval, P.nnz_a * 8, cudaMemcpyDeviceToDevice, h->stream));
    h->have_rs = d_rs != nullptr;
    if (d_rs) {
      h->b_rs.ensure(std::max<int64_t>(P.n, 1) * 8);
      CK(cudaMemcpyAsync(h->b_rs.p, d_rs, P.n * 8, cudaMemcpyDeviceToDevice, h->stream));
    }
    return factor_dispatch(h, check);
  });
}

int mfgpu_factor_scaled(mfgpu_ctx* h, const double* nzval, int32_t scale, int32_t check) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->analyzed) return fail(h, MFGPU_ERR_STATE, "factor before analyze");
  h->f32_values = h->c64_values = false;
  if (scale < MFGPU_SCALE_NONE || scale > MFGPU_SCALE_MAX) return fail(h, MFGPU_ERR_ARGUMENT, "bad scale kind");
  if (h->plan.nnz_a && !nzval) return fail(h, MFGPU_ERR_ARGUMENT, "null values");
  h->factored = h->csc_ready = false;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    const Plan& P = h->plan;
    h->b_ax.ensure(std::max<int64_t>(P.nnz_a, 1) * 8);
    if (P.nnz_a) CK(cudaMemcpyAsync(h->b_ax.p, nzval, P.nnz_a * 8, cudaMemcpyHostToDevice, h->stream));
    h->have_rs = scale != MFGPU_SCALE_NONE;
    if (h->have_rs && P.n) {
      h->b_rs.ensure(std::max<int64_t>(P.n, 1) * 8);
      k_row_scaling<<<grid1(P.n, 256), 256, 0, h->stream>>>(P.n, h->b_csr_ptr.as<int32_t>(), h->b_csr_src.as<int32_t>(),
                                                             h->b_ax.as<double>(), scale, h->b_rs.as<double>());
      CK(cudaGetLastError());
    }
    return factor_dispatch(h, check);
  });
}

int mfgpu_get_row_scaling(mfgpu_ctx* h, double* rs) {
  if (!h || !rs) return MFGPU_ERR_ARGUMENT;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "no factorization");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    const int64_t n = h->plan.n;
    if (!h->have_rs) {
      std::fill(rs, rs + n, 1.0);
      return MFGPU_OK;
    }
    CK(cudaMemcpyAsync(rs, h->b_rs.p, n * 8, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return MFGPU_OK;
  });
}

// Host values (FP64, Float32 values widened, or ComplexF64 as interleaved
// (re, im) doubles) -> factorization.
static int factor_host(mfgpu_ctx* h, const double* nzval, const double* rs, int32_t check, bool f32,
                       bool c64 = false) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->analyzed) return fail(h, MFGPU_ERR_STATE, "factor before analyze");
  if (h->plan.nnz_a && !nzval) return fail(h, MFGPU_ERR_ARGUMENT, "null values");
  // the previous factors stop being valid once A's values are overwritten
  h->factored = h->csc_ready = false;
  h->f32_values = f32;
  h->c64_values = c64;
  const int64_t vb = c64 ? 16 : 8;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    const Plan& P = h->plan;
    h->b_ax.ensure(std::max<int64_t>(P.nnz_a, 1) * vb);
    if (P.nnz_a) CK(cudaMemcpyAsync(h->b_ax.p, nzval, P.nnz_a * vb, cudaMemcpyHostToDevice, h->stream));
    h->have_rs = rs != nullptr;
    if (rs) {
      h->b_rs.ensure(std::max<int64_t>(P.n, 1) * 8);
      CK(cudaMemcpyAsync(h->b_rs.p, rs, P.n * 8, cudaMemcpyHostToDevice, h->stream));
    }
    return factor_dispatch(h, check);
  });
}

int mfgpu_factor(mfgpu_ctx* h, const double* nzval, const double* rs, int32_t check) {
  return factor_host(h, nzval, rs, check, false);
}

int mfgpu_factor_f32(mfgpu_ctx* h, const float* nzval, const float* rs, int32_t check) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->analyzed) return fail(h, MFGPU_ERR_STATE, "factor before analyze");
  const Plan& P = h->plan;
  if (P.nnz_a && !nzval) return fail(h, MFGPU_ERR_ARGUMENT, "null values");
  // Float32 values and scaling widen exactly; the device forms rs * a in
  // FP64 (exact for two Float32 factors) and the FP32 fronts round it once,
  // as a Float32 multiplication would
  std::vector<double> vx(nzval, nzval + P.nnz_a), rsx;
  if (rs) rsx.assign(rs, rs + P.n);
  return factor_host(h, vx.data(), rs ? rsx.data() : nullptr, check, true);
}

int mfgpu_get_factors_f32(mfgpu_ctx* h, int64_t* lcolptr, int64_t* lrowval, float* lnzval, int64_t* ucolptr,
                          int64_t* urowval, float* unzval, int64_t* p, int64_t* q, int64_t* pinv) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "no factorization");
  if (!h->f32_values) return fail(h, MFGPU_ERR_STATE, "the last factorization is not of a Float32 matrix");
  std::vector<double> lx(lnzval ? h->plan.nnz_l : 0), ux(unzval ? h->plan.nnz_u : 0);
  const int rc = mfgpu_get_factors(h, lcolptr, lrowval, lnzval ? lx.data() : nullptr, ucolptr, urowval,
                                   unzval ? ux.data() : nullptr, p, q, pinv);
  if (rc != MFGPU_OK) return rc;
  for (size_t k = 0; k < lx.size(); ++k) lnzval[k] = (float)lx[k];   // FP32 values: exact
  for (size_t k = 0; k < ux.size(); ++k) unzval[k] = (float)ux[k];
  return MFGPU_OK;
}

int mfgpu_solve_f32(mfgpu_ctx* h, int64_t nrhs, const float* b, float* x, int32_t refine) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "solve before factor");
  if (h->c64_factors) return fail(h, MFGPU_ERR_STATE, "the factorization is complex: use mfgpu_solve_c64");
  const int64_t n = h->plan.n;
  if (nrhs < 0 || refine < 0 || (nrhs && n && (!b || !x))) return fail(h, MFGPU_ERR_ARGUMENT, "bad solve sizes");
  if (nrhs == 0 || n == 0) return MFGPU_OK;
  // Float32 b crosses the bus and is widened on the device; x is rounded to
  // Float32 there and copied back
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    const int64_t len = n * nrhs;
    h->b_f32.ensure((size_t)len * 4);
    h->b_b.ensure((size_t)len * 8);
    h->b_x.ensure((size_t)len * 8);
    CK(cudaMemcpyAsync(h->b_f32.p, b, len * 4, cudaMemcpyHostToDevice, st));
    k_convert<float, double><<<grid1(len, 256), 256, 0, st>>>(len, h->b_f32.as<float>(), h->b_b.as<double>());
    solve_dispatch(h, nrhs, h->b_b.as<double>(), n, h->b_x.as<double>(), n, refine);
    k_convert<double, float><<<grid1(len, 256), 256, 0, st>>>(len, h->b_x.as<double>(), h->b_f32.as<float>());
    CK(cudaMemcpyAsync(x, h->b_f32.p, len * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    prof_flush(h);
    return solve_status(h);
  });
}

int mfgpu_factor_sizes(mfgpu_ctx* h, int64_t* out3) {
  if (!h || !out3) return MFGPU_ERR_ARGUMENT;
  if (!h->analyzed) return fail(h, MFGPU_ERR_STATE, "not analyzed");
  out3[0] = h->plan.n;
  out3[1] = h->plan.nnz_l;
  out3[2] = h->plan.nnz_u;
  return MFGPU_OK;
}

// The CSC factors of the last factorization into host buffers; vbytes is
// the size of one value (8, or 16 for ComplexF64 factors).
static int get_factors_impl(mfgpu_ctx* h, int64_t* lcolptr, int64_t* lrowval, void* lnzval, int64_t* ucolptr,
                            int64_t* urowval, void* unzval, int64_t* p, int64_t* q, int64_t* pinv, int64_t vbytes) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "no factorization");
  if (h->c64_factors != (vbytes == 16))
    return fail(h, MFGPU_ERR_STATE, h->c64_factors ? "the factorization is complex: use mfgpu_get_factors_c64"
                                                   : "the factorization is not complex: use mfgpu_get_factors");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    const Plan& P = h->plan;
    cudaStream_t st = h->stream;
    if (lrowval && P.nnz_l) CK(cudaMemcpyAsync(lrowval, h->b_li.p, P.nnz_l * 8, cudaMemcpyDeviceToHost, st));
    if (lnzval && P.nnz_l) CK(cudaMemcpyAsync(lnzval, h->b_lx.p, P.nnz_l * vbytes, cudaMemcpyDeviceToHost, st));
    if (urowval && P.nnz_u) CK(cudaMemcpyAsync(urowval, h->b_ui.p, P.nnz_u * 8, cudaMemcpyDeviceToHost, st));
    if (unzval && P.nnz_u) CK(cudaMemcpyAsync(unzval, h->b_ux.p, P.nnz_u * vbytes, cudaMemcpyDeviceToHost, st));
    std::vector<int32_t> prow(P.n);
    if (P.n) CK(cudaMemcpyAsync(prow.data(), h->b_prow.p, P.n * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int64_t j = 0; j <= P.n; ++j) {
      if (lcolptr) lcolptr[j] = P.lcolptr[j] + 1;
      if (ucolptr) ucolptr[j] = P.ucolptr[j] + 1;
    }
    // p = qf[prow] (src/multifrontal.jl:355-356)
    for (int64_t k = 0; k < P.n; ++k) {
      const int64_t pk = P.qf[prow[k]];
      if (p) p[k] = pk + 1;
      if (q) q[k] = (int64_t)P.qf[k] + 1;
      if (pinv) pinv[pk] = k + 1;
    }
    return MFGPU_OK;
  });
}

int mfgpu_factor_solve(mfgpu_ctx* h, const double* nzval, const double* rs, int32_t check, int64_t nrhs,
                       const double* b, int64_t ldb, double* x, int64_t ldx, int32_t refine) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->analyzed) return fail(h, MFGPU_ERR_STATE, "factor before analyze");
  const int64_t n = h->plan.n;
  if (nrhs < 0 || ldb < n || ldx < n || refine < 0 || (nrhs && n && (!b || !x)))
    return fail(h, MFGPU_ERR_ARGUMENT, "bad solve sizes");
  // the right-hand sides cross the bus on their own stream while the
  // factorization runs (overlapped when b is page-locked)
  const bool copy = nrhs > 0 && n > 0;
  int rc = guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    if (copy) {
      h->b_b.ensure((size_t)n * nrhs * 8);
      h->b_x.ensure((size_t)n * nrhs * 8);
      CK(cudaMemcpy2DAsync(h->b_b.p, n * 8, b, ldb * 8, n * 8, nrhs, cudaMemcpyHostToDevice, h->copy_stream));
      CK(cudaEventRecord(h->ev_copy, h->copy_stream));
    }
    return MFGPU_OK;
  });
  if (rc != MFGPU_OK) return rc;
  rc = factor_host(h, nzval, rs, check, false);
  if (rc != MFGPU_OK || !copy) {
    if (copy) cudaStreamSynchronize(h->copy_stream);   // b's buffer is not reused while the copy runs
    return rc;   // a singular column (check) or an error: no solve
  }
  return guarded(h, [&]() -> int {
    cudaStream_t st = h->stream;
    CK(cudaStreamWaitEvent(st, h->ev_copy, 0));
    solve_dispatch(h, nrhs, h->b_b.as<double>(), n, h->b_x.as<double>(), n, refine);
    CK(cudaMemcpy2DAsync(x, ldx * 8, h->b_x.p, n * 8, n * 8, nrhs, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    prof_flush(h);
    return solve_status(h);
  });
}

int mfgpu_get_factors(mfgpu_ctx* h, int64_t* lcolptr, int64_t* lrowval, double* lnzval, int64_t* ucolptr,
                      int64_t* urowval, double* unzval, int64_t* p, int64_t* q, int64_t* pinv) {
  return get_factors_impl(h, lcolptr, lrowval, lnzval, ucolptr, urowval, unzval, p, q, pinv, 8);
}

int mfgpu_factor_c64(mfgpu_ctx* h, const double* nzval_ri, const double* rs, int32_t check) {
  return factor_host(h, nzval_ri, rs, check, false, true);
}

int mfgpu_get_factors_c64(mfgpu_ctx* h, int64_t* lcolptr, int64_t* lrowval, double* lnzval_ri, int64_t* ucolptr,
                          int64_t* urowval, double* unzval_ri, int64_t* p, int64_t* q, int64_t* pinv) {
  return get_factors_impl(h, lcolptr, lrowval, lnzval_ri, ucolptr, urowval, unzval_ri, p, q, pinv, 16);
}

int mfgpu_solve_c64(mfgpu_ctx* h, int64_t nrhs, const double* b_ri, double* x_ri, int32_t refine) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "solve before factor");
  if (!h->c64_factors) return fail(h, MFGPU_ERR_STATE, "the factorization is not complex: use mfgpu_solve");
  const int64_t n = h->plan.n;
  if (nrhs < 0 || refine < 0 || (nrhs && n && (!b_ri || !x_ri))) return fail(h, MFGPU_ERR_ARGUMENT, "bad solve sizes");
  if (nrhs == 0 || n == 0) return MFGPU_OK;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    const int64_t len = n * nrhs;
    h->b_b.ensure((size_t)len * 16);
    h->b_x.ensure((size_t)len * 16);
    CK(cudaMemcpyAsync(h->b_b.p, b_ri, len * 16, cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(h->ev0, st));
    solve_graph<zc>(h, nrhs, h->b_b.as<zc>(), n, h->b_x.as<zc>(), n, refine);
    CK(cudaEventRecord(h->ev1, st));
    CK(cudaMemcpyAsync(x_ri, h->b_x.p, len * 16, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->t_solve_ms = ms;
    prof_flush(h);
    return solve_status(h);
  });
}

int mfgpu_solve_device(mfgpu_ctx* h, int64_t nrhs, const double* d_b, int64_t ldb, double* d_x, int64_t ldx,
                       int32_t refine) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "solve before factor");
  if (h->c64_factors) return fail(h, MFGPU_ERR_STATE, "the factorization is complex: use mfgpu_solve_c64");
  if (nrhs < 0 || ldb < h->plan.n || ldx < h->plan.n || refine < 0 || (nrhs && h->plan.n && (!d_b || !d_x)))
    return fail(h, MFGPU_ERR_ARGUMENT, "bad solve sizes");
  if (nrhs == 0 || h->plan.n == 0) return MFGPU_OK;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    CK(cudaEventRecord(h->ev0, h->stream));
    solve_dispatch(h, nrhs, d_b, ldb, d_x, ldx, refine);
    CK(cudaEventRecord(h->ev1, h->stream));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->t_solve_ms = ms;
    prof_flush(h);
    return solve_status(h);
  });
}

int mfgpu_solve(mfgpu_ctx* h, int64_t nrhs, const double* b, int64_t ldb, double* x, int64_t ldx, int32_t refine) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "solve before factor");
  if (h->c64_factors) return fail(h, MFGPU_ERR_STATE, "the factorization is complex: use mfgpu_solve_c64");
  const int64_t n = h->plan.n;
  if (nrhs < 0 || ldb < n || ldx < n || refine < 0 || (nrhs && (!b || !x)))
    return fail(h, MFGPU_ERR_ARGUMENT, "bad solve sizes");
  if (nrhs == 0 || n == 0) return MFGPU_OK;
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    h->b_b.ensure((size_t)n * nrhs * 8);
    h->b_x.ensure((size_t)n * nrhs * 8);
    CK(cudaMemcpy2DAsync(h->b_b.p, n * 8, b, ldb * 8, n * 8, nrhs, cudaMemcpyHostToDevice, st));
    solve_dispatch(h, nrhs, h->b_b.as<double>(), n, h->b_x.as<double>(), n, refine);
    CK(cudaMemcpy2DAsync(x, ldx * 8, h->b_x.p, n * 8, n * 8, nrhs, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    prof_flush(h);
    return solve_status(h);
  });
}

int mfgpu_backward_error_device(mfgpu_ctx* h, int64_t nrhs, const double* d_b, int64_t ldb, const double* d_x,
                                int64_t ldx, double* out) {
  if (!h || !out) return MFGPU_ERR_ARGUMENT;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "no matrix values");
  if (h->c64_factors) return fail(h, MFGPU_ERR_STATE, "real vectors only: the factorization is complex");
  if (nrhs < 1 || h->plan.n == 0) {
    *out = 0.0;
    return MFGPU_OK;
  }
  if (!d_b || !d_x || ldb < h->plan.n || ldx < h->plan.n)
    return fail(h, MFGPU_ERR_ARGUMENT, "null vectors or leading dimension below n");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    const Plan& P = h->plan;
    cudaStream_t st = h->stream;
    const int64_t n = P.n;
    h->b_r.ensure(std::max<size_t>((size_t)n * nrhs * 8, 16));
    h->b_err.ensure(std::max<size_t>((size_t)nrhs * 3 * 8, 16));
    h->b_norm.ensure(16);
    CK(cudaMemsetAsync(h->b_err.p, 0, nrhs * 3 * 8, st));
    CK(cudaMemsetAsync(h->b_norm.p, 0, 8, st));
    k_residual<<<grid_residual(n, nrhs), 256, 0, st>>>(n, nrhs, h->b_csr_ptr.as<int32_t>(), h->b_csr_col.as<int32_t>(),
                                                     h->b_csr_src.as<int32_t>(), h->b_ax.as<double>(), d_b, ldb, d_x,
                                                     ldx, h->b_r.as<double>(), n);
    k_bwd_error_parts<<<dim3((unsigned)((n + 255) / 256), (unsigned)std::min<int64_t>(nrhs, 65535)), 256, 0, st>>>(
        n, nrhs, h->b_r.as<double>(), n, d_x, ldx, d_b, ldb, h->b_err.as<unsigned long long>());
    k_norm_inf<<<grid1(n, 256), 256, 0, st>>>(n, h->b_csr_ptr.as<int32_t>(), h->b_csr_src.as<int32_t>(),
                                              h->b_ax.as<double>(), h->b_norm.as<unsigned long long>());
    CK(cudaGetLastError());
    std::vector<double> parts(3 * nrhs);
    double anorm = 0;
    CK(cudaMemcpyAsync(parts.data(), h->b_err.p, nrhs * 3 * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&anorm, h->b_norm.p, 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double worst = 0;
    for (int64_t c = 0; c < nrhs; ++c) worst = worst_eta(worst, parts[3 * c], anorm * parts[3 * c + 1] + parts[3 * c + 2]);
    *out = worst;
    return MFGPU_OK;
  });
}

// ---- autotuner interface ----------------------------------------------------
static void tune_row(float* f, int kind, const GemmTask* t, int64_t count, double flops, double elems,
                     int64_t tiles, int64_t tiles_tc) {
  double m = 0, n = 0, k = 0;
  for (int64_t i = 0; i < count; ++i) {
    m += t[i].m;
    n += t[i].n;
    k += t[i].k;
  }
  const double c = count > 0 ? (double)count : 1.0;
  const double v[kTuneFeatures] = {kind == 0 ? 1.0 : 0.0, kind == 1 ? 1.0 : 0.0, kind == 2 ? 1.0 : 0.0,
                                   std::log10(1 + flops), std::log10(1 + 4.0 * elems), std::log10(1.0 + count),
                                   std::log10(1.0 + tiles), std::log10(1.0 + tiles_tc), std::log10(1 + m / c),
                                   std::log10(1 + n / c), std::log10(1 + k / c)};
  for (int q = 0; q < kTuneFeatures; ++q) f[q] = (float)v[q];
}

int mfgpu_tune_features(mfgpu_ctx* h, int64_t nrhs, int64_t* count, float* feats, int64_t cap) {
  if (!h || !count || nrhs < 1) return MFGPU_ERR_ARGUMENT;
  if (!h->analyzed) return fail(h, MFGPU_ERR_STATE, "tune features before analyze");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    const Plan& P = h->plan;
    build_solve_schedule(h, nrhs, 4);
    const SolveSchedule& S = h->sched;
    std::vector<float> f;
    float row[kTuneFeatures];
    for (const Launch& L : P.launches)
      if (L.kind == kLaunchGemm) {
        tune_row(row, 0, P.gemm_tasks.data() + L.first, L.count, L.flops, L.elems, L.tiles, L.tiles_tc);
        f.insert(f.end(), row, row + kTuneFeatures);
      }
    for (const InvStep& is : P.inv_steps) {
      tune_row(row, 1, P.inv_tasks.data() + is.first, is.count, is.flops, is.elems, is.tiles, is.tiles_tc);
      f.insert(f.end(), row, row + kTuneFeatures);
    }
    for (const auto& st : S.steps)
      if (st.kind == 3) {
        if (st.sp_count)   // the K-chunked form is the one that runs
          tune_row(row, 2, S.sgemms.data() + st.sp_first, st.sp_count, st.flops, st.elems, st.sp_tiles,
                   st.sp_tiles_tc);
        else
          tune_row(row, 2, S.gemms.data() + st.first, st.count, st.flops, st.elems, st.tiles, st.tiles_tc);
        f.insert(f.end(), row, row + kTuneFeatures);
      }
    *count = (int64_t)f.size() / kTuneFeatures;
    if (feats) {
      if (cap < (int64_t)f.size()) return fail(h, MFGPU_ERR_ARGUMENT, "feature buffer too small");
      std::memcpy(feats, f.data(), f.size() * sizeof(float));
    }
    return MFGPU_OK;
  });
}

int mfgpu_tune_set_choice(mfgpu_ctx* h, const int8_t* choice, int64_t count) {
  if (!h || count < 0 || (count && !choice)) return MFGPU_ERR_ARGUMENT;
  for (int64_t i = 0; i < count; ++i)
    if (choice[i] < 0 || choice[i] > 2) return fail(h, MFGPU_ERR_ARGUMENT, "choice must be 0, 1 or 2");
  h->gemm_choice.assign(choice, choice + count);
  ++h->choice_version;
  return MFGPU_OK;
}

int mfgpu_stats_json(mfgpu_ctx* h, char* buf, int64_t cap) {
  if (!h || !buf || cap <= 0) return MFGPU_ERR_ARGUMENT;
  const Plan& P = h->plan;
  int64_t nl = 0, nsmall = 0;
  for (const auto& l : P.launches) {
    ++nl;
    if (l.kind == kLaunchSmall) nsmall += l.count;
  }
  char tmp[2560];
  std::snprintf(tmp, sizeof tmp,
                "{\"n\": %lld, \"nsuper\": %lld, \"levels\": %d, \"nnz_l\": %lld, \"nnz_u\": %lld, "
                "\"max_front\": %d, \"max_pivots\": %d, \"front_elems\": %lld, \"flops\": %.6e, "
                "\"flops_getrf\": %.6e, \"flops_trsm\": %.6e, \"flops_gemm\": %.6e, \"assembly_elem_moves\": %.6e, "
                "\"factor_launches\": %lld, \"small_fronts\": %lld, \"speculative\": %s, \"safe_rerun\": %d, "
                "\"analyze_ms\": %.3f, \"factor_ms\": %.3f, \"solve_ms\": %.3f, \"precision\": \"%s\", "
                "\"status\": %d, \"growth\": %.6e, \"growth_limit\": %.6e, \"refactored_fp64\": %s, "
                "\"flops_inverse\": %.6e, \"lean\": %s, \"pool_elems\": %lld, \"front_elems_full\": %lld, "
                "\"fronts\": %lld, \"merged\": %s, \"flops_exec\": %.6e}",
                (long long)P.n, (long long)(P.merged ? P.ns_orig : P.ns), P.nlevels, (long long)P.nnz_l,
                (long long)P.nnz_u, P.max_nf, P.max_np, (long long)P.front_elems, P.flops_orig, P.flops_getrf,
                P.flops_trsm, P.flops_gemm,
                P.assembly_bytes_per_elem, (long long)nl, (long long)nsmall, P.has_speculative ? "true" : "false",
                h->factor_reruns, h->t_analyze_ms, h->t_factor_ms, h->t_solve_ms,
                h->factor_precision == MFGPU_PRECISION_MIXED ? "mixed" : "fp64", h->last_status, h->growth,
                h->growth_limit, h->refactored_fp64 ? "true" : "false", P.flops_inverse, P.lean ? "true" : "false",
                (long long)P.pool_elems, (long long)P.front_elems_full, (long long)P.ns,
                P.merged ? "true" : "false", P.flops);
  std::string js(tmp);
  js.pop_back();   // reopen the object
  char item[512];
  std::snprintf(item, sizeof item,
                ", \"launches\": %lld, \"graph_replays\": %lld, \"graph_captures\": %lld, \"profiling\": %s, "
                "\"kernels\": {",
                (long long)h->launch_count, (long long)h->graph_replays, (long long)h->graph_captures,
                h->profiling ? "true" : "false");
  js += item;
  bool first = true;
  for (int k = 0; k < KC_COUNT; ++k) {
    const KStat& ks = h->kstat[k];
    if (!ks.launches) continue;
    std::snprintf(item, sizeof item, "%s\"%s\": {\"ms\": %.6f, \"launches\": %lld, \"flops\": %.6e, \"bytes\": %.6e}",
                  first ? "" : ", ", kKernelClassName[k], ks.ms, (long long)ks.launches, ks.flops, ks.bytes);
    js += item;
    first = false;
  }
  js += "}}";
  if ((int64_t)js.size() >= cap) return MFGPU_ERR_ARGUMENT;
  std::memcpy(buf, js.c_str(), js.size() + 1);
  return MFGPU_OK;
}

int mfgpu_launch_records(mfgpu_ctx* h, char* buf, int64_t cap) {
  if (!h || !buf || cap <= 0) return MFGPU_ERR_ARGUMENT;
  std::string js = "[";
  char item[256];
  for (size_t i = 0; i < h->records.size(); ++i) {
    const auto& r = h->records[i];
    std::snprintf(item, sizeof item, "%s[\"%s\", %d, %lld, %.6f, %.6e, %.6e, %d]", i ? ", " : "",
                  kKernelClassName[r.kc], r.level, (long long)r.tasks, r.ms, r.flops, r.bytes, r.tune);
    js += item;
  }
  js += "]";
  if ((int64_t)js.size() >= cap) return (int)std::min<int64_t>(js.size() + 1, INT32_MAX);
  std::memcpy(buf, js.c_str(), js.size() + 1);
  return MFGPU_OK;
}

int mfgpu_set_profiling(mfgpu_ctx* h, int32_t on) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  h->records.clear();
  h->profiling = on != 0;
  h->launch_count = 0;
  for (auto& k : h->kstat) k = KStat{};
  h->pending.clear();
  h->pending_phases.clear();
  h->stamp_next = 0;
  h->evnext = 0;
  return MFGPU_OK;
}

}  // extern "C"

// ===========================================================================
// Backward error without device allocation.
//
// mfgpu_backward_error_device allocates a residual buffer the first time it
// sees a size.  Some callers cannot allocate device memory when they check
// accuracy: services that reserve all device memory when they start (behind a
// caching allocator or a fixed budget), and latency-sensitive loops that must
// not take cudaMalloc's device-wide synchronisation.  This variant never
// stores the residual; per right-hand side it reduces max|b - A x|, max|x|,
// max|b| and ||A||_inf into one file-scope __device__ array of fixed size,
// then forms the error on the device and copies one double to the host.
// ===========================================================================
namespace {

constexpr int64_t kNoAllocMaxRhs = 4096;          // right-hand sides per call
constexpr int kNoAllocMaxDevices = 64;
// [3c]: max|r_c|, [3c+1]: max|x_c|, [3c+2]: max|b_c| (as ordered bits of
// non-negative doubles), [3*max]: ||A||_inf, [3*max+1]: result.
// Every GPU that loads the library holds these 98 KB until the process exits.
__device__ __align__(256) unsigned long long g_noalloc_scratch[3 * kNoAllocMaxRhs + 2];

std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (the current device); the
// symbol's name in host code is only a stand-in, so kernels get this address.
void* noalloc_scratch(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) throw std::invalid_argument("device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_ptr[device] = p;
  }
  return g_noalloc_ptr[device];
}

// Per right-hand side: max|b - A x|, max|x|, max|b| of a 256-row slice of
// one column per CTA (grid: row slices x columns).  The residual of each row
// is formed in registers with k_residual's arithmetic (same order, so the
// same bits) and never stored; the slice is reduced in the CTA and each
// quantity takes one atomicMax per CTA.  A NaN is kept (max_keep_nan).
__global__ void __launch_bounds__(256) k_noalloc_residual_max(int64_t n, int64_t nrhs, const int32_t* __restrict__ rp,
                                                              const int32_t* __restrict__ ci,
                                                              const int32_t* __restrict__ src,
                                                              const double* __restrict__ ax,
                                                              const double* __restrict__ b, int64_t ldb,
                                                              const double* __restrict__ x, int64_t ldx,
                                                              unsigned long long* __restrict__ scratch) {
  __shared__ double red[3][8];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t c = blockIdx.y; c < nrhs; c += gridDim.y) {
    double v[3] = {0.0, 0.0, 0.0};
    if (i < n) {
      double acc = 0.0;
      for (int p = rp[i]; p < rp[i + 1]; ++p) acc += ax[src[p]] * x[ci[p] + c * ldx];
      const double bi = b[i + c * ldb];
      v[0] = fabs(bi - acc);
      v[1] = fabs(x[i + c * ldx]);
      v[2] = fabs(bi);
    }
#pragma unroll
    for (int q = 0; q < 3; ++q)
      for (int o = 16; o > 0; o >>= 1) v[q] = max_keep_nan(v[q], __shfl_xor_sync(0xffffffffu, v[q], o));
    if (lane_id() == 0)
      for (int q = 0; q < 3; ++q) red[q][warp_id()] = v[q];
    __syncthreads();
    if (threadIdx.x < 3) {
      double m = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = max_keep_nan(m, red[threadIdx.x][w]);
      atomicMax(scratch + 3 * c + threadIdx.x, (unsigned long long)__double_as_longlong(m));
    }
    __syncthreads();
  }
}

// The largest backward error over the right-hand sides, folded by
// worst_eta (a NaN in any column makes the result NaN), into the result slot.
__global__ void k_noalloc_finish(int64_t nrhs, unsigned long long* __restrict__ scratch) {
  __shared__ double red[256];
  const double anorm = __longlong_as_double((long long)scratch[3 * kNoAllocMaxRhs]);
  double worst = 0.0;
  for (int64_t c = threadIdx.x; c < nrhs; c += blockDim.x) {
    const double r = __longlong_as_double((long long)scratch[3 * c]);
    const double xn = __longlong_as_double((long long)scratch[3 * c + 1]);
    const double bn = __longlong_as_double((long long)scratch[3 * c + 2]);
    worst = worst_eta(worst, r, anorm * xn + bn);
  }
  red[threadIdx.x] = worst;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = max_keep_nan(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) scratch[3 * kNoAllocMaxRhs + 1] = (unsigned long long)__double_as_longlong(red[0]);
}

}  // namespace

extern "C" int mfgpu_backward_error_noalloc(mfgpu_ctx* h, int64_t nrhs, const double* d_b, int64_t ldb,
                                            const double* d_x, int64_t ldx, double* out) {
  if (!h || !out) return MFGPU_ERR_ARGUMENT;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "no matrix values (factor first)");
  if (h->c64_factors) return fail(h, MFGPU_ERR_STATE, "real vectors only: the factorization is complex");
  if (nrhs < 1 || nrhs > kNoAllocMaxRhs)
    return fail(h, MFGPU_ERR_ARGUMENT, "mfgpu_backward_error_noalloc: nrhs must be in 1.." +
                                           std::to_string(kNoAllocMaxRhs));
  if (h->plan.n == 0) {   // a 0 x 0 system: nothing to launch, as mfgpu_backward_error_device
    *out = 0.0;
    return MFGPU_OK;
  }
  if (!d_b || !d_x) return fail(h, MFGPU_ERR_ARGUMENT, "null vectors");
  if (ldb < h->plan.n || ldx < h->plan.n) return fail(h, MFGPU_ERR_ARGUMENT, "leading dimension below n");
  return guarded(h, [&]() -> int {
    CK(cudaSetDevice(h->device));
    unsigned long long* scratch = static_cast<unsigned long long*>(noalloc_scratch(h->device));
    const Plan& P = h->plan;
    cudaStream_t st = h->stream;
    const int64_t n = P.n;
    CK(cudaMemsetAsync(scratch, 0, sizeof(unsigned long long) * (3 * kNoAllocMaxRhs + 2), st));
    k_noalloc_residual_max<<<dim3((unsigned)((n + 255) / 256), (unsigned)nrhs), 256, 0, st>>>(
        n, nrhs, h->b_csr_ptr.as<int32_t>(), h->b_csr_col.as<int32_t>(), h->b_csr_src.as<int32_t>(),
        h->b_ax.as<double>(), d_b, ldb, d_x, ldx, scratch);
    k_norm_inf<<<grid1(n, 256), 256, 0, st>>>(n, h->b_csr_ptr.as<int32_t>(), h->b_csr_src.as<int32_t>(),
                                              h->b_ax.as<double>(), scratch + 3 * kNoAllocMaxRhs);
    k_noalloc_finish<<<1, 256, 0, st>>>(nrhs, scratch);
    CK(cudaGetLastError());
    unsigned long long bits = 0;
    CK(cudaMemcpyAsync(&bits, scratch + 3 * kNoAllocMaxRhs + 1, sizeof bits, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::memcpy(out, &bits, sizeof bits);
    return MFGPU_OK;
  });
}

// ---- batched systems ------------------------------------------------------
// Many independent systems go through one handle as one block-diagonal
// matrix: each system is ordered by itself and the symbolic pass of the
// block-diagonal pattern under the concatenated orders is a forest holding
// every system's own elimination tree, supernodes and update sets (column
// offsets aside).  Each level-batched launch then factors the fronts of all
// systems at that tree level together, and the per-level sequence is
// replayed from one CUDA graph.  Every system's factors are exactly those of
// splu(A_i; method=:multifrontal) (src/interface.jl:93-120) or of
// multifrontal_lu(A_i; q=colamd_order(A_i)) (src/multifrontal.jl:152).
namespace {

int batch_fetch_factors(mfgpu_ctx* h) {
  auto& B = h->batch;
  if (B.have_factors) return MFGPU_OK;
  const Plan& P = h->plan;
  B.lcolptr.resize(P.n + 1);
  B.ucolptr.resize(P.n + 1);
  B.lrowval.resize(P.nnz_l);
  B.lnzval.resize(P.nnz_l);
  B.urowval.resize(P.nnz_u);
  B.unzval.resize(P.nnz_u);
  B.p.resize(P.n);
  B.q.resize(P.n);
  const int rc = mfgpu_get_factors(h, B.lcolptr.data(), B.lrowval.data(), B.lnzval.data(), B.ucolptr.data(),
                                   B.urowval.data(), B.unzval.data(), B.p.data(), B.q.data(), nullptr);
  if (rc == MFGPU_OK) B.have_factors = true;
  return rc;
}

}  // namespace

extern "C" int mfgpu_batch_analyze(mfgpu_ctx* h, int64_t nsys, const int64_t* n, const int64_t* const* colptr,
                                   const int64_t* const* rowval, int32_t ordering) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  if (nsys < 1 || !n || !colptr || !rowval) return fail(h, MFGPU_ERR_ARGUMENT, "batch: no systems");
  if (ordering != MFGPU_ORDER_AMD && ordering != MFGPU_ORDER_COLAMD)
    return fail(h, MFGPU_ERR_ARGUMENT, "batch: ordering must be MFGPU_ORDER_AMD or MFGPU_ORDER_COLAMD");
  return guarded(h, [&]() -> int {
    auto& B = h->batch;
    B.nsys = 0;
    B.off.clear();
    B.nz_off.clear();
    B.colptr.clear();
    B.rowval.clear();
    B.super_sys.clear();
    B.have_factors = false;
    B.off.assign(nsys + 1, 0);
    B.nz_off.assign(nsys + 1, 0);
    for (int64_t i = 0; i < nsys; ++i) {
      if (n[i] < 1 || !valid_csc(n[i], colptr[i], rowval[i]))
        return fail(h, MFGPU_ERR_ARGUMENT, "batch: system " + std::to_string(i + 1) + " is not a valid square CSC");
      B.off[i + 1] = B.off[i] + n[i];
      B.nz_off[i + 1] = B.nz_off[i] + colptr[i][n[i]] - 1;
    }
    const int64_t N = B.off[nsys];
    B.colptr.resize(N + 1);
    B.rowval.resize(B.nz_off[nsys]);
    B.colptr[0] = 1;
    parallel_for(nsys, [&](int64_t i) {
      const int64_t o = B.off[i], z = B.nz_off[i], ni = n[i];
      for (int64_t j = 1; j <= ni; ++j) B.colptr[o + j] = z + colptr[i][j];
      for (int64_t k = 0; k < colptr[i][ni] - 1; ++k) B.rowval[z + k] = rowval[i][k] + o;
    });
    // orderings and symbolic analyses per system on all host cores, then one
    // block-diagonal forest
    mfgpu_symbolic* sym = nullptr;
    int rc = mfgpu_symbolic_create_batch(nsys, n, colptr, rowval, ordering, &sym);
    if (rc != MFGPU_OK) return fail(h, rc, std::string("batch: symbolic analysis failed: ") + mfgpu_host_last_error());
    std::unique_ptr<mfgpu_symbolic, void (*)(mfgpu_symbolic*)> guard(sym, mfgpu_symbolic_destroy);
    // the forest keeps every system's columns together and in system order
    const auto& S = sym->s;
    const int64_t ns = S.nsuper();
    B.super_sys.resize(ns);
    int64_t sys = 0;
    for (int64_t s = 0; s < ns; ++s) {
      while (S.sstart[s] >= B.off[sys + 1]) ++sys;
      if (S.sstart[s + 1] > B.off[sys + 1]) return fail(h, MFGPU_ERR_INTERNAL, "batch: supernode spans two systems");
      B.super_sys[s] = (int32_t)sys;
    }
    for (int64_t i = 0; i < nsys; ++i)
      for (int64_t k = B.off[i]; k < B.off[i + 1]; ++k)
        if (S.qf[k] < B.off[i] || S.qf[k] >= B.off[i + 1])
          return fail(h, MFGPU_ERR_INTERNAL, "batch: postorder mixes systems");
    rc = mfgpu_analyze_symbolic(h, N, B.colptr.data(), B.rowval.data(), sym);
    if (rc != MFGPU_OK) {
      h->batch.nsys = 0;
      return rc;
    }
    // system of every front (merged fronts stay inside one system's tree)
    const Plan& P = h->plan;
    B.super_sys.resize(P.ns);
    sys = 0;
    for (int64_t x = 0; x < P.ns; ++x) {
      while (P.c1[x] >= B.off[sys + 1]) ++sys;
      B.super_sys[x] = (int32_t)sys;
    }
    B.nsys = nsys;
    return MFGPU_OK;
  });
}

extern "C" int mfgpu_batch_layout(mfgpu_ctx* h, int64_t* nsys, int64_t* col_off, int64_t* nz_off) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  const auto& B = h->batch;
  if (!B.nsys) return fail(h, MFGPU_ERR_STATE, "no batch analyzed");
  if (nsys) *nsys = B.nsys;
  for (int64_t i = 0; i <= B.nsys; ++i) {
    if (col_off) col_off[i] = B.off[i];
    if (nz_off) nz_off[i] = B.nz_off[i];
  }
  return MFGPU_OK;
}

extern "C" int mfgpu_batch_factor(mfgpu_ctx* h, const double* const* nzval, int32_t scale, int32_t check,
                                  int64_t* status) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  auto& B = h->batch;
  if (!B.nsys) return fail(h, MFGPU_ERR_STATE, "batch factor before batch analyze");
  if (!nzval || scale < MFGPU_SCALE_NONE || scale > MFGPU_SCALE_MAX)
    return fail(h, MFGPU_ERR_ARGUMENT, "batch: bad values or scale kind");
  return guarded(h, [&]() -> int {
    const int64_t N = B.off[B.nsys];
    B.nz.ensure(std::max<int64_t>(B.nz_off[B.nsys], 1) * sizeof(double));
    for (int64_t i = 0; i < B.nsys; ++i)
      if (B.nz_off[i + 1] > B.nz_off[i] && !nzval[i])
        return fail(h, MFGPU_ERR_ARGUMENT, "batch: null values for system " + std::to_string(i + 1));
    parallel_for(B.nsys, [&](int64_t i) {
      const int64_t cnt = B.nz_off[i + 1] - B.nz_off[i];
      if (cnt) std::memcpy(B.nz.d() + B.nz_off[i], nzval[i], cnt * sizeof(double));
    });
    (void)N;
    const int rc = mfgpu_factor_scaled(h, B.nz.d(), scale, 0);   // row scaling computed on the device
    if (rc < 0) return rc;
    // per system: the first supernode (postorder) with a zero pivot
    std::vector<int64_t> st(B.nsys, 0);
    int64_t singular = 0;
    const Plan& P = h->plan;
    for (int64_t s = 0; s < (int64_t)h->last_info.size(); ++s) {
      if (h->last_info[s] == INT32_MAX) continue;
      const int32_t sys = B.super_sys[s];
      if (st[sys] == 0) {
        st[sys] = (int64_t)P.c1[s] + h->last_info[s] + 1 - B.off[sys];
        ++singular;
      }
    }
    if (status) std::copy(st.begin(), st.end(), status);
    return check ? (int)singular : MFGPU_OK;
  });
}

extern "C" int mfgpu_batch_solve(mfgpu_ctx* h, int64_t nrhs, const double* const* b, double* const* x,
                                 int32_t refine) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  auto& B = h->batch;
  if (!B.nsys) return fail(h, MFGPU_ERR_STATE, "batch solve before batch analyze");
  if (nrhs < 0 || refine < 0 || (nrhs && (!b || !x))) return fail(h, MFGPU_ERR_ARGUMENT, "batch: bad solve sizes");
  if (nrhs == 0) return MFGPU_OK;
  return guarded(h, [&]() -> int {
    const int64_t N = B.off[B.nsys];
    B.b.ensure(N * nrhs * sizeof(double));
    B.x.ensure(N * nrhs * sizeof(double));
    for (int64_t i = 0; i < B.nsys; ++i)
      if (!b[i] || !x[i]) return fail(h, MFGPU_ERR_ARGUMENT, "batch: null rhs or solution for system " + std::to_string(i + 1));
    parallel_for(B.nsys, [&](int64_t i) {
      const int64_t o = B.off[i], ni = B.off[i + 1] - o;
      for (int64_t k = 0; k < nrhs; ++k) std::memcpy(B.b.d() + k * N + o, b[i] + k * ni, ni * sizeof(double));
    });
    const int rc = mfgpu_solve(h, nrhs, B.b.d(), N, B.x.d(), N, refine);
    if (rc != MFGPU_OK) return rc;
    parallel_for(B.nsys, [&](int64_t i) {
      const int64_t o = B.off[i], ni = B.off[i + 1] - o;
      for (int64_t k = 0; k < nrhs; ++k) std::memcpy(x[i] + k * ni, B.x.d() + k * N + o, ni * sizeof(double));
    });
    return MFGPU_OK;
  });
}

extern "C" int mfgpu_batch_factor_sizes(mfgpu_ctx* h, int64_t sys, int64_t* out3) {
  if (!h || !out3) return MFGPU_ERR_ARGUMENT;
  auto& B = h->batch;
  if (!B.nsys || !h->factored) return fail(h, MFGPU_ERR_STATE, "no batch factorization");
  if (sys < 0 || sys >= B.nsys) return fail(h, MFGPU_ERR_ARGUMENT, "batch: system index out of range");
  const Plan& P = h->plan;
  const int64_t a = B.off[sys], e = B.off[sys + 1];
  out3[0] = e - a;
  out3[1] = (int64_t)P.lcolptr[e] - P.lcolptr[a];
  out3[2] = (int64_t)P.ucolptr[e] - P.ucolptr[a];
  return MFGPU_OK;
}

extern "C" int mfgpu_batch_get_factors(mfgpu_ctx* h, int64_t sys, int64_t* lcolptr, int64_t* lrowval,
                                       double* lnzval, int64_t* ucolptr, int64_t* urowval, double* unzval,
                                       int64_t* p, int64_t* q, int64_t* pinv) {
  if (!h) return MFGPU_ERR_ARGUMENT;
  auto& B = h->batch;
  if (!B.nsys || !h->factored) return fail(h, MFGPU_ERR_STATE, "no batch factorization");
  if (sys < 0 || sys >= B.nsys) return fail(h, MFGPU_ERR_ARGUMENT, "batch: system index out of range");
  return guarded(h, [&]() -> int {
    const int rc = batch_fetch_factors(h);
    if (rc != MFGPU_OK) return rc;
    const int64_t a = B.off[sys], ni = B.off[sys + 1] - a;
    const int64_t l0 = B.lcolptr[a] - 1, u0 = B.ucolptr[a] - 1;
    for (int64_t j = 0; j <= ni; ++j) {
      if (lcolptr) lcolptr[j] = B.lcolptr[a + j] - l0;
      if (ucolptr) ucolptr[j] = B.ucolptr[a + j] - u0;
    }
    const int64_t nl = B.lcolptr[a + ni] - 1 - l0, nu = B.ucolptr[a + ni] - 1 - u0;
    for (int64_t k = 0; k < nl; ++k) {
      if (lrowval) lrowval[k] = B.lrowval[l0 + k] - a;
      if (lnzval) lnzval[k] = B.lnzval[l0 + k];
    }
    for (int64_t k = 0; k < nu; ++k) {
      if (urowval) urowval[k] = B.urowval[u0 + k] - a;
      if (unzval) unzval[k] = B.unzval[u0 + k];
    }
    for (int64_t k = 0; k < ni; ++k) {
      const int64_t pk = B.p[a + k] - a;
      if (p) p[k] = pk;
      if (q) q[k] = B.q[a + k] - a;
      if (pinv) pinv[pk - 1] = k + 1;
    }
    return MFGPU_OK;
  });
}
