// plan.h -- pattern-only analysis that turns a symbolic factorization into
// the device schedule of libmfgpu's numeric factorization and solves.
//
// Everything here depends on the sparsity pattern only (the part of
// src/multifrontal.jl:152-196 that does not touch values): front sizes and
// pool offsets, the map of every entry of V = A[qf,qf] to its front position
// (src/multifrontal.jl:217-231), the extend-add maps of every child
// contribution block (src/multifrontal.jl:45-57, 235-243), the CSC offsets
// of the factors (src/multifrontal.jl:73-104, 278-317), and the level-batched
// launch sequence.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace mfgpu {

// Front size limits of the kernel classes.
constexpr int kSmallFront = 64;      // fronts with nf <= this are factored in one CTA, in shared memory
constexpr int kPanel = 64;           // panel width of the blocked large-front factorization
// Largest pivot block a merged front may get: the explicit pivot-block
// inverses cost (4/3) np^3, so merging into already large supernodes would
// cost more than the hand-overs it saves (64^3 Poisson: 0.31 TFLOP of
// inverses with this limit, 1.06 without).
constexpr int64_t kMergeMaxPivots = 1024;
constexpr int kPivRowsSmem = 256;    // pivot rows a partial-pivoting panel keeps in shared memory
// Pivot-block columns whose panel updates are applied together beyond the
// block (blocked right-looking LU; a multiple of the 64-column panel).
constexpr int32_t kUpdateBlock = 256;
constexpr int kTcTile = 128;         // tile edge of the tensor-core GEMM of the FP32 fronts

enum PanelMode : int32_t {
  kPanelSmemPivot = 0,   // rows k0..np-1 in shared memory, LAPACK partial pivoting
  kPanelSpeculative = 1, // diagonal block only, no interchanges, exact pivot-order check
  kPanelGlobalPivot = 2  // rows k0..np-1 in global memory, LAPACK partial pivoting
};

struct PanelTask {       // one panel step of one large front
  int32_t s;             // supernode
  int32_t k0;            // first panel column
  int32_t mode;          // PanelMode
  int32_t pad;
};

struct TrsmTask {        // triangular solves of one panel step
  int32_t s, k0;
  int32_t r0;            // first row of the L-part solve (k0+kb, or the end of the panel's pivot rows)
  int32_t lrow_tiles;    // 64-row tiles of the L part
  int32_t ucol_tiles;    // 64-column tiles of the U part
  int32_t check;         // speculative: check pivot order on each column's pivot rows
  int64_t tile_base;     // prefix over tasks
};

// A U block of the factor's CSC written from one front column: the rows
// row0 .. row0+rows-1 of the front (one original supernode's pivot rows) go
// to U's CSC at uoff.
struct UBlock {
  int32_t row0, rows;
  int64_t uoff;
};

enum GemmMode : int32_t {
  kGemmSub = 0,          // C = C - A * B
  kGemmSet = 1,          // C = A * B
  kGemmFrom = 2,         // C = D - A * B (D: offset d, leading dimension ldc, same base as C)
  kGemmNeg = 3           // C = -(A * B)
};

struct GemmTask {        // column-major, offsets in elements of the launch's base pointers
  int64_t a, b, c;
  int32_t m, n, k;
  int32_t lda, ldb, ldc;
  int32_t tiles_m, tiles_n;
  int32_t mode;          // GemmMode
  int64_t tile_base;
  int64_t d;             // kGemmFrom: offset of D (same base as C)
  int32_t ldd, pad;      // kGemmFrom: leading dimension of D
};

// A factor GEMM task (FP32 fronts on tensor cores) with its operands split
// once into bf16 parts: byte offsets of the task's A
// and B part tiles in the planes buffer (tiles_m (tiles_n) x kt tiles of
// three kPlaneTileBytes parts each), the prefix of the launch's split units
// ((tiles_m + tiles_n) * kt per task), and its K blocks of 64.
constexpr int64_t kPlaneTileBytes = 128 * 64 * 2;
struct PlaneTask {
  int64_t a_off, b_off;
  int64_t unit_base;
  int32_t kt, pad;
};

// One launch of the blocked inversion of the pivot blocks (both tilings).
struct InvStep {
  int64_t first, count, tiles, tiles_tc;
  double flops, elems;
  int32_t max_k = 0;     // largest K of its tasks
};

enum LaunchKind : int32_t {
  kLaunchSmall = 0,      // fused assemble + factor of small fronts (tasks: supernode ids)
  kLaunchAssemble = 1,   // column-wise assembly of large fronts (front-column range)
  kLaunchPanel = 2,
  kLaunchTrsm = 3,
  kLaunchGemm = 4,
  kLaunchCopyPanels = 5  // lean layout: copy the level's factored panels to the panel pool (front-column range)
};

struct Launch {
  int32_t kind;
  int32_t level;
  int64_t first;         // offset into the task array of this kind (or fc begin)
  int64_t count;         // tasks (or fc count)
  int64_t tiles;         // grid size in tiles for TRSM / GEMM
  int64_t tiles_tc = 0;  // GEMM launches: grid size in 128 x 128 tensor-core tiles
  int32_t rows = 0;      // panel launches: row capacity (threads) of the kernel variant
  int32_t max_k = 0;     // GEMM launches: largest K of its tasks
  double flops = 0;      // algorithmic flops of the launch
  double elems = 0;      // algorithmic element moves (x sizeof(front type) = bytes)
  double extra_bytes = 0;// index / FP64 input bytes
  int64_t split_units = 0, planes_bytes = 0;   // GEMM launches: the operand split (plane_tasks): units, bytes
};

struct Plan {
  int64_t n = 0, ns = 0, nnz_a = 0;
  // per supernode (postorder id)
  std::vector<int32_t> c1, np, nu, nf, height, slot;
  std::vector<int64_t> upd_off, front_off, colbase;
  std::vector<int32_t> child_ptr, child_idx, parent_super;
  // per update-set entry (parallel arrays, sum of nu entries)
  std::vector<int32_t> upd;           // V index of the update row/column
  std::vector<int32_t> rel;           // its position in the parent's front
  std::vector<int64_t> uoff;          // 0-based offset of this (supernode, column) block in U's CSC
  // V = A[qf, qf] built from A's values
  std::vector<int32_t> v_src;         // A.nzval index of each V entry
  std::vector<int32_t> v_srow;        // original row (for Rs)
  std::vector<int32_t> v_frow;        // front row of each V entry
  // per front column, in slot order
  std::vector<int32_t> fc_super;      // owning supernode
  std::vector<int32_t> fc_vbeg, fc_vend;  // V entries assembled into this column
  std::vector<int32_t> fc_ch_ptr;     // children contributions (child, child column)
  std::vector<int32_t> fc_ch;         // pairs, flattened
  int64_t fc_total = 0;
  int64_t front_elems = 0;              // working fronts; the pool also holds panels (lean), inverses, scratch
  int64_t front_elems_full = 0;         // sum of nf^2: every front resident at once
  int64_t pool_elems = 0;               // fronts + panels + inverses + inversion scratch
  // Factored panels, where the solves, the inversion and the CSC scatter read
  // them: the first np columns of the front (leading dimension nf) at
  // lpan_off[s], U12 (np x nu) at u12_off[s] with leading dimension u12 ld =
  // lean ? np : nf.  Without `lean` these point into the resident fronts;
  // with it the fronts' memory is reused once their parent has assembled
  // their contribution block, and every factored front copies its panel to a
  // compact panel pool at the end of its level.
  bool lean = false;
  std::vector<int64_t> lpan_off, u12_off;
  int64_t panel_base = 0, panel_elems = 0;
  // levels / slots
  int32_t nlevels = 0;
  std::vector<int32_t> slot_super;
  std::vector<int32_t> level_slot;    // nlevels+1
  std::vector<int32_t> level_large;   // first large slot of each level
  // factor CSC (0-based pointers)
  std::vector<int64_t> lcolptr, ucolptr;
  int64_t nnz_l = 0, nnz_u = 0;
  // qf (0-based) and original A in CSR for the residual
  std::vector<int32_t> qf;
  std::vector<int32_t> csr_ptr, csr_col, csr_src;
  // inverted 64x64 diagonal blocks of the large fronts' pivot blocks
  std::vector<int64_t> dinv_off;      // per supernode, -1 for small fronts
  int64_t dinv_blocks = 0;
  // explicit inverses of the large fronts' pivot blocks, kept after the
  // fronts in the front pool: inv(L11) (np x np, leading dimension np) at
  // inv_off[s], inv(U11) right after it; the blocked inversion merges the
  // inverted 64 x 64 diagonal blocks pairwise (64 -> 128 -> ...), each merge
  // level one GEMM launch for the products with the off-diagonal block and
  // one for the negated products with the other inverse, through a scratch
  // area after the inverses.
  std::vector<int64_t> inv_off;       // per supernode, -1 for small fronts
  int64_t inv_base = 0, inv_elems = 0, inv_scratch = 0, inv_scratch_elems = 0;
  std::vector<int32_t> inv_blocks;    // (supernode, 64-block) pairs, flattened, for the diagonal-block copy
  std::vector<GemmTask> inv_tasks, inv_tasks_tc;
  std::vector<InvStep> inv_steps;
  double flops_inverse = 0;
  // launch sequences
  std::vector<int32_t> small_tasks;
  std::vector<PanelTask> panel_tasks;
  std::vector<TrsmTask> trsm_tasks;
  std::vector<GemmTask> gemm_tasks;
  std::vector<GemmTask> gemm_tasks_tc;   // the same updates tiled 128 x 128 (FP32 fronts, tensor cores)
  std::vector<PlaneTask> plane_tasks;    // per gemm_tasks_tc entry
  int64_t planes_bytes = 0;              // largest planes buffer of one GEMM launch
  std::vector<Launch> launches;
  bool has_speculative = false;
  // Front merging (execution only).  Chains of supernodes (a child whose
  // columns end right before its parent's) are factored as one front, which
  // saves the child's contribution-block hand-over and the launches of a
  // tree level; the merged front stores the child's logical zeros.  The
  // factor keeps the original supernodes: pivots are searched only among
  // the pivot rows of the column's original supernode (seg_end), and the CSC
  // layout and scatter follow the original structure.  Without merging,
  // seg_end[j] is np of j's front and the o_* arrays stay empty.
  bool merged = false;
  int64_t ns_orig = 0;
  std::vector<int32_t> seg_end;        // per column: front-local end of its pivot-row segment
  std::vector<int32_t> col_orig;       // per column: original supernode
  std::vector<int32_t> o_c1, o_np;     // per original supernode
  std::vector<int64_t> o_upd_off;      // ns_orig + 1
  std::vector<int32_t> o_upd;          // original update sets
  std::vector<int32_t> o_xpos;         // front-local column of each update-set entry
  std::vector<int64_t> fcu_ptr;        // per front column (fc_total + 1)
  std::vector<UBlock> fcu;             // U blocks written from each front column
  double flops_orig = 0;               // flops of the original structure (no merged zeros)
  std::vector<int64_t> front_nv;       // original entries assembled into each front
  // statistics
  double flops = 0, flops_getrf = 0, flops_trsm = 0, flops_gemm = 0;
  double assembly_bytes_per_elem = 0;  // sum of nf^2 + 3 m^2 + nu^2 element moves (x sizeof(T) for bytes)
  int32_t max_nf = 0, max_np = 0;
};

// Checks a caller's symbolic analysis before anything is indexed by it:
// sstart partitions 0..n-1 into nonempty supernodes, upd_ptr is a monotone
// pointer array from 0, every update set holds sorted rows below its
// supernode, parent is an elimination tree (-1 or a later column) and qf a
// permutation.  Throws std::invalid_argument.  Both plan builders call it;
// the consistency of A's pattern with the fronts is checked while the maps
// are built.
void check_symbolic(int64_t n, const int64_t* qf, const int64_t* parent, int64_t ns, const int64_t* sstart,
                    const int64_t* upd_ptr, const int64_t* upd_idx);

// Build the plan.  All inputs 0-based: A pattern (n x n CSC), qf, parent
// (-1 = root), sstart (ns+1), upd_ptr (ns+1), upd_idx.
// `safe` replaces speculative panels by global-memory partial pivoting.
void build_plan(int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf, const int64_t* parent,
                int64_t ns, const int64_t* sstart, const int64_t* upd_ptr, const int64_t* upd_idx, Plan& plan);

// The plan with front merging: the supernodes that amalgamation_marks
// merges (up to max_pivots columns each) are factored as one front; the
// factor's structure, pivot segments and CSC scatter stay those of (sstart,
// upd_ptr, upd_idx).  Falls back to build_plan when nothing merges.
void build_plan_merged(int64_t n, const int64_t* colptr, const int64_t* rowval, const int64_t* qf,
                       const int64_t* parent, int64_t ns, const int64_t* sstart, const int64_t* upd_ptr,
                       const int64_t* upd_idx, Plan& plan, int64_t max_pivots);

// (Re)build the launch sequence: speculative panels, or only pivoting ones.
void build_launches(Plan& plan, bool safe);

// Choose the memory layout: every front resident (lean = false), or working
// fronts placed by lifetime with a compact panel pool (lean = true).  Sets
// front offsets, panel offsets, the inverses' layout and steps, the pool
// size, and rebuilds the launch sequence.
void set_layout(Plan& plan, bool lean);

inline int32_t u12_ld(const Plan& P, int32_t s) { return P.lean ? P.np[s] : P.nf[s]; }

}  // namespace mfgpu
