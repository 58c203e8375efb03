/*
 * cbm_b200.h - C ABI of the B200 CBM (Compressed Binary Matrix) library.
 *
 * A binary adjacency matrix A (N x N) is stored as
 *   - a delta matrix D (CSR, values +-1): row v = A[v] - A[parent(v)], or A[v]
 *     when v hangs from the virtual root;
 *   - a compression tree (a forest over the rows) given as branch offsets and
 *     (parent, child) edges in BFS order per branch.
 * The product is Y = D*X followed by Y[v] += Y[parent(v)] from the roots down.
 *
 * Every function returns CBM_OK (0) or a status code; cbm_status_string()
 * names it.  No function takes or returns framework (torch) types: pointers are
 * plain host or device addresses, sizes are element counts, and `stream` is a
 * cudaStream_t passed as void*.
 *
 * Reference interfaces replaced (paths within cbm4scale/CBM-GPU):
 *   cbm_build / cbm_structure_*       cbm_init_                cbm/cbm_extensions.cpp:60-345
 *   cbm_plan_create                   cusparseCBM::cusparseCBM cbm/cbm.cu:95-142
 *   cbm_plan_destroy                  cusparseCBM::~cusparseCBM cbm/cbm.cu:144-147
 *   cbm_matmul(CBM_OP_VALUES_ADD)     cusparseCBM::matmul_AX_ADX   cbm/cbm.cu:150-207
 *   cbm_matmul(CBM_OP_VALUES_RATIO)   cusparseCBM::matmul_DAX_DADX cbm/cbm.cu:210-268
 *   cbm_matmul(CBM_OP_AX/ADX/DADX)    cbm4mm.matmul / cbm4ad.matmul / cbm4dad.matmul
 *                                     (cbm/cbm4mm.py:53-54, cbm/cbm4ad.py via cbm4mm,
 *                                      cbm/cbm4dad.py:53-54) with the D^-1/2 scaling
 *                                     applied on the fly instead of pre-scaled values
 *                                     (cbm/cbm4ad.py:19-25, cbm/cbm4dad.py:19-34)
 *   cbm_matmul_adjoint                no counterpart: A^T*G in CBM form (autograd)
 *   cbm_s_*_csr_int32                 the cbm_mkl_cpp operators    cbm/cbm_extensions.cpp:351-919
 *                                     (stateless, on the reference's layout; one line each below)
 */
#ifndef CBM_B200_H
#define CBM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  CBM_OK = 0,
  CBM_ERR_INVALID = 1,     /* null pointer, negative size, bad enum */
  CBM_ERR_INDEX = 2,       /* an index outside [0, n) */
  CBM_ERR_ALLOC = 3,       /* host or device allocation failed */
  CBM_ERR_CUDA = 4,        /* a CUDA runtime call failed */
  CBM_ERR_STRUCTURE = 5,   /* not a forest / duplicate child / bad offsets */
  CBM_ERR_DTYPE = 6,       /* unsupported dtype combination */
  CBM_ERR_SHAPE = 7,       /* leading dimension < columns or >= 2^31, aliasing x and y */
  CBM_ERR_TIMEOUT = 8,     /* a device wait ran out (see cbm_plan_error) */
  CBM_ERR_UNSUPPORTED = 9, /* op needs multipliers / values the plan lacks */
  CBM_ERR_WORKSPACE = 10,  /* workspace smaller than cbm_plan_workspace_bytes */
  CBM_ERR_INTERNAL = 11,
  CBM_ERR_TOO_LARGE = 12   /* beyond cbm_matmul_noalloc's fixed scratch (CBM_NOALLOC_MAX_ROWS) */
};

/* ---- dtypes and ops ------------------------------------------------------ */
enum { CBM_F32 = 0, CBM_BF16 = 1 };

enum {
  CBM_OP_AX = 0,          /* Y = A X             (signs only)                     */
  CBM_OP_ADX = 1,         /* Y = A D^-1/2 X      (signs, D[col] on the fly)       */
  CBM_OP_DADX = 2,        /* Y = D^-1/2 A D^-1/2 X (signs, D[col]*D[row], ratio)  */
  CBM_OP_VALUES_ADD = 3,  /* Y = Dv X; Y[v] += Y[u]            (matmul_AX_ADX)   */
  CBM_OP_VALUES_RATIO = 4, /* Y = Dv X; Y[v] += Y[u]*m[v]/m[u]  (matmul_DAX_DADX) */
  CBM_OP_DAD_ADD = 5,      /* entries s*m[col]*m[row], Y[v] += Y[u]: what matmul_AX_ADX
                              computes on the values cbm4dad prepares                 */
  CBM_OP_GIN = 6           /* Y = A X + (1 + eps) X: cbm_matmul_gin only (its workspace
                              query uses this op)                                      */
};

/* ---- construction (host, OpenMP) ----------------------------------------- */
typedef struct cbm_structure cbm_structure;

enum { CBM_BUILD_EXHAUSTIVE = 1 }; /* every pair sharing a column (for checks) */

/* Builds delta matrix + tree from COO (row, col) of a binary N x N matrix.
 * Replaces cbm_init_ (cbm/cbm_extensions.cpp:60-345). n_threads <= 0: all. */
int cbm_build(const int32_t* row, const int32_t* col, int64_t nnz, int64_t n_rows, int64_t alpha,
              int32_t n_threads, int32_t flags, cbm_structure** out);

/* cbm_build with every row's parent restricted to rows of the same cluster
 * (cluster: int32 [n_rows], any ids): the forest is the union of the
 * per-cluster CBMs that the reference's LSH clustering builds one by one
 * (benchmark/clustering_gpu.py:184-195, cbm4mm per cluster), so one plan and
 * one launch serve every cluster.  NULL cluster = cbm_build. */
int cbm_build_clustered(const int32_t* row, const int32_t* col, int64_t nnz, int64_t n_rows, int64_t alpha,
                        const int32_t* cluster, int32_t n_threads, int32_t flags, cbm_structure** out);

/* COO -> CSR with sorted, unique columns per row, the canonical form the
 * constructor works on (the reference's mkl_sparse_convert_csr,
 * cbm/cbm_extensions.cpp:70-98).  flags: CBM_COALESCE_SYMMETRIZE adds every
 * edge's transpose, CBM_COALESCE_DROP_SELF drops (i, i).  ptr: int64 [n+1];
 * out_col: capacity nnz (2 nnz with SYMMETRIZE).  Host, OpenMP. */
enum { CBM_COALESCE_SYMMETRIZE = 1, CBM_COALESCE_DROP_SELF = 2 };
int cbm_coalesce(const int32_t* row, const int32_t* col, int64_t nnz, int64_t n, int32_t flags, int64_t* ptr,
                 int32_t* out_col, int64_t* out_nnz);

/* The six arrays cbm_init_ returns (cbm/cbm_extensions.cpp:301-344), in its
 * order, then extras: the delta matrix as CSR (rows sorted, one block per row),
 * the parent of each node (N = virtual root), and counters. */
enum {
  CBM_S_DELTA_ROW = 0, /* int32 [Z]   child id of each delta entry            */
  CBM_S_DELTA_COL = 1, /* int32 [Z]                                           */
  CBM_S_DELTA_VAL = 2, /* float [Z]   +-1                                     */
  CBM_S_BRANCHES = 3,  /* int32 [B+1] prefix sums of edges per branch         */
  CBM_S_SRC = 4,       /* int32 [E]   parent of each tree edge (BFS order)    */
  CBM_S_DST = 5,       /* int32 [E]   child  of each tree edge                */
  CBM_S_PARENT = 6,    /* int32 [N]                                           */
  CBM_S_CSR_PTR = 7,   /* int32 [N+1]                                         */
  CBM_S_CSR_COL = 8,   /* int32 [Z]                                           */
  CBM_S_CSR_VAL = 9,   /* float [Z]                                           */
  CBM_S_N_CANDIDATES = 100, /* length-only queries */
  CBM_S_TREE_COST = 101,
  CBM_S_NNZ_A = 102,
  CBM_S_SYMMETRIC = 103     /* 1 if A == A^T (then A^T G = A G) */
};
int64_t cbm_structure_len(const cbm_structure* s, int32_t which);
int cbm_structure_copy(const cbm_structure* s, int32_t which, void* dst);
void cbm_structure_free(cbm_structure* s);

/* Host-only check of a delta matrix + tree (CSR row pointers monotone and
 * ending at nnz, columns in range, branch offsets a prefix sum ending at
 * n_edges, parents/children in range, no node with two parents, no cycle).
 * cbm_plan_create runs the same checks.  Host pointers. */
int cbm_validate(const int32_t* row_ptr, const int32_t* col_idx, int64_t n_rows, int64_t n_cols, int64_t nnz,
                 const int32_t* branches, int64_t n_branch_offsets, const int32_t* src, const int32_t* dst,
                 int64_t n_edges);

/* ---- device plan ----------------------------------------------------------- */
typedef struct cbm_plan cbm_plan;

enum {
  CBM_INPUT_DEVICE = 0, /* structure pointers are device addresses */
  CBM_INPUT_HOST = 1    /* structure pointers are host addresses   */
};

/* Uploads the structure in the kernels' layout (rows in tree-level order,
 * column index and sign packed in one word, long rows split in chunks).
 * values (nnz floats) give each entry's sign and, for the VALUES ops, its
 * value; NULL means every entry is +1.  multipliers (N floats, may be NULL)
 * are copied.
 * Replaces cusparseCBM::cusparseCBM (cbm/cbm.cu:95-142). */
int cbm_plan_create(const int32_t* row_ptr, const int32_t* col_idx, const float* values, int64_t n_rows,
                    int64_t n_cols, int64_t nnz, const int32_t* branches, int64_t n_branch_offsets,
                    const int32_t* src, const int32_t* dst, int64_t n_edges, const float* multipliers,
                    int32_t input_kind, void* stream, cbm_plan** out);

/* Copies N multipliers (device pointer) into the plan: D^-1/2 for ADX/DADX. */
int cbm_plan_set_multipliers(cbm_plan* plan, const float* d_multipliers, void* stream);

/* Tuning knobs.  chunk_nnz (>= 32): rows with more entries are summed in
 * chunks of that size by separate teams (host-side re-layout + upload).
 * rows_per_claim (>= 1): consecutive level-0 rows a team takes per queue
 * claim; rows_per_claim_deep (>= 0): the same for rows below level 0, which
 * wait on their parents (0: automatic, one row when more than a quarter of the
 * rows are below level 0, else rows_per_claim).
 * variant: which forward kernel runs on the 16-byte vector path.
 * hot_rows (>= 0): the staged kernel asks L2 to keep the X rows of this many
 * most-gathered columns and to evict the others and the output rows first;
 * 0 turns the cache policies off.  team (0, 8, 16, 32): lanes per row stream
 * in the staged kernel (0: its default; several streams share each warp).
 * Changing chunk_nnz or hot_rows re-lays out the plan (synchronous). */
enum {
  CBM_VARIANT_AUTO = 0,     /* staged where it applies, else register gather; register
                               gather also for rows of at most 512 bytes when most rows
                               hang below tree level 0 */
  CBM_VARIANT_REGISTER = 1, /* X rows gathered into registers, U entries at a time */
  CBM_VARIANT_STAGED = 2,   /* X rows staged through shared memory by cp.async */
  CBM_VARIANT_TMA = 3       /* X rows gathered four at a time by TMA (tile::gather4) into
                               per-team rings; rows of 8, 16 or 32 pieces of 16 bytes, at
                               most 256 elements (else as STAGED) */
};
int cbm_plan_tune(cbm_plan* plan, int32_t chunk_nnz, int32_t rows_per_claim, int32_t rows_per_claim_deep,
                  int32_t variant, int64_t hot_rows, int32_t team, void* stream);

/* How a product is executed (FP32 Y without the GIN term or compensation;
 * other products always run fused).  FUSED: one pass, each row adds its
 * parent's row as soon as it is final.  TWO: a first pass stores every row's
 * delta sum without waiting on parents, a second adds the parent terms in
 * tree-level order; same arithmetic, bit-identical results.  AUTO (default):
 * fused, which measured as fast or faster on every tree tried. */
enum { CBM_PASSES_AUTO = 0, CBM_PASSES_FUSED = 1, CBM_PASSES_TWO = 2 };
int cbm_plan_set_passes(cbm_plan* plan, int32_t passes);

/* Device scratch bytes a call with these operand types needs (0 is possible). */
int64_t cbm_plan_workspace_bytes(const cbm_plan* plan, int32_t op, int64_t n_cols, int32_t x_dtype,
                                 int32_t y_dtype, int32_t adjoint);

/* Y = op(A) X.  x: [n_rows, n_cols] row-major with leading dimension ldx, y
 * likewise with ldy; both device memory, not overlapping.  workspace: device
 * scratch of at least cbm_plan_workspace_bytes() bytes.  Allocates nothing,
 * launches one kernel on `stream` per block of up to 1,024 (FP32 X) or 2,048
 * (BF16 X) columns, does not synchronise.  Calls on one plan must be ordered
 * (one stream, or events): they share the plan's queue state.
 * Replaces matmul_AX_ADX / matmul_DAX_DADX (cbm/cbm.cu:150-268). */
int cbm_matmul(cbm_plan* plan, int32_t op, const void* x, int32_t x_dtype, int64_t ldx, void* y,
               int32_t y_dtype, int64_t ldy, int64_t n_cols, void* workspace, int64_t workspace_bytes,
               void* stream);

/* GIN aggregation Y = A X + (1 + epsilon) X on the CBM product, with the self
 * term fused into the final store (the parent rows propagated down the tree
 * are the A X rows, kept in the workspace).  Square A; X and Y as for
 * cbm_matmul; workspace: cbm_plan_workspace_bytes(plan, CBM_OP_GIN, ...).
 * Each element is fma(1 + epsilon, X[v], (A X)[v]).
 * Replaces s_spmm_update_add_csr_int32 (cbm/cbm_extensions.cpp:498-591), the
 * reference's CPU-only GIN form (its MKL SpMM + update + cblas_saxpy). */
int cbm_matmul_gin(cbm_plan* plan, float epsilon, const void* x, int32_t x_dtype, int64_t ldx, void* y,
                   int32_t y_dtype, int64_t ldy, int64_t n_cols, void* workspace, int64_t workspace_bytes,
                   void* stream);

/* Y = op(A) X for operands in host memory (page-locked for full-speed
 * copies): X is copied in and Y out in column slabs of slab_cols columns (0:
 * one slab), with the host-to-device copy of slab k+1, the product of slab k
 * and the device-to-host copy of slab k-1 overlapped on two copy streams of
 * the plan and `stream` (64 fp32 columns, 256-byte row pieces, is the
 * measured best on B200 over PCIe).  x_host [n_cols(A), n_cols] with leading dimension
 * ldx_host, y_host [n_rows(A), n_cols] with ldy_host; x_dev / y_dev: device
 * buffers of the same shapes, contiguous (the caller's: nothing is
 * allocated); workspace as for cbm_matmul with slab_cols columns.  Returns
 * once everything is queued; `stream` waits for the last copy, so a
 * synchronisation of `stream` makes y_host final.  Calls on one plan must be
 * ordered on one stream.  The reference has no host-operand product (its
 * callers copy with torch before matmul_AX_ADX, cbm/cbm4mm.py:53-54). */
int cbm_matmul_host(cbm_plan* plan, int32_t op, const void* x_host, int32_t x_dtype, int64_t ldx_host,
                    void* y_host, int32_t y_dtype, int64_t ldy_host, int64_t n_cols, int64_t slab_cols,
                    void* x_dev, void* y_dev, void* workspace, int64_t workspace_bytes, void* stream);

/* cbm_matmul_host across calls (0: off, the default).  With it on:
 *  - a call's copy-in of X waits only until the previous call's products have
 *    finished reading the device copy of X (slab by slab when both calls
 *    have the same columns, slab width, dtypes and device buffers), not for
 *    the previous call's copy-out, so copies in and out of consecutive calls
 *    overlap.  The copy-in is not ordered after other work the caller queued
 *    on `stream`: x_host must be complete when the call is made (written by
 *    the host);
 *  - `stream` waits for the call's products only: its copy-out of Y stays
 *    pending.  cbm_plan_host_wait(plan, stream) makes `stream` wait for every
 *    copy-out queued so far; after that a synchronisation of `stream` makes
 *    y_host final.  A call without overlap also ends with `stream` waiting
 *    for every copy-out, as before.
 * Results are unchanged. */
int cbm_plan_set_host_overlap(cbm_plan* plan, int32_t on);

/* `stream` waits for every copy-out of Y queued by cbm_matmul_host calls of
 * this plan (needed after calls with overlap on; no effect otherwise). */
int cbm_plan_host_wait(cbm_plan* plan, void* stream);

/* dX = op(A)^T G (the adjoint of cbm_matmul for CBM_OP_AX/ADX/DADX): a
 * reverse tree propagation (children into parents) then a transposed delta
 * gather.  Same conventions as cbm_matmul.  No counterpart in the reference. */
int cbm_matmul_adjoint(cbm_plan* plan, int32_t op, const void* g, int32_t g_dtype, int64_t ldg, void* dx,
                       int32_t dx_dtype, int64_t lddx, int64_t n_cols, void* workspace,
                       int64_t workspace_bytes, void* stream);

/* Builds the adjoint layout (reverse-propagation lists and the transposed
 * delta matrix) ahead of the first cbm_matmul_adjoint; synchronous. */
int cbm_plan_prepare_adjoint(cbm_plan* plan, void* stream);

/* Precision form (BF16 X): rows at tree depth >= min_depth add their parent's
 * row with compensated arithmetic (an error-free TwoSum per element, the
 * rounding residual carried down the chain in an FP32 workspace row per
 * internal node), so a chain's error stays that of one rounding instead of
 * growing with its depth.  Applies when the tree has more than min_depth
 * levels; such products run on the register-gather kernel.  -1: never;
 * default 64 (below it an FP32 chain's rounding, depth * 2^-24 relative,
 * stays under 4e-6).  FP32 X keeps the reference's plain rounding (parity). */
int cbm_plan_set_compensation(cbm_plan* plan, int32_t min_depth);

/* Limit of every device-side wait, in nanoseconds (default 1 s). */
int cbm_plan_set_timeout(cbm_plan* plan, int64_t ns);

/* Test hook: make queue item `item` wait on `parent_node` (whose ready flag may
 * never be set) to exercise the bounded wait.  -1 removes the parent. */
int cbm_plan_debug_set_parent(cbm_plan* plan, int64_t item, int32_t parent_node, void* stream);

/* Test hook: builds the adjoint layout if needed, rebuilds its transposed
 * delta matrix on the host (a counting sort) and compares it word for word
 * with the one sorted on the device: CBM_OK if equal, CBM_ERR_INTERNAL if not.
 * Synchronous. */
int cbm_plan_debug_check_transpose(cbm_plan* plan, void* stream);

/* Synchronises `stream`, returns the first device-side error recorded since
 * the last call (CBM_OK, CBM_ERR_TIMEOUT, CBM_ERR_INDEX) in *device_status and
 * clears it. info (may be NULL) receives where it happened. */
int cbm_plan_error(cbm_plan* plan, void* stream, int32_t* device_status, int64_t* info);

/* ---- product without allocation ----------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (a plugin inside a process whose allocator owns all of the GPU, a
 * serving loop that must not take cudaMalloc's implicit synchronisation, an
 * extension point that is only handed buffers): Y = A X computed straight from
 * the reference's layout in the caller's device buffers, with no plan and no
 * workspace.  row_ptr/col_idx/values: the delta matrix as CSR (values NULL =
 * all +1); src/dst: the tree edges in BFS order per branch (the reference's
 * mca_src_idx / mca_dst_idx); multipliers NULL gives matmul_AX_ADX, non-NULL
 * matmul_DAX_DADX (cbm/cbm.cu:150-268).  x: [n_cols, n_x_cols] fp32, y:
 * [n_rows, n_x_cols] fp32, both contiguous.  d_status (device int32, may be
 * NULL) receives the device-side status when the work ends (CBM_OK,
 * CBM_ERR_TIMEOUT, CBM_ERR_INDEX).
 * Scratch: a fixed 8 MiB array inside the library, held on every GPU that
 * loads it; n_rows above CBM_NOALLOC_MAX_ROWS returns CBM_ERR_TOO_LARGE.
 * The first call on a device looks up the array's device address (set-up);
 * make that first call before any stream capture.  That address is kept for
 * the life of the process: do not call this entry point after a
 * cudaDeviceReset.  Calls share the array: calls whose kernels overlap on the
 * GPU race.  Row pointers outside 0 <= begin <= end <= row_ptr[n_rows] and
 * column or tree indices out of range are skipped and reported as
 * CBM_ERR_INDEX, a node with two parents as CBM_ERR_STRUCTURE.  Allocates
 * nothing; two kernel launches on `stream`, no synchronisation. */
#define CBM_NOALLOC_MAX_ROWS 1048544
int cbm_matmul_noalloc(const int32_t* row_ptr, const int32_t* col_idx, const float* values, int64_t n_rows,
                       int64_t n_cols, const int32_t* src, const int32_t* dst, int64_t n_edges,
                       const float* multipliers, const float* x, float* y, int64_t n_x_cols, int32_t* d_status,
                       void* stream);

/* ---- the reference's CPU operators on the GPU --------------------------------
 * Stateless GPU counterparts of the eight products the reference's cbm_mkl_cpp
 * module binds (cbm/cbm_extensions.cpp:909-919), on the reference's own
 * layout: no plan, every call reads the caller's arrays.
 *   A [n_rows, n_cols]: MKL's four-array CSR as the reference passes it --
 *     rp_b / rp_e begin and end row pointers (crow[:-1], crow[1:]), col, val
 *     (val NULL: every entry 1); entries lie in [0, nnz).
 *   Tree: branch offsets (n_branch_offsets = branches + 1, a prefix sum from 0
 *     to n_edges) and the (parent src, child dst) edges in BFS order per
 *     branch: cbm_init_'s output (CBM_S_BRANCHES / CBM_S_SRC / CBM_S_DST).
 *     Edges are processed in their listed order, parents before children.
 *   rhs, out: contiguous row-major FP32 with n_rhs_cols columns.
 * All pointers are device addresses.  workspace: device memory of at least
 * cbm_direct_workspace_bytes(rows of out) bytes, 16-byte aligned, zero-filled
 * once before its first use and then kept (a status word, a claim counter and
 * two per-node stamps compared against a per-call value: never cleared again).
 * Calls that share a workspace must be ordered (one stream).  Each call
 * launches on `stream` without synchronising; index errors found on the device
 * (CBM_ERR_INDEX), a node with two parents or bad branch offsets
 * (CBM_ERR_STRUCTURE) and bounded waits that ran out (CBM_ERR_TIMEOUT: a child
 * edge listed before its parent's) are recorded in the workspace and read with
 * cbm_direct_status.
 * Rounding: each row sums its entries in order, one FMA per entry (MKL's order
 * may differ in the last bits); the update adds Y[v] + Y[u]; the fused update
 * adds fma(Y[u], m[v] / m[u], Y[v]) (the reference's CPU rounding,
 * cbm/cbm_extensions.cpp:660-697, not the GPU path's (Y[u] m[v]) / m[u]); the
 * GIN term is fma(1 + epsilon, X, Y) (its cblas_saxpy).  The transposed
 * product adds with atomics: its summation order is not deterministic. */
int64_t cbm_direct_workspace_bytes(int64_t n_rows);

/* Synchronises `stream`, returns the first device-side error the calls on this
 * workspace recorded (CBM_OK if none) and clears it; info (may be NULL)
 * receives the entry, row, edge or branch offset where it happened. */
int cbm_direct_status(void* workspace, void* stream, int32_t* device_status, int64_t* info);

/* out = A rhs.  Replaces s_spmm_csr_int32 (cbm/cbm_extensions.cpp:700-740). */
int cbm_s_spmm_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col, const float* val,
                         int64_t n_rows, int64_t n_cols, int64_t nnz, const float* rhs, int64_t n_rhs_cols,
                         float* out, void* workspace, int64_t workspace_bytes, void* stream);

/* out [n_cols, C] = A^T rhs (rhs [n_rows, C]).  Replaces s_spmm_csr_t_int32
 * (cbm/cbm_extensions.cpp:742-782), which declares A square. */
int cbm_s_spmm_csr_t_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col, const float* val,
                           int64_t n_rows, int64_t n_cols, int64_t nnz, const float* rhs, int64_t n_rhs_cols,
                           float* out, void* workspace, int64_t workspace_bytes, void* stream);

/* out = A rhs + (1 + epsilon) rhs (square A).  Replaces s_spmm_add_csr_int32
 * (cbm/cbm_extensions.cpp:446-492). */
int cbm_s_spmm_add_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col, const float* val,
                             int64_t n_rows, int64_t n_cols, int64_t nnz, const float* rhs, int64_t n_rhs_cols,
                             float epsilon, float* out, void* workspace, int64_t workspace_bytes, void* stream);

/* out = Delta rhs, then out[dst] += out[src] along the tree.  Replaces
 * s_spmm_update_csr_int32 (cbm/cbm_extensions.cpp:351-444). */
int cbm_s_spmm_update_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col, const float* val,
                                int64_t n_rows, int64_t n_cols, int64_t nnz, const float* rhs, int64_t n_rhs_cols,
                                const int32_t* branches, int64_t n_branch_offsets, const int32_t* src,
                                const int32_t* dst, int64_t n_edges, float* out, void* workspace,
                                int64_t workspace_bytes, void* stream);

/* out = Delta rhs, then out[dst] = fma(out[src], m[dst] / m[src], out[dst]).
 * Replaces s_spmm_fused_update_csr_int32 (cbm/cbm_extensions.cpp:593-698). */
int cbm_s_spmm_fused_update_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col,
                                      const float* val, int64_t n_rows, int64_t n_cols, int64_t nnz,
                                      const float* rhs, int64_t n_rhs_cols, const int32_t* branches,
                                      int64_t n_branch_offsets, const int32_t* src, const int32_t* dst,
                                      int64_t n_edges, const float* multiplier, float* out, void* workspace,
                                      int64_t workspace_bytes, void* stream);

/* out = Delta rhs, the update, then out += (1 + epsilon) rhs (square A).
 * Replaces s_spmm_update_add_csr_int32 (cbm/cbm_extensions.cpp:494-591). */
int cbm_s_spmm_update_add_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col,
                                    const float* val, int64_t n_rows, int64_t n_cols, int64_t nnz,
                                    const float* rhs, int64_t n_rhs_cols, float epsilon, const int32_t* branches,
                                    int64_t n_branch_offsets, const int32_t* src, const int32_t* dst,
                                    int64_t n_edges, float* out, void* workspace, int64_t workspace_bytes,
                                    void* stream);

/* out[dst] += out[src] along the tree, in place on out [n_out_rows,
 * n_out_cols].  Replaces s_update_csr_int32 (cbm/cbm_extensions.cpp:784-838). */
int cbm_s_update_csr_int32(const int32_t* branches, int64_t n_branch_offsets, const int32_t* src,
                           const int32_t* dst, int64_t n_edges, float* out, int64_t n_out_rows,
                           int64_t n_out_cols, void* workspace, int64_t workspace_bytes, void* stream);

/* out[dst] = fma(out[src], m[dst] / m[src], out[dst]) along the tree, in place.
 * Replaces s_fused_update_csr_int32 (cbm/cbm_extensions.cpp:841-907). */
int cbm_s_fused_update_csr_int32(const int32_t* branches, int64_t n_branch_offsets, const int32_t* src,
                                 const int32_t* dst, int64_t n_edges, const float* multiplier, float* out,
                                 int64_t n_out_rows, int64_t n_out_cols, void* workspace, int64_t workspace_bytes,
                                 void* stream);

/* Plan statistics (for the bench's algorithmic byte counts). */
enum {
  CBM_P_ROWS = 0,
  CBM_P_COLS = 1,
  CBM_P_NNZ = 2,
  CBM_P_EDGES = 3,
  CBM_P_BRANCHES = 4,
  CBM_P_LEVELS = 5,
  CBM_P_INTERNAL = 6,
  CBM_P_CHUNKS = 7,
  CBM_P_LONG_ROWS = 8,
  CBM_P_UNIT_VALUES = 9,
  CBM_P_GRID = 10,
  CBM_P_LAUNCHES = 11 /* kernels launched by this plan so far */
};
int64_t cbm_plan_stat(const cbm_plan* plan, int32_t which);

void cbm_plan_destroy(cbm_plan* plan);

const char* cbm_status_string(int32_t status);

#ifdef __cplusplus
}
#endif
#endif /* CBM_B200_H */
