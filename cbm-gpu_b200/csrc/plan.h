// The plan object behind the opaque cbm_plan handle (include/cbm_b200.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <nvtx3/nvToolsExt.h>

#include <vector>

#include "kernels.cuh"

// NVTX range over a host-side phase (plan set-up, launches, layouts): named
// spans in an Nsight timeline; a few nanoseconds when no tool is attached.
struct CbmRange {
  explicit CbmRange(const char* name) { nvtxRangePushA(name); }
  ~CbmRange() { nvtxRangePop(); }
  CbmRange(const CbmRange&) = delete;
  CbmRange& operator=(const CbmRange&) = delete;
};

struct cbm_plan {
  int device = 0;
  int64_t n_rows = 0, n_cols = 0, nnz = 0, n_edges = 0, n_branches = 0;
  int64_t n_items = 0, n_internal = 0, levels = 0;
  bool unit_values = true, has_values = false;
  int32_t chunk_nnz = 256;      // split rows longer than this
  int32_t rows_per_claim = 4;   // level-0 rows a team takes per queue claim
  int32_t rows_per_claim_deep = 0;  // rows below level 0 a team takes per claim (0: automatic)
  int64_t n_root = 0;           // rows at level 0 (children of the virtual root)
  int32_t variant = 0;          // CBM_VARIANT_*: forward kernel choice
  int64_t hot_rows = 65536;     // columns whose X rows the staged kernel asks L2 to keep (0: no hints)
  int32_t staged_team = 0;      // lanes per team of the staged kernel (0: its default)
  int32_t passes = 0;           // CBM_PASSES_*: fused product or delta pass + propagation pass
  int64_t launches = 0;
  int64_t last_grid = 0;
  long long timeout_ns = 1000000000ll;  // bounded waits: 1 s
  // BF16 X: rows at tree depth >= comp_depth add their parent with compensated
  // (TwoSum) arithmetic and carry the rounding residual (-1: never)
  int32_t comp_depth = 64;
  std::vector<int64_t> level_start;  // first item of each tree level, [levels + 1]

  // host copies used to rebuild chunk tables and the adjoint layout
  std::vector<int64_t> h_ptr;     // entry offsets per item (level order)
  std::vector<int32_t> h_order;   // node of each item
  std::vector<int32_t> h_parent;  // parent per node (-1: virtual root)
  std::vector<int32_t> h_slot;    // internal slot per node (-1: leaf)
  std::vector<int32_t> h_depth;
  std::vector<uint32_t> h_ent;    // column | sign << 31, item order
  std::vector<float> h_val;       // values in item order (empty when all are +-1)

  // forward layout (device); d_ptr/d_ent/d_val and d_cent/d_cval are the
  // stream layout rebuilt with the chunk size (build_layout)
  int32_t* d_node = nullptr;
  int64_t* d_ptr = nullptr;
  uint32_t* d_ent = nullptr;
  float* d_val = nullptr;
  uint32_t* d_cent = nullptr;
  float* d_cval = nullptr;
  int32_t* d_par = nullptr;
  int32_t* d_par_item = nullptr;
  int32_t* d_self_slot = nullptr;
  int32_t* d_par_slot = nullptr;
  float* d_mult = nullptr;
  unsigned* d_node_flag = nullptr;
  cbm::QueueState* d_qs = nullptr;
  // forward chunks
  int64_t n_chunks = 0, long_rows = 0;
  int32_t* d_chunk0 = nullptr;
  int32_t* d_chunk_item = nullptr;
  int64_t* d_chunk_beg = nullptr;
  int64_t* d_chunk_end = nullptr;
  unsigned* d_chunk_flag = nullptr;
  // claim units of the staged kernel (build_units)
  int64_t n_units = 0;
  int32_t* d_unit = nullptr;
  std::vector<void*> unit_bufs;

  // adjoint layout (built on first use)
  bool adj_built = false;
  int64_t n_rev_items = 0, n_rev_chunks = 0;
  int32_t* d_rev_chunk0 = nullptr;
  int32_t* d_rev_nchunk = nullptr;
  unsigned* d_rev_chunk_flag = nullptr;
  int32_t* d_rev_node = nullptr;   // internal nodes (and chunk items), deepest level first
  int32_t* d_rev_slot = nullptr;
  int64_t* d_rev_ptr = nullptr;    // children lists
  uint32_t* d_rev_ent = nullptr;   // child | internal << 30 (slot if internal)
  unsigned* d_adj_flag = nullptr;  // [n_internal]
  std::vector<int64_t> h_t_ptr;    // transposed delta: entries per column
  int64_t* d_t_ptr = nullptr;
  uint32_t* d_t_ent = nullptr;     // row (or slot) | internal << 30 | sign << 31
  int64_t n_t_chunks = 0;
  int32_t* d_t_chunk0 = nullptr;
  int32_t* d_t_chunk_item = nullptr;
  int64_t* d_t_chunk_beg = nullptr;
  int64_t* d_t_chunk_end = nullptr;
  unsigned* d_t_chunk_flag = nullptr;

  std::vector<void*> bufs, chunk_bufs, adj_bufs, adj_chunk_bufs;

  // host-operand pipeline (cbm_matmul_host): two copy streams and the events
  // that order slabs across them, created on first use
  cudaStream_t h2d = nullptr, d2h = nullptr;
  std::vector<cudaEvent_t> events;
  // overlap across calls (cbm_plan_set_host_overlap).  Events per slab k:
  // events[2 + 3k] copy-in done, [3 + 3k] product done, [4 + 3k] copy-out
  // done; [0] the call's start on the caller's stream, [1] its last copy-out.
  // A call with the previous call's slab layout orders slab by slab against
  // it (its copy-in of slab k after that call's product k, its product k
  // after that call's copy-out k); otherwise against the whole call
  // (host_prev_prod: the last product; events[1]: the last copy-out).  With
  // overlap the caller's stream is released after the products and the
  // copy-out stays pending (host_out_pending) until cbm_plan_host_wait or a
  // call without overlap.
  bool host_overlap = false;
  bool host_prev_valid = false;
  bool host_out_pending = false;
  cudaEvent_t host_prev_prod = nullptr;
  int64_t host_prev_layout[5] = {0, 0, 0, 0, 0};  // columns, slab width, slabs, x and y element bytes
  const void* host_prev_xd = nullptr;
  const void* host_prev_yd = nullptr;
};

namespace cbm {
int cuda_status(cudaError_t e);
void free_all(std::vector<void*>& v);
int build_layout(cbm_plan* P, cudaStream_t st);
int build_units(cbm_plan* P, cudaStream_t st);
int32_t claim_rows(const cbm_plan* P);
int32_t deep_rows_per_claim(const cbm_plan* P);
int sm_count(int device);
int rebuild_adjoint_chunks(cbm_plan* P, cudaStream_t st);
void release_pipeline(cbm_plan* P);
int transpose_on_device(cbm_plan* P, cudaStream_t st);
int matmul_impl(cbm_plan* P, int32_t op, float gin_scale, const void* x, int32_t xdt, int64_t ldx, void* y,
                int32_t ydt, int64_t ldy, int64_t n_cols, void* ws, int64_t ws_bytes, void* stream);
}  // namespace cbm
