// Launch side of the CBM product: operand checks, tile-shape selection, the
// adjoint layout and the host-operand pipeline behind cbm_matmul /
// cbm_matmul_adjoint / cbm_matmul_host.  The kernel instantiations live in the
// launch_*.cu units (launch.cuh).

#include "cbm_b200.h"
#include "launch.cuh"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

namespace cbm {

int sm_count(int device) {
  static std::atomic<int> count[kMaxDevices];
  if (device < 0 || device >= kMaxDevices) return 1;
  int c = count[device].load(std::memory_order_acquire);
  if (c > 0) return c;
  if (cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || c < 1) return 1;
  count[device].store(c, std::memory_order_release);
  return c;
}

namespace {

int64_t round4(int64_t x) { return (x + 3) / 4 * 4; }

// compensated propagation applies to BF16 X on trees deeper than the threshold
bool comp_active(const cbm_plan* P, int32_t xdt) {
  return xdt == CBM_BF16 && P->comp_depth >= 0 && P->levels > P->comp_depth && P->n_internal > 0;
}
int64_t align256(int64_t b) { return (b + 255) / 256 * 256; }

// Columns one launch covers: 32 lanes x 8 vectors x V elements.
int64_t block_cols(int v) { return 32 * 8 * (int64_t)v; }

struct Shape {
  bool vec;
  int v;       // elements per vector
  int64_t cb;  // columns per launch
};

int elem_size(int32_t dt) { return dt == CBM_BF16 ? 2 : 4; }

Shape pick_shape(int32_t xdt, int32_t ydt, const void* x, int64_t ldx, const void* y, int64_t ldy, int64_t c) {
  const int vv = xdt == CBM_BF16 ? 8 : 4;
  const bool aligned = c % vv == 0 && (reinterpret_cast<uintptr_t>(x) % 16 == 0) &&
                       (reinterpret_cast<uintptr_t>(y) % 16 == 0) && (ldx * elem_size(xdt)) % 16 == 0 &&
                       (ldy * elem_size(ydt)) % 16 == 0;
  Shape s;
  s.vec = aligned;
  s.v = aligned ? vv : 1;
  s.cb = block_cols(s.v);
  return s;
}

void team_for(int64_t nvec, int* team, int* vpl) {
  if (nvec >= 32) {
    *team = 32;
    const int64_t need = (nvec + 31) / 32;
    *vpl = need <= 1 ? 1 : need <= 2 ? 2 : need <= 4 ? 4 : 8;
  } else {
    int t = 1;
    while (t < nvec) t <<= 1;
    *team = t;
    *vpl = 1;
  }
}

bool dtype_ok(int32_t xdt, int32_t ydt) {
  return (xdt == CBM_F32 && ydt == CBM_F32) || (xdt == CBM_BF16 && ydt == CBM_F32) ||
         (xdt == CBM_BF16 && ydt == CBM_BF16);
}

// bytes from the first to one past the last element of a [rows, cols] view with leading dimension ld
int64_t extent(int64_t rows, int64_t ld, int64_t cols, int32_t dt) {
  return rows > 0 ? ((rows - 1) * ld + cols) * elem_size(dt) : 0;
}

bool overlaps(const void* a, int64_t abytes, const void* b, int64_t bbytes) {
  const uintptr_t a0 = reinterpret_cast<uintptr_t>(a), b0 = reinterpret_cast<uintptr_t>(b);
  return a0 < b0 + (uintptr_t)bbytes && b0 < a0 + (uintptr_t)abytes;
}

// cuTensorMapEncodeTiled from the driver, found once through the runtime
// (no link-time dependency on libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  }
  return fn;
}

// Tensor map of X for the gather: columns [0, cols) of `rows` rows with a
// leading dimension of ldx elements; box = the whole width, one row high
// (what tile::gather4 takes).  x 16-byte aligned, ldx * size a multiple of 16,
// cols * size a multiple of 16 and cols <= 256 (checked by the caller).
int encode_x_map(CUtensorMap* map, const void* x, int32_t xdt, int64_t rows, int64_t ldx, int64_t cols) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return CBM_ERR_CUDA;
  const int es = xdt == CBM_BF16 ? 2 : 4;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)(ldx * es)};
  const cuuint32_t box[2] = {(cuuint32_t)cols, 1u};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = fn(map, xdt == CBM_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                        const_cast<void*>(x), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE,
                        cols * es >= 256 ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B : CU_TENSOR_MAP_L2_PROMOTION_NONE,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? CBM_OK : CBM_ERR_CUDA;
}

// Team shape of the staged kernel for nvec 16-byte pieces per row.  A lane
// holds at most 32 accumulators (8 pieces of fp32, 4 of bf16).  Default: the
// widest team up to a full warp (one row stream per warp when the row has >= 32
// pieces; narrower rows share a warp between streams that step together);
// `forced` (8, 16 or 32) overrides it where the pieces fit.
bool staged_shape(int64_t nvec, int v, int forced, int* team, int* vpl) {
  const int max_vpl = 32 / v;
  if (nvec < 8 || nvec > 32 * max_vpl) return false;
  int t = 8;
  while (t < 32 && t < nvec) t <<= 1;
  if (forced != 0) {
    if (forced * max_vpl < nvec) return false;
    t = forced;
  }
  int p = 1;
  while (t * p < nvec) p <<= 1;
  *team = t;
  *vpl = p;
  return true;
}

int launch_staged(cbm_plan* P, const FwdArgs& a, int32_t xdt, int32_t ydt, int team, int vpl, cudaStream_t st) {
  if (xdt == CBM_F32) return launch_staged_f32(P, a, team, vpl, st);
  if (ydt == CBM_F32) return launch_staged_bf16_f32(P, a, team, vpl, st);
  return launch_staged_bf16_bf16(P, a, team, vpl, st);
}

// The TMA variant applies to 16-byte-vector rows of a power-of-two number of
// pieces (8 .. 32 per team, at most 256 elements: one TMA box), one or two
// pieces per lane.
bool tma_shape(int64_t nvec, int v, int team, int vpl) {
  return nvec >= 8 && (nvec & (nvec - 1)) == 0 && nvec == (int64_t)team * vpl && nvec * v <= 256 && vpl <= 2;
}

int launch_fwd(cbm_plan* P, const FwdArgs& a, int32_t xdt, int32_t ydt, bool vec, int vpl, bool shallow,
               cudaStream_t st) {
  if (xdt == CBM_F32) return launch_fwd_f32(P, a, vec, vpl, st);
  return launch_fwd_bf16(P, a, ydt, vec, vpl, shallow, st);
}

template <typename T>
int upload(T** dst, const std::vector<T>& src, cudaStream_t st, std::vector<void*>& owned) {
  *dst = nullptr;
  if (src.empty()) return CBM_OK;
  void* p = nullptr;
  if (cudaMalloc(&p, src.size() * sizeof(T)) != cudaSuccess) return CBM_ERR_ALLOC;
  owned.push_back(p);
  if (cudaMemcpyAsync(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return CBM_ERR_CUDA;
  *dst = static_cast<T*>(p);
  return CBM_OK;
}

int zeros_u32(unsigned** dst, int64_t n, cudaStream_t st, std::vector<void*>& owned) {
  *dst = nullptr;
  if (n <= 0) return CBM_OK;
  void* p = nullptr;
  if (cudaMalloc(&p, n * sizeof(unsigned)) != cudaSuccess) return CBM_ERR_ALLOC;
  owned.push_back(p);
  if (cudaMemsetAsync(p, 0, n * sizeof(unsigned), st) != cudaSuccess) return CBM_ERR_CUDA;
  *dst = static_cast<unsigned*>(p);
  return CBM_OK;
}

}  // namespace

int rebuild_adjoint_chunks(cbm_plan* P, cudaStream_t st) {
  if (!P->adj_built) return CBM_OK;
  free_all(P->adj_chunk_bufs);
  std::vector<int32_t> chunk0(P->n_cols, -1), citem;
  std::vector<int64_t> cbeg, cend;
  const int64_t T = P->chunk_nnz;
  for (int64_t j = 0; j < P->n_cols; ++j) {
    const int64_t b = P->h_t_ptr[j], e = P->h_t_ptr[j + 1];
    if (e - b > T) {
      chunk0[j] = (int32_t)citem.size();
      for (int64_t s = b; s < e; s += T) {
        citem.push_back((int32_t)j);
        cbeg.push_back(s);
        cend.push_back(std::min(e, s + T));
      }
    }
  }
  P->n_t_chunks = (int64_t)citem.size();
  int rc;
  if ((rc = upload(&P->d_t_chunk0, chunk0, st, P->adj_chunk_bufs))) return rc;
  if ((rc = upload(&P->d_t_chunk_item, citem, st, P->adj_chunk_bufs))) return rc;
  if ((rc = upload(&P->d_t_chunk_beg, cbeg, st, P->adj_chunk_bufs))) return rc;
  if ((rc = upload(&P->d_t_chunk_end, cend, st, P->adj_chunk_bufs))) return rc;
  if ((rc = zeros_u32(&P->d_t_chunk_flag, P->n_t_chunks, st, P->adj_chunk_bufs))) return rc;
  return cuda_status(cudaStreamSynchronize(st));
}

// Reverse-propagation items (internal nodes, deepest first, with their
// children lists; built on the host) and the transposed delta matrix (sorted
// on the device, transpose.cu), built once per plan.
int build_adjoint(cbm_plan* P, cudaStream_t st) {
  if (P->adj_built) return CBM_OK;
  CbmRange range("cbm build_adjoint");
  if (P->n_rows >= (int64_t)kInternalBit || P->n_cols >= (int64_t)kInternalBit) return CBM_ERR_INVALID;
  const int64_t n = P->n_rows;
  // children lists, by parent
  std::vector<int64_t> cptr(n + 1, 0);
  for (int64_t v = 0; v < n; ++v)
    if (P->h_parent[v] >= 0) cptr[P->h_parent[v] + 1]++;
  for (int64_t v = 0; v < n; ++v) cptr[v + 1] += cptr[v];
  std::vector<int32_t> kids(cptr[n]);
  {
    std::vector<int64_t> fill(cptr.begin(), cptr.end() - 1);
    for (int64_t v = 0; v < n; ++v)
      if (P->h_parent[v] >= 0) kids[fill[P->h_parent[v]]++] = (int32_t)v;
  }
  // internal nodes in reverse item (level) order; a children list longer than
  // kRevChunk is summed in chunk items queued just before its node
  constexpr int64_t kRevChunk = 64;
  std::vector<int32_t> rnode, rslot, rchunk0, rnchunk;
  std::vector<int64_t> rptr(1, 0);
  std::vector<uint32_t> rent;
  int32_t n_rev_chunks = 0;
  for (int64_t i = n - 1; i >= 0; --i) {
    const int32_t w = P->h_order[i];
    if (P->h_slot[w] < 0) continue;
    const int64_t nk = cptr[w + 1] - cptr[w];
    const bool split = nk > kRevChunk;
    const int32_t first = n_rev_chunks;
    for (int64_t k = cptr[w]; k < cptr[w + 1]; ++k) {
      const int32_t c = kids[k];
      rent.push_back(P->h_slot[c] >= 0 ? ((uint32_t)P->h_slot[c] | kInternalBit) : (uint32_t)c);
      if (split && ((k - cptr[w] + 1) % kRevChunk == 0 || k + 1 == cptr[w + 1])) {
        rnode.push_back(-1);  // chunk item
        rslot.push_back(n_rev_chunks++);
        rchunk0.push_back(-1);
        rnchunk.push_back(0);
        rptr.push_back((int64_t)rent.size());
      }
    }
    rnode.push_back(w);
    rslot.push_back(P->h_slot[w]);
    rchunk0.push_back(split ? first : -1);
    rnchunk.push_back(split ? n_rev_chunks - first : 0);
    rptr.push_back((int64_t)rent.size());  // empty range when split
  }
  P->n_rev_items = (int64_t)rnode.size();
  P->n_rev_chunks = n_rev_chunks;
  int rc;
  if ((rc = upload(&P->d_rev_node, rnode, st, P->adj_bufs))) return rc;
  if ((rc = upload(&P->d_rev_chunk0, rchunk0, st, P->adj_bufs))) return rc;
  if ((rc = upload(&P->d_rev_nchunk, rnchunk, st, P->adj_bufs))) return rc;
  if ((rc = zeros_u32(&P->d_rev_chunk_flag, n_rev_chunks, st, P->adj_bufs))) return rc;
  if ((rc = upload(&P->d_rev_slot, rslot, st, P->adj_bufs))) return rc;
  if ((rc = upload(&P->d_rev_ptr, rptr, st, P->adj_bufs))) return rc;
  if ((rc = upload(&P->d_rev_ent, rent, st, P->adj_bufs))) return rc;
  if ((rc = zeros_u32(&P->d_adj_flag, P->n_internal, st, P->adj_bufs))) return rc;
  // transposed delta: column j lists (row v or its slot, sign), sorted on the GPU
  if ((rc = transpose_on_device(P, st))) return rc;
  P->adj_built = true;
  return rebuild_adjoint_chunks(P, st);
}

void release_pipeline(cbm_plan* P) {
  for (cudaEvent_t e : P->events) cudaEventDestroy(e);
  P->events.clear();
  if (P->host_prev_prod) cudaEventDestroy(P->host_prev_prod);
  P->host_prev_prod = nullptr;
  P->host_prev_valid = false;
  P->host_out_pending = false;
  if (P->h2d) cudaStreamDestroy(P->h2d);
  if (P->d2h) cudaStreamDestroy(P->d2h);
  P->h2d = P->d2h = nullptr;
}

// Copy streams (created on the plan's device) and at least `n` events.
int pipeline_ready(cbm_plan* P, size_t n) {
  if (!P->h2d && cudaStreamCreateWithFlags(&P->h2d, cudaStreamNonBlocking) != cudaSuccess) return CBM_ERR_CUDA;
  if (!P->d2h && cudaStreamCreateWithFlags(&P->d2h, cudaStreamNonBlocking) != cudaSuccess) return CBM_ERR_CUDA;
  if (!P->host_prev_prod && cudaEventCreateWithFlags(&P->host_prev_prod, cudaEventDisableTiming) != cudaSuccess)
    return CBM_ERR_CUDA;
  while (P->events.size() < n) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return CBM_ERR_CUDA;
    P->events.push_back(e);
  }
  return CBM_OK;
}

}  // namespace cbm

using namespace cbm;

extern "C" {

int64_t cbm_plan_workspace_bytes(const cbm_plan* P, int32_t op, int64_t n_cols, int32_t x_dtype, int32_t y_dtype,
                                 int32_t adjoint) {
  if (!P || n_cols < 0) return -1;
  const int vv = x_dtype == CBM_BF16 ? 8 : 4;
  const int64_t cols = std::min<int64_t>(n_cols, block_cols(vv));
  const int64_t ldp = round4(cols);
  int64_t rows;
  if (adjoint) {
    // chunk counts of the transposed matrix are only known once built; bound
    // them by nnz / chunk_nnz + n_cols
    const int64_t t_chunks = P->adj_built ? P->n_t_chunks : (2 * P->nnz / P->chunk_nnz + 1);
    rows = P->n_internal + t_chunks + (P->adj_built ? P->n_rev_chunks : P->n_internal);
  } else {
    rows = P->n_chunks + ((y_dtype == CBM_BF16 || op == CBM_OP_GIN) ? P->n_internal : 0) +
           (comp_active(P, x_dtype) ? P->n_internal : 0);
  }
  return align256(rows * ldp * 4) + 256;
}

int cbm_plan_set_host_overlap(cbm_plan* P, int32_t on) {
  if (!P || (on != 0 && on != 1)) return CBM_ERR_INVALID;
  P->host_overlap = on != 0;
  return CBM_OK;
}

int cbm_plan_set_passes(cbm_plan* P, int32_t passes) {
  if (!P || passes < CBM_PASSES_AUTO || passes > CBM_PASSES_TWO) return CBM_ERR_INVALID;
  P->passes = passes;
  return CBM_OK;
}

int cbm_plan_set_timeout(cbm_plan* P, int64_t ns) {
  if (!P || ns <= 0) return CBM_ERR_INVALID;
  P->timeout_ns = ns;
  return CBM_OK;
}

int cbm_plan_debug_set_parent(cbm_plan* P, int64_t item, int32_t parent_node, void* stream) {
  // Test hook: points an item's parent at another node (e.g. a leaf, whose
  // ready flag nothing sets) so that the bounded wait can be exercised.
  if (!P || item < 0 || item >= P->n_items || parent_node < -1 || parent_node >= P->n_rows) return CBM_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaMemcpyAsync(P->d_par + item, &parent_node, sizeof(int32_t), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return CBM_ERR_CUDA;
  const int32_t zero = 0;
  if (cudaMemcpyAsync(P->d_par_slot + item, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return CBM_ERR_CUDA;
  int32_t par_item = -1;
  for (int64_t i = 0; parent_node >= 0 && i < P->n_items; ++i)
    if (P->h_order[i] == parent_node) par_item = (int32_t)i;
  if (cudaMemcpyAsync(P->d_par_item + item, &par_item, sizeof(int32_t), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return CBM_ERR_CUDA;
  return cuda_status(cudaStreamSynchronize(st));
}

int cbm_matmul(cbm_plan* P, int32_t op, const void* x, int32_t xdt, int64_t ldx, void* y, int32_t ydt, int64_t ldy,
               int64_t n_cols, void* ws, int64_t ws_bytes, void* stream) {
  if (op == CBM_OP_GIN) return CBM_ERR_INVALID;  // needs epsilon: cbm_matmul_gin
  return cbm::matmul_impl(P, op, 0.f, x, xdt, ldx, y, ydt, ldy, n_cols, ws, ws_bytes, stream);
}

int cbm_matmul_gin(cbm_plan* P, float epsilon, const void* x, int32_t xdt, int64_t ldx, void* y, int32_t ydt,
                   int64_t ldy, int64_t n_cols, void* ws, int64_t ws_bytes, void* stream) {
  if (P && P->n_rows != P->n_cols) return CBM_ERR_SHAPE;  // X[v] must exist for every row v
  return cbm::matmul_impl(P, CBM_OP_GIN, 1.0f + epsilon, x, xdt, ldx, y, ydt, ldy, n_cols, ws, ws_bytes, stream);
}

}  // extern "C"

namespace cbm {

int matmul_impl(cbm_plan* P, int32_t op, float gin_scale, const void* x, int32_t xdt, int64_t ldx, void* y,
                int32_t ydt, int64_t ldy, int64_t n_cols, void* ws, int64_t ws_bytes, void* stream) {
  CbmRange range("cbm_matmul");
  if (!P || op < CBM_OP_AX || op > CBM_OP_GIN || n_cols < 0) return CBM_ERR_INVALID;
  const bool gin = op == CBM_OP_GIN;
  if (!dtype_ok(xdt, ydt)) return CBM_ERR_DTYPE;
  if (n_cols == 0 || P->n_rows == 0) return CBM_OK;
  if (!x || !y) return CBM_ERR_INVALID;
  if (ldx < n_cols || ldy < n_cols || ldx > INT32_MAX || ldy > INT32_MAX) return CBM_ERR_SHAPE;
  if (overlaps(x, extent(P->n_cols, ldx, n_cols, xdt), y, extent(P->n_rows, ldy, n_cols, ydt))) return CBM_ERR_SHAPE;
  // column multipliers (D[col]) need a square A; the ratio rule of the VALUES
  // op reads row multipliers only, so a rectangular plan (a row shard) may
  // take it with one multiplier per row
  const bool needs_col_mult = op == CBM_OP_ADX || op == CBM_OP_DADX || op == CBM_OP_DAD_ADD;
  const bool needs_mult = needs_col_mult || op == CBM_OP_VALUES_RATIO;
  if (needs_mult && !P->d_mult) return CBM_ERR_UNSUPPORTED;
  if (needs_col_mult && P->n_rows != P->n_cols) return CBM_ERR_UNSUPPORTED;
  if ((op == CBM_OP_VALUES_ADD || op == CBM_OP_VALUES_RATIO) && xdt != CBM_F32) return CBM_ERR_DTYPE;
  const int64_t need = cbm_plan_workspace_bytes(P, op, n_cols, xdt, ydt, 0);
  const bool comp = comp_active(P, xdt);
  const bool state_rows = ydt == CBM_BF16 || gin;  // parents' rows come from pstate
  const bool need_ws = P->n_chunks > 0 || (state_rows && P->n_internal > 0) || comp;
  if (need_ws && (!ws || ws_bytes < need)) return CBM_ERR_WORKSPACE;
  if (ws && reinterpret_cast<uintptr_t>(ws) % 16 != 0) return CBM_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  int scale = SCALE_SIGN, prop = PROP_ADD;
  switch (op) {
    case CBM_OP_AX: break;
    case CBM_OP_ADX: scale = SCALE_DCOL; break;
    case CBM_OP_DADX: scale = SCALE_DCOL_DROW; prop = PROP_RATIO; break;
    case CBM_OP_VALUES_ADD: scale = P->unit_values ? SCALE_SIGN : SCALE_VALUES; break;
    case CBM_OP_VALUES_RATIO:
      scale = P->unit_values ? SCALE_SIGN : SCALE_VALUES;
      prop = PROP_RATIO;
      break;
    case CBM_OP_DAD_ADD: scale = SCALE_DCOL_DROW; break;
    case CBM_OP_GIN: scale = P->unit_values ? SCALE_SIGN : SCALE_VALUES; break;
  }
  const Shape sh = pick_shape(xdt, ydt, x, ldx, y, ldy, n_cols);
  for (int64_t c0 = 0; c0 < n_cols; c0 += sh.cb) {
    const int64_t cols = std::min(sh.cb, n_cols - c0);
    const int64_t nvec = cols / sh.v;
    int team, vpl;
    team_for(nvec, &team, &vpl);
    const int64_t ldp = round4(cols);
    FwdArgs a;
    std::memset(&a, 0, sizeof(a));
    a.n_items = (int32_t)P->n_items;
    a.node = P->d_node;
    a.ptr = P->d_ptr;
    a.ent = P->d_ent;
    a.val = P->d_val;
    a.cent = P->d_cent;
    a.cval = P->d_cval;
    a.par = P->d_par;
    a.par_item = P->d_par_item;
    a.self_slot = P->d_self_slot;
    a.par_slot = P->d_par_slot;
    a.chunk0 = P->d_chunk0;
    a.n_chunks = (int32_t)P->n_chunks;
    a.chunk_item = P->d_chunk_item;
    a.chunk_beg = P->d_chunk_beg;
    a.chunk_end = P->d_chunk_end;
    a.mult = P->d_mult;
    a.node_flag = P->d_node_flag;
    a.chunk_flag = P->d_chunk_flag;
    a.qs = P->d_qs;
    a.x = static_cast<const char*>(x) + c0 * elem_size(xdt);
    a.ldx = ldx;
    a.y = static_cast<char*>(y) + c0 * elem_size(ydt);
    a.ldy = ldy;
    a.nvec = (int32_t)nvec;
    a.ldp = (int32_t)ldp;
    a.partial = static_cast<float*>(ws);
    a.pstate = ws ? static_cast<float*>(ws) + P->n_chunks * ldp : nullptr;
    a.gin = gin ? 1 : 0;
    a.gin_scale = gin_scale;
    a.comp_item0 = (int32_t)P->n_items;
    a.comp_read0 = (int32_t)P->n_items;
    if (comp) {
      a.pcomp = static_cast<float*>(ws) + (P->n_chunks + (state_rows ? P->n_internal : 0)) * ldp;
      a.comp_item0 = (int32_t)P->level_start[P->comp_depth];
      a.comp_read0 = (int32_t)P->level_start[std::min<int64_t>(P->comp_depth + 1, P->levels)];
    }
    a.scale_mode = scale;
    a.prop_mode = prop;
    a.team = team;
    a.rows_per_claim = claim_rows(P);
    a.rows_per_claim_deep = deep_rows_per_claim(P);
    a.n_root = (int32_t)P->n_root;
    a.unit = P->d_unit;
    a.n_units = (int32_t)P->n_units;
    a.hints = P->hot_rows > 0 ? 1 : 0;
    a.timeout_ns = P->timeout_ns;
    a.publish_epoch = 1;
    int s_team = 0, s_vpl = 0;
    // The GIN form runs on the register kernel (its self term and state rows
    // stay out of the staged kernel's registers).  So does AUTO on trees where
    // most rows wait on a parent: there the work is a chain of short waits,
    // and the register kernel's lighter rows finish them sooner (measured on
    // the 170K-node GCN graph, 84 % of rows below level 0: 0.30 -> 0.18 ms at
    // 40 FP32 columns, 0.35 -> 0.23 ms at 128 BF16 columns; the 1M-node and
    // 2.4M-node power-law graphs, 5 % and 40 % below level 0, keep the staged
    // kernel).
    // (rows of at most 512 bytes: the widths measured; wider rows keep the
    // staged kernel, whose ring carries more bytes in flight per lane)
    const bool deep_tree = (P->n_items - P->n_root) * 2 > P->n_items && cols * elem_size(xdt) <= 512;
    // Two passes (FP32 Y, no GIN term, no compensation): every row's delta sum
    // first, with no parent waits, then the parent terms in level order
    // (prop_kernel).  Opt-in: AUTO keeps the fused pass, which measured as
    // fast or faster on every tree tried (the 7-level GCN graph, 40 FP32
    // columns: 179 us fused, 259 us in two passes; a 2,000-deep chain: 4.1 ms
    // either way).
    const bool two_pass = ydt == CBM_F32 && !gin && !comp && P->n_items > P->n_root &&
                          P->passes == CBM_PASSES_TWO;
    if (two_pass) {
      // the first pass waits on nothing: level-0 claim sizes for every row
      a.skip_parent = 1;
      a.publish_epoch = 0;
      a.n_root = a.n_items;
      a.unit = nullptr;
      a.n_units = 0;
    }
    const bool staged = sh.vec && !gin && P->variant != CBM_VARIANT_REGISTER &&
                        !(P->variant == CBM_VARIANT_AUTO && deep_tree && !two_pass) &&
                        staged_shape(nvec, sh.v, P->staged_team, &s_team, &s_vpl);
    const bool tma = staged && P->variant == CBM_VARIANT_TMA && tma_shape(nvec, sh.v, s_team, s_vpl);
    int rc;
    if (comp) {
      rc = launch_fwd_comp(P, a, ydt, sh.vec, vpl, st);
    } else if (tma) {
      CUtensorMap map;
      if ((rc = encode_x_map(&map, a.x, xdt, P->n_cols, ldx, cols))) return rc;
      a.team = s_team;
      a.tma_rb = (int32_t)(nvec * 16);
      rc = launch_tma(P, a, xdt, ydt, s_team, s_vpl, map, st);
    } else if (staged) {
      a.team = s_team;
      rc = launch_staged(P, a, xdt, ydt, s_team, s_vpl, st);
    } else {
      // on such trees level-0 claims of two rows also serve narrow operands
      // better (40 BF16 columns on the GCN graph: 0.26 -> 0.17 ms)
      if (P->variant == CBM_VARIANT_AUTO && deep_tree && !two_pass)
        a.rows_per_claim = std::min<int32_t>(a.rows_per_claim, 2);
      rc = launch_fwd(P, a, xdt, ydt, sh.vec, vpl, !deep_tree || two_pass, st);
    }
    if (rc) return rc;
    if (two_pass) {
      PropArgs pa;
      std::memset(&pa, 0, sizeof(pa));
      pa.n_items = (int32_t)P->n_items;
      pa.n_root = (int32_t)P->n_root;
      pa.node = P->d_node;
      pa.par = P->d_par;
      pa.par_item = P->d_par_item;
      pa.y = static_cast<float*>(a.y);
      pa.ldy = ldy;
      pa.mult = P->d_mult;
      pa.prop_mode = prop;
      pa.node_flag = P->d_node_flag;
      pa.qs = P->d_qs;
      pa.timeout_ns = P->timeout_ns;
      // FP32 rows in 16-byte vectors where Y allows them
      const bool yvec = cols % 4 == 0 && reinterpret_cast<uintptr_t>(a.y) % 16 == 0 && (ldy * 4) % 16 == 0;
      const int64_t ynvec = yvec ? cols / 4 : cols;
      int pteam, pvpl;
      team_for(ynvec, &pteam, &pvpl);
      pa.nvec = (int32_t)ynvec;
      pa.team = pteam;
      if ((rc = launch_prop(P, pa, yvec, pvpl, st))) return rc;
    }
  }
  return CBM_OK;
}

}  // namespace cbm

extern "C" {

int cbm_matmul_host(cbm_plan* P, int32_t op, const void* x_host, int32_t xdt, int64_t ldx_host, void* y_host,
                    int32_t ydt, int64_t ldy_host, int64_t n_cols, int64_t slab_cols, void* x_dev, void* y_dev,
                    void* ws, int64_t ws_bytes, void* stream) {
  CbmRange range("cbm_matmul_host");
  if (!P || n_cols < 0 || slab_cols < 0) return CBM_ERR_INVALID;
  if (!dtype_ok(xdt, ydt)) return CBM_ERR_DTYPE;
  if (n_cols == 0 || P->n_rows == 0) return CBM_OK;
  if (!x_host || !y_host || !x_dev || !y_dev) return CBM_ERR_INVALID;
  if (ldx_host < n_cols || ldy_host < n_cols) return CBM_ERR_SHAPE;
  const int64_t xs = elem_size(xdt), ys = elem_size(ydt);
  // slabs: a multiple of 16 bytes wide in both operands where possible
  int64_t w = slab_cols == 0 ? n_cols : std::min(slab_cols, n_cols);
  const int64_t unit = 16 / std::min(xs, ys);
  if (w < n_cols && w % unit != 0) w = std::min(n_cols, (w + unit - 1) / unit * unit);
  // slab boundaries: w columns each, the last one the remainder.  Narrower
  // first or last slabs (to shorten the copy-in that opens the pipeline and
  // the copy-out that closes it) measured slower on B200: strided copies of
  // 128-byte pieces lose much of their rate while the other direction runs.
  std::vector<int64_t> bounds(1, 0);
  while (n_cols - bounds.back() > w) bounds.push_back(bounds.back() + w);
  bounds.push_back(n_cols);
  const int64_t n_slabs = (int64_t)bounds.size() - 1;
  if (n_slabs > 4096) return CBM_ERR_INVALID;
  // the product's own checks (workspace, multipliers, op) run on the first slab
  int rc = pipeline_ready(P, (size_t)(3 * n_slabs + 2));
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaEvent_t* ev = P->events.data();
  const bool overlap = P->host_overlap;
  const int64_t layout[5] = {n_cols, w, n_slabs, xs, ys};
  const bool same_layout = P->host_prev_valid && std::equal(layout, layout + 5, P->host_prev_layout) &&
                           P->host_prev_xd == x_dev && P->host_prev_yd == y_dev;
  // the copy-out stream starts after the work already queued on the caller's
  // stream.  The copy-in does too, except with overlap after a previous call:
  // then it waits only until that call's products no longer read the device
  // copy of X (slab by slab with the same layout), so it runs under that
  // call's copy-out
  if (cudaEventRecord(ev[0], st) != cudaSuccess) return CBM_ERR_CUDA;
  if (cudaStreamWaitEvent(P->d2h, ev[0], 0) != cudaSuccess) return CBM_ERR_CUDA;
  if (!(overlap && P->host_prev_valid)) {
    if (cudaStreamWaitEvent(P->h2d, ev[0], 0) != cudaSuccess) return CBM_ERR_CUDA;
  } else if (!same_layout) {
    // other buffers or slabs: after the previous call's products and its
    // pending copy-out (the new device buffers may reuse its memory)
    if (cudaStreamWaitEvent(P->h2d, P->host_prev_prod, 0) != cudaSuccess) return CBM_ERR_CUDA;
    if (P->host_out_pending && cudaStreamWaitEvent(P->h2d, ev[1], 0) != cudaSuccess) return CBM_ERR_CUDA;
  }
  // a previous call's copy-out still pending: the products may not overwrite
  // the device copy of Y before it has left (slab by slab with the same layout)
  const bool wait_out = P->host_prev_valid && P->host_out_pending;
  if (wait_out && !same_layout && cudaStreamWaitEvent(st, ev[1], 0) != cudaSuccess) return CBM_ERR_CUDA;
  const char* xh = static_cast<const char*>(x_host);
  char* yh = static_cast<char*>(y_host);
  char* xd = static_cast<char*>(x_dev);
  char* yd = static_cast<char*>(y_dev);
  for (int64_t k = 0; k < n_slabs; ++k) {
    const int64_t c0 = bounds[k], cw = bounds[k + 1] - c0;
    cudaEvent_t in = ev[2 + 3 * k], prod = ev[3 + 3 * k], out = ev[4 + 3 * k];
    // each wait on the previous call's event of slab k is queued before this
    // call records that event again
    if (overlap && same_layout && cudaStreamWaitEvent(P->h2d, prod, 0) != cudaSuccess) return CBM_ERR_CUDA;
    if (cudaMemcpy2DAsync(xd + c0 * xs, n_cols * xs, xh + c0 * xs, ldx_host * xs, cw * xs, P->n_cols,
                          cudaMemcpyHostToDevice, P->h2d) != cudaSuccess)
      return CBM_ERR_CUDA;
    if (cudaEventRecord(in, P->h2d) != cudaSuccess) return CBM_ERR_CUDA;
    if (cudaStreamWaitEvent(st, in, 0) != cudaSuccess) return CBM_ERR_CUDA;
    if (wait_out && same_layout && cudaStreamWaitEvent(st, out, 0) != cudaSuccess) return CBM_ERR_CUDA;
    rc = cbm_matmul(P, op, xd + c0 * xs, xdt, n_cols, yd + c0 * ys, ydt, n_cols, cw, ws, ws_bytes, stream);
    if (rc) return rc;
    if (cudaEventRecord(prod, st) != cudaSuccess) return CBM_ERR_CUDA;
    if (k + 1 == n_slabs && cudaEventRecord(P->host_prev_prod, st) != cudaSuccess) return CBM_ERR_CUDA;
    if (cudaStreamWaitEvent(P->d2h, prod, 0) != cudaSuccess) return CBM_ERR_CUDA;
    if (cudaMemcpy2DAsync(yh + c0 * ys, ldy_host * ys, yd + c0 * ys, n_cols * ys, cw * ys, P->n_rows,
                          cudaMemcpyDeviceToHost, P->d2h) != cudaSuccess)
      return CBM_ERR_CUDA;
    if (cudaEventRecord(out, P->d2h) != cudaSuccess) return CBM_ERR_CUDA;
  }
  if (cudaEventRecord(ev[1], P->d2h) != cudaSuccess) return CBM_ERR_CUDA;
  P->host_prev_valid = true;
  std::copy(layout, layout + 5, P->host_prev_layout);
  P->host_prev_xd = x_dev;
  P->host_prev_yd = y_dev;
  // without overlap the caller's stream resumes once the last slab is back in
  // host memory; with it, once the products are done (the copy-out pending)
  P->host_out_pending = overlap;
  if (!overlap && cudaStreamWaitEvent(st, ev[1], 0) != cudaSuccess) return CBM_ERR_CUDA;
  return CBM_OK;
}

int cbm_plan_host_wait(cbm_plan* P, void* stream) {
  if (!P) return CBM_ERR_INVALID;
  if (!P->host_out_pending || P->events.size() < 2) return CBM_OK;
  return cuda_status(cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), P->events[1], 0));
}

int cbm_plan_prepare_adjoint(cbm_plan* P, void* stream) {
  if (!P) return CBM_ERR_INVALID;
  return build_adjoint(P, static_cast<cudaStream_t>(stream));
}

int cbm_matmul_adjoint(cbm_plan* P, int32_t op, const void* g, int32_t gdt, int64_t ldg, void* dx, int32_t ddt,
                       int64_t lddx, int64_t n_cols, void* ws, int64_t ws_bytes, void* stream) {
  CbmRange range("cbm_matmul_adjoint");
  if (!P || op < CBM_OP_AX || op > CBM_OP_DADX || n_cols < 0) return CBM_ERR_INVALID;
  if (!dtype_ok(gdt, ddt)) return CBM_ERR_DTYPE;
  if (n_cols == 0 || P->n_rows == 0 || P->n_cols == 0) return CBM_OK;
  if (!g || !dx) return CBM_ERR_INVALID;
  if (ldg < n_cols || lddx < n_cols || ldg > INT32_MAX || lddx > INT32_MAX) return CBM_ERR_SHAPE;
  if (overlaps(g, extent(P->n_rows, ldg, n_cols, gdt), dx, extent(P->n_cols, lddx, n_cols, ddt))) return CBM_ERR_SHAPE;
  if ((op == CBM_OP_ADX || op == CBM_OP_DADX) && (!P->d_mult || P->n_rows != P->n_cols)) return CBM_ERR_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = build_adjoint(P, st);
  if (rc) return rc;
  const int64_t need = cbm_plan_workspace_bytes(P, op, n_cols, gdt, ddt, 1);
  const bool need_ws = P->n_internal > 0 || P->n_t_chunks > 0;
  if (need_ws && (!ws || ws_bytes < need)) return CBM_ERR_WORKSPACE;
  if (ws && reinterpret_cast<uintptr_t>(ws) % 16 != 0) return CBM_ERR_INVALID;
  const Shape sh = pick_shape(gdt, ddt, g, ldg, dx, lddx, n_cols);
  for (int64_t c0 = 0; c0 < n_cols; c0 += sh.cb) {
    const int64_t cols = std::min(sh.cb, n_cols - c0);
    const int64_t nvec = cols / sh.v;
    int team, vpl;
    team_for(nvec, &team, &vpl);
    const int64_t ldp = round4(cols);
    float* h = static_cast<float*>(ws);
    float* partial = ws ? h + P->n_internal * ldp : nullptr;                 // transposed chunks
    float* rpartial = ws ? partial + P->n_t_chunks * ldp : nullptr;          // reverse chunks
    const void* gb = static_cast<const char*>(g) + c0 * elem_size(gdt);
    if (P->n_internal > 0) {
      RevArgs r;
      std::memset(&r, 0, sizeof(r));
      r.n_items = (int32_t)P->n_rev_items;
      r.node = P->d_rev_node;
      r.slot = P->d_rev_slot;
      r.ptr = P->d_rev_ptr;
      r.ent = P->d_rev_ent;
      r.chunk0 = P->d_rev_chunk0;
      r.nchunk = P->d_rev_nchunk;
      r.mult = P->d_mult;
      r.scale_g = op == CBM_OP_DADX;
      r.flag = P->d_adj_flag;
      r.chunk_flag = P->d_rev_chunk_flag;
      r.partial = rpartial;
      r.qs = P->d_qs;
      r.g = gb;
      r.ldg = ldg;
      r.h = h;
      r.ldp = (int32_t)ldp;
      r.nvec = (int32_t)nvec;
      r.team = team;
      // every reverse item waits on its children, claimed just before it: one
      // item per claim keeps a wait from holding up the claim's other items
      // (measured on the 170K-node GCN graph: 0.42 -> 0.26 ms at 40 columns)
      r.rows_per_claim = 1;
      r.timeout_ns = P->timeout_ns;
      if ((rc = launch_rev(P, r, gdt, sh.vec, vpl, st))) return rc;
    }
    TrArgs t;
    std::memset(&t, 0, sizeof(t));
    t.n_items = (int32_t)P->n_cols;
    t.ptr = P->d_t_ptr;
    t.ent = P->d_t_ent;
    t.n_chunks = (int32_t)P->n_t_chunks;
    t.chunk0 = P->d_t_chunk0;
    t.chunk_item = P->d_t_chunk_item;
    t.chunk_beg = P->d_t_chunk_beg;
    t.chunk_end = P->d_t_chunk_end;
    t.chunk_flag = P->d_t_chunk_flag;
    t.mult = P->d_mult;
    t.scale_g = op == CBM_OP_DADX;
    t.scale_out = op == CBM_OP_ADX || op == CBM_OP_DADX;
    t.qs = P->d_qs;
    t.g = gb;
    t.ldg = ldg;
    t.h = h;
    t.ldp = (int32_t)ldp;
    t.dx = static_cast<char*>(dx) + c0 * elem_size(ddt);
    t.lddx = lddx;
    t.nvec = (int32_t)nvec;
    t.partial = partial;
    t.team = team;
    t.rows_per_claim = claim_rows(P);
    t.timeout_ns = P->timeout_ns;
    if ((rc = launch_tr(P, t, gdt, ddt, sh.vec, vpl, st))) return rc;
  }
  return CBM_OK;
}

}  // extern "C"
