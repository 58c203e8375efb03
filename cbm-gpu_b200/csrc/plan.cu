// Host side of the CBM product: plan creation (validation + device layout) and
// the C-ABI entry points declared in include/cbm_b200.h.
//
// The reference keeps borrowed pointers to the cuSPARSE CSR and the BFS edge
// list (cbm/cbm.cu:95-142) and allocates a cuSPARSE buffer on every call
// (cbm/cbm.cu:181,203).  A plan instead owns one device copy of the structure
// laid out for the fused kernel:
//
//   items    rows sorted by tree depth (stable by node id): the work queue order
//   ent      column | sign << 31 of every delta entry, rows in item order
//   ptr      int64 offsets of each item's entries
//   par      parent node per item (-1 for children of the virtual root)
//   chunks   long rows split into fixed-size entry ranges, queued before rows
//
// plus the queue state and ready flags.  Calls allocate nothing.

#include "cbm_b200.h"
#include "kernels.cuh"
#include "plan.h"

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

namespace cbm {

int cuda_status(cudaError_t e) { return e == cudaSuccess ? CBM_OK : CBM_ERR_CUDA; }

template <typename T>
int dev_upload(T** dst, const std::vector<T>& src, cudaStream_t st, std::vector<void*>& owned) {
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

template <typename T>
int host_fetch(std::vector<T>& dst, const T* src, int64_t n, bool on_device, cudaStream_t st) {
  dst.resize(n);
  if (n == 0) return CBM_OK;
  if (!src) return CBM_ERR_INVALID;
  if (on_device) {
    if (cudaMemcpyAsync(dst.data(), src, n * sizeof(T), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      return CBM_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CBM_ERR_CUDA;
  } else {
    std::memcpy(dst.data(), src, n * sizeof(T));
  }
  return CBM_OK;
}

void free_all(std::vector<void*>& v) {
  for (void* p : v) cudaFree(p);
  v.clear();
}

// Checks the structure the way the kernels rely on it and returns each node's
// parent (-1: child of the virtual root) and depth.  Host only.
int validate_structure(const int32_t* rp, const int32_t* ci, int64_t n_rows, int64_t n_cols, int64_t nnz,
                       const int32_t* br, int64_t n_branch_offsets, const int32_t* es, const int32_t* ed,
                       int64_t n_edges, std::vector<int32_t>& parent, std::vector<int32_t>& depth) {
  if (n_rows < 0 || n_cols < 0 || nnz < 0 || n_edges < 0 || n_branch_offsets < 0) return CBM_ERR_INVALID;
  if (rp[0] != 0 || rp[n_rows] != nnz) return CBM_ERR_STRUCTURE;
  for (int64_t i = 0; i < n_rows; ++i)
    if (rp[i + 1] < rp[i]) return CBM_ERR_STRUCTURE;
  for (int64_t k = 0; k < nnz; ++k)
    if (ci[k] < 0 || ci[k] >= n_cols) return CBM_ERR_INDEX;
  if (n_branch_offsets > 0) {
    if (br[0] != 0 || br[n_branch_offsets - 1] != n_edges) return CBM_ERR_STRUCTURE;
    for (int64_t b = 0; b + 1 < n_branch_offsets; ++b)
      if (br[b + 1] < br[b]) return CBM_ERR_STRUCTURE;
  } else if (n_edges != 0) {
    return CBM_ERR_STRUCTURE;
  }
  parent.assign(n_rows, -1);
  for (int64_t e = 0; e < n_edges; ++e) {
    const int32_t u = es[e], v = ed[e];
    if (u < 0 || u >= n_rows || v < 0 || v >= n_rows) return CBM_ERR_INDEX;
    if (u == v || parent[v] != -1) return CBM_ERR_STRUCTURE;
    parent[v] = u;
  }
  // depth of every node; a cycle is a structure error
  depth.assign(n_rows, -1);
  std::vector<int32_t> stack;
  std::vector<char> on_stack(n_rows, 0);
  for (int64_t v0 = 0; v0 < n_rows; ++v0) {
    if (depth[v0] >= 0) continue;
    int32_t v = (int32_t)v0;
    stack.clear();
    while (v >= 0 && depth[v] < 0) {
      if (on_stack[v]) return CBM_ERR_STRUCTURE;
      on_stack[v] = 1;
      stack.push_back(v);
      v = parent[v];
    }
    int32_t d = (v >= 0) ? depth[v] : -1;
    for (size_t i = stack.size(); i-- > 0;) {
      depth[stack[i]] = ++d;
      on_stack[stack[i]] = 0;
    }
  }
  return CBM_OK;
}

// Builds the device stream layout for the current chunk size and uploads it:
// rows no longer than chunk_nnz keep their entries in s_ent, contiguous in
// item order (so a run of consecutive items is one contiguous entry range);
// longer rows have no entries there and are summed from c_ent in chunks of
// chunk_nnz entries.
int build_layout(cbm_plan* P, cudaStream_t st) {
  CbmRange range("cbm build_layout");
  free_all(P->chunk_bufs);
  const int64_t n = P->n_items;
  const int64_t T = P->chunk_nnz;
  const bool vals = !P->h_val.empty();
  std::vector<int64_t> sptr(n + 1, 0);
  std::vector<int32_t> chunk0(n, -1), citem;
  std::vector<int64_t> cbeg, cend;
  int64_t long_rows = 0, long_nnz = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t len = P->h_ptr[i + 1] - P->h_ptr[i];
    const bool is_long = len > T;
    sptr[i + 1] = sptr[i] + (is_long ? 0 : len);
    if (is_long) {
      ++long_rows;
      chunk0[i] = (int32_t)citem.size();
      for (int64_t s = 0; s < len; s += T) {
        citem.push_back((int32_t)i);
        cbeg.push_back(long_nnz + s);
        cend.push_back(long_nnz + std::min(len, s + T));
      }
      long_nnz += len;
    }
  }
  if (citem.size() > (size_t)INT32_MAX) return CBM_ERR_INVALID;
  // the hot_rows columns gathered most often get the hot bit (their X rows are
  // kept in L2 by the staged kernel)
  std::vector<uint32_t> hot(P->n_cols, 0u);
  if (P->hot_rows > 0 && P->n_cols > 0) {
    std::vector<int64_t> freq(P->n_cols, 0);
    for (uint32_t e : P->h_ent) freq[e & 0x3fffffffu]++;
    std::vector<int32_t> by(P->n_cols);
    for (int64_t c = 0; c < P->n_cols; ++c) by[c] = (int32_t)c;
    const int64_t k = std::min<int64_t>(P->hot_rows, P->n_cols);
    std::nth_element(by.begin(), by.begin() + (k - 1), by.end(),
                     [&](int32_t a, int32_t b) { return freq[a] > freq[b] || (freq[a] == freq[b] && a < b); });
    for (int64_t i = 0; i < k; ++i)
      if (freq[by[i]] > 1) hot[by[i]] = 0x40000000u;
  }
  std::vector<uint32_t> sent(sptr[n]), cent(long_nnz);
  std::vector<float> sval(vals ? sptr[n] : 0), cval(vals ? long_nnz : 0);
  for (int64_t i = 0, lo = 0; i < n; ++i) {
    const int64_t b = P->h_ptr[i], len = P->h_ptr[i + 1] - b;
    uint32_t* out = chunk0[i] >= 0 ? cent.data() + lo : sent.data() + sptr[i];
    for (int64_t q = 0; q < len; ++q) {
      const uint32_t e = P->h_ent[b + q];
      out[q] = e | hot[e & 0x3fffffffu];
    }
    if (chunk0[i] >= 0) {
      if (vals) std::memcpy(cval.data() + lo, P->h_val.data() + b, len * sizeof(float));
      lo += len;
    } else {
      if (vals) std::memcpy(sval.data() + sptr[i], P->h_val.data() + b, len * sizeof(float));
    }
  }
  P->n_chunks = (int64_t)citem.size();
  P->long_rows = long_rows;
  int rc;
  if ((rc = dev_upload(&P->d_ptr, sptr, st, P->chunk_bufs))) return rc;
  if ((rc = dev_upload(&P->d_ent, sent, st, P->chunk_bufs))) return rc;
  if ((rc = dev_upload(&P->d_val, sval, st, P->chunk_bufs))) return rc;
  if ((rc = dev_upload(&P->d_cent, cent, st, P->chunk_bufs))) return rc;
  if ((rc = dev_upload(&P->d_cval, cval, st, P->chunk_bufs))) return rc;
  if ((rc = dev_upload(&P->d_chunk0, chunk0, st, P->chunk_bufs))) return rc;
  if ((rc = dev_upload(&P->d_chunk_item, citem, st, P->chunk_bufs))) return rc;
  if ((rc = dev_upload(&P->d_chunk_beg, cbeg, st, P->chunk_bufs))) return rc;
  if ((rc = dev_upload(&P->d_chunk_end, cend, st, P->chunk_bufs))) return rc;
  if (P->n_chunks > 0) {
    void* f = nullptr;
    if (cudaMalloc(&f, P->n_chunks * sizeof(unsigned))) return CBM_ERR_ALLOC;
    P->chunk_bufs.push_back(f);
    if (cudaMemsetAsync(f, 0, P->n_chunks * sizeof(unsigned), st)) return CBM_ERR_CUDA;
    P->d_chunk_flag = static_cast<unsigned*>(f);
  } else {
    P->d_chunk_flag = nullptr;
  }
  // chunk flags restart at 0 while the epoch keeps counting: never equal
  if ((rc = build_units(P, st))) return rc;
  return cuda_status(cudaStreamSynchronize(st));
}

// Level-0 rows a team takes per claim: rows_per_claim, cut down on plans with
// fewer rows than that many per resident warp of the GPU (64 per SM).  A
// team's rows run one after another, so a small plan spreads them one per
// team instead (4,096 rows, 64 FP32 columns: 52 -> 17 us per product).
int32_t claim_rows(const cbm_plan* P) {
  const int64_t warps = (int64_t)sm_count(P->device) * 64;
  const int64_t fit = P->n_items / std::max<int64_t>(warps, 1);
  return (int32_t)std::max<int64_t>(1, std::min<int64_t>(P->rows_per_claim, fit));
}

// Rows below level 0 wait on parents claimed just before them; when they are a
// large share of the rows, one-row claims keep that chain short.  Otherwise
// their parents are long finished and larger claims cost less.
int32_t deep_rows_per_claim(const cbm_plan* P) {
  if (P->rows_per_claim_deep > 0) return P->rows_per_claim_deep;
  return (P->n_items - P->n_root) * 4 > P->n_items ? 1 : claim_rows(P);
}

// Claim units of the staged kernel.  Level-0 items (which wait on nothing) are
// grouped greedily into runs whose cost reaches rows_per_claim x the mean
// cost of a level-0 row, at most kMaxUnit items: teams that step together
// then get similar amounts of work.  A row costs its entries plus 4 (its
// finishing work); a split row costs its chunk count plus 4 (its entries are
// summed by chunk teams).  Items below level 0 keep fixed-size claims of
// deep_rows_per_claim items.
int build_units(cbm_plan* P, cudaStream_t st) {
  CbmRange range("cbm build_units");
  constexpr int64_t kMaxUnit = 8;  // items held one per lane by the narrowest team
  free_all(P->unit_bufs);
  P->d_unit = nullptr;
  P->n_units = 0;
  const int64_t n = P->n_items, nr = std::min<int64_t>(P->n_root, n);
  if (n == 0) return CBM_OK;
  const int64_t T = P->chunk_nnz;
  auto cost = [&](int64_t i) {
    const int64_t len = P->h_ptr[i + 1] - P->h_ptr[i];
    return (len > T ? (len + T - 1) / T : len) + 4;
  };
  double total = 0;
  for (int64_t i = 0; i < nr; ++i) total += (double)cost(i);
  const double target = nr > 0 ? claim_rows(P) * total / (double)nr : 0.0;
  std::vector<int32_t> unit(1, 0);
  int64_t i = 0;
  while (i < nr) {
    double c = 0;
    int64_t j = i;
    while (j < nr && j - i < kMaxUnit && (j == i || c + 0.5 * (double)cost(j) <= target)) c += (double)cost(j++);
    unit.push_back((int32_t)j);
    i = j;
  }
  const int64_t rd = std::max<int32_t>(1, std::min<int32_t>(deep_rows_per_claim(P), (int32_t)kMaxUnit));
  for (; i < n; i += rd) unit.push_back((int32_t)std::min(n, i + rd));
  P->n_units = (int64_t)unit.size() - 1;
  return dev_upload(&P->d_unit, unit, st, P->unit_bufs);
}

}  // namespace cbm

using namespace cbm;

extern "C" {

const char* cbm_status_string(int32_t s) {
  switch (s) {
    case CBM_OK: return "ok";
    case CBM_ERR_INVALID: return "invalid argument";
    case CBM_ERR_INDEX: return "index out of range";
    case CBM_ERR_ALLOC: return "allocation failed";
    case CBM_ERR_CUDA: return "CUDA runtime error";
    case CBM_ERR_STRUCTURE: return "invalid compression tree (not a forest, duplicate child or bad branch offsets)";
    case CBM_ERR_DTYPE: return "unsupported dtype combination";
    case CBM_ERR_SHAPE: return "bad shape, leading dimension or overlapping operands";
    case CBM_ERR_TIMEOUT: return "a device wait timed out";
    case CBM_ERR_UNSUPPORTED: return "operation needs multipliers or values the plan does not have";
    case CBM_ERR_WORKSPACE: return "workspace too small";
    case CBM_ERR_INTERNAL: return "internal error";
    case CBM_ERR_TOO_LARGE: return "too many rows for the fixed scratch of cbm_matmul_noalloc";
    default: return "unknown status";
  }
}

int cbm_validate(const int32_t* row_ptr, const int32_t* col_idx, int64_t n_rows, int64_t n_cols, int64_t nnz,
                 const int32_t* branches, int64_t n_branch_offsets, const int32_t* src, const int32_t* dst,
                 int64_t n_edges) {
  if (!row_ptr || (nnz > 0 && !col_idx) || (n_edges > 0 && (!src || !dst)) || (n_branch_offsets > 0 && !branches))
    return CBM_ERR_INVALID;
  std::vector<int32_t> parent, depth;
  return validate_structure(row_ptr, col_idx, n_rows, n_cols, nnz, branches, n_branch_offsets, src, dst, n_edges,
                            parent, depth);
}

int cbm_plan_create(const int32_t* row_ptr, const int32_t* col_idx, const float* values, int64_t n_rows,
                    int64_t n_cols, int64_t nnz, const int32_t* branches, int64_t n_branch_offsets,
                    const int32_t* src, const int32_t* dst, int64_t n_edges, const float* multipliers,
                    int32_t input_kind, void* stream, cbm_plan** out) {
  CbmRange range("cbm_plan_create");
  if (!out) return CBM_ERR_INVALID;
  *out = nullptr;
  if (n_rows < 0 || n_cols < 0 || nnz < 0 || n_edges < 0 || n_branch_offsets < 0) return CBM_ERR_INVALID;
  if (n_rows >= (int64_t)1 << 30 || n_cols >= (int64_t)1 << 30) return CBM_ERR_INVALID;  // 30-bit column field
  if (input_kind != CBM_INPUT_DEVICE && input_kind != CBM_INPUT_HOST) return CBM_ERR_INVALID;
  const bool dev = input_kind == CBM_INPUT_DEVICE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  cbm_plan* P = new (std::nothrow) cbm_plan();
  if (!P) return CBM_ERR_ALLOC;
  auto fail = [&](int rc) {
    free_all(P->unit_bufs);
    free_all(P->chunk_bufs);
    free_all(P->bufs);
    delete P;
    return rc;
  };
  if (cudaGetDevice(&P->device) != cudaSuccess) return fail(CBM_ERR_CUDA);
  P->n_rows = n_rows;
  P->n_cols = n_cols;
  P->nnz = nnz;
  P->n_edges = n_edges;

  std::vector<int32_t> rp, ci, br, es, ed;
  std::vector<float> vals, mult;
  int rc;
  if ((rc = host_fetch(rp, row_ptr, n_rows + 1, dev, st))) return fail(rc);
  if ((rc = host_fetch(ci, col_idx, nnz, dev, st))) return fail(rc);
  if (values) {
    if ((rc = host_fetch(vals, values, nnz, dev, st))) return fail(rc);
  }
  if ((rc = host_fetch(br, branches, n_branch_offsets, dev, st))) return fail(rc);
  if ((rc = host_fetch(es, src, n_edges, dev, st))) return fail(rc);
  if ((rc = host_fetch(ed, dst, n_edges, dev, st))) return fail(rc);
  if (multipliers) {
    if ((rc = host_fetch(mult, multipliers, n_rows, dev, st))) return fail(rc);
  }

  // ---- validation ----
  std::vector<int32_t> parent, depth;
  rc = validate_structure(rp.data(), ci.data(), n_rows, n_cols, nnz, br.data(), n_branch_offsets, es.data(),
                          ed.data(), n_edges, parent, depth);
  if (rc) return fail(rc);
  P->n_branches = n_branch_offsets > 0 ? n_branch_offsets - 1 : 0;
  // ---- level order ----
  int32_t max_depth = 0;
  for (int64_t v = 0; v < n_rows; ++v) max_depth = std::max(max_depth, depth[v]);
  P->levels = n_rows > 0 ? max_depth + 1 : 0;
  P->n_root = 0;
  for (int64_t v = 0; v < n_rows; ++v) P->n_root += depth[v] == 0;
  std::vector<int64_t> lvl_start(max_depth + 2, 0);
  for (int64_t v = 0; v < n_rows; ++v) lvl_start[depth[v] + 1]++;
  for (int32_t l = 0; l <= max_depth; ++l) lvl_start[l + 1] += lvl_start[l];
  P->level_start = lvl_start;
  std::vector<int32_t> order(n_rows);
  {
    std::vector<int64_t> fill(lvl_start.begin(), lvl_start.end() - 1);
    for (int64_t v = 0; v < n_rows; ++v) order[fill[depth[v]]++] = (int32_t)v;
  }
  std::vector<char> has_child(n_rows, 0);
  for (int64_t v = 0; v < n_rows; ++v)
    if (parent[v] >= 0) has_child[parent[v]] = 1;
  std::vector<int32_t> slot(n_rows, -1);
  int64_t n_internal = 0;
  for (int64_t i = 0; i < n_rows; ++i)
    if (has_child[order[i]]) slot[order[i]] = (int32_t)n_internal++;
  P->n_internal = n_internal;

  P->n_items = n_rows;
  std::vector<int32_t> item_node(n_rows), item_par(n_rows), item_self_slot(n_rows), item_par_slot(n_rows),
      item_par_item(n_rows), item_of(n_rows);
  for (int64_t i = 0; i < n_rows; ++i) item_of[order[i]] = (int32_t)i;
  P->h_ptr.assign(n_rows + 1, 0);
  for (int64_t i = 0; i < n_rows; ++i) {
    const int32_t v = order[i];
    item_node[i] = v | (has_child[v] ? (int32_t)0x80000000u : 0);
    item_par[i] = parent[v];
    item_self_slot[i] = slot[v];
    item_par_slot[i] = parent[v] >= 0 ? slot[parent[v]] : -1;
    item_par_item[i] = parent[v] >= 0 ? item_of[parent[v]] : -1;
    P->h_ptr[i + 1] = P->h_ptr[i] + (rp[v + 1] - rp[v]);
  }
  bool unit = true;
  for (int64_t k = 0; k < (int64_t)vals.size(); ++k)
    if (vals[k] != 1.0f && vals[k] != -1.0f) {
      unit = false;
      break;
    }
  P->unit_values = unit;
  P->has_values = !vals.empty();
  std::vector<uint32_t> ent(nnz);
  std::vector<float> lval;
  if (!unit) lval.resize(nnz);
  for (int64_t i = 0; i < n_rows; ++i) {
    const int32_t v = order[i];
    int64_t o = P->h_ptr[i];
    for (int64_t k = rp[v]; k < rp[v + 1]; ++k, ++o) {
      const bool neg = !vals.empty() && std::signbit(vals[k]);
      ent[o] = (uint32_t)ci[k] | (neg ? 0x80000000u : 0u);
      if (!unit) lval[o] = vals[k];
    }
  }
  // keep what the adjoint layout needs
  P->h_order = order;
  P->h_parent = parent;
  P->h_slot = slot;
  P->h_depth = depth;
  P->h_ent.swap(ent);
  P->h_val.swap(lval);

  // ---- upload ----
  if ((rc = dev_upload(&P->d_node, item_node, st, P->bufs))) return fail(rc);
  if ((rc = dev_upload(&P->d_par, item_par, st, P->bufs))) return fail(rc);
  if ((rc = dev_upload(&P->d_par_item, item_par_item, st, P->bufs))) return fail(rc);
  if ((rc = dev_upload(&P->d_self_slot, item_self_slot, st, P->bufs))) return fail(rc);
  if ((rc = dev_upload(&P->d_par_slot, item_par_slot, st, P->bufs))) return fail(rc);
  if (!mult.empty()) {
    if ((rc = dev_upload(&P->d_mult, mult, st, P->bufs))) return fail(rc);
  }
  {
    void* f = nullptr;
    const size_t bytes = std::max<int64_t>(n_rows, 1) * sizeof(unsigned);
    if (cudaMalloc(&f, bytes) != cudaSuccess) return fail(CBM_ERR_ALLOC);
    P->bufs.push_back(f);
    if (cudaMemsetAsync(f, 0, bytes, st) != cudaSuccess) return fail(CBM_ERR_CUDA);
    P->d_node_flag = static_cast<unsigned*>(f);
    if (cudaMalloc(&f, sizeof(QueueState)) != cudaSuccess) return fail(CBM_ERR_ALLOC);
    P->bufs.push_back(f);
    if (cudaMemsetAsync(f, 0, sizeof(QueueState), st) != cudaSuccess) return fail(CBM_ERR_CUDA);
    P->d_qs = static_cast<QueueState*>(f);
  }
  if ((rc = build_layout(P, st))) return fail(rc);
  *out = P;
  return CBM_OK;
}

int cbm_plan_set_multipliers(cbm_plan* P, const float* d_mult, void* stream) {
  if (!P || !d_mult) return CBM_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!P->d_mult && P->n_rows > 0) {
    void* p = nullptr;
    if (cudaMalloc(&p, P->n_rows * sizeof(float)) != cudaSuccess) return CBM_ERR_ALLOC;
    P->bufs.push_back(p);
    P->d_mult = static_cast<float*>(p);
  }
  if (P->n_rows > 0 &&
      cudaMemcpyAsync(P->d_mult, d_mult, P->n_rows * sizeof(float), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
    return CBM_ERR_CUDA;
  return CBM_OK;
}

int cbm_plan_tune(cbm_plan* P, int32_t chunk_nnz, int32_t rows_per_claim, int32_t rows_per_claim_deep,
                  int32_t variant, int64_t hot_rows, int32_t team, void* stream) {
  if (!P || chunk_nnz < 32 || rows_per_claim < 1 || rows_per_claim > 1024 || hot_rows < 0) return CBM_ERR_INVALID;
  if (rows_per_claim_deep < 0 || rows_per_claim_deep > 1024) return CBM_ERR_INVALID;
  const bool deep_changed = rows_per_claim_deep != P->rows_per_claim_deep;
  P->rows_per_claim_deep = rows_per_claim_deep;
  if (team != 0 && team != 8 && team != 16 && team != 32) return CBM_ERR_INVALID;
  P->staged_team = team;
  if (variant < CBM_VARIANT_AUTO || variant > CBM_VARIANT_TMA) return CBM_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaStreamSynchronize(st) != cudaSuccess) return CBM_ERR_CUDA;
  const bool claims_changed = rows_per_claim != P->rows_per_claim;
  P->rows_per_claim = rows_per_claim;
  P->variant = variant;
  if (chunk_nnz != P->chunk_nnz || hot_rows != P->hot_rows) {
    P->chunk_nnz = chunk_nnz;
    P->hot_rows = hot_rows;
    int rc = build_layout(P, st);  // rebuilds the units too
    if (rc) return rc;
    rc = rebuild_adjoint_chunks(P, st);
    if (rc) return rc;
  } else if (claims_changed || deep_changed) {
    int rc = build_units(P, st);
    if (rc) return rc;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CBM_ERR_CUDA;
  }
  return CBM_OK;
}

int cbm_plan_set_compensation(cbm_plan* P, int32_t min_depth) {
  if (!P || min_depth < -1) return CBM_ERR_INVALID;
  P->comp_depth = min_depth;
  return CBM_OK;
}

int cbm_plan_error(cbm_plan* P, void* stream, int32_t* device_status, int64_t* info) {
  if (!P || !device_status) return CBM_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaStreamSynchronize(st) != cudaSuccess) return CBM_ERR_CUDA;
  QueueState q;
  if (cudaMemcpy(&q, P->d_qs, sizeof(q), cudaMemcpyDeviceToHost) != cudaSuccess) return CBM_ERR_CUDA;
  *device_status = q.error;
  if (info) *info = q.error_info;
  if (q.error != 0) {
    const int zero[2] = {0, 0};
    if (cudaMemcpy(&P->d_qs->error, zero, sizeof(int) * 2, cudaMemcpyHostToDevice) != cudaSuccess)
      return CBM_ERR_CUDA;
  }
  return CBM_OK;
}

int64_t cbm_plan_stat(const cbm_plan* P, int32_t which) {
  if (!P) return -1;
  switch (which) {
    case CBM_P_ROWS: return P->n_rows;
    case CBM_P_COLS: return P->n_cols;
    case CBM_P_NNZ: return P->nnz;
    case CBM_P_EDGES: return P->n_edges;
    case CBM_P_BRANCHES: return P->n_branches;
    case CBM_P_LEVELS: return P->levels;
    case CBM_P_INTERNAL: return P->n_internal;
    case CBM_P_CHUNKS: return P->n_chunks;
    case CBM_P_LONG_ROWS: return P->long_rows;
    case CBM_P_UNIT_VALUES: return P->unit_values ? 1 : 0;
    case CBM_P_GRID: return P->last_grid;
    case CBM_P_LAUNCHES: return P->launches;
    default: return -1;
  }
}

void cbm_plan_destroy(cbm_plan* P) {
  if (!P) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != P->device) cudaSetDevice(P->device);
  release_pipeline(P);
  free_all(P->unit_bufs);
  free_all(P->chunk_bufs);
  free_all(P->adj_bufs);
  free_all(P->adj_chunk_bufs);
  free_all(P->bufs);
  if (cur >= 0 && cur != P->device) cudaSetDevice(cur);
  delete P;
}

}  // extern "C"
