// The reference's CPU operators (the cbm_mkl_cpp module,
// cbm/cbm_extensions.cpp:351-919) as stateless GPU products on the reference's
// own layout.
//
// The reference binds eight products over a CSR matrix given by begin/end row
// pointers (MKL's four-array CSR) and, for the CBM forms, the compression tree
// as branch offsets plus (parent, child) edges in BFS order per branch.  They
// keep no state between calls, so neither do these: every call reads the
// caller's arrays directly (no plan, no re-layout, no upload).  The only
// memory they need beyond their operands is a caller-owned workspace of
// 256 + 8 N bytes: a status word and a claim counter, and per node a
// "has a parent" stamp and a "row is final" stamp.  Stamps are compared with a
// per-call value from a process-wide counter, so the workspace is never
// cleared between calls (it must be zero-filled once, before its first use).
//
// Kernels (all on the caller's stream, none synchronises):
//   direct_mark    every tree edge: stamp its child; check indices, that no
//                  node has two parents and that the branch offsets are a
//                  prefix sum ending at the edge count; zero the claim counter.
//   direct_spmm    Y[i] = sum_k val_k X[col_k] over row i's entries in order
//                  (one FMA per entry, the order of the oracle's restatement;
//                  MKL's own summation order may differ in the last bits), a
//                  team of lanes per row with 16-byte gathers of X rows;
//                  optionally + (1 + eps) X[i] fused into the store.
//   direct_update  tree edges claimed in their listed order (parents precede
//                  children in BFS order, so the earliest unfinished edge
//                  never waits): wait (bounded) until the parent row is final
//                  when the parent has a parent itself, then
//                  Y[v] = Y[v] + Y[u]                     (update)
//                  Y[v] = fma(Y[u], m[v] / m[u], Y[v])    (fused update, the
//                  rounding of cbm/cbm_extensions.cpp:660-697), and mark v final.
//   direct_spmm_t  Y = A^T X: each row's X row scattered into the rows of its
//                  columns with vector atomic adds (order not deterministic).
//   direct_axpy    Y += (1 + eps) X element-wise (the reference's cblas_saxpy),
//                  after the update of the GIN form.

#include "cbm_b200.h"
#include "launch.cuh"

#include <atomic>

namespace cbm {
namespace {

constexpr int kDirectThreads = 256;
constexpr int64_t kDirectHeader = 256;  // QueueState, padded

struct DirectArgs {
  const int32_t* rp_b;
  const int32_t* rp_e;
  const int32_t* col;
  const float* val;  // NULL: every entry 1
  int64_t n_rows, n_cols, nnz;
  const float* x;  // [n_x_rows, c]
  float* y;        // [n_rows (n_cols for the transpose), c]
  int64_t c;
  float self_scale;
  int32_t self_term;  // y = fma(self_scale, x[i], (A x)[i]) in the SpMM store
  const int32_t* branches;
  int64_t n_branch_offsets;
  const int32_t* src;
  const int32_t* dst;
  int64_t n_edges;
  const float* mult;  // NULL: plain update
  QueueState* qs;     // workspace header
  unsigned* has_parent;
  unsigned* ready;
  unsigned epoch;
  long long timeout_ns;
};

__device__ __forceinline__ void record(QueueState* qs, int code, long long info) {
  if (atomicCAS(&qs->error, 0, code) == 0) qs->error_info = info;
}

__global__ void __launch_bounds__(kDirectThreads) direct_mark(const DirectArgs a) {
  if (blockIdx.x == 0 && threadIdx.x == 0) a.qs->next_row = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < a.n_edges; e += stride) {
    const int32_t u = a.src[e], v = a.dst[e];
    if (u < 0 || u >= a.n_rows || v < 0 || v >= a.n_rows || u == v) {
      record(a.qs, CBM_ERR_INDEX, e);
      continue;
    }
    if (atomicExch(a.has_parent + v, a.epoch) == a.epoch) record(a.qs, CBM_ERR_STRUCTURE, e);  // two parents
  }
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n_branch_offsets; i += stride) {
    const int32_t b = a.branches[i];
    const bool bad = b < 0 || b > a.n_edges || (i == 0 && b != 0) ||
                     (i == a.n_branch_offsets - 1 && b != a.n_edges) || (i > 0 && a.branches[i - 1] > b);
    if (bad) record(a.qs, CBM_ERR_STRUCTURE, i);
  }
}

// Team of TL lanes per row; lane owns VPL vectors of V floats per pass of
// TL * VPL * V columns.
template <int TL, int VPL, int V>
__global__ void __launch_bounds__(kDirectThreads, 4) direct_spmm(const DirectArgs a) {
  constexpr int kTeams = kDirectThreads / TL;
  constexpr int U = (VPL * V >= 8) ? 4 : 8;  // entries whose gathers are in flight together
  constexpr int64_t kPass = (int64_t)TL * VPL * V;
  const int tl = threadIdx.x % TL;
  const int64_t n_teams = (int64_t)gridDim.x * kTeams;
  for (int64_t row = (int64_t)blockIdx.x * kTeams + threadIdx.x / TL; row < a.n_rows; row += n_teams) {
    int64_t b = a.rp_b[row], e = a.rp_e[row];
    if (b < 0 || e < b || e > a.nnz) {
      if (tl == 0) record(a.qs, CBM_ERR_INDEX, row);
      b = e = 0;
    }
    for (int64_t c0 = 0; c0 < a.c; c0 += kPass) {
      float acc[VPL][V];
#pragma unroll
      for (int q = 0; q < VPL; ++q)
#pragma unroll
        for (int j = 0; j < V; ++j) acc[q][j] = 0.f;
      // wide rows (groups of 4): the next group's columns and values are
      // loaded while the current group's X rows are gathered; narrow rows
      // (groups of 8) load each group's own at its start, which keeps their
      // registers within four blocks per SM
      constexpr bool kPrefetch = U == 4;
      int32_t pc[U];
      float pw[U];
      auto fetch = [&](int64_t k) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const bool in = k + u < e;
          pc[u] = in ? __ldg(a.col + k + u) : 0;
          pw[u] = (in && a.val) ? __ldg(a.val + k + u) : 1.f;
        }
      };
      if (kPrefetch && b < e) fetch(b);
      for (int64_t k0 = b; k0 < e; k0 += U) {
        const int n = (int)((e - k0) < U ? (e - k0) : U);
        int64_t off[U];
        float w[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          off[u] = -1;
          w[u] = 0.f;
          if (u < n) {
            const int32_t cj = kPrefetch ? pc[u] : __ldg(a.col + k0 + u);
            if (cj < 0 || cj >= a.n_cols) {
              if (tl == 0) record(a.qs, CBM_ERR_INDEX, k0 + u);
            } else {
              off[u] = (int64_t)cj * a.c;
              w[u] = kPrefetch ? pw[u] : (a.val ? __ldg(a.val + k0 + u) : 1.f);
            }
          }
        }
        if (kPrefetch && k0 + U < e) fetch(k0 + U);
        float xv[U][VPL][V];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
          for (int q = 0; q < VPL; ++q) {
            const int64_t cc = c0 + ((int64_t)q * TL + tl) * V;
            if (off[u] >= 0 && cc < a.c) {
              Vec<float, V>::load(a.x + off[u] + cc, xv[u][q]);
            } else {
#pragma unroll
              for (int j = 0; j < V; ++j) xv[u][q][j] = 0.f;
            }
          }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (off[u] >= 0)
#pragma unroll
            for (int q = 0; q < VPL; ++q)
#pragma unroll
              for (int j = 0; j < V; ++j) acc[q][j] = fmaf(w[u], xv[u][q][j], acc[q][j]);
      }
#pragma unroll
      for (int q = 0; q < VPL; ++q) {
        const int64_t cc = c0 + ((int64_t)q * TL + tl) * V;
        if (cc >= a.c) continue;
        if (a.self_term) {
          float xs[V];
          Vec<float, V>::load(a.x + row * a.c + cc, xs);
#pragma unroll
          for (int j = 0; j < V; ++j) acc[q][j] = fmaf(a.self_scale, xs[j], acc[q][j]);
        }
        store_vec<float, V>(a.y + row * a.c + cc, acc[q]);
      }
    }
  }
}

template <int TL, int VPL, int V>
__global__ void __launch_bounds__(kDirectThreads) direct_update(const DirectArgs a) {
  constexpr int64_t kPass = (int64_t)TL * VPL * V;
  const int tl = threadIdx.x % TL;
  const int lane = threadIdx.x & 31;
  const unsigned tmask = TL == 32 ? 0xffffffffu : (((1u << TL) - 1u) << (lane / TL * TL));
  for (;;) {
    unsigned base = 0;
    if (tl == 0) base = atomicAdd(&a.qs->next_row, 1u);
    base = __shfl_sync(tmask, base, 0, TL);
    if ((int64_t)base >= a.n_edges) break;
    const int64_t e = base;
    const int32_t u = a.src[e], v = a.dst[e];
    if (u < 0 || u >= a.n_rows || v < 0 || v >= a.n_rows || u == v) continue;  // recorded by direct_mark
    bool ok = true;
    if (a.has_parent[u] == a.epoch) ok = wait_flag(a.ready + u, a.epoch, a.qs, a.timeout_ns, e);
    if (ok) {
      const float r = a.mult ? __fdiv_rn(a.mult[v], a.mult[u]) : 1.f;
      const float* yu = a.y + (int64_t)u * a.c;
      float* yv = a.y + (int64_t)v * a.c;
      for (int64_t c0 = 0; c0 < a.c; c0 += kPass) {
#pragma unroll
        for (int q = 0; q < VPL; ++q) {
          const int64_t cc = c0 + ((int64_t)q * TL + tl) * V;
          if (cc >= a.c) continue;
          float pu[V], pv[V];
          load_f32_cg<V>(yu + cc, pu);
          load_f32_cg<V>(yv + cc, pv);
#pragma unroll
          for (int j = 0; j < V; ++j) pv[j] = a.mult ? fmaf(pu[j], r, pv[j]) : __fadd_rn(pv[j], pu[j]);
          store_f32<V>(yv + cc, pv);
        }
      }
    }
    // v is marked final even after a failed wait, so that no wait on it hangs
    __threadfence();
    __syncwarp(tmask);
    if (tl == 0) st_release(a.ready + v, a.epoch);
  }
}

template <int TL, int VPL, int V>
__global__ void __launch_bounds__(kDirectThreads) direct_spmm_t(const DirectArgs a) {
  constexpr int kTeams = kDirectThreads / TL;
  constexpr int64_t kPass = (int64_t)TL * VPL * V;
  const int tl = threadIdx.x % TL;
  const int64_t n_teams = (int64_t)gridDim.x * kTeams;
  for (int64_t row = (int64_t)blockIdx.x * kTeams + threadIdx.x / TL; row < a.n_rows; row += n_teams) {
    int64_t b = a.rp_b[row], e = a.rp_e[row];
    if (b < 0 || e < b || e > a.nnz) {
      if (tl == 0) record(a.qs, CBM_ERR_INDEX, row);
      continue;
    }
    if (b == e) continue;
    for (int64_t c0 = 0; c0 < a.c; c0 += kPass) {
      float xr[VPL][V];
#pragma unroll
      for (int q = 0; q < VPL; ++q) {
        const int64_t cc = c0 + ((int64_t)q * TL + tl) * V;
        if (cc < a.c) {
          Vec<float, V>::load(a.x + row * a.c + cc, xr[q]);
        } else {
#pragma unroll
          for (int j = 0; j < V; ++j) xr[q][j] = 0.f;
        }
      }
      for (int64_t k = b; k < e; ++k) {
        const int32_t cj = __ldg(a.col + k);
        if (cj < 0 || cj >= a.n_cols) {
          if (tl == 0 && c0 == 0) record(a.qs, CBM_ERR_INDEX, k);
          continue;
        }
        const float w = a.val ? __ldg(a.val + k) : 1.f;
        float* yr = a.y + (int64_t)cj * a.c;
#pragma unroll
        for (int q = 0; q < VPL; ++q) {
          const int64_t cc = c0 + ((int64_t)q * TL + tl) * V;
          if (cc >= a.c) continue;
          if constexpr (V == 4) {
            atomicAdd(reinterpret_cast<float4*>(yr + cc),
                      make_float4(w * xr[q][0], w * xr[q][1], w * xr[q][2], w * xr[q][3]));
          } else {
            atomicAdd(yr + cc, w * xr[q][0]);
          }
        }
      }
    }
  }
}

template <int V>
__global__ void __launch_bounds__(kDirectThreads) direct_axpy(const DirectArgs a) {
  const int64_t n = a.n_rows * a.c / V;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float xs[V], ys[V];
    Vec<float, V>::load(a.x + i * V, xs);
    load_f32_cg<V>(a.y + i * V, ys);
#pragma unroll
    for (int j = 0; j < V; ++j) ys[j] = fmaf(a.self_scale, xs[j], ys[j]);
    store_f32<V>(a.y + i * V, ys);
  }
}

int current_device() {
  int d = 0;
  return cudaGetDevice(&d) == cudaSuccess ? d : -1;
}

template <typename K>
int launch_direct(GridCache& cache, K kern, const DirectArgs& a, cudaStream_t st) {
  const int grid = cached_grid(cache, kern, current_device(), kDirectThreads, 0);
  if (grid <= 0) return CBM_ERR_CUDA;
  kern<<<grid, kDirectThreads, 0, st>>>(a);
  return cuda_status(cudaGetLastError());
}

enum DirectKernel { K_SPMM = 0, K_UPDATE = 1, K_SPMM_T = 2 };

template <int TL, int VPL, int V>
int launch_shape(int which, const DirectArgs& a, cudaStream_t st) {
  static GridCache c_spmm, c_update, c_spmm_t;
  switch (which) {
    case K_SPMM: return launch_direct(c_spmm, direct_spmm<TL, VPL, V>, a, st);
    case K_UPDATE: return launch_direct(c_update, direct_update<TL, VPL, V>, a, st);
    default: return launch_direct(c_spmm_t, direct_spmm_t<TL, VPL, V>, a, st);
  }
}

// Lanes per row and vectors per lane for c columns: 16-byte vectors when the
// operands allow them, a full warp per row from 32 vectors on, two vectors
// per lane from 64 on (passes of 256 columns), else the smallest power-of-two
// team that covers the row.
int launch_kernel(int which, const DirectArgs& a, bool vec, cudaStream_t st) {
  if (!vec) return launch_shape<32, 1, 1>(which, a, st);
  const int64_t nvec = a.c / 4;
  if (nvec >= 64) return launch_shape<32, 2, 4>(which, a, st);
  if (nvec > 16) return launch_shape<32, 1, 4>(which, a, st);
  if (nvec > 8) return launch_shape<16, 1, 4>(which, a, st);
  if (nvec > 4) return launch_shape<8, 1, 4>(which, a, st);
  if (nvec > 2) return launch_shape<4, 1, 4>(which, a, st);
  if (nvec > 1) return launch_shape<2, 1, 4>(which, a, st);
  return launch_shape<1, 1, 4>(which, a, st);
}

std::atomic<unsigned> g_call_epoch{0};

unsigned next_epoch() {
  unsigned e = g_call_epoch.fetch_add(1u) + 1u;
  if (e == 0) e = g_call_epoch.fetch_add(1u) + 1u;  // 0 is the zero-filled workspace's value
  return e;
}

bool aligned16(const void* p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; }

// One call: optional SpMM (or its transpose), optional tree update, optional
// trailing (1 + eps) X term.
struct DirectCall {
  bool spmm = false, transpose = false, update = false, axpy = false;
  const int32_t* rp_b = nullptr;
  const int32_t* rp_e = nullptr;
  const int32_t* col = nullptr;
  const float* val = nullptr;
  int64_t n_rows = 0, n_cols = 0, nnz = 0;
  const float* x = nullptr;
  int64_t c = 0;
  float self_scale = 1.f;
  const int32_t* branches = nullptr;
  int64_t n_branch_offsets = 0;
  const int32_t* src = nullptr;
  const int32_t* dst = nullptr;
  int64_t n_edges = 0;
  const float* mult = nullptr;
  float* y = nullptr;
  int64_t n_y_rows = 0;
  void* ws = nullptr;
  int64_t ws_bytes = 0;
  void* stream = nullptr;
};

int run(const DirectCall& k) {
  CbmRange range("cbm direct product");
  if (k.n_rows < 0 || k.n_cols < 0 || k.nnz < 0 || k.c < 0 || k.n_edges < 0 || k.n_branch_offsets < 0 ||
      k.n_y_rows < 0)
    return CBM_ERR_INVALID;
  if (!k.ws || k.ws_bytes < cbm_direct_workspace_bytes(k.n_y_rows) || !aligned16(k.ws)) return CBM_ERR_WORKSPACE;
  if (k.spmm && k.n_rows > 0 && (!k.rp_b || !k.rp_e || (k.nnz > 0 && !k.col))) return CBM_ERR_INVALID;
  if (k.update && k.n_edges > 0 && (!k.src || !k.dst)) return CBM_ERR_INVALID;
  if (k.update && k.n_branch_offsets > 0 && !k.branches) return CBM_ERR_INVALID;
  if (k.n_rows >= INT32_MAX || k.n_cols >= INT32_MAX || k.nnz >= INT32_MAX) return CBM_ERR_TOO_LARGE;
  if (k.c == 0 || k.n_y_rows == 0) return CBM_OK;
  if (!k.y || ((k.spmm || k.axpy) && !k.x)) return CBM_ERR_INVALID;
  // x and y must not overlap (the update reads and writes y in place)
  if (k.x) {
    const int64_t x_rows = k.transpose ? k.n_rows : (k.spmm ? k.n_cols : k.n_y_rows);
    const uintptr_t x0 = reinterpret_cast<uintptr_t>(k.x), y0 = reinterpret_cast<uintptr_t>(k.y);
    const uintptr_t xb = (uintptr_t)(x_rows * k.c * 4), yb = (uintptr_t)(k.n_y_rows * k.c * 4);
    if (x0 < y0 + yb && y0 < x0 + xb) return CBM_ERR_SHAPE;
  }
  cudaStream_t st = static_cast<cudaStream_t>(k.stream);
  DirectArgs a;
  memset(&a, 0, sizeof(a));
  a.rp_b = k.rp_b;
  a.rp_e = k.rp_e;
  a.col = k.col;
  a.val = k.val;
  a.n_rows = k.spmm ? k.n_rows : k.n_y_rows;
  a.n_cols = k.n_cols;
  a.nnz = k.nnz;
  a.x = k.x;
  a.y = k.y;
  a.c = k.c;
  a.self_scale = k.self_scale;
  a.branches = k.branches;
  a.n_branch_offsets = k.n_branch_offsets;
  a.src = k.src;
  a.dst = k.dst;
  a.n_edges = k.n_edges;
  a.mult = k.mult;
  a.qs = static_cast<QueueState*>(k.ws);
  a.has_parent = reinterpret_cast<unsigned*>(static_cast<char*>(k.ws) + kDirectHeader);
  a.ready = a.has_parent + k.n_y_rows;
  a.epoch = next_epoch();
  a.timeout_ns = 1000000000ll;
  const bool vec = k.c % 4 == 0 && aligned16(k.y) && (!k.x || aligned16(k.x));
  int rc;
  const bool tree = k.update && (k.n_edges > 0 || k.n_branch_offsets > 0);
  if (tree) {
    // the tree's nodes are the output rows
    a.n_rows = k.n_y_rows;
    direct_mark<<<sm_count(current_device()) * 4, kDirectThreads, 0, st>>>(a);
    if ((rc = cuda_status(cudaGetLastError()))) return rc;
    a.n_rows = k.spmm ? k.n_rows : k.n_y_rows;
  }
  if (k.spmm && k.transpose) {
    if (cudaMemsetAsync(k.y, 0, (size_t)(k.n_y_rows * k.c * 4), st) != cudaSuccess) return CBM_ERR_CUDA;
    if ((rc = launch_kernel(K_SPMM_T, a, vec, st))) return rc;
  } else if (k.spmm) {
    // GIN without a tree: (1 + eps) X fused into the SpMM's store
    a.self_term = k.axpy && !tree;
    if ((rc = launch_kernel(K_SPMM, a, vec, st))) return rc;
    a.self_term = 0;
  }
  if (tree && k.n_edges > 0) {
    a.n_rows = k.n_y_rows;
    if ((rc = launch_kernel(K_UPDATE, a, vec, st))) return rc;
  }
  if (k.axpy && (tree || !k.spmm)) {
    a.n_rows = k.n_y_rows;
    static GridCache c4, c1;
    rc = vec ? launch_direct(c4, direct_axpy<4>, a, st) : launch_direct(c1, direct_axpy<1>, a, st);
    if (rc) return rc;
  }
  return CBM_OK;
}

}  // namespace
}  // namespace cbm

using cbm::DirectCall;

extern "C" {

int64_t cbm_direct_workspace_bytes(int64_t n_rows) {
  if (n_rows < 0) return -1;
  return (cbm::kDirectHeader + 8 * n_rows + 255) / 256 * 256;
}

int cbm_direct_status(void* workspace, void* stream, int32_t* device_status, int64_t* info) {
  if (!workspace || !device_status) return CBM_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cbm::QueueState qs;
  if (cudaMemcpyAsync(&qs, workspace, sizeof(qs), cudaMemcpyDeviceToHost, st) != cudaSuccess) return CBM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return CBM_ERR_CUDA;
  *device_status = qs.error;
  if (info) *info = qs.error_info;
  if (qs.error != 0) {
    // clear the status (error and error_info) for the next calls
    if (cudaMemsetAsync(&static_cast<cbm::QueueState*>(workspace)->error, 0, 16, st) != cudaSuccess)
      return CBM_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return CBM_ERR_CUDA;
  }
  return CBM_OK;
}

int cbm_s_spmm_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col, const float* val,
                         int64_t n_rows, int64_t n_cols, int64_t nnz, const float* rhs, int64_t n_rhs_cols,
                         float* out, void* workspace, int64_t workspace_bytes, void* stream) {
  DirectCall k;
  k.spmm = true;
  k.rp_b = rp_b, k.rp_e = rp_e, k.col = col, k.val = val, k.n_rows = n_rows, k.n_cols = n_cols, k.nnz = nnz;
  k.x = rhs, k.c = n_rhs_cols, k.y = out, k.n_y_rows = n_rows;
  k.ws = workspace, k.ws_bytes = workspace_bytes, k.stream = stream;
  return cbm::run(k);
}

int cbm_s_spmm_csr_t_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col, const float* val,
                           int64_t n_rows, int64_t n_cols, int64_t nnz, const float* rhs, int64_t n_rhs_cols,
                           float* out, void* workspace, int64_t workspace_bytes, void* stream) {
  DirectCall k;
  k.spmm = true;
  k.transpose = true;
  k.rp_b = rp_b, k.rp_e = rp_e, k.col = col, k.val = val, k.n_rows = n_rows, k.n_cols = n_cols, k.nnz = nnz;
  k.x = rhs, k.c = n_rhs_cols, k.y = out, k.n_y_rows = n_cols;
  k.ws = workspace, k.ws_bytes = workspace_bytes, k.stream = stream;
  return cbm::run(k);
}

int cbm_s_spmm_add_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col, const float* val,
                             int64_t n_rows, int64_t n_cols, int64_t nnz, const float* rhs, int64_t n_rhs_cols,
                             float epsilon, float* out, void* workspace, int64_t workspace_bytes, void* stream) {
  if (n_rows != n_cols) return CBM_ERR_SHAPE;  // X[i] must exist for every row i
  DirectCall k;
  k.spmm = true;
  k.axpy = true;
  k.self_scale = 1.0f + epsilon;
  k.rp_b = rp_b, k.rp_e = rp_e, k.col = col, k.val = val, k.n_rows = n_rows, k.n_cols = n_cols, k.nnz = nnz;
  k.x = rhs, k.c = n_rhs_cols, k.y = out, k.n_y_rows = n_rows;
  k.ws = workspace, k.ws_bytes = workspace_bytes, k.stream = stream;
  return cbm::run(k);
}

int cbm_s_spmm_update_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col, const float* val,
                                int64_t n_rows, int64_t n_cols, int64_t nnz, const float* rhs, int64_t n_rhs_cols,
                                const int32_t* branches, int64_t n_branch_offsets, const int32_t* src,
                                const int32_t* dst, int64_t n_edges, float* out, void* workspace,
                                int64_t workspace_bytes, void* stream) {
  DirectCall k;
  k.spmm = true;
  k.update = true;
  k.rp_b = rp_b, k.rp_e = rp_e, k.col = col, k.val = val, k.n_rows = n_rows, k.n_cols = n_cols, k.nnz = nnz;
  k.x = rhs, k.c = n_rhs_cols, k.y = out, k.n_y_rows = n_rows;
  k.branches = branches, k.n_branch_offsets = n_branch_offsets, k.src = src, k.dst = dst, k.n_edges = n_edges;
  k.ws = workspace, k.ws_bytes = workspace_bytes, k.stream = stream;
  return cbm::run(k);
}

int cbm_s_spmm_fused_update_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col,
                                      const float* val, int64_t n_rows, int64_t n_cols, int64_t nnz,
                                      const float* rhs, int64_t n_rhs_cols, const int32_t* branches,
                                      int64_t n_branch_offsets, const int32_t* src, const int32_t* dst,
                                      int64_t n_edges, const float* multiplier, float* out, void* workspace,
                                      int64_t workspace_bytes, void* stream) {
  if (!multiplier && n_edges > 0) return CBM_ERR_INVALID;
  DirectCall k;
  k.spmm = true;
  k.update = true;
  k.mult = multiplier;
  k.rp_b = rp_b, k.rp_e = rp_e, k.col = col, k.val = val, k.n_rows = n_rows, k.n_cols = n_cols, k.nnz = nnz;
  k.x = rhs, k.c = n_rhs_cols, k.y = out, k.n_y_rows = n_rows;
  k.branches = branches, k.n_branch_offsets = n_branch_offsets, k.src = src, k.dst = dst, k.n_edges = n_edges;
  k.ws = workspace, k.ws_bytes = workspace_bytes, k.stream = stream;
  return cbm::run(k);
}

int cbm_s_spmm_update_add_csr_int32(const int32_t* rp_b, const int32_t* rp_e, const int32_t* col,
                                    const float* val, int64_t n_rows, int64_t n_cols, int64_t nnz,
                                    const float* rhs, int64_t n_rhs_cols, float epsilon, const int32_t* branches,
                                    int64_t n_branch_offsets, const int32_t* src, const int32_t* dst,
                                    int64_t n_edges, float* out, void* workspace, int64_t workspace_bytes,
                                    void* stream) {
  if (n_rows != n_cols) return CBM_ERR_SHAPE;
  DirectCall k;
  k.spmm = true;
  k.update = true;
  k.axpy = true;
  k.self_scale = 1.0f + epsilon;
  k.rp_b = rp_b, k.rp_e = rp_e, k.col = col, k.val = val, k.n_rows = n_rows, k.n_cols = n_cols, k.nnz = nnz;
  k.x = rhs, k.c = n_rhs_cols, k.y = out, k.n_y_rows = n_rows;
  k.branches = branches, k.n_branch_offsets = n_branch_offsets, k.src = src, k.dst = dst, k.n_edges = n_edges;
  k.ws = workspace, k.ws_bytes = workspace_bytes, k.stream = stream;
  return cbm::run(k);
}

int cbm_s_update_csr_int32(const int32_t* branches, int64_t n_branch_offsets, const int32_t* src,
                           const int32_t* dst, int64_t n_edges, float* out, int64_t n_out_rows,
                           int64_t n_out_cols, void* workspace, int64_t workspace_bytes, void* stream) {
  DirectCall k;
  k.update = true;
  k.y = out, k.n_y_rows = n_out_rows, k.c = n_out_cols;
  k.branches = branches, k.n_branch_offsets = n_branch_offsets, k.src = src, k.dst = dst, k.n_edges = n_edges;
  k.ws = workspace, k.ws_bytes = workspace_bytes, k.stream = stream;
  return cbm::run(k);
}

int cbm_s_fused_update_csr_int32(const int32_t* branches, int64_t n_branch_offsets, const int32_t* src,
                                 const int32_t* dst, int64_t n_edges, const float* multiplier, float* out,
                                 int64_t n_out_rows, int64_t n_out_cols, void* workspace, int64_t workspace_bytes,
                                 void* stream) {
  if (!multiplier && n_edges > 0) return CBM_ERR_INVALID;
  DirectCall k;
  k.update = true;
  k.mult = multiplier;
  k.y = out, k.n_y_rows = n_out_rows, k.c = n_out_cols;
  k.branches = branches, k.n_branch_offsets = n_branch_offsets, k.src = src, k.dst = dst, k.n_edges = n_edges;
  k.ws = workspace, k.ws_bytes = workspace_bytes, k.stream = stream;
  return cbm::run(k);
}

}  // extern "C"
