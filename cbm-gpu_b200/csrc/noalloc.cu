// cbm_matmul_noalloc: the CBM product for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc: a plugin loaded into a host process
// whose allocator already owns all of the GPU's memory, a serving loop that
// must not take cudaMalloc's implicit device synchronisation, or an extension
// point that is only ever handed buffers.  cbm_plan_create allocates (the
// plan's device layout) and cbm_matmul wants a caller-allocated workspace;
// this entry point needs neither.  It reads the delta matrix and the tree in
// the reference's own layout (CSR + BFS edge list) straight from the caller's
// buffers and keeps its scratch (queue counters, a status word, and per row a
// parent mark and a ready flag) in one fixed array compiled into this file.
//
// The array is a file-scope __device__ variable, zero-filled when the module
// loads: every GPU that loads this library holds its 8 MiB until the process
// exits.  Calls share it and it keeps the last call's contents: every call
// zeroes the queue counters before using them and clears the status word after
// reporting it; the parent marks and ready flags are compared against a stamp
// unique to the call (a process-wide counter on the host), so they need no
// clearing, and a call that stopped half-way cannot leave marks that the next
// call mistakes for its own.  Calls whose kernels overlap on the GPU (two
// streams, no ordering between them) race on the array and give wrong
// results.  Host code cannot use the array's name as a device address (on the
// host it names a host-side stand-in); the device address is fetched once per
// device with cudaGetSymbolAddress, with that device current, on the first
// call made on that device, and kept for the life of the process: after a
// cudaDeviceReset the module, and with it the array, is loaded anew at another
// address, so this entry point must not be used after a device reset.
//
// Two kernels on the caller's stream:
//   1. every row: Y[v] = sum_k val_k * X[col_k] (sequential FMAs per row, the
//      order cbm_matmul uses for rows it does not split; a row whose pointers
//      are not 0 <= begin <= end <= nnz is recorded and written as zeros), and
//      a mark on every node that has a parent (a second parent is recorded);
//   2. every tree edge (u, v), in the given BFS order, taken from a work queue:
//      wait (bounded) until u is final if u has a parent, then
//      Y[v] += Y[u]   or   Y[v] += Y[u] * m[v] / m[u]   (cbm/cbm.cu:54, :88),
//      and mark v final.

#include "cbm_b200.h"
#include "kernels.cuh"

#include <atomic>
#include <mutex>

namespace {

constexpr int64_t kScratchBytes = int64_t(8) << 20;  // 8 MiB per device
constexpr int64_t kHeaderBytes = 256;                // queue state
constexpr int64_t kMaxRows = (kScratchBytes - kHeaderBytes) / 8;  // two flags per row
constexpr int kMaxDevices = 64;
constexpr int kWarps = 8;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set-up on the
// first call per device).
int scratch_address(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return CBM_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return CBM_ERR_INVALID;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CBM_ERR_CUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return CBM_OK;
}

struct NoAllocArgs {
  const int32_t* row_ptr;
  const int32_t* col_idx;
  const float* values;
  int64_t n_rows, n_cols;
  const int32_t* src;
  const int32_t* dst;
  int64_t n_edges;
  const float* mult;
  const float* x;
  float* y;
  int64_t c;
  unsigned char* scratch;
  int32_t* status;
  unsigned stamp;  // unique to the call: marks and flags equal to it are this call's
  long long timeout_ns;
};

std::atomic<unsigned> g_stamp{0};

unsigned next_stamp() {
  unsigned s = g_stamp.fetch_add(1u) + 1u;
  if (s == 0) s = g_stamp.fetch_add(1u) + 1u;  // 0 is the zero-filled array's value
  return s;
}

__device__ __forceinline__ cbm::QueueState* state(const NoAllocArgs& a) {
  return reinterpret_cast<cbm::QueueState*>(a.scratch);
}
__device__ __forceinline__ unsigned* has_parent(const NoAllocArgs& a) {
  return reinterpret_cast<unsigned*>(a.scratch + kHeaderBytes);
}
__device__ __forceinline__ unsigned* ready(const NoAllocArgs& a) {
  return reinterpret_cast<unsigned*>(a.scratch + kHeaderBytes) + a.n_rows;
}

__device__ void record(cbm::QueueState* qs, int code, long long info) {
  if (atomicCAS(&qs->error, 0, code) == 0) qs->error_info = info;
}

// Kernel 1: delta rows, warp per row, 128 columns per pass; parent marks.
__global__ void __launch_bounds__(kWarps * 32) noalloc_rows(const NoAllocArgs a) {
  cbm::QueueState* qs = state(a);
  const unsigned target = a.stamp;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
  const int64_t n_warps = (int64_t)gridDim.x * kWarps;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    // the array keeps the previous call's contents: kernel 2's queue counters
    // must start at zero (kernel 2 starts after this kernel ends)
    qs->next_row = 0;
    qs->next_chunk = 0;
    qs->done_blocks = 0;
  }
  unsigned* hp = has_parent(a);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < a.n_edges;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = a.dst[e];
    if (v >= 0 && v < a.n_rows && atomicExch(hp + v, target) == target) record(qs, CBM_ERR_STRUCTURE, e);
  }
  const int64_t nnz = a.n_rows > 0 ? a.row_ptr[a.n_rows] : 0;
  for (int64_t row = warp; row < a.n_rows; row += n_warps) {
    int64_t b = a.row_ptr[row], e = a.row_ptr[row + 1];
    if (b < 0 || e < b || e > nnz) {
      if (lane == 0) record(qs, CBM_ERR_INDEX, row);
      b = e = 0;  // the row is written as zeros
    }
    for (int64_t c0 = 0; c0 < a.c; c0 += 128) {
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      for (int64_t base = b; base < e; base += 32) {
        const int64_t k = base + lane;
        int32_t col = 0;
        float val = 0.f;
        if (k < e) {
          col = a.col_idx[k];
          val = a.values ? a.values[k] : 1.f;
          if (col < 0 || col >= a.n_cols) {
            record(qs, CBM_ERR_INDEX, k);
            col = -1;  // skipped: nothing is read for it
          }
        }
        const int cnt = (int)((e - base) < 32 ? (e - base) : 32);
        for (int j = 0; j < cnt; ++j) {
          const int32_t cj = __shfl_sync(0xffffffffu, col, j);
          const float vj = __shfl_sync(0xffffffffu, val, j);
          if (cj < 0) continue;
          const float* xr = a.x + (int64_t)cj * a.c;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int64_t cc = c0 + lane + 32 * q;
            if (cc < a.c) acc[q] = fmaf(vj, __ldg(xr + cc), acc[q]);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int64_t cc = c0 + lane + 32 * q;
        if (cc < a.c) a.y[row * a.c + cc] = acc[q];
      }
    }
  }
}

// Kernel 2: tree edges from a work queue, in the given order.
__global__ void __launch_bounds__(kWarps * 32) noalloc_edges(const NoAllocArgs a) {
  cbm::QueueState* qs = state(a);
  const unsigned target = a.stamp;
  const int lane = threadIdx.x & 31;
  const unsigned* hp = has_parent(a);
  unsigned* rd = ready(a);
  constexpr unsigned kClaim = 4;
  for (;;) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&qs->next_row, kClaim);
    base = __shfl_sync(0xffffffffu, base, 0);
    if ((int64_t)base >= a.n_edges) break;
    for (unsigned r = 0; r < kClaim && (int64_t)(base + r) < a.n_edges; ++r) {
      const int64_t e = base + r;
      const int32_t u = a.src[e], v = a.dst[e];
      if (u < 0 || u >= a.n_rows || v < 0 || v >= a.n_rows) {
        if (lane == 0) record(qs, CBM_ERR_INDEX, e);
        continue;
      }
      bool ok = true;
      if (hp[u] == target) ok = cbm::wait_flag(rd + u, target, qs, a.timeout_ns, e);
      if (ok) {
        const float* yu = a.y + (int64_t)u * a.c;
        float* yv = a.y + (int64_t)v * a.c;
        const float mv = a.mult ? a.mult[v] : 1.f;
        const float mu = a.mult ? a.mult[u] : 1.f;
        for (int64_t cc = lane; cc < a.c; cc += 32) {
          const float pu = __ldcg(yu + cc);
          const float pv = __ldcg(yv + cc);
          yv[cc] = a.mult ? __fadd_rn(pv, __fdiv_rn(__fmul_rn(pu, mv), mu)) : __fadd_rn(pv, pu);
        }
      }
      __threadfence();
      __syncwarp();
      if (lane == 0) cbm::st_release(rd + v, target);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&qs->done_blocks, 1u);
    if (prev == gridDim.x - 1) {
      // report the status, then clear it for the next call
      if (a.status) *a.status = *(volatile int*)&qs->error;
      qs->error = 0;
      qs->error_info = 0;
      qs->next_row = 0;
      qs->done_blocks = 0;
      __threadfence();
    }
  }
}

int grid_of(const void* kernel) {
  int dev = 0, sms = 1, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kWarps * 32, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return sms * per_sm;
}

}  // namespace

extern "C" int cbm_matmul_noalloc(const int32_t* row_ptr, const int32_t* col_idx, const float* values,
                                  int64_t n_rows, int64_t n_cols, const int32_t* src, const int32_t* dst,
                                  int64_t n_edges, const float* multipliers, const float* x, float* y,
                                  int64_t n_x_cols, int32_t* d_status, void* stream) {
  if (n_rows < 0 || n_cols < 0 || n_edges < 0 || n_x_cols < 0) return CBM_ERR_INVALID;
  if (n_rows > kMaxRows) return CBM_ERR_TOO_LARGE;
  if (n_edges > 0 && n_edges >= n_rows) return CBM_ERR_STRUCTURE;  // a forest has fewer edges than nodes
  if (n_rows > 0 && (!row_ptr || !y || (n_x_cols > 0 && n_cols > 0 && !x))) return CBM_ERR_INVALID;
  if (n_edges > 0 && (!src || !dst)) return CBM_ERR_INVALID;
  if (!col_idx && n_rows > 0) return CBM_ERR_INVALID;
  void* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  NoAllocArgs a;
  a.row_ptr = row_ptr;
  a.col_idx = col_idx;
  a.values = values;
  a.n_rows = n_rows;
  a.n_cols = n_cols;
  a.src = src;
  a.dst = dst;
  a.n_edges = n_edges;
  a.mult = multipliers;
  a.x = x;
  a.y = y;
  a.c = n_x_cols;
  a.scratch = static_cast<unsigned char*>(scratch);
  a.status = d_status;
  a.stamp = next_stamp();
  a.timeout_ns = 1000000000ll;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  noalloc_rows<<<grid_of(reinterpret_cast<const void*>(noalloc_rows)), kWarps * 32, 0, st>>>(a);
  if (cudaGetLastError() != cudaSuccess) return CBM_ERR_CUDA;
  noalloc_edges<<<grid_of(reinterpret_cast<const void*>(noalloc_edges)), kWarps * 32, 0, st>>>(a);
  if (cudaGetLastError() != cudaSuccess) return CBM_ERR_CUDA;
  return CBM_OK;
}
