// Device code of the CBM product: one persistent kernel per product.
//
//   Y[v] = sum_k s_k * X[col_k]   (the delta row of v)          cbm/cbm.cu:184-189
//        + Y[parent(v)]            (tree propagation)            cbm/cbm.cu:25-57
//        or + Y[parent(v)] * m[v] / m[parent(v)]                 cbm/cbm.cu:59-91
//
// The reference runs a cuSPARSE SpMM over all rows, then walks each tree branch
// serially in one thread block.  Here a single kernel does both in one pass:
// rows are taken from a device work queue in tree-level order, a team of lanes
// gathers the row's X rows with 16-byte loads, adds the parent's finished row
// (waiting on the parent's ready flag, a bounded wait), and writes Y[v] once.
// Rows longer than the chunk size are summed in chunks by other teams first
// (chunk items precede row items in the queue) and combined in a fixed order.
//
// Progress: items are claimed in queue order by running warps, every item
// depends only on earlier items, and each team finishes its items in claim
// order, so the earliest unfinished item never waits: no deadlock for any grid
// size.  Every wait is still bounded (globaltimer), recording CBM_ERR_TIMEOUT.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace cbm {

constexpr int kThreads = 256;

enum ScaleMode : int {
  SCALE_SIGN = 0,       // s
  SCALE_DCOL = 1,       // s * m[col]
  SCALE_DCOL_DROW = 2,  // (s * m[col]) * m[row]
  SCALE_VALUES = 3      // stored value
};
enum PropMode : int { PROP_ADD = 0, PROP_RATIO = 1 };

struct QueueState {
  unsigned int next_chunk;
  unsigned int next_row;
  unsigned int done_blocks;
  unsigned int epoch;
  int error;
  int pad;
  long long error_info;
};

struct FwdArgs {
  // rows in level order
  int32_t n_items;
  const int32_t* node;       // node id per item; bit 31 set: node has children
  const int64_t* ptr;        // [n_items + 1]
  const uint32_t* ent;       // column | sign << 31
  const float* val;          // values (SCALE_VALUES) or null
  const int32_t* par;        // parent node id, -1 for children of the virtual root
  const int32_t* self_slot;  // internal-node slot of the item's node, -1 if leaf
  const int32_t* par_slot;   // internal-node slot of the parent, -1
  const int32_t* chunk0;     // first chunk of a split row, -1
  // chunks of long rows
  int32_t n_chunks;
  const int32_t* chunk_item;
  const int64_t* chunk_beg;
  const int64_t* chunk_end;
  // state
  const float* mult;
  unsigned int* node_flag;   // [n_rows], ready epoch of internal nodes
  unsigned int* chunk_flag;  // [n_chunks]
  QueueState* qs;
  // operands
  const void* x;
  int64_t ldx;
  void* y;
  int64_t ldy;
  int32_t nvec;        // vectors per row (columns / V)
  int32_t ldp;         // floats per row of partial / parent-state scratch
  float* partial;      // [n_chunks, ldp]
  float* pstate;       // [n_internal, ldp] fp32 parent rows when Y is bf16
  int32_t scale_mode;
  int32_t prop_mode;
  int32_t team;        // lanes per row: 1, 2, 4, 8, 16 or 32
  int32_t rows_per_claim;
  long long timeout_ns;
};

// ---- memory-model helpers ----------------------------------------------------
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr long long kMaxSpins = 1ll << 22;

// Bounded wait until *flag == target.  Records the first failure in qs.
// Once any wait of the launch has failed, later waits give up at once, so a
// launch ends within about one timeout whatever goes wrong.
static __device__ __noinline__ bool wait_flag(const unsigned int* flag, unsigned int target, QueueState* qs,
                                              long long timeout_ns, long long info) {
  if (ld_acquire(flag) == target) return true;
  if (*(volatile int*)&qs->error != 0) return false;
  const unsigned long long t0 = global_ns();
  unsigned int ns = 32;
  for (long long it = 0; it < kMaxSpins; ++it) {
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
    if (ld_acquire(flag) == target) return true;
    if ((long long)(global_ns() - t0) > timeout_ns) break;
    if ((it & 63) == 63 && *(volatile int*)&qs->error != 0) return false;
  }
  if (atomicCAS(&qs->error, 0, 8 /* CBM_ERR_TIMEOUT */) == 0) qs->error_info = info;
  return false;
}

// ---- vector loads / stores ---------------------------------------------------
template <typename T, int V>
struct Vec;

template <>
struct Vec<float, 4> {
  static __device__ __forceinline__ void load(const float* p, float (&o)[4]) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
  }
};
template <>
struct Vec<float, 1> {
  static __device__ __forceinline__ void load(const float* p, float (&o)[1]) { o[0] = __ldg(p); }
};
template <>
struct Vec<__nv_bfloat16, 8> {
  static __device__ __forceinline__ void load(const __nv_bfloat16* p, float (&o)[8]) {
    const uint4 t = __ldg(reinterpret_cast<const uint4*>(p));
    const uint32_t w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      o[2 * i] = __uint_as_float(w[i] << 16);
      o[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
    }
  }
};
template <>
struct Vec<__nv_bfloat16, 1> {
  static __device__ __forceinline__ void load(const __nv_bfloat16* p, float (&o)[1]) {
    const unsigned short b = __ldg(reinterpret_cast<const unsigned short*>(p));
    o[0] = __uint_as_float(((uint32_t)b) << 16);
  }
};

// store V floats as T
template <typename T, int V>
__device__ __forceinline__ void store_vec(T* p, const float (&v)[V]);

template <>
__device__ __forceinline__ void store_vec<float, 4>(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
template <>
__device__ __forceinline__ void store_vec<float, 8>(float* p, const float (&v)[8]) {
  reinterpret_cast<float4*>(p)[0] = make_float4(v[0], v[1], v[2], v[3]);
  reinterpret_cast<float4*>(p)[1] = make_float4(v[4], v[5], v[6], v[7]);
}
template <>
__device__ __forceinline__ void store_vec<float, 1>(float* p, const float (&v)[1]) {
  *p = v[0];
}
template <>
__device__ __forceinline__ void store_vec<__nv_bfloat16, 8>(__nv_bfloat16* p, const float (&v)[8]) {
  __nv_bfloat162 h[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<uint4*>(p) = *reinterpret_cast<const uint4*>(h);
}
template <>
__device__ __forceinline__ void store_vec<__nv_bfloat16, 1>(__nv_bfloat16* p, const float (&v)[1]) {
  *p = __float2bfloat16_rn(v[0]);
}

// fp32 scratch rows (partials, parent state): L2-coherent loads after an acquire
template <int V>
__device__ __forceinline__ void load_f32_cg(const float* p, float (&o)[V]) {
  if constexpr (V % 4 == 0) {
#pragma unroll
    for (int i = 0; i < V / 4; ++i) {
      const float4 t = __ldcg(reinterpret_cast<const float4*>(p) + i);
      o[4 * i] = t.x; o[4 * i + 1] = t.y; o[4 * i + 2] = t.z; o[4 * i + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int i = 0; i < V; ++i) o[i] = __ldcg(p + i);
  }
}
template <int V>
__device__ __forceinline__ void store_f32(float* p, const float (&v)[V]) {
  if constexpr (V % 4 == 0) {
#pragma unroll
    for (int i = 0; i < V / 4; ++i)
      reinterpret_cast<float4*>(p)[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
  } else {
#pragma unroll
    for (int i = 0; i < V; ++i) p[i] = v[i];
  }
}
// parent row stored as T (Y itself): L2-coherent load
template <typename T, int V>
__device__ __forceinline__ void load_y_cg(const T* p, float (&o)[V]) {
  if constexpr (sizeof(T) == 4) {
    load_f32_cg<V>(reinterpret_cast<const float*>(p), o);
  } else {
    // bf16 parent rows are never read: the fp32 parent state is used instead
#pragma unroll
    for (int i = 0; i < V; ++i) o[i] = 0.f;
  }
}

template <int VPL, int V>
__host__ __device__ constexpr int unroll_for() {
  return (32 / (VPL * V)) < 1 ? 1 : ((32 / (VPL * V)) > 8 ? 8 : (32 / (VPL * V)));
}

// acc += sum over entries [beg, end) of scale_k * X[col_k]
template <typename XT, int VPL, int V>
__device__ __forceinline__ void gather_range(float (&acc)[VPL][V], const XT* __restrict__ x, int64_t ldx, int nvec,
                                             const uint32_t* __restrict__ ent, const float* __restrict__ val,
                                             int64_t beg, int64_t end, int scale_mode,
                                             const float* __restrict__ mult, float dv, int tl, int TL,
                                             unsigned tmask) {
  constexpr int U = unroll_for<VPL, V>();
  for (int64_t base = beg; base < end; base += TL) {
    const int64_t idx = base + tl;
    uint32_t e = 0;
    float sc = 0.f;
    if (idx < end) {
      e = __ldg(ent + idx);
      const uint32_t c = e & 0x7fffffffu;
      const float sgn = (e >> 31) ? -1.f : 1.f;
      if (scale_mode == SCALE_SIGN) {
        sc = sgn;
      } else if (scale_mode == SCALE_DCOL) {
        sc = sgn * __ldg(mult + c);
      } else if (scale_mode == SCALE_DCOL_DROW) {
        sc = __fmul_rn(sgn * __ldg(mult + c), dv);
      } else {
        sc = __ldg(val + idx);
      }
    }
    const int cnt = (int)((end - base) < TL ? (end - base) : TL);
    for (int j = 0; j < cnt; j += U) {
      float buf[U][VPL][V];
      float s[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint32_t eu = __shfl_sync(tmask, e, j + u < cnt ? j + u : 0, TL);
        s[u] = __shfl_sync(tmask, sc, j + u < cnt ? j + u : 0, TL);
        const XT* row = x + (int64_t)(eu & 0x7fffffffu) * ldx;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = tl + v * TL;
          if (j + u < cnt && vi < nvec) {
            Vec<XT, V>::load(row + (int64_t)vi * V, buf[u][v]);
          } else {
#pragma unroll
            for (int k = 0; k < V; ++k) buf[u][v][k] = 0.f;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (j + u < cnt) {
#pragma unroll
          for (int v = 0; v < VPL; ++v)
#pragma unroll
            for (int k = 0; k < V; ++k) acc[v][k] = fmaf(s[u], buf[u][v][k], acc[v][k]);
        }
      }
    }
  }
}

template <typename XT, typename YT, int VPL, int V>
__device__ __forceinline__ void fwd_chunk(const FwdArgs& a, int k, unsigned epoch, int tl, int TL, unsigned tmask) {
  float acc[VPL][V];
#pragma unroll
  for (int v = 0; v < VPL; ++v)
#pragma unroll
    for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
  const int item = a.chunk_item[k];
  const int node = a.node[item] & 0x7fffffff;
  const float dv = (a.scale_mode == SCALE_DCOL_DROW) ? __ldg(a.mult + node) : 1.f;
  gather_range<XT, VPL, V>(acc, static_cast<const XT*>(a.x), a.ldx, a.nvec, a.ent, a.val, a.chunk_beg[k],
                           a.chunk_end[k], a.scale_mode, a.mult, dv, tl, TL, tmask);
  float* prow = a.partial + (int64_t)k * a.ldp;
#pragma unroll
  for (int v = 0; v < VPL; ++v) {
    const int vi = tl + v * TL;
    if (vi < a.nvec) store_f32<V>(prow + vi * V, acc[v]);
  }
  __threadfence();
  __syncwarp(tmask);
  if (tl == 0) st_release(a.chunk_flag + k, epoch);
}

template <typename XT, typename YT, int VPL, int V>
__device__ __forceinline__ void fwd_row(const FwdArgs& a, int item, unsigned epoch, int tl, int TL, unsigned tmask) {
  float acc[VPL][V];
#pragma unroll
  for (int v = 0; v < VPL; ++v)
#pragma unroll
    for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
  const int nodew = a.node[item];
  const int node = nodew & 0x7fffffff;
  const bool internal = nodew < 0;
  const bool need_dv = (a.scale_mode == SCALE_DCOL_DROW) || (a.prop_mode == PROP_RATIO);
  const float dv = need_dv ? __ldg(a.mult + node) : 1.f;
  const int c0 = a.chunk0[item];
  if (c0 < 0) {
    gather_range<XT, VPL, V>(acc, static_cast<const XT*>(a.x), a.ldx, a.nvec, a.ent, a.val, a.ptr[item],
                             a.ptr[item + 1], a.scale_mode, a.mult, dv, tl, TL, tmask);
  } else {
    for (int k = c0; k < a.n_chunks && a.chunk_item[k] == item; ++k) {
      if (!wait_flag(a.chunk_flag + k, epoch, a.qs, a.timeout_ns, (long long)k)) continue;
      const float* prow = a.partial + (int64_t)k * a.ldp;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int vi = tl + v * TL;
        if (vi < a.nvec) {
          float t[V];
          load_f32_cg<V>(prow + vi * V, t);
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = __fadd_rn(acc[v][q], t[q]);
        }
      }
    }
  }
  const int p = a.par[item];
  // after a failed (timed-out) wait the parent is left out; the error is recorded
  if (p >= 0 && wait_flag(a.node_flag + p, epoch, a.qs, a.timeout_ns, (long long)node)) {
    const float dp = (a.prop_mode == PROP_RATIO) ? __ldg(a.mult + p) : 1.f;
    const int ps = a.par_slot[item];
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
      const int vi = tl + v * TL;
      if (vi < a.nvec) {
        float yp[V];
        if constexpr (sizeof(YT) == 4) {
          load_y_cg<YT, V>(static_cast<const YT*>(a.y) + (int64_t)p * a.ldy + (int64_t)vi * V, yp);
        } else {
          load_f32_cg<V>(a.pstate + (int64_t)ps * a.ldp + vi * V, yp);
        }
        if (a.prop_mode == PROP_RATIO) {
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = __fadd_rn(acc[v][q], __fdiv_rn(__fmul_rn(yp[q], dv), dp));
        } else {
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = __fadd_rn(acc[v][q], yp[q]);
        }
      }
    }
  }
  YT* yrow = static_cast<YT*>(a.y) + (int64_t)node * a.ldy;
#pragma unroll
  for (int v = 0; v < VPL; ++v) {
    const int vi = tl + v * TL;
    if (vi < a.nvec) store_vec<YT, V>(yrow + (int64_t)vi * V, acc[v]);
  }
  if (internal) {
    if constexpr (sizeof(YT) != 4) {
      float* srow = a.pstate + (int64_t)a.self_slot[item] * a.ldp;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int vi = tl + v * TL;
        if (vi < a.nvec) store_f32<V>(srow + vi * V, acc[v]);
      }
    }
    __threadfence();
    __syncwarp(tmask);
    if (tl == 0) st_release(a.node_flag + node, epoch);
  }
}

__device__ __forceinline__ void finish_block(QueueState* qs, unsigned epoch) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&qs->done_blocks, 1u);
    if (prev == gridDim.x - 1) {
      qs->next_chunk = 0;
      qs->next_row = 0;
      qs->done_blocks = 0;
      __threadfence();
      atomicExch(&qs->epoch, epoch);
    }
  }
}

template <typename XT, typename YT, int VPL, int V>
__global__ void __launch_bounds__(kThreads) fwd_kernel(const FwdArgs a) {
  const int lane = threadIdx.x & 31;
  const int TL = a.team;
  const int team = lane / TL;
  const int tl = lane & (TL - 1);
  const int teams = 32 / TL;
  const unsigned tmask = (TL == 32) ? 0xffffffffu : (((1u << TL) - 1u) << (team * TL));
  const unsigned epoch = *(volatile unsigned*)&a.qs->epoch + 1u;

  if (a.n_chunks > 0) {
    for (;;) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(&a.qs->next_chunk, (unsigned)teams);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= (unsigned)a.n_chunks) break;
      const unsigned k = base + team;
      if (k < (unsigned)a.n_chunks) fwd_chunk<XT, YT, VPL, V>(a, (int)k, epoch, tl, TL, tmask);
      __syncwarp();
    }
  }
  const unsigned per_claim = (unsigned)(teams * a.rows_per_claim);
  for (;;) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&a.qs->next_row, per_claim);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= (unsigned)a.n_items) break;
    for (int r = 0; r < a.rows_per_claim; ++r) {
      const unsigned item = base + team + (unsigned)(r * teams);
      if (item >= (unsigned)a.n_items) break;
      fwd_row<XT, YT, VPL, V>(a, (int)item, epoch, tl, TL, tmask);
    }
    __syncwarp();
  }
  finish_block(a.qs, epoch);
}

// ============================================================================
// Adjoint: dX = Delta^T P^T G' with P the tree-prefix operator (A = P Delta).
//   reverse pass   H[w] = G'[w] + sum over children c of H[c]   (deepest first)
//   transposed     dX[j] = m[j]^(ADX/DADX) * sum over (v, j, s) of s * H[v]
// with G' = m o G for DADX.  Leaves are not materialised: their H is G'.
// ============================================================================
constexpr uint32_t kInternalBit = 0x40000000u;
constexpr uint32_t kIndexMask = 0x3fffffffu;

struct RevArgs {
  int32_t n_items;       // internal nodes, deepest level first
  const int32_t* node;
  const int32_t* slot;
  const int64_t* ptr;    // children lists
  const uint32_t* ent;   // child | internal bit (slot then)
  const float* mult;
  int32_t scale_g;       // G' = m o G
  unsigned int* flag;    // [n_internal]
  QueueState* qs;
  const void* g;
  int64_t ldg;
  float* h;              // [n_internal, ldp]
  int32_t ldp;
  int32_t nvec;
  int32_t team;
  int32_t rows_per_claim;
  long long timeout_ns;
};

struct TrArgs {
  int32_t n_items;       // columns of Delta
  const int64_t* ptr;
  const uint32_t* ent;   // row | internal bit (slot then) | sign << 31
  int32_t n_chunks;
  const int32_t* chunk0;
  const int32_t* chunk_item;
  const int64_t* chunk_beg;
  const int64_t* chunk_end;
  unsigned int* chunk_flag;
  const float* mult;
  int32_t scale_g;       // leaves read m[v] * G[v]
  int32_t scale_out;     // dX[j] *= m[j]
  QueueState* qs;
  const void* g;
  int64_t ldg;
  const float* h;
  int32_t ldp;
  void* dx;
  int64_t lddx;
  int32_t nvec;
  float* partial;
  int32_t team;
  int32_t rows_per_claim;
  long long timeout_ns;
};

// acc += sum over entries of s * (internal ? H[slot] : scale * G[row]).  With
// wait != 0 each internal entry's ready flag is awaited first.
template <typename GT, int VPL, int V>
__device__ __forceinline__ void gather_dual(float (&acc)[VPL][V], const GT* __restrict__ g, int64_t ldg,
                                            const float* __restrict__ h, int ldp, int nvec,
                                            const uint32_t* __restrict__ ent, int64_t beg, int64_t end,
                                            const float* __restrict__ mult, bool scale_g, bool signed_ent,
                                            const unsigned int* flag, unsigned epoch, QueueState* qs,
                                            long long timeout_ns, int tl, int TL, unsigned tmask) {
  constexpr int U = unroll_for<VPL, V>();
  for (int64_t base = beg; base < end; base += TL) {
    const int64_t idx = base + tl;
    uint32_t e = 0;
    float sc = 0.f;
    if (idx < end) {
      e = __ldg(ent + idx);
      const uint32_t r = e & kIndexMask;
      const float sgn = (signed_ent && (e >> 31)) ? -1.f : 1.f;
      if (e & kInternalBit) {
        sc = sgn;
        if (flag) wait_flag(flag + r, epoch, qs, timeout_ns, (long long)r);
      } else {
        sc = scale_g ? sgn * __ldg(mult + r) : sgn;
      }
    }
    if (flag) __syncwarp(tmask);
    const int cnt = (int)((end - base) < TL ? (end - base) : TL);
    for (int j = 0; j < cnt; j += U) {
      float buf[U][VPL][V];
      float s[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int src = j + u < cnt ? j + u : 0;
        const uint32_t eu = __shfl_sync(tmask, e, src, TL);
        s[u] = __shfl_sync(tmask, sc, src, TL);
        const uint32_t r = eu & kIndexMask;
        const bool in = (eu & kInternalBit) != 0;
        if (in && flag && j + u < cnt) {
          // every lane acquires the flag itself before reading the row
          wait_flag(flag + r, epoch, qs, timeout_ns, (long long)r);
        }
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = tl + v * TL;
          if (j + u < cnt && vi < nvec) {
            if (in) {
              load_f32_cg<V>(h + (int64_t)r * ldp + vi * V, buf[u][v]);
            } else {
              Vec<GT, V>::load(g + (int64_t)r * ldg + (int64_t)vi * V, buf[u][v]);
            }
          } else {
#pragma unroll
            for (int k = 0; k < V; ++k) buf[u][v][k] = 0.f;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (j + u < cnt) {
#pragma unroll
          for (int v = 0; v < VPL; ++v)
#pragma unroll
            for (int k = 0; k < V; ++k) acc[v][k] = fmaf(s[u], buf[u][v][k], acc[v][k]);
        }
      }
    }
  }
}

template <typename GT, int VPL, int V>
__global__ void __launch_bounds__(kThreads) rev_kernel(const RevArgs a) {
  const int lane = threadIdx.x & 31;
  const int TL = a.team;
  const int team = lane / TL;
  const int tl = lane & (TL - 1);
  const int teams = 32 / TL;
  const unsigned tmask = (TL == 32) ? 0xffffffffu : (((1u << TL) - 1u) << (team * TL));
  const unsigned epoch = *(volatile unsigned*)&a.qs->epoch + 1u;
  const GT* g = static_cast<const GT*>(a.g);
  const unsigned per_claim = (unsigned)(teams * a.rows_per_claim);
  for (;;) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&a.qs->next_row, per_claim);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= (unsigned)a.n_items) break;
    for (int rr = 0; rr < a.rows_per_claim; ++rr) {
      const unsigned item = base + team + (unsigned)(rr * teams);
      if (item >= (unsigned)a.n_items) break;
      const int w = a.node[item];
      const int ws = a.slot[item];
      float acc[VPL][V];
      const float sw = a.scale_g ? __ldg(a.mult + w) : 1.f;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int vi = tl + v * TL;
        if (vi < a.nvec) {
          float t[V];
          Vec<GT, V>::load(g + (int64_t)w * a.ldg + (int64_t)vi * V, t);
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = __fmul_rn(sw, t[q]);
        } else {
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
        }
      }
      gather_dual<GT, VPL, V>(acc, g, a.ldg, a.h, a.ldp, a.nvec, a.ent, a.ptr[item], a.ptr[item + 1], a.mult,
                              a.scale_g != 0, false, a.flag, epoch, a.qs, a.timeout_ns, tl, TL, tmask);
      float* hrow = a.h + (int64_t)ws * a.ldp;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int vi = tl + v * TL;
        if (vi < a.nvec) store_f32<V>(hrow + vi * V, acc[v]);
      }
      __threadfence();
      __syncwarp(tmask);
      if (tl == 0) st_release(a.flag + ws, epoch);
    }
    __syncwarp();
  }
  finish_block(a.qs, epoch);
}

template <typename GT, typename DT, int VPL, int V>
__global__ void __launch_bounds__(kThreads) tr_kernel(const TrArgs a) {
  const int lane = threadIdx.x & 31;
  const int TL = a.team;
  const int team = lane / TL;
  const int tl = lane & (TL - 1);
  const int teams = 32 / TL;
  const unsigned tmask = (TL == 32) ? 0xffffffffu : (((1u << TL) - 1u) << (team * TL));
  const unsigned epoch = *(volatile unsigned*)&a.qs->epoch + 1u;
  const GT* g = static_cast<const GT*>(a.g);
  if (a.n_chunks > 0) {
    for (;;) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(&a.qs->next_chunk, (unsigned)teams);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= (unsigned)a.n_chunks) break;
      const unsigned k = base + team;
      if (k < (unsigned)a.n_chunks) {
        float acc[VPL][V];
#pragma unroll
        for (int v = 0; v < VPL; ++v)
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
        gather_dual<GT, VPL, V>(acc, g, a.ldg, a.h, a.ldp, a.nvec, a.ent, a.chunk_beg[k], a.chunk_end[k],
                                a.mult, a.scale_g != 0, true, nullptr, epoch, a.qs, a.timeout_ns, tl, TL,
                                tmask);
        float* prow = a.partial + (int64_t)k * a.ldp;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = tl + v * TL;
          if (vi < a.nvec) store_f32<V>(prow + vi * V, acc[v]);
        }
        __threadfence();
        __syncwarp(tmask);
        if (tl == 0) st_release(a.chunk_flag + k, epoch);
      }
      __syncwarp();
    }
  }
  const unsigned per_claim = (unsigned)(teams * a.rows_per_claim);
  for (;;) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&a.qs->next_row, per_claim);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= (unsigned)a.n_items) break;
    for (int rr = 0; rr < a.rows_per_claim; ++rr) {
      const unsigned item = base + team + (unsigned)(rr * teams);
      if (item >= (unsigned)a.n_items) break;
      float acc[VPL][V];
#pragma unroll
      for (int v = 0; v < VPL; ++v)
#pragma unroll
        for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
      const int c0 = a.chunk0[item];
      if (c0 < 0) {
        gather_dual<GT, VPL, V>(acc, g, a.ldg, a.h, a.ldp, a.nvec, a.ent, a.ptr[item], a.ptr[item + 1], a.mult,
                                a.scale_g != 0, true, nullptr, epoch, a.qs, a.timeout_ns, tl, TL, tmask);
      } else {
        for (int k = c0; k < a.n_chunks && a.chunk_item[k] == (int)item; ++k) {
          if (!wait_flag(a.chunk_flag + k, epoch, a.qs, a.timeout_ns, (long long)k)) continue;
          const float* prow = a.partial + (int64_t)k * a.ldp;
#pragma unroll
          for (int v = 0; v < VPL; ++v) {
            const int vi = tl + v * TL;
            if (vi < a.nvec) {
              float t[V];
              load_f32_cg<V>(prow + vi * V, t);
#pragma unroll
              for (int q = 0; q < V; ++q) acc[v][q] = __fadd_rn(acc[v][q], t[q]);
            }
          }
        }
      }
      const float so = a.scale_out ? __ldg(a.mult + item) : 1.f;
      DT* drow = static_cast<DT*>(a.dx) + (int64_t)item * a.lddx;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int vi = tl + v * TL;
        if (vi < a.nvec) {
          if (a.scale_out) {
#pragma unroll
            for (int q = 0; q < V; ++q) acc[v][q] = __fmul_rn(acc[v][q], so);
          }
          store_vec<DT, V>(drow + (int64_t)vi * V, acc[v]);
        }
      }
    }
    __syncwarp();
  }
  finish_block(a.qs, epoch);
}

}  // namespace cbm
