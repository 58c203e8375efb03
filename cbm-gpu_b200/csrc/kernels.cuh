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

#include <cuda.h>  // CUtensorMap (the TMA descriptor type)
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <climits>

namespace cbm {

constexpr int kThreads = 256;

// Forward entry word: column in bits 0-29, bit 30 set for the columns gathered
// most often (L2 keeps their X rows), bit 31 the sign.
constexpr uint32_t kColMask = 0x3fffffffu;
constexpr uint32_t kHotBit = 0x40000000u;

// Element offset of row r with leading dimension ld (below 2^31, which the
// host checks): one widening 32 x 32 -> 64-bit multiply per gathered row
// instead of a 64-bit one.
__device__ __forceinline__ uint64_t row_off(uint32_t r, int64_t ld) { return (uint64_t)r * (uint32_t)ld; }

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
  const int32_t* par_item;   // queue position of the parent's item, -1
  const int32_t* self_slot;  // internal-node slot of the item's node, -1 if leaf
  const int32_t* par_slot;   // internal-node slot of the parent, -1
  const int32_t* chunk0;     // first chunk of a split row, -1
  // chunks of long rows (entries in cent / cval)
  const uint32_t* cent;
  const float* cval;
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
  int32_t rows_per_claim;       // level-0 rows a team takes per claim
  int32_t rows_per_claim_deep;  // rows below level 0 a team takes per claim
  int32_t n_root;               // items [0, n_root) are level 0 (no parent)
  // staged kernel with several teams per warp: claims of one unit per team,
  // unit u = items [unit[u], unit[u + 1]) (at most 8), level-0 units balanced
  // by entries (null, or full-warp teams: claims of rows_per_claim /
  // rows_per_claim_deep items)
  const int32_t* unit;
  int32_t n_units;
  int32_t hints;       // L2 cache policies on (staged kernel)
  // compensated propagation (register kernel, COMP = true): items from
  // comp_item0 on (tree depth >= the plan's threshold) add their parent term
  // with an error-free sum and carry the rounding residual; items from
  // comp_read0 on (depth >= threshold + 1) read their parent's residual row
  int32_t comp_item0;
  int32_t comp_read0;
  float* pcomp;        // [n_internal, ldp] residual rows of internal nodes
  int32_t tma_rb;      // TMA variant: bytes of one gathered row (nvec * 16)
  // GIN form (register kernel only): Y[v] = (A X)[v] + gin_scale * X[v]
  // (gin_scale = 1 + epsilon), the self term added in the final store only;
  // internal nodes then keep their (A X) rows in pstate for their children,
  // as with BF16 Y
  int32_t gin;
  float gin_scale;
  // first pass of a two-pass product (FP32 Y): rows store their delta sums
  // only (no parent term, no ready flags); prop_kernel adds the parents
  int32_t skip_parent;
  int32_t publish_epoch;  // the last block publishes the launch epoch (0: a pass that another follows)
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

// evict-first (streaming) stores of V floats as T
template <typename T, int V>
__device__ __forceinline__ void store_vec_cs(T* p, const float (&v)[V]) {
  if constexpr (sizeof(T) == 4 && V % 4 == 0) {
#pragma unroll
    for (int i = 0; i < V / 4; ++i)
      __stcs(reinterpret_cast<float4*>(p) + i, make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]));
  } else if constexpr (sizeof(T) == 2 && V == 8) {
    __nv_bfloat162 h[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    __stcs(reinterpret_cast<uint4*>(p), *reinterpret_cast<const uint4*>(h));
  } else {
    store_vec<T, V>(p, v);
  }
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

// acc += sum over entries [beg, end) of scale_k * X[col_k], UF entries' gathers
// in flight per lane (0: unroll_for's choice); OFF32: X holds fewer than 2^32
// elements, so a row's offset is 32-bit element arithmetic
template <typename XT, int VPL, int V, int UF = 0, bool OFF32 = false>
__device__ __forceinline__ void gather_range(float (&acc)[VPL][V], const XT* __restrict__ x, int64_t ldx, int nvec,
                                             const uint32_t* __restrict__ ent, const float* __restrict__ val,
                                             int64_t beg, int64_t end, int scale_mode,
                                             const float* __restrict__ mult, float dv, int tl, int TL,
                                             unsigned tmask) {
  constexpr int U = UF > 0 ? UF : unroll_for<VPL, V>();
  for (int64_t base = beg; base < end; base += TL) {
    const int64_t idx = base + tl;
    uint32_t e = 0;
    float sc = 0.f;
    if (idx < end) {
      e = __ldg(ent + idx);
      const uint32_t c = e & kColMask;
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
        const XT* row = OFF32 ? x + (uint32_t)((eu & kColMask) * (uint32_t)ldx) : x + row_off(eu & kColMask, ldx);
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

// Resident blocks per SM of the register kernel.  Rows of one 16-byte vector
// per lane are latency-bound where X is L2-resident, and more warps hide more
// of the latency, at the cost of registers (gathers in flight).  Measured on
// B200, bit-identical results either way:
//   X and Y of one type: 4 blocks (at most 64 registers) with two gathers in
//     flight per lane (170K-node GCN graph: 128 BF16 columns 0.235 -> 0.210
//     ms, 128 FP32 0.311 -> 0.258, 40 FP32 0.180 -> 0.162);
//   BF16 X, FP32 Y: 3 blocks (at most 85 registers) where most rows wait on a
//     parent (GCN graph, 40 columns: 0.160 ms against 0.196 with 2 blocks and
//     0.210 with 4); WIDE, taken on shallower trees: 4 blocks with two in
//     flight (512-graph batch, 64 columns: 4.87 ms against 5.44 with 3 blocks
//     and 7.53 with 2).
template <typename XT, typename YT, int VPL, bool COMP, bool WIDE>
__host__ __device__ constexpr int fwd_min_blocks() {
  return (VPL != 1 || COMP) ? 1 : ((sizeof(XT) == sizeof(YT) || WIDE) ? 4 : 3);
}
template <typename XT, typename YT, int VPL, bool COMP, bool WIDE>
__host__ __device__ constexpr int fwd_in_flight() {
  return fwd_min_blocks<XT, YT, VPL, COMP, WIDE>() == 4 ? 2 : 0;  // 0: unroll_for's choice
}

template <typename XT, typename YT, int VPL, int V, bool COMP = false, bool WIDE = false, bool OFF32 = false>
__device__ __forceinline__ void fwd_chunk(const FwdArgs& a, int k, unsigned epoch, int tl, int TL, unsigned tmask) {
  float acc[VPL][V];
#pragma unroll
  for (int v = 0; v < VPL; ++v)
#pragma unroll
    for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
  const int item = a.chunk_item[k];
  const int node = a.node[item] & 0x7fffffff;
  const float dv = (a.scale_mode == SCALE_DCOL_DROW) ? __ldg(a.mult + node) : 1.f;
  gather_range<XT, VPL, V, fwd_in_flight<XT, YT, VPL, COMP, WIDE>(), OFF32>(
      acc, static_cast<const XT*>(a.x), a.ldx, a.nvec, a.cent, a.cval, a.chunk_beg[k], a.chunk_end[k],
      a.scale_mode, a.mult, dv, tl, TL, tmask);
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

// out = gin_scale * X[node] + acc (one rounding) for the GIN form, else acc
template <typename XT, int V>
__device__ __forceinline__ void gin_self(const FwdArgs& a, int node, int vi, const float (&acc)[V], float (&out)[V]) {
  if (a.gin) {
    float xs[V];
    Vec<XT, V>::load(static_cast<const XT*>(a.x) + (int64_t)node * a.ldx + (int64_t)vi * V, xs);
#pragma unroll
    for (int q = 0; q < V; ++q) out[q] = fmaf(a.gin_scale, xs[q], acc[q]);
  } else {
#pragma unroll
    for (int q = 0; q < V; ++q) out[q] = acc[q];
  }
}

// s + e == a + b exactly (Knuth's TwoSum; explicit roundings, no contraction)
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  const float bp = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bp)), __fsub_rn(b, bp));
}

template <typename XT, typename YT, int VPL, int V, bool COMP = false, bool WIDE = false, bool OFF32 = false>
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
    gather_range<XT, VPL, V, fwd_in_flight<XT, YT, VPL, COMP, WIDE>(), OFF32>(
        acc, static_cast<const XT*>(a.x), a.ldx, a.nvec, a.ent, a.val, a.ptr[item], a.ptr[item + 1],
        a.scale_mode, a.mult, dv, tl, TL, tmask);
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
  const int p = a.skip_parent ? -1 : a.par[item];
  // compensated arithmetic for this row, a residual to read from the parent
  const bool cmode = COMP && item >= a.comp_item0;
  const bool cread = COMP && item >= a.comp_read0;
  float cres[VPL][V];  // unused (and removed by the compiler) without COMP
#pragma unroll
  for (int v = 0; v < VPL; ++v)
#pragma unroll
    for (int q = 0; q < V; ++q) cres[v][q] = 0.f;
  // after a failed (timed-out) wait the parent is left out; the error is recorded
  if (p >= 0 && wait_flag(a.node_flag + p, epoch, a.qs, a.timeout_ns, (long long)node)) {
    const float dp = (a.prop_mode == PROP_RATIO) ? __ldg(a.mult + p) : 1.f;
    const int ps = a.par_slot[item];
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
      const int vi = tl + v * TL;
      if (vi < a.nvec) {
        float yp[V];
        if (sizeof(YT) == 4 && !a.gin) {
          load_y_cg<YT, V>(static_cast<const YT*>(a.y) + (int64_t)p * a.ldy + (int64_t)vi * V, yp);
        } else {
          load_f32_cg<V>(a.pstate + (int64_t)ps * a.ldp + vi * V, yp);
        }
        if (COMP && cmode) {
          // parent value = yp + rp (rp: its residual); add with TwoSum and keep
          // the rounding errors (of the ratio's product and quotient too)
          float rp[V];
          if (cread) {
            load_f32_cg<V>(a.pcomp + (int64_t)ps * a.ldp + vi * V, rp);
          } else {
#pragma unroll
            for (int q = 0; q < V; ++q) rp[q] = 0.f;
          }
#pragma unroll
          for (int q = 0; q < V; ++q) {
            float t = yp[q], r = rp[q];
            if (a.prop_mode == PROP_RATIO) {
              const float prod = __fmul_rn(yp[q], dv);
              const float pe = fmaf(yp[q], dv, -prod);     // prod + pe == yp * dv
              t = __fdiv_rn(prod, dp);
              const float qe = __fdiv_rn(fmaf(-t, dp, prod), dp);  // t + qe ~ prod / dp
              r = __fadd_rn(__fdiv_rn(fmaf(r, dv, pe), dp), qe);
            }
            float s_, e_;
            two_sum(acc[v][q], t, s_, e_);
            acc[v][q] = s_;
            cres[v][q] = __fadd_rn(r, e_);
          }
        } else if (a.prop_mode == PROP_RATIO) {
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = __fadd_rn(acc[v][q], __fdiv_rn(__fmul_rn(yp[q], dv), dp));
        } else {
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = __fadd_rn(acc[v][q], yp[q]);
        }
      }
    }
  }
  if (COMP && cmode) {
    // the row's value is acc + cres, rounded once; its residual is kept for
    // the children of an internal node
#pragma unroll
    for (int v = 0; v < VPL; ++v)
#pragma unroll
      for (int q = 0; q < V; ++q) {
        float s_, e_;
        two_sum(acc[v][q], cres[v][q], s_, e_);
        acc[v][q] = s_;
        cres[v][q] = e_;
      }
    if (internal) {
      float* crow = a.pcomp + (int64_t)a.self_slot[item] * a.ldp;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int vi = tl + v * TL;
        if (vi < a.nvec) store_f32<V>(crow + vi * V, cres[v]);
      }
    }
  }
  YT* yrow = static_cast<YT*>(a.y) + (int64_t)node * a.ldy;
#pragma unroll
  for (int v = 0; v < VPL; ++v) {
    const int vi = tl + v * TL;
    if (vi < a.nvec) {
      float out[V];
      gin_self<XT, V>(a, node, vi, acc[v], out);
      store_vec<YT, V>(yrow + (int64_t)vi * V, out);
    }
  }
  if (internal && !a.skip_parent) {
    if (sizeof(YT) != 4 || a.gin) {
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

// The last block to finish resets the queue counters and, unless another pass
// of the same product follows, publishes the launch epoch.
__device__ __forceinline__ void finish_block(QueueState* qs, unsigned epoch, bool publish = true) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(&qs->done_blocks, 1u);
    if (prev == gridDim.x - 1) {
      qs->next_chunk = 0;
      qs->next_row = 0;
      qs->done_blocks = 0;
      __threadfence();
      if (publish) atomicExch(&qs->epoch, epoch);
    }
  }
}

template <typename XT, typename YT, int VPL, int V, bool COMP = false, bool WIDE = false, bool OFF32 = false>
__global__ void __launch_bounds__(kThreads, (fwd_min_blocks<XT, YT, VPL, COMP, WIDE>()))
    fwd_kernel(const FwdArgs a) {
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
      if (k < (unsigned)a.n_chunks) fwd_chunk<XT, YT, VPL, V, COMP, WIDE, OFF32>(a, (int)k, epoch, tl, TL, tmask);
      __syncwarp();
    }
  }
  // claims of rows_per_claim rows per team while the queue is in level 0, of
  // rows_per_claim_deep below it (sized by where the warp's last claim fell)
  unsigned last = 0;
  for (;;) {
    const int R = last < (unsigned)a.n_root ? a.rows_per_claim : a.rows_per_claim_deep;
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&a.qs->next_row, (unsigned)(teams * R));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= (unsigned)a.n_items) break;
    last = base;
    for (int r = 0; r < R; ++r) {
      const unsigned item = base + team + (unsigned)(r * teams);
      if (item >= (unsigned)a.n_items) break;
      fwd_row<XT, YT, VPL, V, COMP, WIDE, OFF32>(a, (int)item, epoch, tl, TL, tmask);
    }
    __syncwarp();
  }
  finish_block(a.qs, epoch, a.publish_epoch != 0);
}

// ============================================================================
// Second pass of a two-pass product (FP32 Y): the first pass (fwd_kernel or
// fwd_stream_kernel with skip_parent) left every row's delta sum in Y; this
// pass adds the parent term to the rows below tree level 0, in level order
// (items [n_root, n_items)): wait (bounded) until the parent is final when it
// is itself below level 0, then
//   Y[v] = Y[v] + Y[u]                 (PROP_ADD)
//   Y[v] = Y[v] + (Y[u] m[v]) / m[u]   (PROP_RATIO, cbm/cbm.cu:88)
// the same additions, in the same order, as the one-pass kernels, so results
// are bit-identical.  A deep tree's rows then gather X without waiting on
// their parents, and the waits left here are short (no gathers behind them).
// ============================================================================
struct PropArgs {
  int32_t n_items;
  int32_t n_root;
  const int32_t* node;
  const int32_t* par;
  const int32_t* par_item;
  float* y;
  int64_t ldy;
  int32_t nvec;
  const float* mult;
  int32_t prop_mode;
  unsigned int* node_flag;
  QueueState* qs;
  int32_t team;
  long long timeout_ns;
};

template <int VPL, int V>
__global__ void __launch_bounds__(kThreads) prop_kernel(const PropArgs a) {
  const int lane = threadIdx.x & 31;
  const int TL = a.team;
  const int team = lane / TL;
  const int tl = lane & (TL - 1);
  const int teams = 32 / TL;
  const unsigned tmask = (TL == 32) ? 0xffffffffu : (((1u << TL) - 1u) << (team * TL));
  const unsigned epoch = *(volatile unsigned*)&a.qs->epoch + 1u;
  const unsigned n_deep = (unsigned)(a.n_items - a.n_root);
  for (;;) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&a.qs->next_row, (unsigned)teams);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n_deep) break;
    const unsigned k = base + team;
    if (k < n_deep) {
      const int item = a.n_root + (int)k;
      const int nodew = a.node[item];
      const int node = nodew & 0x7fffffff;
      const int p = a.par[item];
      bool ok = p >= 0;
      if (ok && a.par_item[item] >= a.n_root)
        ok = wait_flag(a.node_flag + p, epoch, a.qs, a.timeout_ns, (long long)node);
      if (ok) {
        const bool ratio = a.prop_mode == PROP_RATIO;
        const float dv = ratio ? __ldg(a.mult + node) : 1.f;
        const float dp = ratio ? __ldg(a.mult + p) : 1.f;
        const float* yp_row = a.y + (int64_t)p * a.ldy;
        float* yv_row = a.y + (int64_t)node * a.ldy;
        // passes of TL * VPL vectors cover rows of any width
        for (int vb = 0; vb < a.nvec; vb += TL * VPL) {
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = vb + tl + v * TL;
          if (vi < a.nvec) {
            float yp[V], yv[V];
            load_f32_cg<V>(yp_row + vi * V, yp);
            load_f32_cg<V>(yv_row + vi * V, yv);
            if (ratio) {
#pragma unroll
              for (int q = 0; q < V; ++q) yv[q] = __fadd_rn(yv[q], __fdiv_rn(__fmul_rn(yp[q], dv), dp));
            } else {
#pragma unroll
              for (int q = 0; q < V; ++q) yv[q] = __fadd_rn(yv[q], yp[q]);
            }
            store_f32<V>(yv_row + vi * V, yv);
          }
        }
        }
      }
      if (nodew < 0) {
        // marked final even after a failed wait, so that no wait on it hangs
        __threadfence();
        __syncwarp(tmask);
        if (tl == 0) st_release(a.node_flag + node, epoch);
      }
    }
    __syncwarp();
  }
  finish_block(a.qs, epoch);
}

// ============================================================================
// Staged variant of the forward kernel (16-byte vector path, teams of >= 8
// lanes).  The work a team claims is a run of consecutive items, and the
// stream layout stores their entries contiguously, so the team walks one flat
// entry range.  X rows are fetched with cp.async into a per-thread ring of S
// slots in shared memory, S entries ahead of the consumer, independent of row
// boundaries: S gathers stay in flight without holding registers.  Each lane
// copies and later reads only its own 16-byte pieces, so the only waits are
// the lane's own cp.async groups.  Column indices come in batches of TL (one
// coalesced load per batch), three batches in flight; the items' metadata for
// a claim is held one item per lane.  Rows are finished (chunk partials,
// parent, store, ready flag) when the consumer crosses their end.
// ============================================================================
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16_hint(void* smem, const void* gmem, uint64_t policy) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "l"(policy)
               : "memory");
}
// copies `bytes` (16 or 0) and zero-fills the rest: a copy that may be empty
// without a branch (the address must still point into the operand)
__device__ __forceinline__ void cp_async16_hint_n(void* smem, const void* gmem, unsigned bytes, uint64_t policy) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2, %3;" ::"r"(s), "l"(gmem), "r"(bytes),
               "l"(policy)
               : "memory");
}
// the same without an L2 policy
__device__ __forceinline__ void cp_async16_n(void* smem, const void* gmem, unsigned bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---- TMA (tile::gather4) and mbarrier helpers ------------------------------
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// makes initialised barriers visible to the TMA unit (the async proxy)
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// four rows r0..r3 of a 2-D tensor (box: all columns from col0, one row high)
// into dst, one after another; completion counted on bar
__device__ __forceinline__ void tma_gather4(void* dst, const CUtensorMap* map, int col0, int r0, int r1, int r2, int r3,
                                            uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7], %8;" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(col0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(smem_u32(bar)),
      "l"(policy)
      : "memory");
}
// Bounded wait for a barrier phase: try_wait (which itself suspends for a
// while) until the phase completes or timeout_ns pass.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, long long timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (long long it = 0; it < kMaxSpins; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((long long)(global_ns() - t0) > timeout_ns) break;
  }
  return false;
}

template <typename XT, int V>
__device__ __forceinline__ void unpack16(const uint4& r, float (&o)[V]) {
  if constexpr (sizeof(XT) == 4) {
    o[0] = __uint_as_float(r.x);
    o[1] = __uint_as_float(r.y);
    o[2] = __uint_as_float(r.z);
    o[3] = __uint_as_float(r.w);
  } else {
    const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      o[2 * i] = __uint_as_float(w[i] << 16);
      o[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
    }
  }
}

// Scale of one entry before the row factor: s, s * m[col] (both for
// SCALE_DCOL and SCALE_DCOL_DROW, whose consumer then multiplies by m[row]) or
// the stored value.
__device__ __forceinline__ float entry_scale(uint32_t e, int64_t idx, bool valid, int scale_mode, const float* mult,
                                             const float* val) {
  if (!valid) return 0.f;
  const float sgn = (e >> 31) ? -1.f : 1.f;
  if (scale_mode == SCALE_SIGN) return sgn;
  if (scale_mode == SCALE_VALUES) return __ldg(val + idx);
  return sgn * __ldg(mult + (e & kColMask));
}

// One team's pipelined pass over the `len` entries ent[k0, k0 + len).  With
// lockstep every lane of the warp calls it (a team with nothing to do passes
// len = 0).
// Positions are 32-bit and relative to k0; batches of TL entries start at
// multiples of TL.  next_end() gives the relative position where the
// current item ends (INT_MAX when none is left); on_end(acc) finishes it,
// resets acc and advances, updating row_dv (the row factor: m[row] under
// SCALE_DCOL_DROW, exactly 1 otherwise).
template <typename XT, int TL, int VPL, int V, int S, int BLOCK, bool OFF32, bool HINTS, typename NextEnd,
          typename OnEnd>
__device__ __forceinline__ void stream_pass(const XT* __restrict__ x, int64_t ldx, int nvec,
                                            const uint32_t* __restrict__ ent, const float* __restrict__ val,
                                            int64_t k0, int len, int scale_mode, const float* __restrict__ mult,
                                            uint4* __restrict__ ring, int tl, unsigned tmask, NextEnd next_end,
                                            OnEnd on_end, const float& row_dv, bool hints, bool lockstep) {
  static_assert(S <= TL && TL % S == 0, "ring depth must divide the team size");
  uint64_t pol_keep, pol_stream;
  if (hints) {
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol_keep));
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol_stream));
  } else {
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol_keep));
    pol_stream = pol_keep;
  }
  const uint32_t* ent0 = ent + k0;
  const float* val0 = val ? val + k0 : nullptr;
  const XT* xl = x + (int64_t)tl * V;  // this lane's first element of any row
  uint4* my = ring + threadIdx.x;      // this thread's ring: slot s, piece v at my[(s * VPL + v) * BLOCK]
  bool piece_ok[VPL];
#pragma unroll
  for (int v = 0; v < VPL; ++v) piece_ok[v] = tl + v * TL < nvec;

  // three batches of TL entries: A (holds the consumer position), B, C
  int bA = 0;
  uint32_t eA = 0, eB = 0, eC = 0;
  float sA = 0.f, sB = 0.f;
  {
    const int ia = tl, ib = TL + tl, ic = 2 * TL + tl;
    if (ia < len) eA = __ldcs(ent0 + ia);
    if (ib < len) eB = __ldcs(ent0 + ib);
    if (ic < len) eC = __ldcs(ent0 + ic);
    sA = entry_scale(eA, ia, ia < len, scale_mode, mult, val0);
    sB = entry_scale(eB, ib, ib < len, scale_mode, mult, val0);
  }
  // X row of entry word e from a lane's base: with OFF32 (X holds fewer than
  // 2^32 elements) a 32-bit element offset and one scaled add, else 64-bit
  auto row_at = [&](const XT* base, uint32_t e) -> const XT* {
    if constexpr (OFF32) {
      return base + (uint32_t)((e & kColMask) * (uint32_t)ldx);
    } else {
      return base + row_off(e & kColMask, ldx);
    }
  };
  // entry p's pieces into ring slot sp (no commit).  One piece per lane
  // (narrow rows): branch-free.  An entry past the stream's end (its word is
  // 0, so the address is X's first row) copies 0 bytes and zero-fills the
  // slot.  A lane without a piece (a row narrower than the team) copies the
  // first 16 bytes of the row, a valid address, into a slot whose sums no
  // store reads (every store is limited to the row's pieces); so the
  // per-entry code tests only the stream's end, with a constant size.
  // Several pieces per lane: pieces outside the row and entries past the end
  // are skipped (the slots keep old data, never read).
  const XT* xp = piece_ok[0] ? xl : x;
  auto produce = [&](int p, uint4* sp) {
    // HINTS: the entry's hot bit picks its L2 policy; without (a plan with
    // no hot set) the copies carry no policy and need no per-entry choice
    if constexpr (VPL == 1) {
      const bool inA = p < bA + TL;
      const uint32_t e = __shfl_sync(tmask, inA ? eA : eB, p & (TL - 1), TL);
      const XT* row = row_at(xp, e);
      if constexpr (HINTS) {
        const uint64_t pol = (e & kHotBit) ? pol_keep : pol_stream;
        cp_async16_hint_n(sp, row, p < len ? 16u : 0u, pol);
      } else {
        cp_async16_n(sp, row, p < len ? 16u : 0u);
      }
    } else if (p < len) {
      const bool inA = p < bA + TL;
      const uint32_t e = __shfl_sync(tmask, inA ? eA : eB, p & (TL - 1), TL);
      const XT* row = row_at(xl, e);
      const uint64_t pol = (e & kHotBit) ? pol_keep : pol_stream;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        if (piece_ok[v]) {
          if constexpr (HINTS) {
            cp_async16_hint(sp + v * BLOCK, row + v * TL * V, pol);
          } else {
            cp_async16(sp + v * BLOCK, row + v * TL * V);
          }
        }
      }
    }
  };
  // Entries move in groups of U (one cp.async group each, S / U groups in
  // flight); a group without a row end inside is consumed by straight-line
  // code (all U scales, then all U pieces, then the FMAs), one with a row end
  // (or past the stream's end) entry by entry.
  constexpr int U = S >= 8 ? 4 : 2;
  constexpr int G = S / U;
  static_assert(S % U == 0 && TL % U == 0, "groups must tile the ring and the batches");
#pragma unroll
  for (int j = 0; j < S; ++j) {
    produce(j, my + j * (VPL * BLOCK));
    if (j % U == U - 1) cp_async_commit();
  }

  float acc[VPL][V];
#pragma unroll
  for (int v = 0; v < VPL; ++v)
#pragma unroll
    for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
  int end_at = next_end();
  int slot = 0;  // ring slot of entry k (a multiple of U)
  // With lockstep, all teams of the warp step together (to the warp's longest
  // stream) so that one instruction serves every team, finished teams idling.
  // Only when no team waits on a row another team of the warp produces in the
  // same pass (the caller checks): a wait would then block the producer at
  // the per-step warp barrier.
  // (a full-warp team is alone in its warp: no lockstep, every step active)
  const bool ls = TL < 32 && lockstep;
  const int wlen = ls ? __reduce_max_sync(0xffffffffu, len) : len;
  auto consume = [&](int kk, uint4* sp, bool active) {
    float sc = __fmul_rn(__shfl_sync(tmask, sA, kk & (TL - 1), TL), row_dv);
#pragma unroll
    for (int v = 0; v < VPL; ++v) {
      if (piece_ok[v] && active) {
        float t[V];
        unpack16<XT, V>(sp[v * BLOCK], t);
#pragma unroll
        for (int q = 0; q < V; ++q) acc[v][q] = fmaf(sc, t[q], acc[v][q]);
      }
    }
  };
  for (int k = 0; k < wlen; k += U) {
    if (k == bA + TL) {
      // rotate: A <- B (scales ready), B <- C (scales now), load a new C
      bA += TL;
      eA = eB;
      sA = sB;
      eB = eC;
      const int ib = bA + TL + tl, ic = bA + 2 * TL + tl;
      sB = entry_scale(eB, ib, ib < len, scale_mode, mult, val0);
      eC = ic < len ? __ldcs(ent0 + ic) : 0u;
    }
    cp_async_wait<G - 1>();
    uint4* sp = my + slot * (VPL * BLOCK);
    if (k + U <= len && end_at >= k + U) {
      // row_dv is m[row] under SCALE_DCOL_DROW and exactly 1 otherwise
      if constexpr (VPL == 1) {
        // all U scales, then all U pieces, then the FMAs (lanes outside the
        // row add their placeholder pieces to accumulators no store reads)
        float sc[U];
        uint4 raw[U];
#pragma unroll
        for (int u = 0; u < U; ++u) sc[u] = __fmul_rn(__shfl_sync(tmask, sA, (k + u) & (TL - 1), TL), row_dv);
#pragma unroll
        for (int u = 0; u < U; ++u) raw[u] = sp[u * BLOCK];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          float t[V];
          unpack16<XT, V>(raw[u], t);
#pragma unroll
          for (int q = 0; q < V; ++q) acc[0][q] = fmaf(sc[u], t[q], acc[0][q]);
        }
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u) consume(k + u, sp + u * (VPL * BLOCK), true);
      }
    } else {
      for (int u = 0; u < U; ++u) {
        const int kk = k + u;
        const bool active = kk < len;
        if (active) {
          while (kk == end_at) {
            on_end(acc);
            end_at = next_end();
          }
        }
        consume(kk, sp + u * (VPL * BLOCK), active);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) produce(k + S + u, sp + u * (VPL * BLOCK));
    cp_async_commit();
    slot = (slot + U == S) ? 0 : slot + U;
    if (ls) __syncwarp();
  }
  cp_async_wait<0>();
  while (end_at <= len) {
    on_end(acc);
    end_at = next_end();
  }
  if (ls) __syncwarp();
}

// TMA variant of stream_pass: the team's rows come in groups of four by one
// tile::gather4 copy (issued by the team's first lane) into the team's ring of
// G slots of four rows, completion counted on one mbarrier per slot.
// Every lane owns every piece of a row here (nvec == TL * VPL, rows of 16-byte
// multiples, 128-byte multiples per row), so a lane reads pieces tl + v * TL of
// each gathered row.  The summation order is stream_pass's (sequential FMAs
// per row).  A wait that runs out records CBM_ERR_TIMEOUT and stops further
// copies; the copies already issued are waited for (bounded) before return.
template <typename XT, int TL, int VPL, int V, int G, typename NextEnd, typename OnEnd>
__device__ __forceinline__ void stream_pass_tma(const CUtensorMap* tmap, int rb, const uint32_t* __restrict__ ent,
                                                const float* __restrict__ val, int64_t k0, int len, int scale_mode,
                                                const float* __restrict__ mult, uint8_t* tring, uint64_t* tbar,
                                                unsigned& phase, int tl, unsigned tmask, NextEnd next_end,
                                                OnEnd on_end, const float& row_dv, bool hints, bool lockstep,
                                                QueueState* qs, long long timeout_ns) {
  static_assert(G >= 2 && (G & (G - 1)) == 0 && 4 * G <= TL, "G slots of four rows, 4G entries within two batches");
  uint64_t pol_keep, pol_stream;
  if (hints) {
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol_keep));
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol_stream));
  } else {
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(pol_keep));
    pol_stream = pol_keep;
  }
  const uint32_t* ent0 = ent + k0;
  const float* val0 = val ? val + k0 : nullptr;
  // a failure earlier in this launch: no more copies (the results are void)
  bool broken = *(volatile int*)&qs->error != 0;

  int bA = 0;
  uint32_t eA = 0, eB = 0, eC = 0;
  float sA = 0.f, sB = 0.f;
  {
    const int ia = tl, ib = TL + tl, ic = 2 * TL + tl;
    if (ia < len) eA = __ldcs(ent0 + ia);
    if (ib < len) eB = __ldcs(ent0 + ib);
    if (ic < len) eC = __ldcs(ent0 + ic);
    sA = entry_scale(eA, ia, ia < len, scale_mode, mult, val0);
    sB = entry_scale(eB, ib, ib < len, scale_mode, mult, val0);
  }
  int issued = 0;  // groups issued so far (group g: entries 4g .. 4g + 3)
  // entries of group g lie in batches A and B: the consumer is at 4g - 4G or
  // later, and 4G <= TL
  auto issue = [&](int g) {
    const int p0 = 4 * g;
    if (p0 >= len || broken) return;
    uint32_t e4[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int p = p0 + u < len ? p0 + u : len - 1;  // padding repeats the last row
      e4[u] = __shfl_sync(tmask, p < bA + TL ? eA : eB, p & (TL - 1), TL);
    }
    if (tl == 0) {
      const int sl = g & (G - 1);
      const uint64_t pol = ((e4[0] | e4[1] | e4[2] | e4[3]) & kHotBit) ? pol_keep : pol_stream;
      fence_proxy_async();
      mbar_expect_tx(tbar + sl, 4u * (unsigned)rb);
      tma_gather4(tring + (size_t)sl * 4 * rb, tmap, 0, (int)(e4[0] & kColMask), (int)(e4[1] & kColMask),
                  (int)(e4[2] & kColMask), (int)(e4[3] & kColMask), tbar + sl, pol);
    }
    issued = g + 1;
  };
#pragma unroll
  for (int g = 0; g < G; ++g) issue(g);

  float acc[VPL][V];
#pragma unroll
  for (int v = 0; v < VPL; ++v)
#pragma unroll
    for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
  int end_at = next_end();
  const bool ls = TL < 32 && lockstep;
  const int wlen = ls ? __reduce_max_sync(0xffffffffu, len) : len;
  int waited = 0;  // groups waited for
  auto consume = [&](int kk, const uint8_t* rowp, bool active) {
    const float sc = __fmul_rn(__shfl_sync(tmask, sA, kk & (TL - 1), TL), row_dv);
    if (active) {
      const uint4* pr = reinterpret_cast<const uint4*>(rowp) + tl;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        float t[V];
        unpack16<XT, V>(pr[v * TL], t);
#pragma unroll
        for (int q = 0; q < V; ++q) acc[v][q] = fmaf(sc, t[q], acc[v][q]);
      }
    }
  };
  for (int k = 0; k < wlen; k += 4) {
    if (k == bA + TL) {
      bA += TL;
      eA = eB;
      sA = sB;
      eB = eC;
      const int ib = bA + TL + tl, ic = bA + 2 * TL + tl;
      sB = entry_scale(eB, ib, ib < len, scale_mode, mult, val0);
      eC = ic < len ? __ldcs(ent0 + ic) : 0u;
    }
    const int g = k >> 2;
    const int sl = g & (G - 1);
    if (k < len && g < issued) {
      if (mbar_wait_bounded(tbar + sl, (phase >> sl) & 1u, timeout_ns)) {
        phase ^= 1u << sl;
      } else if (!broken) {
        broken = true;
        if (tl == 0 && atomicCAS(&qs->error, 0, 8 /* CBM_ERR_TIMEOUT */) == 0) qs->error_info = -1 - (long long)g;
      }
      waited = g + 1;
    }
    const uint8_t* slot = tring + (size_t)sl * 4 * rb;
    if (k + 4 <= len && end_at >= k + 4) {
      float sc[4];
      uint4 raw[4][VPL];
#pragma unroll
      for (int u = 0; u < 4; ++u) sc[u] = __fmul_rn(__shfl_sync(tmask, sA, (k + u) & (TL - 1), TL), row_dv);
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < VPL; ++v) raw[u][v] = reinterpret_cast<const uint4*>(slot + u * rb)[tl + v * TL];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          float t[V];
          unpack16<XT, V>(raw[u][v], t);
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = fmaf(sc[u], t[q], acc[v][q]);
        }
    } else {
      for (int u = 0; u < 4; ++u) {
        const int kk = k + u;
        const bool active = kk < len;
        if (active) {
          while (kk == end_at) {
            on_end(acc);
            end_at = next_end();
          }
        }
        consume(kk, slot + u * rb, active);
      }
    }
    // every lane of the team is done with the slot before it is refilled
    __syncwarp(tmask);
    issue(g + G);
    if (ls) __syncwarp();
  }
  // after a failure: wait (bounded) for the copies still in flight
  for (int g = waited; g < issued; ++g) {
    const int sl = g & (G - 1);
    if (mbar_wait_bounded(tbar + sl, (phase >> sl) & 1u, timeout_ns)) phase ^= 1u << sl;
  }
  while (end_at <= len) {
    on_end(acc);
    end_at = next_end();
  }
  if (ls) __syncwarp();
}

// TMA = true: rows arrive by tile::gather4 copies into per-team rings (the
// dynamic shared memory then holds BLOCK / TL teams x S / 4 slots of four
// rows of tma_rb bytes, followed by one mbarrier per slot: S entries in flight
// per team, as in the cp.async ring); `tmap` describes
// X (columns [0, nvec * V), every row, one-row box).  TMA = false: the
// per-thread cp.async ring of stream_pass (tmap unused).
template <typename XT, typename YT, int TL, int VPL, int V, int S, int BLOCK, bool TMA = false, bool OFF32 = false,
          bool HINTS = true>
__global__ void __launch_bounds__(BLOCK) fwd_stream_kernel(const FwdArgs a, const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(128) uint4 ring[];
  const int lane = threadIdx.x & 31;
  const int team = lane / TL;
  const int tl = lane & (TL - 1);
  constexpr int teams = 32 / TL;
  const unsigned tmask = (TL == 32) ? 0xffffffffu : (((1u << TL) - 1u) << (team * TL));
  const unsigned epoch = *(volatile unsigned*)&a.qs->epoch + 1u;
  const XT* x = static_cast<const XT*>(a.x);
  const bool hints = a.hints != 0;
  float ch_dv = 1.f;
  // TMA rings and barriers of this thread's team
  uint8_t* tring = nullptr;
  uint64_t* tbar = nullptr;
  unsigned tphase = 0;
  constexpr int G = S / 4;
  if constexpr (TMA) {
    constexpr int n_teams = BLOCK / TL;
    const int bt = threadIdx.x / TL;
    uint8_t* base = reinterpret_cast<uint8_t*>(ring);
    tring = base + (size_t)bt * G * 4 * a.tma_rb;
    tbar = reinterpret_cast<uint64_t*>(base + (size_t)n_teams * G * 4 * a.tma_rb) + bt * G;
    if (tl == 0) {
#pragma unroll
      for (int g = 0; g < G; ++g) mbar_init(tbar + g, 1);
      mbar_init_fence();
    }
    __syncwarp(tmask);
  }

  // ---- chunks of long rows: one chunk per team per claim ----
  if (a.n_chunks > 0) {
    for (;;) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(&a.qs->next_chunk, (unsigned)teams);
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= (unsigned)a.n_chunks) break;
      const unsigned k = base + team;
      const bool have = k < (unsigned)a.n_chunks;
      int64_t cb = 0;
      int clen = 0;
      if (have) {
        const int item = a.chunk_item[k];
        const int node = a.node[item] & 0x7fffffff;
        ch_dv = (a.scale_mode == SCALE_DCOL_DROW) ? __ldg(a.mult + node) : 1.f;
        cb = a.chunk_beg[k];
        clen = (int)(a.chunk_end[k] - cb);
      }
      bool done = !have;
      auto next_end = [&]() -> int { return done ? INT_MAX : clen; };
      auto on_end = [&](float (&acc)[VPL][V]) {
        float* prow = a.partial + (int64_t)k * a.ldp;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = tl + v * TL;
          if (vi < a.nvec) store_f32<V>(prow + vi * V, acc[v]);
        }
        __threadfence();
        __syncwarp(tmask);
        if (tl == 0) st_release(a.chunk_flag + k, epoch);
        done = true;
      };
      // chunks depend on nothing: always in lockstep
      if constexpr (TMA) {
        stream_pass_tma<XT, TL, VPL, V, G>(&tmap, a.tma_rb, a.cent, a.cval, cb, clen, a.scale_mode, a.mult, tring, tbar,
                                        tphase, tl, tmask, next_end, on_end, ch_dv, hints, true, a.qs, a.timeout_ns);
      } else {
        stream_pass<XT, TL, VPL, V, S, BLOCK, OFF32, HINTS>(x, a.ldx, a.nvec, a.cent, a.cval, cb, clen, a.scale_mode, a.mult,
                                              ring, tl, tmask, next_end, on_end, ch_dv, hints, true);
      }
    }
  }

  // ---- rows: a team takes R consecutive items per claim: rows_per_claim while
  // the queue is in level 0, rows_per_claim_deep below it (sized by where the
  // warp's last claim fell)
  const bool need_dv = (a.scale_mode == SCALE_DCOL_DROW) || (a.prop_mode == PROP_RATIO);
  const int64_t hi = a.n_items;
  unsigned last = 0;
  for (;;) {
    // this team's items [i0, i1); base: the first item of the warp's claim
    int64_t i0, i1;
    unsigned base;
    // units pay off where teams share a warp (they step together); a full-warp
    // team keeps the plain claims (one dependent load fewer per claim)
    if (TL < 32 && a.unit) {
      unsigned claimed = 0;
      if (lane == 0) claimed = atomicAdd(&a.qs->next_row, (unsigned)teams);
      const unsigned ub = __shfl_sync(0xffffffffu, claimed, 0);
      if (ub >= (unsigned)a.n_units) break;
      const unsigned u = ub + team;
      base = (unsigned)a.unit[ub];
      i0 = u < (unsigned)a.n_units ? a.unit[u] : hi;
      i1 = u < (unsigned)a.n_units ? a.unit[u + 1] : hi;
    } else {
      const int Rp = last < (unsigned)a.n_root ? a.rows_per_claim : a.rows_per_claim_deep;
      const int R = Rp < TL ? Rp : TL;
      unsigned claimed = 0;
      if (lane == 0) claimed = atomicAdd(&a.qs->next_row, (unsigned)(teams * R));
      base = __shfl_sync(0xffffffffu, claimed, 0);
      if ((int64_t)base >= hi) break;
      last = base;
      i0 = (int64_t)base + (int64_t)team * R;
      i1 = (i0 + R < hi) ? i0 + R : hi;
    }
    {
      const int nit = i0 < hi ? (int)(i1 - i0) : 0;
      const int64_t k0 = nit > 0 ? a.ptr[i0] : 0;
      // item metadata, one item per lane; ends relative to k0
      int m_node = 0, m_par = -1, m_chunk = -1, m_pslot = -1, m_sslot = -1, m_end = 0;
      float m_dv = 1.f;
      bool dep_in_claim = false;
      if (tl < nit) {
        const int64_t it = i0 + tl;
        m_node = a.node[it];
        m_par = a.skip_parent ? -1 : a.par[it];
        dep_in_claim = m_par >= 0 && a.par_item[it] >= (int)base;
        m_chunk = a.chunk0[it];
        m_pslot = a.par_slot[it];
        m_sslot = a.self_slot[it];
        m_end = (int)(a.ptr[it + 1] - k0);
        if (need_dv) m_dv = __ldg(a.mult + (m_node & 0x7fffffff));
      }
      const int len = nit > 0 ? __shfl_sync(tmask, m_end, nit - 1, TL) : 0;
      int cur = 0;  // item (relative) the consumer is in
      const bool drow = a.scale_mode == SCALE_DCOL_DROW;
      float row_dv = drow ? __shfl_sync(tmask, m_dv, 0, TL) : 1.f;
      auto next_end = [&]() -> int { return cur < nit ? __shfl_sync(tmask, m_end, cur, TL) : INT_MAX; };
      // Parent rows are fetched ahead: the parent's ready flag of item i+1 is
      // acquired when item i starts, and if it was set, item i+1's parent row is
      // loaded into registers when item i+1 starts; the row end then finds it
      // there.  A flag not yet set falls back to the bounded wait at the end.
      bool pf_ok = false;
      float pbuf[VPL][V];
      // claims without any parent skip this bookkeeping
      const bool any_parent = __any_sync(tmask, tl < nit && m_par >= 0);
      auto acquire_for = [&](int it) -> unsigned {
        if (!any_parent || it >= nit) return 0u;
        const int p = __shfl_sync(tmask, m_par, it, TL);
        return p >= 0 ? ld_acquire(a.node_flag + p) : 0u;
      };
      auto prefetch = [&](int it, unsigned fval) {
        pf_ok = false;
        if (!any_parent || it >= nit) return;
        const int p = __shfl_sync(tmask, m_par, it, TL);
        const int ps = __shfl_sync(tmask, m_pslot, it, TL);
        if (p < 0 || fval != epoch) return;
        pf_ok = true;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = tl + v * TL;
          if (vi < a.nvec) {
            if constexpr (sizeof(YT) == 4) {
              load_y_cg<YT, V>(static_cast<const YT*>(a.y) + (int64_t)p * a.ldy + (int64_t)vi * V, pbuf[v]);
            } else {
              load_f32_cg<V>(a.pstate + (int64_t)ps * a.ldp + vi * V, pbuf[v]);
            }
          }
        }
      };
      unsigned flag_next;
      {
        const unsigned f0 = acquire_for(0);
        flag_next = acquire_for(1);
        prefetch(0, f0);
      }
      auto on_end = [&](float (&acc)[VPL][V]) {
        const int nodew = __shfl_sync(tmask, m_node, cur, TL);
        const int node = nodew & 0x7fffffff;
        const int c0 = __shfl_sync(tmask, m_chunk, cur, TL);
        const int p = __shfl_sync(tmask, m_par, cur, TL);
        const int ps = __shfl_sync(tmask, m_pslot, cur, TL);
        const int ss = __shfl_sync(tmask, m_sslot, cur, TL);
        const float dv = __shfl_sync(tmask, m_dv, cur, TL);
        if (c0 >= 0) {
          const int item = (int)(i0 + cur);
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
        if (p >= 0 && (pf_ok || wait_flag(a.node_flag + p, epoch, a.qs, a.timeout_ns, (long long)node))) {
          const float dp = (a.prop_mode == PROP_RATIO) ? __ldg(a.mult + p) : 1.f;
#pragma unroll
          for (int v = 0; v < VPL; ++v) {
            const int vi = tl + v * TL;
            if (vi < a.nvec) {
              float yp[V];
              if (pf_ok) {
#pragma unroll
                for (int q = 0; q < V; ++q) yp[q] = pbuf[v][q];
              } else if constexpr (sizeof(YT) == 4) {
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
        // leaves are not read again by this kernel: stream them past L2 (not
        // in a first pass, whose rows the second pass reads back)
        const bool stream_y = hints && nodew >= 0 && !a.skip_parent;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = tl + v * TL;
          if (vi < a.nvec) {
            if (stream_y)
              store_vec_cs<YT, V>(yrow + (int64_t)vi * V, acc[v]);
            else
              store_vec<YT, V>(yrow + (int64_t)vi * V, acc[v]);
          }
        }
        if (nodew < 0 && !a.skip_parent) {
          if constexpr (sizeof(YT) != 4) {
            float* srow = a.pstate + (int64_t)ss * a.ldp;
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
#pragma unroll
        for (int v = 0; v < VPL; ++v)
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
        ++cur;
        const float next_dv = __shfl_sync(tmask, m_dv, cur < nit ? cur : 0, TL);
        row_dv = drow ? next_dv : 1.f;
        const unsigned f_cur = flag_next;
        flag_next = acquire_for(cur + 1);
        prefetch(cur, f_cur);
      };
      // a parent row inside this warp's claim: let the teams run independently
      const bool lockstep = !__any_sync(0xffffffffu, dep_in_claim);
      if constexpr (TMA) {
        stream_pass_tma<XT, TL, VPL, V, G>(&tmap, a.tma_rb, a.ent, a.val, k0, len, a.scale_mode, a.mult, tring, tbar,
                                        tphase, tl, tmask, next_end, on_end, row_dv, hints, lockstep, a.qs,
                                        a.timeout_ns);
      } else {
        stream_pass<XT, TL, VPL, V, S, BLOCK, OFF32, HINTS>(x, a.ldx, a.nvec, a.ent, a.val, k0, len, a.scale_mode, a.mult, ring,
                                              tl, tmask, next_end, on_end, row_dv, hints, lockstep);
      }
    }
  }
  finish_block(a.qs, epoch, a.publish_epoch != 0);
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
  // items, deepest level first: for each internal node its chunk items (long
  // children lists), then the node item
  int32_t n_items;
  const int32_t* node;   // node id, or -1 for a chunk item
  const int32_t* slot;   // node item: internal slot; chunk item: chunk id
  const int64_t* ptr;    // children (or chunk) ranges in ent
  const uint32_t* ent;   // child | internal bit (slot then)
  const int32_t* chunk0; // node item: first chunk id, -1 when not split
  const int32_t* nchunk; // node item: number of chunks
  const float* mult;
  int32_t scale_g;       // G' = m o G
  unsigned int* flag;    // [n_internal]
  unsigned int* chunk_flag;  // [chunks]
  float* partial;        // [chunks, ldp]
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
        // each lane acquires the flag of its own entry; the team barrier below
        // orders every lane's later reads of those rows after these acquires
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
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = tl + v * TL;
          if (j + u < cnt && vi < nvec) {
            if (in) {
              load_f32_cg<V>(h + row_off(r, ldp) + vi * V, buf[u][v]);
            } else {
              Vec<GT, V>::load(g + row_off(r, ldg) + (int64_t)vi * V, buf[u][v]);
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

// acc += sum over entries of s * (internal ? H[slot] : scale * G[row]) with the
// whole warp on one entry range: G = 32 / TL groups of TL lanes, group g takes
// the entries g, g + G, g + 2G, ... of each batch of 32, and the groups' sums
// are added at the end (shuffles across the group bits), so every lane holds
// the total.  Rows narrower than a warp then keep all 32 lanes on one column
// instead of splitting the warp between columns whose lists differ in length.
// The sum's order differs from the one-team order; the adjoint is held to
// FP64 and finite-difference bounds, not to the forward's order.
template <typename GT, int VPL, int V>
__device__ __forceinline__ void gather_dual_split(float (&acc)[VPL][V], const GT* __restrict__ g, int64_t ldg,
                                                  const float* __restrict__ h, int ldp, int nvec,
                                                  const uint32_t* __restrict__ ent, int64_t beg, int64_t end,
                                                  const float* __restrict__ mult, bool scale_g, int lane, int TL) {
  constexpr int U = unroll_for<VPL, V>();
  const int grp = lane / TL;
  const int tl = lane & (TL - 1);
  const int G = 32 / TL;
  for (int64_t base = beg; base < end; base += 32) {
    const int64_t idx = base + lane;
    uint32_t e = 0;
    float sc = 0.f;
    if (idx < end) {
      e = __ldg(ent + idx);
      const uint32_t r = e & kIndexMask;
      const float sgn = (e >> 31) ? -1.f : 1.f;
      sc = (e & kInternalBit) ? sgn : (scale_g ? sgn * __ldg(mult + r) : sgn);
    }
    const int cnt = (int)((end - base) < 32 ? (end - base) : 32);
    for (int j = 0; j < cnt; j += G * U) {  // the same trip count on every lane
      float buf[U][VPL][V];
      float s[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int jj = j + u * G + grp;
        const uint32_t eu = __shfl_sync(0xffffffffu, e, jj < cnt ? jj : 0);
        s[u] = __shfl_sync(0xffffffffu, sc, jj < cnt ? jj : 0);
        const uint32_t r = eu & kIndexMask;
        const bool in = (eu & kInternalBit) != 0;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = tl + v * TL;
          if (jj < cnt && vi < nvec) {
            if (in) {
              load_f32_cg<V>(h + row_off(r, ldp) + vi * V, buf[u][v]);
            } else {
              Vec<GT, V>::load(g + row_off(r, ldg) + (int64_t)vi * V, buf[u][v]);
            }
          } else {
#pragma unroll
            for (int k = 0; k < V; ++k) buf[u][v][k] = 0.f;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (j + u * G + grp < cnt) {
#pragma unroll
          for (int v = 0; v < VPL; ++v)
#pragma unroll
            for (int k = 0; k < V; ++k) acc[v][k] = fmaf(s[u], buf[u][v][k], acc[v][k]);
        }
      }
    }
  }
  for (int off = TL; off < 32; off <<= 1) {
#pragma unroll
    for (int v = 0; v < VPL; ++v)
#pragma unroll
      for (int k = 0; k < V; ++k) acc[v][k] += __shfl_xor_sync(0xffffffffu, acc[v][k], off);
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
      if (w >= 0) {
        // node item: its own G' row
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
        // partial sums of its chunks, in order
        const int c0 = a.chunk0[item];
        for (int k = c0, ke = c0 + (c0 >= 0 ? a.nchunk[item] : 0); k < ke; ++k) {
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
      } else {
#pragma unroll
        for (int v = 0; v < VPL; ++v)
#pragma unroll
          for (int q = 0; q < V; ++q) acc[v][q] = 0.f;
      }
      gather_dual<GT, VPL, V>(acc, g, a.ldg, a.h, a.ldp, a.nvec, a.ent, a.ptr[item], a.ptr[item + 1], a.mult,
                              a.scale_g != 0, false, a.flag, epoch, a.qs, a.timeout_ns, tl, TL, tmask);
      float* orow = (w >= 0) ? a.h + (int64_t)ws * a.ldp : a.partial + (int64_t)ws * a.ldp;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int vi = tl + v * TL;
        if (vi < a.nvec) store_f32<V>(orow + vi * V, acc[v]);
      }
      __threadfence();
      __syncwarp(tmask);
      if (tl == 0) st_release((w >= 0 ? a.flag : a.chunk_flag) + ws, epoch);
    }
    __syncwarp();
  }
  finish_block(a.qs, epoch);
}

// SPLIT (rows narrower than a warp): one item per warp, its entries spread
// over the warp's lane groups (gather_dual_split); group 0 writes the result.
template <typename GT, typename DT, int VPL, int V, bool SPLIT = false>
__global__ void __launch_bounds__(kThreads) tr_kernel(const TrArgs a) {
  const int lane = threadIdx.x & 31;
  const int TL = a.team;
  const int team = SPLIT ? 0 : lane / TL;
  const int tl = lane & (TL - 1);
  const int teams = SPLIT ? 1 : 32 / TL;
  const bool writer = !SPLIT || lane < TL;
  const unsigned tmask = (SPLIT || TL == 32) ? 0xffffffffu : (((1u << TL) - 1u) << (team * TL));
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
        if constexpr (SPLIT) {
          gather_dual_split<GT, VPL, V>(acc, g, a.ldg, a.h, a.ldp, a.nvec, a.ent, a.chunk_beg[k], a.chunk_end[k],
                                        a.mult, a.scale_g != 0, lane, TL);
        } else {
          gather_dual<GT, VPL, V>(acc, g, a.ldg, a.h, a.ldp, a.nvec, a.ent, a.chunk_beg[k], a.chunk_end[k],
                                  a.mult, a.scale_g != 0, true, nullptr, epoch, a.qs, a.timeout_ns, tl, TL,
                                  tmask);
        }
        float* prow = a.partial + (int64_t)k * a.ldp;
#pragma unroll
        for (int v = 0; v < VPL; ++v) {
          const int vi = tl + v * TL;
          if (writer && vi < a.nvec) store_f32<V>(prow + vi * V, acc[v]);
        }
        __threadfence();
        __syncwarp(tmask);
        if (SPLIT ? lane == 0 : tl == 0) st_release(a.chunk_flag + k, epoch);
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
        if constexpr (SPLIT) {
          gather_dual_split<GT, VPL, V>(acc, g, a.ldg, a.h, a.ldp, a.nvec, a.ent, a.ptr[item], a.ptr[item + 1],
                                        a.mult, a.scale_g != 0, lane, TL);
        } else {
          gather_dual<GT, VPL, V>(acc, g, a.ldg, a.h, a.ldp, a.nvec, a.ent, a.ptr[item], a.ptr[item + 1], a.mult,
                                  a.scale_g != 0, true, nullptr, epoch, a.qs, a.timeout_ns, tl, TL, tmask);
        }
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
      // an empty column contributes nothing; do not scale it (m may be inf there)
      const bool empty = c0 < 0 && a.ptr[item] == a.ptr[item + 1];
      const float so = (a.scale_out && !empty) ? __ldg(a.mult + item) : 1.f;
      DT* drow = static_cast<DT*>(a.dx) + (int64_t)item * a.lddx;
#pragma unroll
      for (int v = 0; v < VPL; ++v) {
        const int vi = tl + v * TL;
        if (writer && vi < a.nvec) {
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
