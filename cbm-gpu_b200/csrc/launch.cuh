// Kernel launchers.  Each launch_*.cu translation unit instantiates the
// kernels of one family and operand type pair through these templates, so the
// library's ~130 kernel instantiations compile in parallel; matmul.cu holds
// the host logic and calls the per-unit entry points declared at the end.
#pragma once

#include <atomic>
#include <cstring>

#include "cbm_b200.h"
#include "kernels.cuh"
#include "plan.h"

namespace cbm {

constexpr int kMaxDevices = 64;
// staged kernel: ring of S slots of VPL 16-byte pieces per thread, blocks of
// 128 threads
constexpr int kStagedBlock = 128;

// Multiprocessor count of `device`, looked up once per device (thread-safe).
int sm_count(int device);

// Grid of one kernel instantiation per device: resident blocks per SM x SMs,
// computed on first use.  Threads that race compute the same value, and the
// slots are atomic and indexed by device, so a launch never takes another
// device's grid.
struct GridCache {
  std::atomic<int> grid[kMaxDevices];
};

template <typename K>
int cached_grid(GridCache& c, K kernel, int device, int block, int smem) {
  if (device < 0 || device >= kMaxDevices) return 0;
  int g = c.grid[device].load(std::memory_order_acquire);
  if (g > 0) return g;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess) return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  g = per_sm * sm_count(device);
  c.grid[device].store(g, std::memory_order_release);
  return g;
}

template <typename XT, typename YT, int VPL, int V, bool COMP = false, bool WIDE = false>
int launch_fwd_t(cbm_plan* P, const FwdArgs& a, cudaStream_t st) {
  static GridCache cache[2];
  // BF16 X with fewer than 2^32 elements takes 32-bit row offsets (measured
  // faster there; FP32 X keeps the widening multiply)
  bool off32 = false;
  auto kern = fwd_kernel<XT, YT, VPL, V, COMP, WIDE, false>;
  if constexpr (sizeof(XT) == 2) {
    off32 = (uint64_t)P->n_cols * (uint64_t)a.ldx <= 0xffffffffull;
    if (off32) kern = fwd_kernel<XT, YT, VPL, V, COMP, WIDE, true>;
  }
  const int grid = cached_grid(cache[off32 ? 1 : 0], kern, P->device, kThreads, 0);
  if (grid <= 0) return CBM_ERR_CUDA;
  kern<<<grid, kThreads, 0, st>>>(a);
  P->launches++;
  P->last_grid = grid;
  return cuda_status(cudaGetLastError());
}

template <typename XT, typename YT, int TL, int VPL, int V, int S, bool TMA = false>
int launch_stream_t(cbm_plan* P, const FwdArgs& a, const CUtensorMap& map, cudaStream_t st) {
  constexpr int n_teams = kStagedBlock / TL;
  // 32-bit X row offsets when every row offset of X fits them (X rows =
  // the plan's columns)
  const bool off32 = (uint64_t)P->n_cols * (uint64_t)a.ldx <= 0xffffffffull;
  auto kern = fwd_stream_kernel<XT, YT, TL, VPL, V, S, kStagedBlock, TMA, false>;
  int grid;
  int smem;
  if constexpr (TMA) {
    // the ring's size follows the row width: no cached grid (opt-in variant)
    smem = n_teams * (S / 4) * (4 * a.tma_rb + 8);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
      return CBM_ERR_CUDA;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kStagedBlock, smem) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    grid = per_sm * sm_count(P->device);
  } else {
    // a plan without a hot set (hints off) takes copies without L2 policies
    // (the 64-bit form keeps the policy kernel: policies are then all normal)
    static GridCache cache[3];
    const int form = !off32 ? 0 : a.hints ? 1 : 2;
    if (form == 1) kern = fwd_stream_kernel<XT, YT, TL, VPL, V, S, kStagedBlock, false, true, true>;
    if (form == 2) kern = fwd_stream_kernel<XT, YT, TL, VPL, V, S, kStagedBlock, false, true, false>;
    smem = S * VPL * kStagedBlock * 16;
    grid = cached_grid(cache[form], kern, P->device, kStagedBlock, smem);
    if (grid <= 0) return CBM_ERR_CUDA;
  }
  kern<<<grid, kStagedBlock, smem, st>>>(a, map);
  P->launches++;
  P->last_grid = grid;
  return cuda_status(cudaGetLastError());
}

template <typename XT, typename YT, int TL>
int launch_staged_team(cbm_plan* P, const FwdArgs& a, int vpl, const CUtensorMap& map, cudaStream_t st) {
  constexpr int V = 16 / (int)sizeof(XT);
  // one piece per lane: a deeper ring (16 slots, 32 KiB per block) keeps as
  // many bytes in flight as two pieces in 8 slots
  constexpr int S1 = TL >= 16 ? 16 : 8;
  switch (vpl) {
    case 1: return launch_stream_t<XT, YT, TL, 1, V, S1>(P, a, map, st);
    case 2: return launch_stream_t<XT, YT, TL, 2, V, 8>(P, a, map, st);
    case 4: return launch_stream_t<XT, YT, TL, 4, V, 8>(P, a, map, st);
    default:
      if constexpr (V == 4) return launch_stream_t<XT, YT, TL, 8, V, 4>(P, a, map, st);
      return CBM_ERR_INTERNAL;
  }
}

template <typename XT, typename YT>
int launch_staged_any(cbm_plan* P, const FwdArgs& a, int team, int vpl, cudaStream_t st) {
  CUtensorMap none;
  memset(&none, 0, sizeof(none));
  if (team == 8) return launch_staged_team<XT, YT, 8>(P, a, vpl, none, st);
  if (team == 16) return launch_staged_team<XT, YT, 16>(P, a, vpl, none, st);
  return launch_staged_team<XT, YT, 32>(P, a, vpl, none, st);
}

// TMA variant: every lane owns every piece (nvec == team * vpl), one or two
// pieces per lane; ring depths as in the cp.async variant.
template <typename XT, typename YT>
int launch_tma_any(cbm_plan* P, const FwdArgs& a, int team, int vpl, const CUtensorMap& map, cudaStream_t st) {
  constexpr int V = 16 / (int)sizeof(XT);
  if (team == 8 && vpl == 1) return launch_stream_t<XT, YT, 8, 1, V, 8, true>(P, a, map, st);
  if (team == 16 && vpl == 1) return launch_stream_t<XT, YT, 16, 1, V, 16, true>(P, a, map, st);
  if (team == 32 && vpl == 1) return launch_stream_t<XT, YT, 32, 1, V, 16, true>(P, a, map, st);
  if (team == 32 && vpl == 2) return launch_stream_t<XT, YT, 32, 2, V, 8, true>(P, a, map, st);
  return CBM_ERR_INTERNAL;
}

template <typename XT, typename YT, int V, bool COMP = false>
int launch_fwd_v(cbm_plan* P, const FwdArgs& a, int vpl, cudaStream_t st) {
  switch (vpl) {
    case 1: return launch_fwd_t<XT, YT, 1, V, COMP>(P, a, st);
    case 2: return launch_fwd_t<XT, YT, 2, V, COMP>(P, a, st);
    case 4: return launch_fwd_t<XT, YT, 4, V, COMP>(P, a, st);
    default: return launch_fwd_t<XT, YT, 8, V, COMP>(P, a, st);
  }
}

template <typename GT, int VPL, int V>
int launch_rev_t(cbm_plan* P, const RevArgs& a, cudaStream_t st) {
  static GridCache cache;
  auto kern = rev_kernel<GT, VPL, V>;
  const int grid = cached_grid(cache, kern, P->device, kThreads, 0);
  if (grid <= 0) return CBM_ERR_CUDA;
  kern<<<grid, kThreads, 0, st>>>(a);
  P->launches++;
  return cuda_status(cudaGetLastError());
}

template <typename GT, typename DT, int VPL, int V, bool SPLIT = false>
int launch_tr_t(cbm_plan* P, const TrArgs& a, cudaStream_t st) {
  static GridCache cache;
  auto kern = tr_kernel<GT, DT, VPL, V, SPLIT>;
  const int grid = cached_grid(cache, kern, P->device, kThreads, 0);
  if (grid <= 0) return CBM_ERR_CUDA;
  kern<<<grid, kThreads, 0, st>>>(a);
  P->launches++;
  return cuda_status(cudaGetLastError());
}

template <int VPL, int V>
int launch_prop_t(cbm_plan* P, const PropArgs& a, cudaStream_t st) {
  static GridCache cache;
  auto kern = prop_kernel<VPL, V>;
  const int grid = cached_grid(cache, kern, P->device, kThreads, 0);
  if (grid <= 0) return CBM_ERR_CUDA;
  kern<<<grid, kThreads, 0, st>>>(a);
  P->launches++;
  return cuda_status(cudaGetLastError());
}

// ---- per-unit entry points (launch_*.cu) ------------------------------------------
int launch_staged_f32(cbm_plan* P, const FwdArgs& a, int team, int vpl, cudaStream_t st);
int launch_staged_bf16_f32(cbm_plan* P, const FwdArgs& a, int team, int vpl, cudaStream_t st);
int launch_staged_bf16_bf16(cbm_plan* P, const FwdArgs& a, int team, int vpl, cudaStream_t st);
int launch_tma(cbm_plan* P, const FwdArgs& a, int32_t xdt, int32_t ydt, int team, int vpl, const CUtensorMap& map,
               cudaStream_t st);
int launch_fwd_f32(cbm_plan* P, const FwdArgs& a, bool vec, int vpl, cudaStream_t st);
// wide: on trees where few rows wait on a parent, one-vector rows of BF16 X
// and FP32 Y take the 4-block instantiation (fwd_min_blocks)
int launch_fwd_bf16(cbm_plan* P, const FwdArgs& a, int32_t ydt, bool vec, int vpl, bool wide, cudaStream_t st);
// compensated propagation: BF16 X only (the precision form), register kernel
int launch_fwd_comp(cbm_plan* P, const FwdArgs& a, int32_t ydt, bool vec, int vpl, cudaStream_t st);
// second pass of a two-pass product (FP32 Y)
int launch_prop(cbm_plan* P, const PropArgs& a, bool vec, int vpl, cudaStream_t st);
int launch_rev(cbm_plan* P, const RevArgs& a, int32_t gdt, bool vec, int vpl, cudaStream_t st);
int launch_tr(cbm_plan* P, const TrArgs& a, int32_t gdt, int32_t ddt, bool vec, int vpl, cudaStream_t st);

}  // namespace cbm
