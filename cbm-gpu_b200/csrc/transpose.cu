// The transposed delta matrix of the adjoint (dX = Delta^T H), built once per
// plan on the GPU.
//
// Column j of Delta lists, in increasing row order, one word per entry:
//   (internal ? slot | kInternalBit : row) | sign << 31
// so that the transposed gather reads H (the reverse-propagated rows) for
// internal nodes and G' for leaves.  Built by a key-value radix sort on the
// device: key (column << 32 | row), value the word above; the column counts
// come from a histogram and a scan.  The reference has no backward pass; its
// CPU transposed SpMM (s_spmm_csr_t_int32, cbm/cbm_extensions.cpp:741-782)
// hands the transpose to MKL instead.
//
// cbm_plan_debug_check_transpose rebuilds the same index on the host (a
// counting sort) and compares it with the device's, word for word.

#include "cbm_b200.h"
#include "kernels.cuh"
#include "plan.h"

#include <cub/cub.cuh>

#include <vector>

namespace cbm {
namespace {

// one warp per item (row in level order): sort keys, values and column counts
__global__ void transpose_keys(const int64_t* __restrict__ ptr, const int32_t* __restrict__ order,
                               const int32_t* __restrict__ slot, const uint32_t* __restrict__ ent, int64_t n_items,
                               unsigned long long* __restrict__ keys, uint32_t* __restrict__ vals,
                               unsigned long long* __restrict__ counts) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x / 32);
  for (int64_t i = (int64_t)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; i < n_items; i += warps) {
    const int32_t v = order[i];
    const uint32_t rv = slot[v] >= 0 ? ((uint32_t)slot[v] | kInternalBit) : (uint32_t)v;
    for (int64_t k = ptr[i] + lane; k < ptr[i + 1]; k += 32) {
      const uint32_t e = ent[k];
      const uint32_t c = e & 0x7fffffffu;
      keys[k] = ((unsigned long long)c << 32) | (uint32_t)v;
      vals[k] = rv | (e & 0x80000000u);
      atomicAdd(counts + c, 1ull);
    }
  }
}

template <typename T>
int temp_upload(T** dst, const std::vector<T>& src, cudaStream_t st, std::vector<void*>& owned) {
  *dst = nullptr;
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(src.size(), 1) * sizeof(T)) != cudaSuccess) return CBM_ERR_ALLOC;
  owned.push_back(p);
  if (!src.empty() &&
      cudaMemcpyAsync(p, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return CBM_ERR_CUDA;
  *dst = static_cast<T*>(p);
  return CBM_OK;
}

void* temp_alloc(size_t bytes, std::vector<void*>& owned) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) return nullptr;
  owned.push_back(p);
  return p;
}

int bits_for(int64_t x) {
  int b = 0;
  while (b < 63 && ((int64_t)1 << b) <= x) ++b;
  return b;
}

}  // namespace

// Column pointers (into h_t_ptr, on the host too: the chunk tables need them)
// and the entry words (P->d_t_ptr, P->d_t_ent, owned by adj_bufs).
int transpose_on_device(cbm_plan* P, cudaStream_t st) {
  CbmRange range("cbm transpose_on_device");
  const int64_t n = P->n_items, z = P->nnz, nc = P->n_cols;
  std::vector<void*> tmp;
  auto done = [&](int rc) {
    cudaStreamSynchronize(st);
    free_all(tmp);
    return rc;
  };
  int64_t* d_ptr = nullptr;
  int32_t *d_order = nullptr, *d_slot = nullptr;
  uint32_t* d_ent = nullptr;
  int rc;
  if ((rc = temp_upload(&d_ptr, P->h_ptr, st, tmp))) return done(rc);
  if ((rc = temp_upload(&d_order, P->h_order, st, tmp))) return done(rc);
  if ((rc = temp_upload(&d_slot, P->h_slot, st, tmp))) return done(rc);
  if ((rc = temp_upload(&d_ent, P->h_ent, st, tmp))) return done(rc);
  auto* keys = static_cast<unsigned long long*>(temp_alloc(z * sizeof(unsigned long long), tmp));
  auto* keys_out = static_cast<unsigned long long*>(temp_alloc(z * sizeof(unsigned long long), tmp));
  auto* vals = static_cast<uint32_t*>(temp_alloc(z * sizeof(uint32_t), tmp));
  auto* counts = static_cast<unsigned long long*>(temp_alloc((nc + 1) * sizeof(unsigned long long), tmp));
  if (!keys || !keys_out || !vals || !counts) return done(CBM_ERR_ALLOC);
  // owned outputs
  void* tp = nullptr;
  if (cudaMalloc(&tp, (nc + 1) * sizeof(int64_t)) != cudaSuccess) return done(CBM_ERR_ALLOC);
  P->adj_bufs.push_back(tp);
  P->d_t_ptr = static_cast<int64_t*>(tp);
  P->d_t_ent = nullptr;
  if (z > 0) {
    void* te = nullptr;
    if (cudaMalloc(&te, z * sizeof(uint32_t)) != cudaSuccess) return done(CBM_ERR_ALLOC);
    P->adj_bufs.push_back(te);
    P->d_t_ent = static_cast<uint32_t*>(te);
  }
  if (cudaMemsetAsync(counts, 0, (nc + 1) * sizeof(unsigned long long), st) != cudaSuccess) return done(CBM_ERR_CUDA);
  if (cudaMemsetAsync(P->d_t_ptr, 0, sizeof(int64_t), st) != cudaSuccess) return done(CBM_ERR_CUDA);
  if (z > 0) {
    const int blocks = (int)std::min<int64_t>((n + 7) / 8, 148 * 16);
    transpose_keys<<<std::max(blocks, 1), 256, 0, st>>>(d_ptr, d_order, d_slot, d_ent, n, keys, vals, counts);
    if (cudaGetLastError() != cudaSuccess) return done(CBM_ERR_CUDA);
    // stable sort by (column, row): rows ascend within each column
    const int end_bit = 32 + bits_for(nc);
    size_t tb = 0;
    if (cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys_out, vals, P->d_t_ent, (int64_t)z, 0, end_bit,
                                        st) != cudaSuccess)
      return done(CBM_ERR_CUDA);
    void* t = temp_alloc(tb, tmp);
    if (!t) return done(CBM_ERR_ALLOC);
    if (cub::DeviceRadixSort::SortPairs(t, tb, keys, keys_out, vals, P->d_t_ent, (int64_t)z, 0, end_bit, st) !=
        cudaSuccess)
      return done(CBM_ERR_CUDA);
  }
  if (nc > 0) {
    // t_ptr[j + 1] = counts[0] + ... + counts[j]
    size_t tb = 0;
    if (cub::DeviceScan::InclusiveSum(nullptr, tb, counts, P->d_t_ptr + 1, (int64_t)nc, st) != cudaSuccess)
      return done(CBM_ERR_CUDA);
    void* t = temp_alloc(tb, tmp);
    if (!t) return done(CBM_ERR_ALLOC);
    if (cub::DeviceScan::InclusiveSum(t, tb, counts, P->d_t_ptr + 1, (int64_t)nc, st) != cudaSuccess)
      return done(CBM_ERR_CUDA);
  }
  P->h_t_ptr.assign(nc + 1, 0);
  if (cudaMemcpyAsync(P->h_t_ptr.data(), P->d_t_ptr, (nc + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, st) !=
      cudaSuccess)
    return done(CBM_ERR_CUDA);
  return done(cuda_status(cudaStreamSynchronize(st)));
}

// The same index by a counting sort on the host (rows visited in node order).
void transpose_on_host(const cbm_plan* P, std::vector<int64_t>& tptr, std::vector<uint32_t>& tent) {
  const int64_t n = P->n_items;
  tptr.assign(P->n_cols + 1, 0);
  for (int64_t k = 0; k < P->nnz; ++k) tptr[(P->h_ent[k] & 0x7fffffffu) + 1]++;
  for (int64_t j = 0; j < P->n_cols; ++j) tptr[j + 1] += tptr[j];
  tent.assign(P->nnz, 0);
  std::vector<int64_t> fill(tptr.begin(), tptr.end() - 1);
  std::vector<int64_t> item_of(n);
  for (int64_t i = 0; i < n; ++i) item_of[P->h_order[i]] = i;
  for (int64_t v = 0; v < n; ++v) {
    const int64_t i = item_of[v];
    const uint32_t rv = P->h_slot[v] >= 0 ? ((uint32_t)P->h_slot[v] | kInternalBit) : (uint32_t)v;
    for (int64_t k = P->h_ptr[i]; k < P->h_ptr[i + 1]; ++k) {
      const uint32_t e = P->h_ent[k];
      tent[fill[e & 0x7fffffffu]++] = rv | (e & 0x80000000u);
    }
  }
}

}  // namespace cbm

using namespace cbm;

extern "C" int cbm_plan_debug_check_transpose(cbm_plan* P, void* stream) {
  if (!P) return CBM_ERR_INVALID;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = cbm_plan_prepare_adjoint(P, stream);
  if (rc) return rc;
  std::vector<int64_t> tptr, dptr(P->n_cols + 1);
  std::vector<uint32_t> tent, dent(P->nnz);
  transpose_on_host(P, tptr, tent);
  if (cudaMemcpyAsync(dptr.data(), P->d_t_ptr, dptr.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st) !=
      cudaSuccess)
    return CBM_ERR_CUDA;
  if (P->nnz > 0 &&
      cudaMemcpyAsync(dent.data(), P->d_t_ent, dent.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess)
    return CBM_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return CBM_ERR_CUDA;
  return (tptr == dptr && tent == dent && tptr == P->h_t_ptr) ? CBM_OK : CBM_ERR_INTERNAL;
}
