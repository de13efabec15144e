// Device construction of the CSR pattern of a cell integral.
//
// Same result as the host builder (fe_sparsity.cpp): the DOLFINx
// SparsityPattern of the cell integral -- sorted unique block columns per
// block row -- unrolled to scalar AIJ exactly as create_cuda_matrix does
// (la/petsc.cpp:45-65).  For callers that create many meshes (a request
// server, many-mesh batches) the host build dominates setup; here
//   k_pair_keys   one key R * n1 + C per (cell, local row, local col)
//   radix sort + unique (CUB) -> the block pattern in row-major order
//   k_block_count block row lengths, exclusive scan -> block row pointers
//   k_unroll_rows / k_unroll_cols   scalar row_ptr, col and the diagonal
//                 slots, every scalar row of block row R holding
//                 bs1 * len(R) columns.
#include <cub/cub.cuh>

#include <algorithm>

#include "fe_internal.h"

namespace fe {
namespace {

unsigned grid1(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

__global__ void k_pair_keys(const int32_t* __restrict__ d0, const int32_t* __restrict__ d1, int64_t num_cells,
                            int k0, int k1, uint64_t n1, uint64_t* __restrict__ keys) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t kk = (int64_t)k0 * k1;
  if (t >= num_cells * kk) return;
  const int64_t c = t / kk;
  const int e = (int)(t - c * kk);
  const int i = e / k1, j = e - i * k1;
  keys[t] = (uint64_t)(uint32_t)d0[c * k0 + i] * n1 + (uint64_t)(uint32_t)d1[c * k1 + j];
}

__global__ void k_block_count(const uint64_t* __restrict__ ukeys, const int* __restrict__ nu_ptr, uint64_t n1,
                              int32_t* __restrict__ rcount) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= *nu_ptr) return;
  atomicAdd(rcount + (int64_t)(ukeys[t] / n1), 1);
}

__global__ void k_unroll_rows(const int32_t* __restrict__ bptr, int64_t nR, int bs0, int bs1,
                              int32_t* __restrict__ row_ptr) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r > nR * bs0) return;
  if (r == nR * bs0) {
    row_ptr[r] = bs0 * bs1 * bptr[nR];
    return;
  }
  const int64_t R = r / bs0;
  const int a = (int)(r - R * bs0);
  const int32_t L = bptr[R + 1] - bptr[R];
  row_ptr[r] = bs0 * bs1 * bptr[R] + a * L * bs1;
}

__global__ void k_unroll_cols(const uint64_t* __restrict__ ukeys, const int* __restrict__ nu_ptr, uint64_t n1,
                              const int32_t* __restrict__ bptr, const int32_t* __restrict__ row_ptr, int bs0,
                              int bs1, int32_t* __restrict__ col, int32_t* __restrict__ diag) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= *nu_ptr) return;
  const uint64_t key = ukeys[t];
  const int64_t R = (int64_t)(key / n1);
  const int32_t C = (int32_t)(key - (uint64_t)R * n1);
  const int32_t p = (int32_t)(t - bptr[R]);
  for (int a = 0; a < bs0; ++a) {
    const int64_t r = R * bs0 + a;
    const int32_t base = row_ptr[r] + p * bs1;
    for (int b = 0; b < bs1; ++b) {
      const int32_t c = C * bs1 + b;
      col[base + b] = c;
      if (c == r) diag[r] = base + b;
    }
  }
}

__global__ void k_fill_i32(int32_t* __restrict__ v, int64_t n, int32_t x) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) v[t] = x;
}

}  // namespace

void build_pattern_device(const fe_dofmap_s& rows, const fe_dofmap_s& cols, cudaStream_t s, fe_sparsity_s& sp) {
  const int64_t C = rows.num_cells;
  const int64_t nR = rows.num_blocks, nC = cols.num_blocks;
  const int64_t npairs = C * rows.k * cols.k;
  FE_REQUIRE(npairs < INT32_MAX, "too many cell couplings for the device pattern build");
  sp.num_rows = nR * rows.bs;
  sp.num_cols = nC * cols.bs;
  const uint64_t n1 = (uint64_t)std::max<int64_t>(1, nC);
  int end_bit = 1;
  while (end_bit < 64 && ((uint64_t)1 << end_bit) < (uint64_t)std::max<int64_t>(1, nR) * n1) ++end_bit;

  DevBuf<int32_t> bptr(nR + 1);
  DevBuf<int> nu(1);
  DevBuf<uint64_t> ukeys;
  FE_CUDA(cudaMemsetAsync(bptr.p, 0, (nR + 1) * sizeof(int32_t), s));
  FE_CUDA(cudaMemsetAsync(nu.p, 0, sizeof(int), s));
  if (npairs > 0) {
    DevBuf<uint64_t> keys(npairs), sorted(npairs);
    k_pair_keys<<<grid1(npairs, 256), 256, 0, s>>>(rows.dofs.p, cols.dofs.p, C, rows.k, cols.k, n1, keys.p);
    FE_CUDA(cudaGetLastError());
    size_t tb = 0;
    FE_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys.p, sorted.p, (int)npairs, 0, end_bit, s));
    size_t tu = 0;
    FE_CUDA(cub::DeviceSelect::Unique(nullptr, tu, sorted.p, keys.p, nu.p, (int)npairs, s));
    DevBuf<unsigned char> temp(std::max(tb, tu));
    FE_CUDA(cub::DeviceRadixSort::SortKeys(temp.p, tb, keys.p, sorted.p, (int)npairs, 0, end_bit, s));
    FE_CUDA(cub::DeviceSelect::Unique(temp.p, tu, sorted.p, keys.p, nu.p, (int)npairs, s));
    int hnu = 0;
    FE_CUDA(cudaMemcpyAsync(&hnu, nu.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    FE_CUDA(cudaStreamSynchronize(s));
    ukeys.alloc(std::max(1, hnu));
    if (hnu) FE_CUDA(cudaMemcpyAsync(ukeys.p, keys.p, (size_t)hnu * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    const int64_t bnnz = hnu;
    if ((int64_t)bnnz * rows.bs * cols.bs > INT32_MAX)
      FE_FAIL(FE_ERR_ARG, "pattern has " + std::to_string(bnnz * rows.bs * cols.bs) + " entries (> int32)");
    if (bnnz) {
      k_block_count<<<grid1(bnnz, 256), 256, 0, s>>>(ukeys.p, nu.p, n1, bptr.p);
      FE_CUDA(cudaGetLastError());
    }
    size_t ts = 0;
    FE_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, ts, bptr.p, bptr.p, (int)(nR + 1), s));
    DevBuf<unsigned char> tscan(std::max<size_t>(1, ts));
    FE_CUDA(cub::DeviceScan::ExclusiveSum(tscan.p, ts, bptr.p, bptr.p, (int)(nR + 1), s));
    FE_CUDA(cudaStreamSynchronize(s));  // keys, sorted and the temporaries are freed on return
  }
  int hnu = 0;
  FE_CUDA(cudaMemcpyAsync(&hnu, nu.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  FE_CUDA(cudaStreamSynchronize(s));
  const int64_t nnz = (int64_t)hnu * rows.bs * cols.bs;
  sp.nnz = nnz;
  const int64_t nrows = sp.num_rows;
  sp.row_ptr.alloc(nrows + 1);
  sp.col.alloc(std::max<int64_t>(1, nnz));
  sp.diag.alloc(std::max<int64_t>(1, nrows));
  k_unroll_rows<<<grid1(nrows + 1, 256), 256, 0, s>>>(bptr.p, nR, rows.bs, cols.bs, sp.row_ptr.p);
  FE_CUDA(cudaGetLastError());
  if (nrows) {
    k_fill_i32<<<grid1(nrows, 256), 256, 0, s>>>(sp.diag.p, nrows, -1);
    FE_CUDA(cudaGetLastError());
  }
  if (hnu) {
    k_unroll_cols<<<grid1(hnu, 256), 256, 0, s>>>(ukeys.p, nu.p, n1, bptr.p, sp.row_ptr.p, rows.bs, cols.bs,
                                                  sp.col.p, sp.diag.p);
    FE_CUDA(cudaGetLastError());
  }
  sp.host_row_ptr.resize(nrows + 1);
  FE_CUDA(cudaMemcpyAsync(sp.host_row_ptr.data(), sp.row_ptr.p, (nrows + 1) * sizeof(int32_t),
                          cudaMemcpyDeviceToHost, s));
  FE_CUDA(cudaStreamSynchronize(s));  // bptr, nu and ukeys are freed on return
}

}  // namespace fe
