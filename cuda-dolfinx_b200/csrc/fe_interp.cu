// Same-map interpolation between Lagrange spaces on one mesh: u1 = I u0.
//
// The reference (CUDACoefficient::interpolate,
// cpp/cudolfinx/fem/CUDACoefficient.h:64-83 -> interpolate_same_map,
// cpp/cudolfinx/fem/CUDAInterpolate.cu) gathers every cell's source values
// into a temporary [cells x n0] array, multiplies by the n1 x n0
// interpolation matrix for every cell and scatters the [cells x n1] result,
// so a dof shared by several cells is written by each of them (the last write
// wins) and two temporaries are allocated per call.  Here every target dof is
// computed once, from an owner cell: the lowest (cell, local dof) that lists
// it, found once per target dofmap with an atomicMin.  One thread per target
// dof; the matrix travels in the kernel parameters; the result is
// deterministic and written with coalesced stores.
#include <cuda_runtime.h>

#include <climits>

#include "fe_internal.h"

namespace fe {
namespace {

constexpr int kInterpMax = 20 * 20;

__global__ void k_owner_fill(int32_t* __restrict__ owner, int64_t n) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) owner[t] = INT_MAX;
}

__global__ void k_owner_min(const int32_t* __restrict__ dofs, int64_t num_entries, int32_t* __restrict__ owner) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= num_entries) return;
  const int32_t d = dofs[t];
  if (d >= 0) atomicMin(owner + d, (int32_t)t);
}

struct InterpArgs {
  const int32_t* __restrict__ owner;
  const int32_t* __restrict__ dofs0;
  const double* __restrict__ u0;
  double* __restrict__ u1;
  int64_t num_blocks;
  int k1, k0, bs;
  double im[kInterpMax];  // [k1][k0] row-major
};

__global__ void __launch_bounds__(256) k_interpolate(const InterpArgs a) {
  const int64_t d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (d >= a.num_blocks) return;
  const int32_t e = __ldg(a.owner + d);
  if (e == INT_MAX) return;  // listed by no cell: left unchanged
  const int64_t c = e / a.k1;
  const int i = (int)(e - c * a.k1);
  const int32_t* src = a.dofs0 + c * a.k0;
  for (int q = 0; q < a.bs; ++q) {
    double acc = 0.0;
    for (int j = 0; j < a.k0; ++j) acc += a.im[i * a.k0 + j] * __ldg(a.u0 + (int64_t)__ldg(src + j) * a.bs + q);
    a.u1[d * a.bs + q] = acc;
  }
}

unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void interpolate(fe_dofmap_s& target, double* u1, const fe_dofmap_s& source, const double* u0, const double* im,
                 cudaStream_t s) {
  if (target.k * source.k > kInterpMax) FE_FAIL(FE_ERR_ARG, "interpolation matrix larger than 20 x 20");
  // owners are int32 (cell, local dof) entry indices
  FE_REQUIRE(target.num_cells * (int64_t)target.k <= (int64_t)INT_MAX,
             "interpolation target dofmap has more than 2^31-1 (cell, dof) entries");
  if (!target.owner.p && target.num_blocks) {
    target.owner.alloc(target.num_blocks);
    k_owner_fill<<<blocks_for(target.num_blocks, 256), 256, 0, s>>>(target.owner.p, target.num_blocks);
    FE_CUDA(cudaGetLastError());
    const int64_t n = target.num_cells * target.k;
    if (n) {
      k_owner_min<<<blocks_for(n, 256), 256, 0, s>>>(target.dofs.p, n, target.owner.p);
      FE_CUDA(cudaGetLastError());
    }
  }
  if (!target.num_blocks) return;
  InterpArgs a{};
  a.owner = target.owner.p;
  a.dofs0 = source.dofs.p;
  a.u0 = u0;
  a.u1 = u1;
  a.num_blocks = target.num_blocks;
  a.k1 = target.k;
  a.k0 = source.k;
  a.bs = target.bs;
  for (int t = 0; t < target.k * source.k; ++t) a.im[t] = im[t];
  k_interpolate<<<blocks_for(target.num_blocks, 256), 256, 0, s>>>(a);
  FE_CUDA(cudaGetLastError());
}

}  // namespace fe
