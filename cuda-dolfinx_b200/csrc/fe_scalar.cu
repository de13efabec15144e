// Scalar assembly (functionals): int f dx, int k |grad u|^2 dx for P1 / P2 u,
// int g ds over exterior facets, int jump(u)^2 dS over interior facets.
//
// The reference generates cell / exterior-facet / interior-facet scalar
// kernels that add every thread's partial value into the result with one
// FP64 atomicAdd (CUDAFormIntegral.cpp:66-266, scalar_reduction), so the sum's
// rounding depends on scheduling.  Here the reduction has a fixed order: a
// fixed grid strides over the cells (or facets), each block reduces its
// threads' partials with a fixed shuffle tree and a fixed warp order into one
// partial per block, and one block sums the partials in index order -- the
// value is bitwise reproducible on a given GPU.
#include <cuda_runtime.h>

#include <algorithm>

#include "fe_element_code.cuh"
#include "fe_internal.h"

namespace fe {
namespace {

constexpr int kScalarThreads = 256;

struct ScalarArgs {
  int kind;
  int64_t num_items;
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  // coefficient 0 (f, g or k)
  int c0kind;
  double c0const;
  const double* __restrict__ c0v;
  const int32_t* __restrict__ c0map;
  // coefficient 1 (u of the energy functionals)
  const double* __restrict__ u;
  const int32_t* __restrict__ umap;
  // facets ((cell, facet) pairs; interior facets: (cell0, facet0, cell1, facet1))
  const int2* __restrict__ facets;
  const int4* __restrict__ quads;
  double* __restrict__ partial;
};

struct Geo {
  double K[3][3];
  double adet;
};

__device__ __forceinline__ void tet_geometry(const double* __restrict__ x, int4 v, Geo& g) {
  double J[3][3];
  const int vv[3] = {v.y, v.z, v.w};
#pragma unroll
  for (int cc = 0; cc < 3; ++cc)
#pragma unroll
    for (int r = 0; r < 3; ++r) J[r][cc] = __ldg(x + 3 * (int64_t)vv[cc] + r) - __ldg(x + 3 * (int64_t)v.x + r);
  const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  const double id = 1.0 / det;
  g.K[0][0] = c00 * id;
  g.K[1][0] = c01 * id;
  g.K[2][0] = c02 * id;
  g.K[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  g.K[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  g.K[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  g.K[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  g.K[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  g.K[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  g.adet = fabs(det);
}

__device__ __forceinline__ double coef0_cell(const ScalarArgs& a, int64_t c) {
  return a.c0kind == FE_COEFF_DG0 ? __ldg(a.c0v + c) : a.c0const;
}

// sum over the facet of g times the facet area / 3 per facet vertex: the
// exact integral of a P1 g over a triangle is area * (g0 + g1 + g2) / 3
__device__ double facet_value(const ScalarArgs& a, int64_t t) {
  const int2 cf = __ldg(a.facets + t);
  const int64_t c = cf.x;
  const int f = cf.y;
  const int4 v = __ldg(reinterpret_cast<const int4*>(a.geom) + c);
  const int vv[4] = {v.x, v.y, v.z, v.w};
  int loc[3], n = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (q != f) loc[n++] = q;
  double p[3][3];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int d = 0; d < 3; ++d) p[q][d] = __ldg(a.x + 3 * (int64_t)vv[loc[q]] + d);
  const double u[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
  const double w[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
  const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
  const double area = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
  if (a.c0kind == FE_COEFF_P1) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 3; ++q) s += __ldg(a.c0v + __ldg(a.c0map + 4 * c + loc[q]));
    return area * s * (1.0 / 3.0);
  }
  return area * coef0_cell(a, c);
}

// int jump(u)^2 dS over interior facet t: DG0 u: |F| (u0 - u1)^2; a vertex
// field (DG1 / P1 through a 4-dof map): the jump is linear on the facet with
// vertex values d_p, and int (sum_p d_p lambda_p)^2 = |F| (sum d_p^2 + (sum d_p)^2) / 12
__device__ double jump_value(const ScalarArgs& a, int64_t t) {
  const int4 q = __ldg(a.quads + t);
  const int4 g0 = __ldg(reinterpret_cast<const int4*>(a.geom) + q.x);
  const int4 g1 = __ldg(reinterpret_cast<const int4*>(a.geom) + q.z);
  const int v0[4] = {g0.x, g0.y, g0.z, g0.w}, v1[4] = {g1.x, g1.y, g1.z, g1.w};
  int loc0[3], loc1[3], n = 0;
#pragma unroll
  for (int u = 0; u < 4; ++u)
    if (u != q.y) loc0[n++] = u;
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    loc1[p] = 0;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (u != q.w && v1[u] == v0[loc0[p]]) loc1[p] = u;
  }
  double P[3][3];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int d = 0; d < 3; ++d) P[p][d] = __ldg(a.x + 3 * (int64_t)v0[loc0[p]] + d);
  const double e1[3] = {P[1][0] - P[0][0], P[1][1] - P[0][1], P[1][2] - P[0][2]};
  const double e2[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
  const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
               cz = e1[0] * e2[1] - e1[1] * e2[0];
  const double area = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
  if (a.c0kind == FE_COEFF_P1) {
    double s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      const double d = __ldg(a.c0v + __ldg(a.c0map + 4 * (int64_t)q.x + loc0[p])) -
                       __ldg(a.c0v + __ldg(a.c0map + 4 * (int64_t)q.z + loc1[p]));
      s1 += d;
      s2 += d * d;
    }
    return area * (s2 + s1 * s1) * (1.0 / 12.0);
  }
  if (a.c0kind == FE_COEFF_DG0) {
    const double d = __ldg(a.c0v + q.x) - __ldg(a.c0v + q.z);
    return area * d * d;
  }
  return 0.0;  // a constant has no jump
}

__device__ double cell_value(const ScalarArgs& a, int64_t c) {
  if (a.kind == FE_FORM_FACET_INTEGRAL) return facet_value(a, c);
  if (a.kind == FE_FORM_JUMP_NORM) return jump_value(a, c);
  Geo g;
  tet_geometry(a.x, __ldg(reinterpret_cast<const int4*>(a.geom) + c), g);
  const double vol = g.adet * (1.0 / 6.0);
  if (a.kind == FE_FORM_INTEGRAL) {
    if (a.c0kind == FE_COEFF_P1) {
      const int4 m = __ldg(reinterpret_cast<const int4*>(a.c0map) + c);
      return vol * 0.25 * (__ldg(a.c0v + m.x) + __ldg(a.c0v + m.y) + __ldg(a.c0v + m.z) + __ldg(a.c0v + m.w));
    }
    return vol * coef0_cell(a, c);
  }
  const double k = coef0_cell(a, c);
  if (a.kind == FE_FORM_P1_ENERGY) {
    const int4 m = __ldg(reinterpret_cast<const int4*>(a.umap) + c);
    const double u0 = __ldg(a.u + m.x), du[3] = {__ldg(a.u + m.y) - u0, __ldg(a.u + m.z) - u0,
                                                 __ldg(a.u + m.w) - u0};
    // grad u = K^T (u1 - u0, u2 - u0, u3 - u0)
    double gr[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) gr[b] = g.K[0][b] * du[0] + g.K[1][b] * du[1] + g.K[2][b] * du[2];
    return k * vol * (gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2]);
  }
  // P2 energy: u_e^T A_e u_e with the P2 stiffness element matrix
  double ue[10];
#pragma unroll
  for (int i = 0; i < 10; ++i) ue[i] = __ldg(a.u + __ldg(a.umap + 10 * c + i));
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  double gq[6];
#pragma unroll
  for (int s = 0; s < 6; ++s)
    gq[s] = g.adet * (g.K[pa[s]][0] * g.K[pb[s]][0] + g.K[pa[s]][1] * g.K[pb[s]][1] + g.K[pa[s]][2] * g.K[pb[s]][2]);
  double e = 0.0;
  p2_stiffness_const<double>(gq, [&](int i, int j, double v) { e += (i == j ? 1.0 : 2.0) * v * ue[i] * ue[j]; });
  return k * e;
}

// deterministic block sum: fixed shuffle tree per warp, warps in index order
__device__ double block_reduce(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
  return s;
}

__global__ void __launch_bounds__(kScalarThreads) k_scalar(const ScalarArgs a) {
  __shared__ double sh[kScalarThreads / 32];
  double v = 0.0;
  for (int64_t c = blockIdx.x * (int64_t)kScalarThreads + threadIdx.x; c < a.num_items;
       c += (int64_t)gridDim.x * kScalarThreads)
    v += cell_value(a, c);
  const double s = block_reduce(v, sh);
  if (threadIdx.x == 0) a.partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kScalarThreads) k_scalar_final(double* __restrict__ partial, int n) {
  __shared__ double sh[kScalarThreads / 32];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += kScalarThreads) v += partial[i];
  const double s = block_reduce(v, sh);
  if (threadIdx.x == 0) partial[n] = s;
}

}  // namespace

bool is_scalar_kind(int kind) {
  return kind == FE_FORM_INTEGRAL || kind == FE_FORM_P1_ENERGY || kind == FE_FORM_P2_ENERGY ||
         kind == FE_FORM_FACET_INTEGRAL || kind == FE_FORM_JUMP_NORM;
}

double assemble_scalar(fe_form_s& f, cudaStream_t s) {
  const int grid = std::max(1, f.ctx->num_sms * 4);
  if (f.scalar_partial.n < (size_t)grid + 1) f.scalar_partial.alloc(grid + 1);
  ScalarArgs a{};
  a.kind = f.kind;
  a.num_items =
      (f.kind == FE_FORM_FACET_INTEGRAL || f.kind == FE_FORM_JUMP_NORM) ? f.num_facets : f.mesh->num_cells;
  a.x = f.mesh->x.p;
  a.geom = f.mesh->geom.p;
  const Coefficient& c0 = f.coeff[0];
  a.c0kind = c0.kind < 0 ? FE_COEFF_CONSTANT : c0.kind;
  a.c0const = c0.kind < 0 ? 1.0 : c0.constant[0];
  a.c0v = c0.values;
  a.c0map = c0.map ? c0.map->dofs.p : nullptr;
  const Coefficient& c1 = f.coeff[1];
  a.u = c1.values;
  a.umap = c1.map ? c1.map->dofs.p : nullptr;
  a.facets = reinterpret_cast<const int2*>(f.facets.p);
  a.quads = reinterpret_cast<const int4*>(f.facets.p);
  a.partial = f.scalar_partial.p;
  k_scalar<<<grid, kScalarThreads, 0, s>>>(a);
  FE_CUDA(cudaGetLastError());
  k_scalar_final<<<1, kScalarThreads, 0, s>>>(f.scalar_partial.p, grid);
  FE_CUDA(cudaGetLastError());
  double h = 0.0;
  FE_CUDA(cudaMemcpyAsync(&h, f.scalar_partial.p + grid, sizeof(double), cudaMemcpyDeviceToHost, s));
  FE_CUDA(cudaStreamSynchronize(s));
  return h;
}

}  // namespace fe
