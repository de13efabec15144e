// Exterior-facet integrals (ds): Robin-type mass alpha*u*v*ds on P1/P2,
// Neumann loads g*v*ds on P1/P2 and traction t.v*ds on vector P2.
//
// The reference generates these from FFCx exterior-facet tabulate_tensor
// bodies: vector assembly CUDAFormIntegral.cpp:361-447, matrix assembly
// :1667-1793, lifting :721-837.  Facets come as (cell, local facet) pairs (the
// exterior-facet integration domain; facet f is opposite vertex f) and the
// element tensor is indexed by the cell's local dofs, so the matrix kernel
// scatters through the cell's byte map exactly like the cell kernels.  The
// facet reference tensors are exact rational integrals (generated tables):
// only the dofs on the facet carry values.
#include <cuda_runtime.h>

#define FE_FACET_TABLES
#include "fe_element_code.cuh"
#include "fe_internal.h"

namespace fe {
namespace {

struct FacetArgs {
  int64_t num_facets;
  const int2* __restrict__ facets;  // (cell, local facet)
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  const int32_t* __restrict__ dofs;
  int bs;
  // coefficient: alpha (mass) or g / t (loads)
  int ckind;
  double cconst[3];
  const double* __restrict__ cvals;
  const int32_t* __restrict__ cmap;
  // matrix
  const uint8_t* __restrict__ pos;
  const int32_t* __restrict__ row_ptr;
  const uint8_t* __restrict__ bc0;
  const uint8_t* __restrict__ bc1;
  double* __restrict__ values;
  // vector / lifting
  double* __restrict__ b;
  int64_t num_values;
  const double* __restrict__ g;
  const double* __restrict__ x0;
  double scale;
};

// area of facet f of cell c (the triangle of the three other vertices)
__device__ __forceinline__ double facet_area(const FacetArgs& a, int64_t c, int f) {
  const int4 v = __ldg(reinterpret_cast<const int4*>(a.geom) + c);
  const int vv[4] = {v.x, v.y, v.z, v.w};
  int t[3], n = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q)
    if (q != f) t[n++] = vv[q];
  double p[3][3];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int d = 0; d < 3; ++d) p[q][d] = __ldg(a.x + 3 * (int64_t)t[q] + d);
  const double u[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
  const double w[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
  const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
  return 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
}

template <int DEG>
struct FacetTab;
template <>
struct FacetTab<1> {
  static constexpr int K = 4, ND = 3;
  static __device__ __forceinline__ int dof(int f, int q) { return kFacetDofsP1[f][q]; }
  static __device__ __forceinline__ double mass(int f, int p, int q) { return kFacetMassP1[f][p][q]; }
  static __device__ __forceinline__ double load(int f, int p) { return kFacetLoadP1[f][p]; }
  static __device__ __forceinline__ double loadw(int f, int m, int p) { return kFacetLoadWP1[f][m][p]; }
};
template <>
struct FacetTab<2> {
  static constexpr int K = 10, ND = 6;
  static __device__ __forceinline__ int dof(int f, int q) { return kFacetDofsP2[f][q]; }
  static __device__ __forceinline__ double mass(int f, int p, int q) { return kFacetMassP2[f][p][q]; }
  static __device__ __forceinline__ double load(int f, int p) { return kFacetLoadP2[f][p]; }
  static __device__ __forceinline__ double loadw(int f, int m, int p) { return kFacetLoadWP2[f][m][p]; }
};

// scalar facet coefficient of cell c: constant or the cell's DG0 value
__device__ __forceinline__ double facet_scalar(const FacetArgs& a, int64_t c) {
  return a.ckind == FE_COEFF_DG0 ? __ldg(a.cvals + c) : a.cconst[0];
}

template <int DEG>
__global__ void k_facet_mass(const FacetArgs a) {
  using T = FacetTab<DEG>;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.num_facets) return;
  const int2 cf = __ldg(a.facets + t);
  const int64_t c = cf.x;
  const int f = cf.y;
  const double s = facet_area(a, c, f) * facet_scalar(a, c);
  int R[T::ND], rp[T::ND];
  bool mr[T::ND], mc[T::ND];
#pragma unroll
  for (int p = 0; p < T::ND; ++p) {
    R[p] = __ldg(a.dofs + c * T::K + T::dof(f, p));
    rp[p] = __ldg(a.row_ptr + R[p]);
    mr[p] = a.bc0 && a.bc0[R[p]];
    mc[p] = a.bc1 && a.bc1[R[p]];
  }
  const uint8_t* pc = a.pos + c * (T::K * T::K);
#pragma unroll
  for (int p = 0; p < T::ND; ++p)
#pragma unroll
    for (int q = 0; q < T::ND; ++q) {
      if (mr[p] || mc[q]) continue;
      const int i = T::dof(f, p), j = T::dof(f, q);
      atomicAdd(a.values + rp[p] + __ldg(pc + i * T::K + j), s * T::mass(f, p, q));
    }
}

// scalar facet load: constant / DG0 g (cell value) or P1 g through its dofmap
template <int DEG>
__global__ void k_facet_load(const FacetArgs a) {
  using T = FacetTab<DEG>;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.num_facets) return;
  const int2 cf = __ldg(a.facets + t);
  const int64_t c = cf.x;
  const int f = cf.y;
  const double area = facet_area(a, c, f);
  double gv[4] = {0.0, 0.0, 0.0, 0.0};
  const bool p1 = a.ckind == FE_COEFF_P1;
  if (p1) {
    const int4 m = __ldg(reinterpret_cast<const int4*>(a.cmap) + c);
    gv[0] = __ldg(a.cvals + m.x);
    gv[1] = __ldg(a.cvals + m.y);
    gv[2] = __ldg(a.cvals + m.z);
    gv[3] = __ldg(a.cvals + m.w);
  }
  const double s = p1 ? area : area * facet_scalar(a, c);
#pragma unroll
  for (int p = 0; p < T::ND; ++p) {
    double v;
    if (p1) {
      v = 0.0;
#pragma unroll
      for (int m = 0; m < 4; ++m) v = fma(gv[m], T::loadw(f, m, p), v);
    } else {
      v = T::load(f, p);
    }
    const int64_t R = __ldg(a.dofs + c * T::K + T::dof(f, p));
    if (R < a.num_values) atomicAdd(a.b + R, s * v);
  }
}

// vector-P2 traction load t.v ds, t constant or DG0 (3 values per cell)
__global__ void k_facet_traction(const FacetArgs a) {
  using T = FacetTab<2>;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.num_facets) return;
  const int2 cf = __ldg(a.facets + t);
  const int64_t c = cf.x;
  const int f = cf.y;
  const double area = facet_area(a, c, f);
  double tv[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) tv[q] = a.ckind == FE_COEFF_DG0 ? __ldg(a.cvals + 3 * c + q) : a.cconst[q];
#pragma unroll
  for (int p = 0; p < T::ND; ++p) {
    const int64_t R = __ldg(a.dofs + c * T::K + T::dof(f, p));
    const double w = area * T::load(f, p);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      if (3 * R + q < a.num_values) atomicAdd(a.b + 3 * R + q, w * tv[q]);
  }
}

// lifting of a facet mass form: b[rows] -= scale * A_f[rows, bc cols] (g - x0)
template <int DEG>
__global__ void k_facet_lift(const FacetArgs a) {
  using T = FacetTab<DEG>;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.num_facets) return;
  const int2 cf = __ldg(a.facets + t);
  const int64_t c = cf.x;
  const int f = cf.y;
  int R[T::ND];
  bool any = false;
  double dv[T::ND];
#pragma unroll
  for (int p = 0; p < T::ND; ++p) {
    R[p] = __ldg(a.dofs + c * T::K + T::dof(f, p));
    const bool m = a.bc1[R[p]] != 0;
    any |= m;
    dv[p] = m ? (a.g[R[p]] - (a.x0 ? a.x0[R[p]] : 0.0)) : 0.0;
  }
  if (!any) return;
  const double s = facet_area(a, c, f) * facet_scalar(a, c);
#pragma unroll
  for (int p = 0; p < T::ND; ++p) {
    double be = 0.0;
#pragma unroll
    for (int q = 0; q < T::ND; ++q) be = fma(T::mass(f, p, q), dv[q], be);
    if (be != 0.0 && R[p] < a.num_values) atomicAdd(a.b + R[p], -a.scale * s * be);
  }
}

unsigned fgrid(int64_t n) { return (unsigned)((n + 127) / 128); }

FacetArgs base_args(const fe_form_s& f) {
  FacetArgs a{};
  a.num_facets = f.num_facets;
  a.facets = reinterpret_cast<const int2*>(f.facets.p);
  a.x = f.mesh->x.p;
  a.geom = f.mesh->geom.p;
  a.dofs = f.V0->dofs.p;
  a.bs = f.V0->bs;
  const Coefficient& k = f.coeff[0];
  a.ckind = k.kind < 0 ? FE_COEFF_CONSTANT : k.kind;
  for (int q = 0; q < 3; ++q) a.cconst[q] = k.kind < 0 ? 1.0 : k.constant[q];
  a.cvals = k.values;
  a.cmap = k.map ? k.map->dofs.p : nullptr;
  return a;
}

}  // namespace

bool is_facet_kind(int kind) {
  return kind == FE_FORM_FFCX_EXTERIOR || kind == FE_FORM_P1_FACET_MASS || kind == FE_FORM_P2_FACET_MASS || kind == FE_FORM_P1_FACET_LOAD ||
         kind == FE_FORM_P2_FACET_LOAD || kind == FE_FORM_VP2_FACET_LOAD;
}

void assemble_matrix_facets(const fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1,
                            cudaStream_t s) {
  if (f.num_facets == 0) return;
  FacetArgs a = base_args(f);
  a.pos = f.pos.p;
  a.row_ptr = f.sp->row_ptr.p;
  a.bc0 = bc0 ? bc0->markers.p : nullptr;
  a.bc1 = bc1 ? bc1->markers.p : nullptr;
  a.values = values;
  if (f.kind == FE_FORM_P1_FACET_MASS) k_facet_mass<1><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  else k_facet_mass<2><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  FE_CUDA(cudaGetLastError());
}

void assemble_vector_facets(const fe_form_s& f, double* b, int64_t num_values, cudaStream_t s) {
  if (f.num_facets == 0) return;
  FacetArgs a = base_args(f);
  a.b = b;
  a.num_values = num_values;
  if (f.kind == FE_FORM_P1_FACET_LOAD) k_facet_load<1><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  else if (f.kind == FE_FORM_P2_FACET_LOAD) k_facet_load<2><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  else k_facet_traction<<<fgrid(f.num_facets), 128, 0, s>>>(a);
  FE_CUDA(cudaGetLastError());
}

void lifting_facets(const fe_form_s& f, const fe_bc_s& bc, const double* x0, double scale, double* b,
                    int64_t num_values, cudaStream_t s) {
  if (f.num_facets == 0) return;
  FacetArgs a = base_args(f);
  a.bc1 = bc.markers.p;
  a.g = bc.g.p;
  a.x0 = x0;
  a.scale = scale;
  a.b = b;
  a.num_values = num_values;
  if (f.kind == FE_FORM_P1_FACET_MASS) k_facet_lift<1><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  else k_facet_lift<2><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  FE_CUDA(cudaGetLastError());
}

}  // namespace fe
