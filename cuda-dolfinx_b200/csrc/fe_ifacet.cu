// Interior-facet integrals (dS) of discontinuous spaces: the jump penalty
// alpha*jump(u)*jump(v)*dS on DG0 / DG1, the average load g*avg(v)*dS and
// lifting of the jump penalty.
//
// The reference generates these from FFCx interior-facet tabulate_tensor
// bodies: vector assembly CUDAFormIntegral.cpp:451-522, matrix assembly
// :1988-2103; the element tensor couples the dofs of the two cells (a
// "macro" cell: cell0's dofs, then cell1's) and FFCx aligns the two cells'
// quadrature points with facet permutations.  Here a facet comes as
// (cell0, local facet0, cell1, local facet1); the kernel matches the facet's
// vertices in the two cells by their global index, so no permutation data is
// needed, and the tensors are closed-form: on a triangle of area |F|,
// int_F lambda_p lambda_q = |F| (1 + delta_pq) / 12 and int_F lambda_p = |F| / 3
// for the facet's barycentric coordinates.  One thread per facet; the matrix
// scatters through a per-facet byte map of the macro couplings.
#include <cuda_runtime.h>

#include <type_traits>

#include "fe_internal.h"

namespace fe {
namespace {

struct IFArgs {
  int kind;
  int64_t num_facets;
  const int4* __restrict__ quads;      // (cell0, facet0, cell1, facet1)
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  const int32_t* __restrict__ macro0;  // [F][2k] test dofs: cell0's, then cell1's
  const int32_t* __restrict__ macro1;  // [F][2k] trial dofs
  // coefficient alpha (jump) or g (load): constant or DG0 (averaged over the two cells)
  int ckind;
  double cconst;
  const double* __restrict__ cvals;
  // matrix
  const uint8_t* __restrict__ pos;     // [F][2k][2k]
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
  unsigned* err;
};

__device__ __forceinline__ double facet_coef(const IFArgs& a, int4 q) {
  return a.ckind == FE_COEFF_DG0 ? 0.5 * (__ldg(a.cvals + q.x) + __ldg(a.cvals + q.z)) : a.cconst;
}

// Area of the shared facet; loc0[p] / loc1[p] = local vertex of cell0 / cell1
// holding facet vertex p.  False (and the error word set) if the two local
// facets are not the same triangle.
__device__ bool shared_facet(const IFArgs& a, int4 q, double& area, int loc0[3], int loc1[3]) {
  const int4 g0 = __ldg(reinterpret_cast<const int4*>(a.geom) + q.x);
  const int4 g1 = __ldg(reinterpret_cast<const int4*>(a.geom) + q.z);
  const int v0[4] = {g0.x, g0.y, g0.z, g0.w}, v1[4] = {g1.x, g1.y, g1.z, g1.w};
  int n = 0;
#pragma unroll
  for (int t = 0; t < 4; ++t)
    if (t != q.y) loc0[n++] = t;
#pragma unroll
  for (int p = 0; p < 3; ++p) {
    loc1[p] = -1;
#pragma unroll
    for (int t = 0; t < 4; ++t)
      if (t != q.w && v1[t] == v0[loc0[p]]) loc1[p] = t;
    if (loc1[p] < 0) {
      atomicOr(a.err, DEV_ERR_FACET);
      return false;
    }
  }
  double P[3][3];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int d = 0; d < 3; ++d) P[p][d] = __ldg(a.x + 3 * (int64_t)v0[loc0[p]] + d);
  const double u[3] = {P[1][0] - P[0][0], P[1][1] - P[0][1], P[1][2] - P[0][2]};
  const double w[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
  const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
  area = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
  return true;
}

// The jump tensor entry (I, J) of the macro dofs, written for compile-time I
// and J: fp[I] is the facet vertex that macro dof I sits on (-1 for the
// vertex opposite the facet; DG0: 0 for both cells), the sign is + for cell0's
// dofs and - for cell1's.  Keeping every index compile-time keeps the
// per-facet arrays in registers.
template <int K, int I, int J>
__device__ __forceinline__ double jump_entry(double s, const int fp[2 * K]) {
  constexpr double sign = ((I < K) == (J < K)) ? 1.0 : -1.0;
  if constexpr (K == 1) {
    return sign * s;
  } else {
    if (fp[I] < 0 || fp[J] < 0) return 0.0;
    return sign * s * (fp[I] == fp[J] ? (2.0 / 12.0) : (1.0 / 12.0));
  }
}

template <int K, int I, int J, typename F>
__device__ __forceinline__ void for_each_entry(F&& f) {
  if constexpr (I < 2 * K) {
    if constexpr (J < 2 * K) {
      f(std::integral_constant<int, I>{}, std::integral_constant<int, J>{});
      for_each_entry<K, I, J + 1>(f);
    } else {
      for_each_entry<K, I + 1, 0>(f);
    }
  }
}

template <int K>
__global__ void __launch_bounds__(128) k_ifacet_jump(const IFArgs a) {
  constexpr int M = 2 * K;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.num_facets) return;
  const int4 q = __ldg(a.quads + t);
  double area;
  int loc0[3], loc1[3];
  if (!shared_facet(a, q, area, loc0, loc1)) return;
  const double s = area * facet_coef(a, q);
  // facet vertex of each macro dof
  int fp[M];
#pragma unroll
  for (int I = 0; I < M; ++I) fp[I] = K == 1 ? 0 : -1;
  if constexpr (K == 4) {
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        if (loc0[p] == v) fp[v] = p;
        if (loc1[p] == v) fp[K + v] = p;
      }
  }
  int rp[M];
  unsigned mr = 0, mc = 0;
#pragma unroll
  for (int I = 0; I < M; ++I) {
    const int r = __ldg(a.macro0 + t * M + I), c = __ldg(a.macro1 + t * M + I);
    rp[I] = __ldg(a.row_ptr + r);
    mr |= (a.bc0 && __ldg(a.bc0 + r) ? 1u : 0u) << I;
    mc |= (a.bc1 && __ldg(a.bc1 + c) ? 1u : 0u) << I;
  }
  const uint8_t* p = a.pos + t * (M * M);
  double* __restrict__ vals = a.values;
  for_each_entry<K, 0, 0>([&](auto ic, auto jc) {
    constexpr int I = decltype(ic)::value, J = decltype(jc)::value;
    const double v = jump_entry<K, I, J>(s, fp);
    if (v != 0.0 && !(((mr >> I) | (mc >> J)) & 1u)) atomicAdd(vals + rp[I] + __ldg(p + I * M + J), v);
  });
}

template <int K>
__global__ void __launch_bounds__(128) k_ifacet_lift(const IFArgs a) {
  constexpr int M = 2 * K;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.num_facets) return;
  double dv[M], be[M];
  bool any = false;
#pragma unroll
  for (int J = 0; J < M; ++J) {
    const int c = __ldg(a.macro1 + t * M + J);
    const bool m = __ldg(a.bc1 + c) != 0;
    dv[J] = m ? __ldg(a.g + c) - (a.x0 ? __ldg(a.x0 + c) : 0.0) : 0.0;
    be[J] = 0.0;
    any |= m;
  }
  if (!any) return;
  const int4 q = __ldg(a.quads + t);
  double area;
  int loc0[3], loc1[3];
  if (!shared_facet(a, q, area, loc0, loc1)) return;
  const double s = area * facet_coef(a, q);
  int fp[M];
#pragma unroll
  for (int I = 0; I < M; ++I) fp[I] = K == 1 ? 0 : -1;
  if constexpr (K == 4) {
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int p = 0; p < 3; ++p) {
        if (loc0[p] == v) fp[v] = p;
        if (loc1[p] == v) fp[K + v] = p;
      }
  }
  for_each_entry<K, 0, 0>([&](auto ic, auto jc) {
    constexpr int I = decltype(ic)::value, J = decltype(jc)::value;
    be[I] += jump_entry<K, I, J>(s, fp) * dv[J];
  });
#pragma unroll
  for (int I = 0; I < M; ++I) {
    const int64_t r = __ldg(a.macro0 + t * M + I);
    if (be[I] != 0.0 && r >= 0 && r < a.num_values) atomicAdd(a.b + r, -a.scale * be[I]);
  }
}

template <int K>
__global__ void __launch_bounds__(128) k_ifacet_avg_load(const IFArgs a) {
  constexpr int M = 2 * K;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.num_facets) return;
  const int4 q = __ldg(a.quads + t);
  double area;
  int loc0[3], loc1[3];
  if (!shared_facet(a, q, area, loc0, loc1)) return;
  const double g = facet_coef(a, q);
  auto add = [&](int I, double v) {
    const int64_t r = __ldg(a.macro0 + t * M + I);
    if (r >= 0 && r < a.num_values) atomicAdd(a.b + r, v);
  };
  if constexpr (K == 1) {
    add(0, 0.5 * g * area);
    add(1, 0.5 * g * area);
  } else {
    const double v = g * area * (0.5 / 3.0);
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      add(loc0[p], v);
      add(K + loc1[p], v);
    }
  }
}

unsigned fgrid(int64_t n) { return (unsigned)((n + 127) / 128); }

IFArgs base_args(const fe_form_s& f) {
  IFArgs a{};
  a.kind = f.kind;
  a.num_facets = f.num_facets;
  a.quads = reinterpret_cast<const int4*>(f.facets.p);
  a.x = f.mesh->x.p;
  a.geom = f.mesh->geom.p;
  a.macro0 = f.macro0.p;
  a.macro1 = f.macro1.p ? f.macro1.p : f.macro0.p;
  const Coefficient& k = f.coeff[0];
  a.ckind = k.kind < 0 ? FE_COEFF_CONSTANT : k.kind;
  a.cconst = k.kind < 0 ? 1.0 : k.constant[0];
  a.cvals = k.values;
  a.err = device_error_word(f.ctx);
  return a;
}

bool dg1(int kind) { return kind == FE_FORM_DG1_JUMP || kind == FE_FORM_DG1_AVG_LOAD; }

}  // namespace

bool is_ifacet_kind(int kind) {
  return kind == FE_FORM_FFCX_INTERIOR || kind == FE_FORM_DG0_JUMP || kind == FE_FORM_DG1_JUMP || kind == FE_FORM_DG0_AVG_LOAD ||
         kind == FE_FORM_DG1_AVG_LOAD;
}

void assemble_matrix_ifacets(const fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1,
                             cudaStream_t s) {
  if (f.num_facets == 0) return;
  IFArgs a = base_args(f);
  a.pos = f.pos.p;
  a.row_ptr = f.sp->row_ptr.p;
  a.bc0 = bc0 ? bc0->markers.p : nullptr;
  a.bc1 = bc1 ? bc1->markers.p : nullptr;
  a.values = values;
  if (dg1(f.kind)) k_ifacet_jump<4><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  else k_ifacet_jump<1><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  FE_CUDA(cudaGetLastError());
}

void assemble_vector_ifacets(const fe_form_s& f, double* b, int64_t num_values, cudaStream_t s) {
  if (f.num_facets == 0) return;
  IFArgs a = base_args(f);
  a.b = b;
  a.num_values = num_values;
  if (dg1(f.kind)) k_ifacet_avg_load<4><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  else k_ifacet_avg_load<1><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  FE_CUDA(cudaGetLastError());
}

void lifting_ifacets(const fe_form_s& f, const fe_bc_s& bc, const double* x0, double scale, double* b,
                     int64_t num_values, cudaStream_t s) {
  if (f.num_facets == 0) return;
  IFArgs a = base_args(f);
  a.bc1 = bc.markers.p;
  a.g = bc.g.p;
  a.x0 = x0;
  a.scale = scale;
  a.b = b;
  a.num_values = num_values;
  if (dg1(f.kind)) k_ifacet_lift<4><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  else k_ifacet_lift<1><<<fgrid(f.num_facets), 128, 0, s>>>(a);
  FE_CUDA(cudaGetLastError());
}

}  // namespace fe
