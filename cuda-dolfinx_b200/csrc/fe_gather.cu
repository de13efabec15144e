// Deterministic matrix assembly: sorted-slot segmented reduction.
//
// The reference has only the FP64-atomic scatter (CUDAFormIntegral.cpp:
// 1103-1226), whose summation order changes from run to run.  This variant
// gives bitwise-reproducible CSR values:
//   plan (once per form + pattern):
//     every element-matrix entry (cell c, local scalar entry e) is one
//     contribution with id e*num_cells + c; contributions are counting-sorted
//     by CSR slot and each slot's list is ordered by id;
//   assemble:
//     k_elem_*    element tensors of all cells -> E[e*num_cells + c] (FP64)
//     k_gather    per CSR row, per slot: value = sum of E over the slot's
//                 list in list order, BC rows/cols masked, written once (the
//                 zero pass and the BC skip of the reference are fused here)
//     set_diagonal as in the atomic variant.
#include <cuda_runtime.h>

#include <algorithm>

#include "fe_element_code.cuh"
#include "fe_internal.h"

fe_form_s::fe_form_s() = default;
fe_form_s::~fe_form_s() = default;

void fe::reset_gather_plan(fe_form_s& f) {
  f.gather.reset();
  reset_tile_plan(f);
  reset_row_plan(f);
  reset_block_plan(f);
  reset_batch_plan(f);
}

namespace fe {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// Exclusive scan of one tile per block; block totals to `sums`.
__global__ void __launch_bounds__(kScanThreads) k_scan_tile(int32_t* __restrict__ data, int64_t n,
                                                             int32_t* __restrict__ sums) {
  __shared__ int32_t warp_tot[kScanThreads / 32];
  const int64_t base = blockIdx.x * (int64_t)kScanTile + threadIdx.x * (int64_t)kScanItems;
  int32_t v[kScanItems];
  int32_t local = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    v[q] = (base + q < n) ? data[base + q] : 0;
    local += v[q];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int32_t incl = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int32_t t = warp_tot[lane];
    int32_t ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t y = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += y;
    }
    warp_tot[lane] = ti - t;  // exclusive warp offsets
    if (lane == 31 && sums) sums[blockIdx.x] = ti;
  }
  __syncthreads();
  int32_t run = warp_tot[wid] + incl - local;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    if (base + q < n) data[base + q] = run;
    run += v[q];
  }
}

__global__ void k_scan_add(int32_t* __restrict__ data, int64_t n, const int32_t* __restrict__ offs) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) data[i] += offs[i / kScanTile];
}

// In-place exclusive scan of n int32 values.
void scan_exclusive(int32_t* data, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    k_scan_tile<<<1, kScanThreads, 0, s>>>(data, n, nullptr);
    FE_CUDA(cudaGetLastError());
    return;
  }
  DevBuf<int32_t> sums(tiles);
  k_scan_tile<<<(unsigned)tiles, kScanThreads, 0, s>>>(data, n, sums.p);
  FE_CUDA(cudaGetLastError());
  scan_exclusive(sums.p, tiles, s);
  k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(data, n, sums.p);
  FE_CUDA(cudaGetLastError());
  FE_CUDA(cudaStreamSynchronize(s));  // `sums` is freed on return
}

struct SlotArgs {
  int64_t num_cells;
  const int32_t* __restrict__ dofs0;
  const int32_t* __restrict__ dofs1;
  int k0, k1, bs;
  const uint8_t* __restrict__ pos;
  const int32_t* __restrict__ row_ptr;
};

// CSR slot of scalar entry (ii, jj) of cell c
__device__ __forceinline__ int32_t slot_of(const SlotArgs& a, int64_t c, int ii, int jj) {
  const int i = ii / a.bs, ca = ii % a.bs, j = jj / a.bs, cb = jj % a.bs;
  const int64_t R = a.dofs0[c * a.k0 + i];
  const int32_t lo = a.row_ptr[R * a.bs + ca];
  return lo + a.bs * (int32_t)a.pos[(c * a.k0 + i) * a.k1 + j] + cb;
}

__global__ void k_count(const SlotArgs a, int32_t* __restrict__ cnt) {
  const int K = a.k0 * a.bs;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.num_cells * K * K) return;
  const int64_t e = t / a.num_cells, c = t % a.num_cells;
  atomicAdd(cnt + slot_of(a, c, (int)(e / K), (int)(e % K)), 1);
}

__global__ void k_fill(const SlotArgs a, int32_t* __restrict__ cursor, int32_t* __restrict__ contrib) {
  const int K = a.k0 * a.bs;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= a.num_cells * K * K) return;
  const int64_t e = t / a.num_cells, c = t % a.num_cells;
  const int32_t q = atomicAdd(cursor + slot_of(a, c, (int)(e / K), (int)(e % K)), 1);
  contrib[q] = (int32_t)t;
}

// order each slot's list by contribution id (lists are short: <= ~24 for the
// supported elements)
__global__ void k_sort_segments(const int32_t* __restrict__ seg, int64_t nnz, int32_t* __restrict__ contrib) {
  const int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (s >= nnz) return;
  const int32_t lo = seg[s], hi = seg[s + 1];
  for (int32_t i = lo + 1; i < hi; ++i) {
    const int32_t v = contrib[i];
    int32_t j = i - 1;
    while (j >= lo && contrib[j] > v) {
      contrib[j + 1] = contrib[j];
      --j;
    }
    contrib[j + 1] = v;
  }
}

// ---- element tensors, entry-major --------------------------------------
struct ElemArgs {
  int64_t num_cells;
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  int coef0_kind;
  const double* __restrict__ c0;
  const int32_t* __restrict__ c0map;
  double c0const;
  int coef1_kind;
  const double* __restrict__ c1;
  double c1const;
  double* __restrict__ E;
};

struct Geo {
  double K[3][3];
  double adet;
};

__device__ __forceinline__ void geo(const double* __restrict__ x, const int32_t* __restrict__ geom, int64_t c,
                                    Geo& g) {
  const int4 v = __ldg(reinterpret_cast<const int4*>(geom) + c);
  const int vv[4] = {v.x, v.y, v.z, v.w};
  double J[3][3];
#pragma unroll
  for (int cc = 0; cc < 3; ++cc)
#pragma unroll
    for (int r = 0; r < 3; ++r) J[r][cc] = __ldg(x + 3 * (int64_t)vv[cc + 1] + r) - __ldg(x + 3 * (int64_t)vv[0] + r);
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

__device__ __forceinline__ double cellcoef(int kind, const double* v, double cst, int64_t c) {
  return kind == FE_COEFF_DG0 ? __ldg(v + c) : cst;
}

__global__ void k_elem_p1(const ElemArgs a) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= a.num_cells) return;
  Geo g;
  geo(a.x, a.geom, c, g);
  double G[4][3];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    G[1][b] = g.K[0][b];
    G[2][b] = g.K[1][b];
    G[3][b] = g.K[2][b];
    G[0][b] = -(g.K[0][b] + g.K[1][b] + g.K[2][b]);
  }
  double kc;
  if (a.coef0_kind == FE_COEFF_P1) {  // P1 coefficient: its cell mean (constant gradients)
    const int4 km = __ldg(reinterpret_cast<const int4*>(a.c0map) + c);
    kc = 0.25 * ((__ldg(a.c0 + km.x) + __ldg(a.c0 + km.y)) + (__ldg(a.c0 + km.z) + __ldg(a.c0 + km.w)));
  } else {
    kc = cellcoef(a.coef0_kind, a.c0, a.c0const, c);
  }
  const double s = g.adet * (1.0 / 6.0) * kc;
  const int64_t N = a.num_cells;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = i; j < 4; ++j) {
      const double v = s * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]);
      a.E[(i * 4 + j) * N + c] = v;
      if (i != j) a.E[(j * 4 + i) * N + c] = v;
    }
}

// mass matrices (P1: K = 4, P2: K = 10) with a constant / DG0 / P1 coefficient
template <int K, int COEF>
__global__ void k_elem_mass(const ElemArgs a) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= a.num_cells) return;
  Geo g;
  geo(a.x, a.geom, c, g);
  const int64_t N = a.num_cells;
  double* __restrict__ E = a.E;
  auto emit = [&](int i, int j, double v) {
    E[(i * K + j) * N + c] = v;
    if (i != j) E[(j * K + i) * N + c] = v;
  };
  if constexpr (COEF == FE_COEFF_P1) {
    const int4 km = __ldg(reinterpret_cast<const int4*>(a.c0map) + c);
    const double cq[4] = {g.adet * __ldg(a.c0 + km.x), g.adet * __ldg(a.c0 + km.y), g.adet * __ldg(a.c0 + km.z),
                          g.adet * __ldg(a.c0 + km.w)};
    if constexpr (K == 4) p1_mass_p1coef<double>(cq, emit);
    else p2_mass_p1coef<double>(cq, emit);
  } else {
    const double sc = g.adet * cellcoef(a.coef0_kind, a.c0, a.c0const, c);
    if constexpr (K == 4) p1_mass_const<double>(sc, emit);
    else p2_mass_const<double>(sc, emit);
  }
}

// vector-P2 mass: all 900 entries (the gather reads every entry), zero
// between different components
template <int COEF>
__global__ void k_elem_vmass(const ElemArgs a) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= a.num_cells) return;
  Geo g;
  geo(a.x, a.geom, c, g);
  const int64_t N = a.num_cells;
  double* __restrict__ E = a.E;
  for (int e = 0; e < 900; ++e) E[e * N + c] = 0.0;
  auto emit = [&](int i, int j, double v) {
#pragma unroll
    for (int ca = 0; ca < 3; ++ca) {
      const int ii = 3 * i + ca, jj = 3 * j + ca;
      E[(ii * 30 + jj) * N + c] = v;
      if (ii != jj) E[(jj * 30 + ii) * N + c] = v;
    }
  };
  if constexpr (COEF == FE_COEFF_P1) {
    const int4 km = __ldg(reinterpret_cast<const int4*>(a.c0map) + c);
    const double cq[4] = {g.adet * __ldg(a.c0 + km.x), g.adet * __ldg(a.c0 + km.y), g.adet * __ldg(a.c0 + km.z),
                          g.adet * __ldg(a.c0 + km.w)};
    p2_mass_p1coef<double>(cq, emit);
  } else {
    p2_mass_const<double>(g.adet * cellcoef(a.coef0_kind, a.c0, a.c0const, c), emit);
  }
}

template <int COEF, typename T>
__global__ void k_elem_p2(const ElemArgs a) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= a.num_cells) return;
  Geo g;
  geo(a.x, a.geom, c, g);
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  double Gh[6];
#pragma unroll
  for (int s = 0; s < 6; ++s)
    Gh[s] = g.adet * (g.K[pa[s]][0] * g.K[pb[s]][0] + g.K[pa[s]][1] * g.K[pb[s]][1] + g.K[pa[s]][2] * g.K[pb[s]][2]);
  const int64_t N = a.num_cells;
  double* __restrict__ E = a.E;
  auto emit = [&](int i, int j, double v) {
    E[(i * 10 + j) * N + c] = v;
    if (i != j) E[(j * 10 + i) * N + c] = v;
  };
  if constexpr (COEF == FE_COEFF_P1) {
    const int4 km = __ldg(reinterpret_cast<const int4*>(a.c0map) + c);
    const double k[4] = {__ldg(a.c0 + km.x), __ldg(a.c0 + km.y), __ldg(a.c0 + km.z), __ldg(a.c0 + km.w)};
    T q[24];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int s = 0; s < 6; ++s) q[m * 6 + s] = (T)(k[m] * Gh[s]);
    p2_stiffness_p1coef<T>(q, emit);
  } else {
    const double k = cellcoef(a.coef0_kind, a.c0, a.c0const, c);
    T gq[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
    p2_stiffness_const<T>(gq, emit);
  }
}

template <typename T>
__global__ void k_elem_p3(const ElemArgs a) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= a.num_cells) return;
  Geo g;
  geo(a.x, a.geom, c, g);
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  const double k = cellcoef(a.coef0_kind, a.c0, a.c0const, c);
  T gq[6];
#pragma unroll
  for (int s = 0; s < 6; ++s) {
    const double gh =
        g.adet * (g.K[pa[s]][0] * g.K[pb[s]][0] + g.K[pa[s]][1] * g.K[pb[s]][1] + g.K[pa[s]][2] * g.K[pb[s]][2]);
    gq[s] = (T)(k * gh);
  }
  const int64_t N = a.num_cells;
  double* __restrict__ E = a.E;
  p3_stiffness_const<T>(gq, [&](int i, int j, double v) {
    E[(i * 20 + j) * N + c] = v;
    if (i != j) E[(j * 20 + i) * N + c] = v;
  });
}

template <typename T>
__global__ void k_elem_vp2(const ElemArgs a) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= a.num_cells) return;
  Geo g;
  geo(a.x, a.geom, c, g);
  const double lam = cellcoef(a.coef0_kind, a.c0, a.c0const, c);
  const double mu = cellcoef(a.coef1_kind, a.c1, a.c1const, c);
  const int64_t N = a.num_cells;
  double* __restrict__ E = a.E;
#pragma unroll 1
  for (int blk = 0; blk < 6; ++blk) {
    const int ca = blk < 3 ? blk : (blk == 5 ? 1 : 0);
    const int cb = blk < 3 ? blk : (blk == 3 ? 1 : 2);
    T W[9];
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        double kk = 0.0;
        if (ca == cb) kk = g.K[p][0] * g.K[q][0] + g.K[p][1] * g.K[q][1] + g.K[p][2] * g.K[q][2];
        W[p * 3 + q] = (T)(g.adet * (mu * (kk + g.K[p][cb] * g.K[q][ca]) + lam * g.K[p][ca] * g.K[q][cb]));
      }
    auto emit = [&](int i, int j, double v) {
      const int ii = 3 * i + ca, jj = 3 * j + cb;
      E[(ii * 30 + jj) * N + c] = v;
      if (ii != jj) E[(jj * 30 + ii) * N + c] = v;
    };
    if (ca == cb)
      p2_block_upper<T>(W, emit);
    else
      p2_block_full<T>(W, emit);
  }
}

// One CSR row per 16-lane group: value = (zero ? 0 : old) + sum of the slot's
// contributions (skipped if the row or the column is BC-marked).
__global__ void k_gather(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col, int64_t num_rows,
                         const int32_t* __restrict__ seg, const int32_t* __restrict__ contrib,
                         const double* __restrict__ E, const uint8_t* __restrict__ bc0,
                         const uint8_t* __restrict__ bc1, int zero, double* __restrict__ values) {
  const int64_t gid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t r = gid >> 4;
  const int lane = threadIdx.x & 15;
  if (r >= num_rows) return;
  const bool rmask = bc0 && bc0[r];
  const int32_t lo = row_ptr[r], hi = row_ptr[r + 1];
  for (int32_t s = lo + lane; s < hi; s += 16) {
    double v = zero ? 0.0 : values[s];
    if (!rmask && !(bc1 && bc1[col[s]])) {
      const int32_t qa = seg[s], qb = seg[s + 1];
      double acc = 0.0;
      for (int32_t q = qa; q < qb; ++q) acc += E[contrib[q]];
      v += acc;
    }
    values[s] = v;
  }
}

unsigned blocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

void ensure_gather_plan(fe_form_s& f, cudaStream_t s) {
  if (f.gather) return;
  const int64_t C = f.mesh->num_cells;
  const int bs = f.V0->bs;
  const int K = f.V0->k * bs;
  const int64_t ncontrib = C * K * K;
  if (ncontrib > INT32_MAX) FE_FAIL(FE_ERR_ARG, "too many element entries for the sorted-slot plan");
  SlotArgs sa{C, f.V0->dofs.p, f.V1->dofs.p, f.V0->k, f.V1->k, bs, f.pos.p, f.sp->row_ptr.p};
  auto G = std::make_unique<fe_form_s::Gather>();
  const int64_t nnz = f.sp->nnz;
  G->num_contrib = ncontrib;
  G->K = K;
  G->seg.alloc(nnz + 1);
  G->contrib.alloc(std::max<int64_t>(1, ncontrib));
  FE_CUDA(cudaMemsetAsync(G->seg.p, 0, (nnz + 1) * sizeof(int32_t), s));
  if (ncontrib) {
    k_count<<<blocks(ncontrib, 256), 256, 0, s>>>(sa, G->seg.p);
    FE_CUDA(cudaGetLastError());
  }
  scan_exclusive(G->seg.p, nnz + 1, s);
  DevBuf<int32_t> cursor(nnz + 1);
  FE_CUDA(cudaMemcpyAsync(cursor.p, G->seg.p, (nnz + 1) * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
  if (ncontrib) {
    k_fill<<<blocks(ncontrib, 256), 256, 0, s>>>(sa, cursor.p, G->contrib.p);
    FE_CUDA(cudaGetLastError());
  }
  if (nnz) {
    k_sort_segments<<<blocks(nnz, 256), 256, 0, s>>>(G->seg.p, nnz, G->contrib.p);
    FE_CUDA(cudaGetLastError());
  }
  FE_CUDA(cudaStreamSynchronize(s));  // cursor is freed on return
  f.gather = std::move(G);
}

void assemble_matrix_gather(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, double diagonal,
                            bool zero, cudaStream_t s) {
  const int64_t C = f.mesh->num_cells;
  ensure_gather_plan(f, s);
  if (!f.gather->E.p) f.gather->E.alloc(std::max<int64_t>(1, f.gather->num_contrib));
  auto& G = *f.gather;
  ElemArgs ea{};
  ea.num_cells = C;
  ea.x = f.mesh->x.p;
  ea.geom = f.mesh->geom.p;
  const Coefficient& k0 = f.coeff[0];
  const Coefficient& k1 = f.coeff[1];
  ea.coef0_kind = k0.kind < 0 ? FE_COEFF_CONSTANT : k0.kind;
  ea.c0 = k0.values;
  ea.c0map = k0.map ? k0.map->dofs.p : nullptr;
  ea.c0const = k0.kind < 0 ? 1.0 : k0.constant[0];
  ea.coef1_kind = k1.kind < 0 ? FE_COEFF_CONSTANT : k1.kind;
  ea.c1 = k1.values;
  ea.c1const = k1.kind < 0 ? 1.0 : k1.constant[0];
  ea.E = G.E.p;
  if (C) {
    const unsigned grid = blocks(C, 128);
    switch (f.kind) {
      case FE_FORM_P1_STIFFNESS:
        k_elem_p1<<<grid, 128, 0, s>>>(ea);
        break;
      case FE_FORM_P2_STIFFNESS:
        if (f.precision == FE_PREC_FP32) {
          if (ea.coef0_kind == FE_COEFF_P1) k_elem_p2<FE_COEFF_P1, float><<<grid, 128, 0, s>>>(ea);
          else k_elem_p2<FE_COEFF_DG0, float><<<grid, 128, 0, s>>>(ea);
        } else {
          if (ea.coef0_kind == FE_COEFF_P1) k_elem_p2<FE_COEFF_P1, double><<<grid, 128, 0, s>>>(ea);
          else k_elem_p2<FE_COEFF_DG0, double><<<grid, 128, 0, s>>>(ea);
        }
        break;
      case FE_FORM_VP2_ELASTICITY:
        if (f.precision == FE_PREC_FP32) k_elem_vp2<float><<<grid, 128, 0, s>>>(ea);
        else k_elem_vp2<double><<<grid, 128, 0, s>>>(ea);
        break;
      case FE_FORM_P1_MASS:
        if (ea.coef0_kind == FE_COEFF_P1) k_elem_mass<4, FE_COEFF_P1><<<grid, 128, 0, s>>>(ea);
        else k_elem_mass<4, FE_COEFF_DG0><<<grid, 128, 0, s>>>(ea);
        break;
      case FE_FORM_P2_MASS:
        if (ea.coef0_kind == FE_COEFF_P1) k_elem_mass<10, FE_COEFF_P1><<<grid, 128, 0, s>>>(ea);
        else k_elem_mass<10, FE_COEFF_DG0><<<grid, 128, 0, s>>>(ea);
        break;
      case FE_FORM_VP2_MASS:
        if (ea.coef0_kind == FE_COEFF_P1) k_elem_vmass<FE_COEFF_P1><<<grid, 128, 0, s>>>(ea);
        else k_elem_vmass<FE_COEFF_DG0><<<grid, 128, 0, s>>>(ea);
        break;
      case FE_FORM_P3_STIFFNESS:
        if (f.precision == FE_PREC_FP32) k_elem_p3<float><<<grid, 128, 0, s>>>(ea);
        else k_elem_p3<double><<<grid, 128, 0, s>>>(ea);
        break;
      default:
        FE_FAIL(FE_ERR_ARG, "not a bilinear form");
    }
    FE_CUDA(cudaGetLastError());
  }
  const int64_t nrows = f.sp->num_rows;
  if (nrows) {
    k_gather<<<blocks(nrows * 16, 256), 256, 0, s>>>(f.sp->row_ptr.p, f.sp->col.p, nrows, G.seg.p, G.contrib.p,
                                                       G.E.p, bc0 ? bc0->markers.p : nullptr,
                                                       bc1 ? bc1->markers.p : nullptr, zero ? 1 : 0, values);
    FE_CUDA(cudaGetLastError());
  }
  if (bc0) launch_set_diagonal(*f.sp, *bc0, diagonal, values, s);
}

}  // namespace fe
