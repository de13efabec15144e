// sm_100a assembly kernels: element tensors + scatter through the cell-to-slot
// map, vector assembly, lifting, set_bc, set_diagonal, slot-map construction.
//
// Reference counterparts (NVRTC string templates, one thread per cell, binary
// search per element entry, FP64 atomicAdd):
//   matrix   cpp/cudolfinx/fem/CUDAFormIntegral.cpp:1103-1226
//   vector   cpp/cudolfinx/fem/CUDAFormIntegral.cpp:270-357
//   lifting  cpp/cudolfinx/fem/CUDAFormIntegral.cpp:603-717
//   utils    cpp/cudolfinx/fem/CUDAAssembler.cpp:38-164
//
// Here the column search is replaced by a per-cell byte map `pos` built once
// (block position of column dof j inside block row dof i), the slot is
// row_ptr[bs*dof_i + a] + bs*pos + b, element tensors use the symmetric half
// only, and coefficients are gathered in-kernel (no separate packing pass).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <memory>
#include <type_traits>
#include <vector>

#include "fe_element_code.cuh"
#include "fe_internal.h"

namespace fe {
namespace {

constexpr int kBlock = 128;  // threads (= cells) per CTA for thread-per-cell kernels

__device__ __forceinline__ void raise_err(unsigned* err, unsigned bit) { atomicOr(err, bit); }

struct CoefDev {
  int kind;            // fe_coeff_kind
  const double* v;     // DG0: [cells*ncomp]; P1: [nodes]
  const int32_t* map;  // P1: [cells*4]
  double c[3];         // constant
};

CoefDev to_dev(const Coefficient* c) {
  CoefDev d{};
  if (!c || c->kind < 0) {
    d.kind = FE_COEFF_CONSTANT;
    d.c[0] = d.c[1] = d.c[2] = 1.0;
    return d;
  }
  d.kind = c->kind;
  d.v = c->values;
  d.map = c->map ? c->map->dofs.p : nullptr;
  for (int i = 0; i < 3; ++i) d.c[i] = c->constant[i];
  return d;
}

// cellwise scalar value of a DG0 / constant coefficient
__device__ __forceinline__ double coef_cell(const CoefDev& k, int64_t c) {
  return k.kind == FE_COEFF_DG0 ? __ldg(k.v + c) : k.c[0];
}

// mean over the cell of a constant / DG0 / P1 coefficient (the exact factor of
// a P1 stiffness entry: the gradients are constant on the cell)
__device__ __forceinline__ double coef_mean(const CoefDev& k, int64_t c) {
  if (k.kind == FE_COEFF_P1) {
    const int4 m = __ldg(reinterpret_cast<const int4*>(k.map) + c);
    return 0.25 * ((__ldg(k.v + m.x) + __ldg(k.v + m.y)) + (__ldg(k.v + m.z) + __ldg(k.v + m.w)));
  }
  return coef_cell(k, c);
}

// ---------------------------------------------------------------------------
// Geometry of an affine tetrahedron: K = J^{-1}, |det J|
// ---------------------------------------------------------------------------
struct CellGeo {
  double K[3][3];
  double adet;
};

__device__ __forceinline__ void cell_geometry(const double* __restrict__ x, int4 v, CellGeo& g) {
  double x0[3], J[3][3];
  const int vv[3] = {v.y, v.z, v.w};
#pragma unroll
  for (int r = 0; r < 3; ++r) x0[r] = __ldg(x + 3 * (int64_t)v.x + r);
#pragma unroll
  for (int cc = 0; cc < 3; ++cc)
#pragma unroll
    for (int r = 0; r < 3; ++r) J[r][cc] = __ldg(x + 3 * (int64_t)vv[cc] + r) - x0[r];
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

__device__ __forceinline__ int4 load_geom(const int32_t* __restrict__ geom, int64_t c) {
  return __ldg(reinterpret_cast<const int4*>(geom) + c);
}

// Ghat_s = adet * (K K^T)_s, s over (00,11,22,01,02,12)
__device__ __forceinline__ void ghat(const CellGeo& g, double G[6]) {
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int s = 0; s < 6; ++s)
    G[s] = g.adet * (g.K[pa[s]][0] * g.K[pb[s]][0] + g.K[pa[s]][1] * g.K[pb[s]][1] +
                     g.K[pa[s]][2] * g.K[pb[s]][2]);
}

// P1 reference gradients dotted with K: grad phi_i = K^T ghat_i
__device__ __forceinline__ void p1_grads(const CellGeo& g, double G[4][3]) {
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    G[1][b] = g.K[0][b];
    G[2][b] = g.K[1][b];
    G[3][b] = g.K[2][b];
    G[0][b] = -(g.K[0][b] + g.K[1][b] + g.K[2][b]);
  }
}

// Stage a tile of the byte map into shared memory.  The map buffer is padded
// to a multiple of 16 bytes and tiles start at multiples of 16 bytes.
template <int BYTES_PER_CELL>
__device__ __forceinline__ void stage_pos(uint8_t* spos, const uint8_t* __restrict__ pos, int64_t c0,
                                          int ncell) {
  const uint4* src = reinterpret_cast<const uint4*>(pos + c0 * BYTES_PER_CELL);
  uint4* dst = reinterpret_cast<uint4*>(spos);
  const int nvec = (ncell * BYTES_PER_CELL + 15) / 16;
  for (int t = threadIdx.x; t < nvec; t += blockDim.x) dst[t] = __ldg(src + t);
}

struct MatArgs {
  int64_t num_cells;
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  const int32_t* __restrict__ dofs0;
  const int32_t* __restrict__ dofs1;
  const uint8_t* __restrict__ pos;
  const int32_t* __restrict__ row_ptr;
  const uint8_t* __restrict__ bc0;
  const uint8_t* __restrict__ bc1;
  CoefDev c0, c1;
  double* __restrict__ values;
  int upper;  // symmetric form + pattern: one reduction per unique entry, into the upper triangle
};

// ---------------------------------------------------------------------------
// P1 stiffness, one thread per cell, FP64 atomics
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT) k_mat_p1_atomic(const MatArgs a) {
  const int64_t c = blockIdx.x * (int64_t)NT + threadIdx.x;
  if (c >= a.num_cells) return;
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  double G[4][3];
  p1_grads(g, G);
  const double s = g.adet * (1.0 / 6.0) * coef_mean(a.c0, c);
  const int4 d0 = __ldg(reinterpret_cast<const int4*>(a.dofs0) + c);
  const int4 d1 = (a.dofs1 == a.dofs0) ? d0 : __ldg(reinterpret_cast<const int4*>(a.dofs1) + c);
  const int r[4] = {d0.x, d0.y, d0.z, d0.w};
  const int cl[4] = {d1.x, d1.y, d1.z, d1.w};
  const uint4 pw = __ldg(reinterpret_cast<const uint4*>(a.pos) + c);
  const uint32_t pws[4] = {pw.x, pw.y, pw.z, pw.w};
  // masked rows / columns: BC dofs and dofs outside a restriction (-1)
  unsigned mr = 0, mc = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    mr |= (r[i] < 0 || (a.bc0 && __ldg(a.bc0 + r[i])) ? 1u : 0u) << i;
    mc |= (cl[i] < 0 || (a.bc1 && __ldg(a.bc1 + cl[i])) ? 1u : 0u) << i;
  }
  int rp[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) rp[i] = r[i] < 0 ? 0 : __ldg(a.row_ptr + r[i]);
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = i; j < 4; ++j) {
      const double v = s * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]);
      const int sij = rp[i] + ((pws[i] >> (8 * j)) & 0xffu), sji = rp[j] + ((pws[j] >> (8 * i)) & 0xffu);
      const unsigned mij = (mr >> i) | (mc >> j), mji = (mr >> j) | (mc >> i);
      if (a.upper) {
        // one reduction per unique entry, into the upper triangle (the lower
        // one is filled from it afterwards); the target is a select, so the
        // warp issues one RED instead of two half-masked ones
        const bool lo = i == j || r[i] < r[j];
        if (!((lo ? mij : mji) & 1u)) atomicAdd(a.values + (lo ? sij : sji), v);
        continue;
      }
      if (!(mij & 1u)) atomicAdd(a.values + sij, v);
      if (i != j && !(mji & 1u)) atomicAdd(a.values + sji, v);
    }
}

// ---------------------------------------------------------------------------
// P2 stiffness, one thread per cell, FP64 atomics
// ---------------------------------------------------------------------------
// NT cells per CTA; STAGE: the CTA's byte maps staged in shared memory with
// 16-byte loads, else each thread reads its cell's bytes from global memory
template <int COEF, typename T, int NT = kBlock, bool STAGE = true>
__global__ void __launch_bounds__(NT) k_mat_p2_atomic(const MatArgs a) {
  __shared__ __align__(16) uint8_t spos[STAGE ? NT * 100 : 16];
  const int64_t c0 = blockIdx.x * (int64_t)NT;
  const int64_t left = a.num_cells - c0;
  const int ncell = left < NT ? (int)left : NT;
  if constexpr (STAGE) {
    stage_pos<100>(spos, a.pos, c0, ncell);
    __syncthreads();
  }
  if ((int)threadIdx.x >= ncell) return;
  const int64_t c = c0 + threadIdx.x;
  const uint8_t* p = STAGE ? spos + threadIdx.x * 100 : a.pos + c * 100;

  const int4 gv = load_geom(a.geom, c);
  CellGeo g;
  cell_geometry(a.x, gv, g);
  double Gh[6];
  ghat(g, Gh);

  int rp[10], rd[10];
  unsigned mr = 0, mc = 0;
  const int32_t* d0 = a.dofs0 + c * 10;
  const int32_t* d1 = a.dofs1 + c * 10;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    // masked rows / columns: BC dofs and dofs outside a restriction (-1)
    const int r = __ldg(d0 + i), cc = __ldg(d1 + i);
    rd[i] = r;
    rp[i] = r < 0 ? 0 : __ldg(a.row_ptr + r);
    mr |= (r < 0 || (a.bc0 && __ldg(a.bc0 + r)) ? 1u : 0u) << i;
    mc |= (cc < 0 || (a.bc1 && __ldg(a.bc1 + cc)) ? 1u : 0u) << i;
  }
  double* __restrict__ vals = a.values;
  const bool upper = a.upper != 0;
  auto emit = [&](int i, int j, double v) {
    const unsigned mij = (mr >> i) | (mc >> j), mji = (mr >> j) | (mc >> i);
    if (upper) {
      // one RED per unique entry, target chosen by a select (no divergence)
      const bool lo = i == j || rd[i] < rd[j];
      const int slot = lo ? rp[i] + p[i * 10 + j] : rp[j] + p[j * 10 + i];
      if (!((lo ? mij : mji) & 1u)) atomicAdd(vals + slot, v);
      return;
    }
    if (!(mij & 1u)) atomicAdd(vals + rp[i] + p[i * 10 + j], v);
    if (i != j && !(mji & 1u)) atomicAdd(vals + rp[j] + p[j * 10 + i], v);
  };
  if constexpr (COEF == FE_COEFF_P1) {
    const int4 km = __ldg(reinterpret_cast<const int4*>(a.c0.map) + c);
    const double k[4] = {__ldg(a.c0.v + km.x), __ldg(a.c0.v + km.y), __ldg(a.c0.v + km.z),
                         __ldg(a.c0.v + km.w)};
    T q[24];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int s = 0; s < 6; ++s) q[m * 6 + s] = (T)(k[m] * Gh[s]);
    p2_stiffness_p1coef<T>(q, emit);
  } else {
    const double k = coef_cell(a.c0, c);
    T gq[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
    p2_stiffness_const<T>(gq, emit);
  }
}

// ---------------------------------------------------------------------------
// P2 stiffness with the reductions coalesced per warp ("coalesced" variant).
// The L2 applies FP64 reductions per 32-byte sector: on B200 one warp
// instruction whose 32 reductions land in 32 sectors runs at ~210 G/s, with
// 2 per sector at ~400 G/s, with 4 at ~500 G/s.  In the thread-per-cell
// scatter each lane reduces into its own cell's rows, so an instruction
// touches ~30 sectors.  Here each thread still computes one cell's element
// tensor, but writes its 55 unique entries to shared memory; the warp then
// issues its 32 cells' 3200 reductions cell by cell, row by row, consecutive
// lanes on consecutive columns of a row: the 10 entries of a cell's row lie
// in one CSR row, ~1.8 per sector.
// ---------------------------------------------------------------------------
constexpr int kCoalThreads = 64;

// STAGE: the CTA's byte maps copied to shared memory first (6.4 KB), else
// fetched as words and handed out by shuffles in the reduction loop, which
// leaves room for a seventh CTA per SM (measured slower on B200: P2 n=96
// 2.66 against 2.46 ms)
template <bool STAGE>
struct P2CoalSmem {
  __align__(16) uint8_t spos[STAGE ? kCoalThreads * 100 : 16];
  double sE[kCoalThreads * 55];
  int32_t srp[kCoalThreads * 10];  // row start of each local row, -1 for a masked row
  uint16_t smc[kCoalThreads];      // masked columns of each cell
};

// the 64 cells from c0: element tensors, then the warp-ordered reductions
template <int COEF, typename T, bool STAGE>
__device__ __forceinline__ void p2_coal_tile(const MatArgs& a, const int64_t c0, P2CoalSmem<STAGE>& S) {
  constexpr int NT = kCoalThreads;
  uint8_t* spos = S.spos;
  double* sE = S.sE;
  int32_t* srp = S.srp;
  uint16_t* smc = S.smc;
  const int64_t left = a.num_cells - c0;
  const int ncell = left < NT ? (int)left : NT;
  const int tid = threadIdx.x, lane = tid & 31, w0 = tid & ~31;
  const int wcells = ncell - w0 < 0 ? 0 : (ncell - w0 < 32 ? ncell - w0 : 32);
  if constexpr (STAGE) {
    // each warp stages its own cells' byte maps (from a 16-byte boundary:
    // (c0 + w0) * 100 is a multiple of 3200; the map buffer is padded to 16)
    const uint4* src = reinterpret_cast<const uint4*>(a.pos + (c0 + w0) * 100);
    uint4* dst = reinterpret_cast<uint4*>(spos + w0 * 100);
    const int nvec = (wcells * 100 + 15) / 16;
    for (int t = lane; t < nvec; t += 32) dst[t] = __ldg(src + t);
  }
  if (tid < ncell) {
    const int64_t c = c0 + tid;
    CellGeo g;
    cell_geometry(a.x, load_geom(a.geom, c), g);
    double Gh[6];
    ghat(g, Gh);
    const int32_t* d0 = a.dofs0 + c * 10;
    const int32_t* d1 = a.dofs1 + c * 10;
    unsigned mc = 0;
#pragma unroll
    for (int i = 0; i < 10; ++i) {
      // masked rows / columns: BC dofs and dofs outside a restriction (-1)
      const int r = __ldg(d0 + i), cc = __ldg(d1 + i);
      const bool mrow = r < 0 || (a.bc0 && __ldg(a.bc0 + r));
      srp[tid * 10 + i] = mrow ? -1 : __ldg(a.row_ptr + r);
      mc |= (cc < 0 || (a.bc1 && __ldg(a.bc1 + cc)) ? 1u : 0u) << i;
    }
    smc[tid] = (uint16_t)mc;
    double* E = sE + tid * 55;
    auto emit = [&](int i, int j, double v) { E[i * (21 - i) / 2 + (j - i)] = v; };
    if constexpr (COEF == FE_COEFF_P1) {
      const int4 km = __ldg(reinterpret_cast<const int4*>(a.c0.map) + c);
      const double k[4] = {__ldg(a.c0.v + km.x), __ldg(a.c0.v + km.y), __ldg(a.c0.v + km.z),
                           __ldg(a.c0.v + km.w)};
      T q[24];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int s2 = 0; s2 < 6; ++s2) q[m * 6 + s2] = (T)(k[m] * Gh[s2]);
      p2_stiffness_p1coef<T>(q, emit);
    } else {
      const double k = coef_cell(a.c0, c);
      T gq[6];
#pragma unroll
      for (int s2 = 0; s2 < 6; ++s2) gq[s2] = (T)(k * Gh[s2]);
      p2_stiffness_const<T>(gq, emit);
    }
  }
  __syncwarp();  // the warp's staged byte maps and its cells' entries
  // lanes 10*h + j (h = 0..2, j = 0..9) take column j of row 3*r + h of one
  // cell, for r = 0..3: four instructions per cell, each on three rows; the
  // entry indices of a lane are the same for every cell
  const int h = lane / 10, j = lane - 10 * h;
  int ei[4], eu[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = 3 * r + h;
    const int lo = i < j ? i : j, hi = i < j ? j : i;
    const bool ok = lane < 30 && i < 10;
    ei[r] = ok ? i : -1;
    eu[r] = lo * (21 - lo) / 2 + (hi - lo);
  }
  double* __restrict__ vals = a.values;
  if constexpr (STAGE) {
#pragma unroll 2
    for (int q = w0; q < w0 + wcells; ++q) {
      const bool cmask = (smc[q] >> j) & 1u;
      const int32_t* rq = srp + q * 10;
      const uint8_t* pq = spos + q * 100;
      const double* Eq = sE + q * 55;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (ei[r] < 0 || cmask) continue;
        const int rs = rq[ei[r]];
        if (rs < 0) continue;
        atomicAdd(vals + rs + pq[ei[r] * 10 + j], Eq[eu[r]]);
      }
    }
  } else {
    // the slot bytes unstaged: lane w < 25 loads word w of a cell's 25 (one
    // coalesced 100-byte load per cell, one cell ahead, into alternating
    // registers), and byte b = 10 ei + j comes from lane b / 4 by a shuffle
    auto word_of = [&](int q) -> uint32_t {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(a.pos + (c0 + q) * 100);  // 100 c: 4-byte aligned
      return lane < 25 ? __ldg(src + lane) : 0u;
    };
    int bi[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) bi[r] = ei[r] < 0 ? 0 : ei[r] * 10 + j;
    auto cell = [&](int q, uint32_t w) {
      const bool cmask = (smc[q] >> j) & 1u;
      const int32_t* rq = srp + q * 10;
      const double* Eq = sE + q * 55;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const uint32_t word = __shfl_sync(0xffffffffu, w, bi[r] >> 2);
        if (ei[r] < 0 || cmask) continue;
        const int rs = rq[ei[r]];
        if (rs < 0) continue;
        atomicAdd(vals + rs + ((word >> (8 * (bi[r] & 3))) & 0xffu), Eq[eu[r]]);
      }
    };
    const int qend = w0 + wcells;
    uint32_t wa = 0u, wb = 0u;
    if (wcells > 0) wa = word_of(w0);
    for (int q = w0; q < qend; q += 2) {
      if (q + 1 < qend) wb = word_of(q + 1);
      cell(q, wa);
      if (q + 1 >= qend) break;
      if (q + 2 < qend) wa = word_of(q + 2);
      cell(q + 1, wb);
    }
  }
}

// 6 CTAs per SM, as many as the staged shared memory allows: the register cap
// is then 168 (the P1-coefficient kernel takes 168 instead of 128; measured
// 1 % faster at P2 n=96 than with the cap of 7 CTAs)
template <int COEF, typename T, bool STAGE>
__global__ void __launch_bounds__(kCoalThreads, STAGE ? 6 : 7) k_mat_p2_coal(const MatArgs a) {
  __shared__ P2CoalSmem<STAGE> S;
  p2_coal_tile<COEF, T, STAGE>(a, blockIdx.x * (int64_t)kCoalThreads, S);
}

// ---------------------------------------------------------------------------
// Mass matrices c*u*v*dx (P1: K = 4, P2: K = 10), one thread per cell, FP64
// atomics.  Only |det J| and the coefficient enter the element tensor.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double cell_adet(const double* __restrict__ x, int4 v) {
  double x0[3], J[3][3];
  const int vv[3] = {v.y, v.z, v.w};
#pragma unroll
  for (int r = 0; r < 3; ++r) x0[r] = __ldg(x + 3 * (int64_t)v.x + r);
#pragma unroll
  for (int cc = 0; cc < 3; ++cc)
#pragma unroll
    for (int r = 0; r < 3; ++r) J[r][cc] = __ldg(x + 3 * (int64_t)vv[cc] + r) - x0[r];
  return fabs(J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) +
              J[0][1] * (J[1][2] * J[2][0] - J[1][0] * J[2][2]) +
              J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]));
}

// emit(i, j, value) for the unique entries i <= j of cell c's mass matrix
template <int K, int COEF, typename Emit>
__device__ __forceinline__ void mass_element(const CoefDev& k, int64_t c, double adet, Emit&& emit) {
  static_assert(K == 4 || K == 10, "P1 or P2 mass");
  if constexpr (COEF == FE_COEFF_P1) {
    const int4 km = __ldg(reinterpret_cast<const int4*>(k.map) + c);
    const double cq[4] = {adet * __ldg(k.v + km.x), adet * __ldg(k.v + km.y), adet * __ldg(k.v + km.z),
                          adet * __ldg(k.v + km.w)};
    if constexpr (K == 4) p1_mass_p1coef<double>(cq, emit);
    else p2_mass_p1coef<double>(cq, emit);
  } else {
    const double sc = adet * coef_cell(k, c);
    if constexpr (K == 4) p1_mass_const<double>(sc, emit);
    else p2_mass_const<double>(sc, emit);
  }
}

template <int K, int COEF>
__global__ void __launch_bounds__(kBlock) k_mat_mass(const MatArgs a) {
  __shared__ __align__(16) uint8_t spos[kBlock * K * K];
  const int64_t c0 = blockIdx.x * (int64_t)kBlock;
  const int64_t left = a.num_cells - c0;
  const int ncell = left < kBlock ? (int)left : kBlock;
  stage_pos<K * K>(spos, a.pos, c0, ncell);
  __syncthreads();
  if ((int)threadIdx.x >= ncell) return;
  const int64_t c = c0 + threadIdx.x;
  const uint8_t* p = spos + threadIdx.x * K * K;
  const double adet = cell_adet(a.x, load_geom(a.geom, c));
  int rp[K], rd[K];
  unsigned mr = 0, mc = 0;
  const int32_t* d0 = a.dofs0 + c * K;
  const int32_t* d1 = a.dofs1 + c * K;
#pragma unroll
  for (int i = 0; i < K; ++i) {
    // masked rows / columns: BC dofs and dofs outside a restriction (-1)
    const int r = __ldg(d0 + i), cc = __ldg(d1 + i);
    rd[i] = r;
    rp[i] = r < 0 ? 0 : __ldg(a.row_ptr + r);
    mr |= (r < 0 || (a.bc0 && __ldg(a.bc0 + r)) ? 1u : 0u) << i;
    mc |= (cc < 0 || (a.bc1 && __ldg(a.bc1 + cc)) ? 1u : 0u) << i;
  }
  double* __restrict__ vals = a.values;
  const bool upper = a.upper != 0;
  mass_element<K, COEF>(a.c0, c, adet, [&](int i, int j, double v) {
    const unsigned mij = (mr >> i) | (mc >> j), mji = (mr >> j) | (mc >> i);
    if (upper) {
      const bool lo = i == j || rd[i] < rd[j];
      const int slot = lo ? rp[i] + p[i * K + j] : rp[j] + p[j * K + i];
      if (!((lo ? mij : mji) & 1u)) atomicAdd(vals + slot, v);
      return;
    }
    if (!(mij & 1u)) atomicAdd(vals + rp[i] + p[i * K + j], v);
    if (i != j && !(mji & 1u)) atomicAdd(vals + rp[j] + p[j * K + i], v);
  });
}

// vector-P2 mass rho*inner(u, v)*dx: component a of node i couples with
// component a of node j only, by the scalar P2 mass entry
template <int COEF>
__global__ void __launch_bounds__(kBlock) k_mat_vmass(const MatArgs a) {
  __shared__ __align__(16) uint8_t spos[kBlock * 100];
  const int64_t c0 = blockIdx.x * (int64_t)kBlock;
  const int64_t left = a.num_cells - c0;
  const int ncell = left < kBlock ? (int)left : kBlock;
  stage_pos<100>(spos, a.pos, c0, ncell);
  __syncthreads();
  if ((int)threadIdx.x >= ncell) return;
  const int64_t c = c0 + threadIdx.x;
  const uint8_t* p = spos + threadIdx.x * 100;
  const double adet = cell_adet(a.x, load_geom(a.geom, c));
  int rp[10], L[10], rd[10];
  unsigned mr = 0, mc = 0;
  const int32_t* d0 = a.dofs0 + c * 10;
  const int32_t* d1 = a.dofs1 + c * 10;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const int R = __ldg(d0 + i);
    const int C = __ldg(d1 + i);
    rd[i] = R;
    rp[i] = R < 0 ? 0 : __ldg(a.row_ptr + 3 * R);
    L[i] = R < 0 ? 0 : __ldg(a.row_ptr + 3 * R + 1) - rp[i];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      mr |= (R < 0 || (a.bc0 && __ldg(a.bc0 + 3 * R + q)) ? 1u : 0u) << (3 * i + q);
      mc |= (C < 0 || (a.bc1 && __ldg(a.bc1 + 3 * C + q)) ? 1u : 0u) << (3 * i + q);
    }
  }
  double* __restrict__ vals = a.values;
  const bool upper = a.upper != 0;
  mass_element<10, COEF>(a.c0, c, adet, [&](int i, int j, double v) {
#pragma unroll
    for (int ca = 0; ca < 3; ++ca) {
      const int ri = 3 * rd[i] + ca, rj = 3 * rd[j] + ca;
      const unsigned mij = (mr >> (3 * i + ca)) | (mc >> (3 * j + ca));
      const unsigned mji = (mr >> (3 * j + ca)) | (mc >> (3 * i + ca));
      if (upper) {
        const bool lo = ri <= rj;
        const int slot = lo ? rp[i] + ca * L[i] + 3 * p[i * 10 + j] + ca : rp[j] + ca * L[j] + 3 * p[j * 10 + i] + ca;
        if (!((lo ? mij : mji) & 1u)) atomicAdd(vals + slot, v);
        continue;
      }
      if (!(mij & 1u)) atomicAdd(vals + rp[i] + ca * L[i] + 3 * p[i * 10 + j] + ca, v);
      if (i != j && !(mji & 1u)) atomicAdd(vals + rp[j] + ca * L[j] + 3 * p[j * 10 + i] + ca, v);
    }
  });
}

// ---------------------------------------------------------------------------
// P3 stiffness (20 dofs, 210 unique entries), one thread per cell, FP64
// atomics.  The 400-byte map rows of a 64-cell tile are staged in shared
// memory with a one-word pad per cell (101 words apart: consecutive threads
// read different banks).
// ---------------------------------------------------------------------------
constexpr int kBlockP3 = 64;
constexpr int kP3Words = 101;  // 100 map words + 1 pad word per cell

template <typename T>
__global__ void __launch_bounds__(kBlockP3) k_mat_p3_atomic(const MatArgs a) {
  __shared__ uint32_t spw[kBlockP3 * kP3Words];
  const int64_t c0 = blockIdx.x * (int64_t)kBlockP3;
  const int64_t left = a.num_cells - c0;
  const int ncell = left < kBlockP3 ? (int)left : kBlockP3;
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(a.pos + c0 * 400);
    for (int w = threadIdx.x; w < ncell * 100; w += kBlockP3) spw[(w / 100) * kP3Words + w % 100] = __ldg(src + w);
  }
  __syncthreads();
  if ((int)threadIdx.x >= ncell) return;
  const int64_t c = c0 + threadIdx.x;
  const uint8_t* p = reinterpret_cast<const uint8_t*>(spw + threadIdx.x * kP3Words);

  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  double Gh[6];
  ghat(g, Gh);

  int rp[20], rd[20];
  unsigned mr = 0, mc = 0;
  const int32_t* d0 = a.dofs0 + c * 20;
  const int32_t* d1 = a.dofs1 + c * 20;
#pragma unroll
  for (int i = 0; i < 20; ++i) {
    // masked rows / columns: BC dofs and dofs outside a restriction (-1)
    const int r = __ldg(d0 + i), cc = __ldg(d1 + i);
    rd[i] = r;
    rp[i] = r < 0 ? 0 : __ldg(a.row_ptr + r);
    mr |= (r < 0 || (a.bc0 && __ldg(a.bc0 + r)) ? 1u : 0u) << i;
    mc |= (cc < 0 || (a.bc1 && __ldg(a.bc1 + cc)) ? 1u : 0u) << i;
  }
  double* __restrict__ vals = a.values;
  const bool upper = a.upper != 0;
  // upper mode keeps the two predicated REDs per entry (one of them active
  // in each lane): choosing the slot by a select, as the other kernels do,
  // measured slower for P3 on B200 (P3 n=48: 2.23 vs 1.79 ms)
  auto emit = [&](int i, int j, double v) {
    const bool do_ij = !upper || i == j || rd[i] < rd[j];
    const bool do_ji = i != j && (!upper || rd[j] < rd[i]);
    if (do_ij && !(((mr >> i) | (mc >> j)) & 1u)) atomicAdd(vals + rp[i] + p[i * 20 + j], v);
    if (do_ji && !(((mr >> j) | (mc >> i)) & 1u)) atomicAdd(vals + rp[j] + p[j * 20 + i], v);
  };
  const double k = coef_cell(a.c0, c);
  T gq[6];
#pragma unroll
  for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
  p3_stiffness_const<T>(gq, emit);
}

// ---------------------------------------------------------------------------
// P3 stiffness (cellwise-constant coefficient, FP64) with the reductions
// coalesced per warp ("coalesced" variant, the FP64 P3 default).  The
// 210-entry element tensor is too large to stage per cell, so each thread
// computes only its cell's geometry, g[s] = k * Ghat_s (6 doubles), row
// starts and column masks; the warp then walks its 32 cells and evaluates
// the 400 entries of each in 13 rounds, lane l of round r on entry
// e = 32r + l = 20i + j: value = sum_s g[s] * kP3GradGradSym[s*400 + e] (the
// terms of p3_stiffness_const; one term order for (i, j) and (j, i), so the
// element matrix is exactly symmetric).  Consecutive lanes take consecutive
// columns of one or two element rows, so an instruction's reductions fall in
// two CSR rows and share L2 sectors, and no transpose pass is needed.
// ---------------------------------------------------------------------------
constexpr int kP3CoalThreads = 128;

__global__ void __launch_bounds__(kP3CoalThreads) k_mat_p3_coal(const MatArgs a) {
  constexpr int NT = kP3CoalThreads;
  __shared__ double stab[2400];        // s-major: conflict-free for consecutive entries
  __shared__ double sg[NT * 6];
  __shared__ int32_t srp[NT * 20];     // row start of each local row, -1 for a masked row
  __shared__ uint32_t smc[NT];         // masked columns of each cell
  const int tid = threadIdx.x, lane = tid & 31, w0 = tid & ~31;
  for (int t = tid; t < 2400; t += NT) stab[t] = kP3GradGradSym[t];
  const int64_t c0 = blockIdx.x * (int64_t)NT;
  const int64_t left = a.num_cells - c0;
  const int ncell = left < NT ? (int)left : NT;
  const int wcells = ncell - w0 < 0 ? 0 : (ncell - w0 < 32 ? ncell - w0 : 32);
  if (tid < ncell) {
    const int64_t c = c0 + tid;
    CellGeo g;
    cell_geometry(a.x, load_geom(a.geom, c), g);
    double Gh[6];
    ghat(g, Gh);
    const double k = coef_cell(a.c0, c);
#pragma unroll
    for (int q = 0; q < 6; ++q) sg[tid * 6 + q] = k * Gh[q];
    const int32_t* d0 = a.dofs0 + c * 20;
    const int32_t* d1 = a.dofs1 + c * 20;
    uint32_t mc = 0;
#pragma unroll
    for (int i = 0; i < 20; ++i) {
      // masked rows / columns: BC dofs and dofs outside a restriction (-1)
      const int r = __ldg(d0 + i), cc = __ldg(d1 + i);
      const bool mrow = r < 0 || (a.bc0 && __ldg(a.bc0 + r));
      srp[tid * 20 + i] = mrow ? -1 : __ldg(a.row_ptr + r);
      mc |= (cc < 0 || (a.bc1 && __ldg(a.bc1 + cc)) ? 1u : 0u) << i;
    }
    smc[tid] = mc;
  }
  __syncthreads();  // the table; each warp's cells need only their warp
  // a cell's 400 slot bytes as 100 words, word w = lane + 32k in register k
  // of the lane (coalesced 128-byte loads), fetched one cell ahead; entry e
  // of round r is byte e % 4 of word e / 4 = 8r + lane / 4, held by lane
  // 8 (r % 4) + lane / 4 in register r / 4
  auto load_words = [&](int64_t c, uint32_t w[4]) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(a.pos + c * 400);  // 400 c is a multiple of 16
#pragma unroll
    for (int k = 0; k < 4; ++k) w[k] = (lane + 32 * k < 100) ? __ldg(src + lane + 32 * k) : 0u;
  };
  double* __restrict__ vals = a.values;
  // the 400 entries of the warp's local cell q from the words w
  auto cell_rounds = [&](int q, const uint32_t w[4]) {
    const double* gq = sg + q * 6;
    const double g0 = gq[0], g1 = gq[1], g2 = gq[2], g3 = gq[3], g4 = gq[4], g5 = gq[5];
    const uint32_t mc = smc[q];
    const int32_t* rq = srp + q * 20;
#pragma unroll
    for (int r = 0; r < 13; ++r) {
      const uint32_t word = __shfl_sync(0xffffffffu, w[r / 4], 8 * (r % 4) + lane / 4);
      const int e = 32 * r + lane;
      if (e >= 400) continue;
      const int i = e / 20, j = e - 20 * (e / 20);
      const int rs = rq[i];
      if (rs < 0 || ((mc >> j) & 1u)) continue;
      const double* tp = stab + e;
      const double v = fma(g2, tp[800], fma(g1, tp[400], g0 * tp[0])) +
                       fma(g5, tp[2000], fma(g4, tp[1600], g3 * tp[1200]));
      atomicAdd(vals + rs + ((word >> (8 * (lane & 3))) & 0xffu), v);
    }
  };
  // two word buffers in turn, each filled one cell ahead of its use (no
  // register copy that would wait for the load)
  uint32_t wa[4] = {0u, 0u, 0u, 0u}, wb[4] = {0u, 0u, 0u, 0u};
  const int qend = w0 + wcells;
  if (wcells > 0) load_words(c0 + w0, wa);
  for (int q = w0; q < qend; q += 2) {
    if (q + 1 < qend) load_words(c0 + q + 1, wb);
    cell_rounds(q, wa);
    if (q + 1 >= qend) break;
    if (q + 2 < qend) load_words(c0 + q + 2, wa);
    cell_rounds(q + 1, wb);
  }
}

// ---------------------------------------------------------------------------
// Vector-P2 elasticity (bs = 3), one thread per cell, FP64 atomics
// A[(i,a),(j,b)] = sum_pq W_ab[p][q] R0[p][q][i][j],
// W_ab[p][q] = |det| (mu (delta_ab (KK^T)_pq + K_pb K_qa) + lam K_pa K_qb)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void elasticity_weights(const CellGeo& g, double lam, double mu, int a, int b,
                                                   T W[9]) {
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      double kk = 0.0;
      if (a == b) kk = g.K[p][0] * g.K[q][0] + g.K[p][1] * g.K[q][1] + g.K[p][2] * g.K[q][2];
      W[p * 3 + q] = (T)(g.adet * (mu * (kk + g.K[p][b] * g.K[q][a]) + lam * g.K[p][a] * g.K[q][b]));
    }
}

template <typename T, typename EmitAB>
__device__ __forceinline__ void elasticity_blocks(const CellGeo& g, double lam, double mu, EmitAB&& emit_ab) {
#pragma unroll 1
  for (int blk = 0; blk < 6; ++blk) {
    const int a = blk < 3 ? blk : (blk == 3 ? 0 : (blk == 4 ? 0 : 1));
    const int b = blk < 3 ? blk : (blk == 3 ? 1 : 2);
    T W[9];
    elasticity_weights<T>(g, lam, mu, a, b, W);
    auto emit = [&](int i, int j, double v) { emit_ab(a, b, i, j, v); };
    if (a == b)
      p2_block_upper<T>(W, emit);
    else
      p2_block_full<T>(W, emit);
  }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_mat_vp2_atomic(const MatArgs a) {
  __shared__ __align__(16) uint8_t spos[kBlock * 100];
  const int64_t c0 = blockIdx.x * (int64_t)kBlock;
  const int64_t left = a.num_cells - c0;
  const int ncell = left < kBlock ? (int)left : kBlock;
  stage_pos<100>(spos, a.pos, c0, ncell);
  __syncthreads();
  if ((int)threadIdx.x >= ncell) return;
  const int64_t c = c0 + threadIdx.x;
  const uint8_t* p = spos + threadIdx.x * 100;

  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  const double lam = coef_cell(a.c0, c), mu = coef_cell(a.c1, c);

  int rp[10], L[10], rd[10];
  unsigned mr = 0, mc = 0;
  const int32_t* d0 = a.dofs0 + c * 10;
  const int32_t* d1 = a.dofs1 + c * 10;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    // masked rows / columns: BC dofs and nodes outside a restriction (-1)
    const int R = __ldg(d0 + i);
    const int C = __ldg(d1 + i);
    rd[i] = R;
    rp[i] = R < 0 ? 0 : __ldg(a.row_ptr + 3 * R);
    L[i] = R < 0 ? 0 : __ldg(a.row_ptr + 3 * R + 1) - rp[i];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      mr |= (R < 0 || (a.bc0 && __ldg(a.bc0 + 3 * R + q)) ? 1u : 0u) << (3 * i + q);
      mc |= (C < 0 || (a.bc1 && __ldg(a.bc1 + 3 * C + q)) ? 1u : 0u) << (3 * i + q);
    }
  }
  double* __restrict__ vals = a.values;
  const bool upper = a.upper != 0;
  elasticity_blocks<T>(g, lam, mu, [&](int ca, int cb, int i, int j, double v) {
    // scalar rows 3*rd[i]+ca and 3*rd[j]+cb; upper mode keeps the entry in the
    // upper triangle (the diagonal entry when they coincide)
    const int ri = 3 * rd[i] + ca, rj = 3 * rd[j] + cb;
    const unsigned mij = (mr >> (3 * i + ca)) | (mc >> (3 * j + cb));
    const unsigned mji = (mr >> (3 * j + cb)) | (mc >> (3 * i + ca));
    if (upper) {
      // one RED per unique entry, target chosen by a select (no divergence)
      const bool lo = ri <= rj;
      const int slot = lo ? rp[i] + ca * L[i] + 3 * p[i * 10 + j] + cb : rp[j] + cb * L[j] + 3 * p[j * 10 + i] + ca;
      if (!((lo ? mij : mji) & 1u)) atomicAdd(vals + slot, v);
      return;
    }
    if (!(mij & 1u)) atomicAdd(vals + rp[i] + ca * L[i] + 3 * p[i * 10 + j] + cb, v);
    if (!(ca == cb && i == j) && !(mji & 1u)) atomicAdd(vals + rp[j] + cb * L[j] + 3 * p[j * 10 + i] + ca, v);
  });
}

// ---------------------------------------------------------------------------
// Vector-P2 elasticity with the reductions coalesced per warp (the vector-P2
// default).  Entry (row (i,a), column (j,b)) of the 30x30 element matrix is
// sum_pq C_ij^pq W^ab_pq with C_ij^pq = int_ref d_p phi_i d_q phi_j (the
// table kP2GradGrad) and W^ab the 9 geometric weights of component block
// (a, b) (elasticity_weights).  One thread per cell computes the 6 weight
// blocks a <= b into shared memory; the warp then walks its 32 cells: one
// instruction per element row (i, a), lane 3j + b on column (j, b), so the
// 30 reductions land on the 10 consecutive slot triples of one CSR row
// (~2 per 32-byte sector, against 1 for the thread-per-cell scatter) and no
// transpose pass is needed.  Every entry is evaluated from its
// upper-triangle form (the pair's smaller (node, component) as the row), in
// one term order, so the element matrix is exactly symmetric.  With FP32
// weights the diagonal entries of each 3x3 node block are, as in the
// thread-per-cell kernel, minus the FP64 sum of the block row's FP32
// off-diagonal entries (exact row sums: rigid translations stay in the null
// space); by symmetry each lane accumulates that sum as its column sum.
// ---------------------------------------------------------------------------
constexpr int kVCoalThreads = 64;

template <typename T>
__global__ void __launch_bounds__(kVCoalThreads) k_mat_vp2_coal(const MatArgs a) {
  constexpr int NT = kVCoalThreads;
  constexpr bool kRowSums = sizeof(T) == 4;
  __shared__ T sC[900];
  __shared__ T sW[NT * 54];                         // per cell: blocks (00,11,22,01,02,12) x 9
  __shared__ __align__(16) uint8_t spos[NT * 100];
  __shared__ int32_t srp[NT * 10];                  // scalar row 3R of local node i (component 0)
  __shared__ int32_t sL[NT * 10];                   // its length (the rows 3R+1, 3R+2 follow)
  __shared__ uint32_t smr[NT], smc[NT];             // masked rows / columns, bit 3i + component
  const int tid = threadIdx.x, lane = tid & 31, w0 = tid & ~31;
  for (int t = tid; t < 900; t += NT) sC[t] = (T)kP2GradGrad[t];
  const int64_t c0 = blockIdx.x * (int64_t)NT;
  const int64_t left = a.num_cells - c0;
  const int ncell = left < NT ? (int)left : NT;
  const int wcells = ncell - w0 < 0 ? 0 : (ncell - w0 < 32 ? ncell - w0 : 32);
  {
    // each warp stages its own cells' byte maps ((c0 + w0) * 100 is a multiple of 16)
    const uint4* src = reinterpret_cast<const uint4*>(a.pos + (c0 + w0) * 100);
    uint4* dst = reinterpret_cast<uint4*>(spos + w0 * 100);
    const int nvec = (wcells * 100 + 15) / 16;
    for (int t = lane; t < nvec; t += 32) dst[t] = __ldg(src + t);
  }
  if (tid < ncell) {
    const int64_t c = c0 + tid;
    CellGeo g;
    cell_geometry(a.x, load_geom(a.geom, c), g);
    const double lam = coef_cell(a.c0, c), mu = coef_cell(a.c1, c);
#pragma unroll 1
    for (int blk = 0; blk < 6; ++blk) {  // rolled: unrolled it takes 144 registers (FP32) instead of 108
      const int ca = blk < 3 ? blk : (blk == 5 ? 1 : 0);
      const int cb = blk < 3 ? blk : (blk == 3 ? 1 : 2);
      elasticity_weights<T>(g, lam, mu, ca, cb, sW + tid * 54 + blk * 9);
    }
    const int32_t* d0 = a.dofs0 + c * 10;
    const int32_t* d1 = a.dofs1 + c * 10;
    uint32_t mr = 0, mc = 0;
#pragma unroll
    for (int i = 0; i < 10; ++i) {
      // masked rows / columns: BC dofs and nodes outside a restriction (-1)
      const int R = __ldg(d0 + i), C = __ldg(d1 + i);
      const int32_t r0 = R < 0 ? 0 : __ldg(a.row_ptr + 3 * R);
      srp[tid * 10 + i] = r0;
      sL[tid * 10 + i] = R < 0 ? 0 : __ldg(a.row_ptr + 3 * R + 1) - r0;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        mr |= (R < 0 || (a.bc0 && __ldg(a.bc0 + 3 * R + q)) ? 1u : 0u) << (3 * i + q);
        mc |= (C < 0 || (a.bc1 && __ldg(a.bc1 + 3 * C + q)) ? 1u : 0u) << (3 * i + q);
      }
    }
    smr[tid] = mr;
    smc[tid] = mc;
  }
  __syncthreads();  // the C table; the warp's own cells need only their warp
  // lanes 30 and 31 run along (the shuffles below take the whole warp) on
  // column (0, 0) without reducing
  const bool lane_on = lane < 30;
  const int j = lane_on ? lane / 3 : 0, b = lane_on ? lane - 3 * (lane / 3) : 0;
  // stored block of components (u, v), u <= v
  auto blk_of = [](int u, int v) { return u == v ? u : (u + v == 1 ? 3 : (u + v == 2 ? 4 : 5)); };
  double* __restrict__ vals = a.values;
  for (int q = w0; q < w0 + wcells; ++q) {
    // W^{ab} and W^{ba} of this lane's column component b, for a = 0..2
    const T* Wc = sW + q * 54;
    T Wab[3][9], Wba[3][9];
#pragma unroll
    for (int ca = 0; ca < 3; ++ca) {
      const int lo = ca < b ? ca : b, hi = ca < b ? b : ca;
      const T* Wb = Wc + 9 * blk_of(lo, hi);
#pragma unroll
      for (int pq = 0; pq < 9; ++pq) {
        const int tq = (pq % 3) * 3 + pq / 3;  // transposed index
        Wab[ca][pq] = ca <= b ? Wb[pq] : Wb[tq];
        Wba[ca][pq] = b <= ca ? Wb[pq] : Wb[tq];
      }
    }
    const uint32_t mr = smr[q], mc = smc[q];
    const bool cmask = !lane_on || ((mc >> (3 * j + b)) & 1u);
    const int32_t* rq = srp + q * 10;
    const int32_t* lq = sL + q * 10;
    const uint8_t* pq8 = spos + q * 100;
    double cs[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
    for (int i = 0; i < 10; ++i) {
      const int rs = rq[i], len = lq[i];
      const int slot0 = rs + 3 * pq8[i * 10 + j] + b;
      // the pair's upper form takes row (i, ca) when (i, ca) <= (j, b), else
      // row (j, b): its C row is C_ij for i < j and C_ji for i > j (the same
      // row for i == j), whatever the components
      const T* Cp = sC + (i <= j ? i * 10 + j : j * 10 + i) * 9;
      T cr[9];
#pragma unroll
      for (int pq = 0; pq < 9; ++pq) cr[pq] = Cp[pq];
#pragma unroll
      for (int ca = 0; ca < 3; ++ca) {
        const bool up = i < j || (i == j && ca <= b);
        // two partial sums (a fixed order, so both lanes of a symmetric pair
        // compute the same value)
        T v0 = T(0), v1 = T(0);
#pragma unroll
        for (int pq = 0; pq < 9; pq += 2) v0 = fma(cr[pq], up ? Wab[ca][pq] : Wba[ca][pq], v0);
#pragma unroll
        for (int pq = 1; pq < 9; pq += 2) v1 = fma(cr[pq], up ? Wab[ca][pq] : Wba[ca][pq], v1);
        const T v = v0 + v1;
        if (kRowSums && i == j) continue;  // node-block diagonals come from the row sums
        if (kRowSums) cs[ca] += (double)v;
        if (!cmask && !((mr >> (3 * i + ca)) & 1u)) atomicAdd(vals + slot0 + ca * len, (double)v);
      }
    }
    if constexpr (kRowSums) {
      // cs[ca] = column sum of block (ca, b) at column j = row sum of block
      // (b, ca) at row j (the element is exactly symmetric).  Entry (row
      // (j, b), column (j, ca)) = -1/2 (row sum + column sum of block (b, ca)),
      // the column sum being lane (j, ca)'s cs[b]: the node block stays
      // symmetric and its rows sum to zero up to the FP32 rounding of one term
      const int rs = rq[j], len = lq[j];
      const int slot = rs + b * len + 3 * pq8[j * 10 + j];
#pragma unroll
      for (int ca = 0; ca < 3; ++ca) {
        const int src = 3 * j + ca;
        const double o0 = __shfl_sync(0xffffffffu, cs[0], src), o1 = __shfl_sync(0xffffffffu, cs[1], src),
                     o2 = __shfl_sync(0xffffffffu, cs[2], src);
        const double other = b == 0 ? o0 : (b == 1 ? o1 : o2);
        if (lane_on && !((mr >> (3 * j + b)) & 1u) && !((mc >> (3 * j + ca)) & 1u))
          atomicAdd(vals + slot + ca, -0.5 * (cs[ca] + other));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Utilities
// ---------------------------------------------------------------------------
__global__ void k_zero(double* __restrict__ v, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if ((reinterpret_cast<uintptr_t>(v) & 15) == 0) {
    double2* v2 = reinterpret_cast<double2*>(v);
    const int64_t n2 = n / 2;
    for (int64_t t = i; t < n2; t += stride) v2[t] = make_double2(0.0, 0.0);
    if (i == 0 && (n & 1)) v[n - 1] = 0.0;
  } else {
    for (int64_t t = i; t < n; t += stride) v[t] = 0.0;
  }
}

// The zero pass and set_diagonal in one launch, for kernels that never
// reduce into a BC row (the element scatters skip them): block b owns the
// slots [b*chunk, (b+1)*chunk), zeroes them, then stores `value` on the
// diagonal slots of the owned BC rows that fall in its range -- dslot (sorted
// ascending) from bstart[b] to bstart[b+1], both precomputed per pattern and
// BC -- so the same block writes both and no ordering across blocks is needed.
__global__ void __launch_bounds__(256) k_zero_diag(double* __restrict__ v, int64_t n, int64_t chunk,
                                                   const int32_t* __restrict__ dslot,
                                                   const int32_t* __restrict__ bstart, double value) {
  const int64_t lo = blockIdx.x * chunk;
  const int64_t hi = lo + chunk < n ? lo + chunk : n;
  if (lo >= hi) return;
  // chunk is even and v is 16-byte aligned: double2 stores over [lo, hi)
  double2* v2 = reinterpret_cast<double2*>(v + lo);
  const int64_t n2 = (hi - lo) / 2;
  for (int64_t t = threadIdx.x; t < n2; t += blockDim.x) v2[t] = make_double2(0.0, 0.0);
  if (threadIdx.x == 0 && ((hi - lo) & 1)) v[hi - 1] = 0.0;
  if (!dslot) return;
  const int32_t k0 = __ldg(bstart + blockIdx.x), k1 = __ldg(bstart + blockIdx.x + 1);
  if (k0 == k1) return;
  __syncthreads();  // the zeros of this range before its diagonal values
  for (int32_t k = k0 + threadIdx.x; k < k1; k += blockDim.x) v[__ldg(dslot + k)] = value;
}

// set_diagonal (CUDAAssembler.cpp:131-164) with the diagonal slot precomputed
__global__ void k_set_diagonal(const int32_t* __restrict__ dofs, int64_t n_owned,
                               const int32_t* __restrict__ diag, int64_t num_rows, double value,
                               double* __restrict__ values) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n_owned) return;
  const int32_t r = dofs[t];
  if (r < 0 || r >= num_rows) return;
  const int32_t s = diag[r];
  if (s >= 0) values[s] = value;
}

// Strictly-lower slot counts per row (diag[r] - row_ptr[r]); -1 when a row
// has no diagonal entry.
__global__ void k_lower_count(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ diag,
                              int64_t num_rows, int32_t* __restrict__ cnt) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= num_rows) return;
  const int32_t d = diag[r];
  cnt[r] = d < 0 ? -1 : d - row_ptr[r];
}

// One pair per strictly-lower slot (r, c), c < r: {the slot, the slot of
// (c, r)}, the latter by binary search in row c; a missing transpose entry
// sets *bad.
__global__ void k_lower_pairs(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                              const int32_t* __restrict__ lower_ptr, int64_t num_rows, int2* __restrict__ pairs,
                              int* __restrict__ bad) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= num_rows) return;
  const int32_t lo = row_ptr[r], n = lower_ptr[r + 1] - lower_ptr[r], base = lower_ptr[r];
  for (int32_t t = 0; t < n; ++t) {
    const int32_t c = col[lo + t];
    int32_t a = row_ptr[c], b = row_ptr[c + 1] - 1, hit = -1;
    while (a <= b) {
      const int32_t m = (a + b) >> 1;
      const int32_t v = col[m];
      if (v == (int32_t)r) {
        hit = m;
        break;
      }
      if (v < (int32_t)r) a = m + 1;
      else b = m - 1;
    }
    if (hit < 0) atomicOr(bad, 1);
    pairs[base + t] = make_int2(lo + t, hit < 0 ? lo + t : hit);
  }
}

// values[pair.x] = values[pair.y] for every strictly-lower slot.  Pairs and
// stores are coalesced; the mirror reads are the only scattered accesses and
// the kernel is bound by their latency, so each thread takes kMirrorUnroll
// pairs 32 apart (every load and store instruction of a warp still covers
// consecutive pairs) and issues all of its gathers before its stores.
constexpr int kMirrorUnroll = 4;

__global__ void __launch_bounds__(256) k_mirror_pairs(const int2* __restrict__ pairs, int64_t n,
                                                      double* __restrict__ values) {
  constexpr int U = kMirrorUnroll;
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = warp * 32 * U; base < n; base += nwarps * 32 * U) {
    int2 p[U];
    double v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t k = base + u * 32 + lane;
      p[u] = k < n ? __ldg(pairs + k) : make_int2(-1, -1);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) v[u] = p[u].x >= 0 ? values[p[u].y] : 0.0;
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (p[u].x >= 0) values[p[u].x] = v[u];
  }
}

// Block size 3: per block row I, the number of node blocks on or below the
// diagonal (block position of column 3I in row 3I, plus one); -1 if the three
// rows of the block row differ in length or the diagonal is missing.
__global__ void k_lower_count3(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ diag,
                               int64_t num_block_rows, int32_t* __restrict__ cnt) {
  const int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (I >= num_block_rows) return;
  const int64_t r = 3 * I;
  const int32_t lo = row_ptr[r], len = row_ptr[r + 1] - lo;
  const int32_t d = diag[r];
  const bool same = row_ptr[r + 2] - row_ptr[r + 1] == len && row_ptr[r + 3] - row_ptr[r + 2] == len;
  cnt[I] = (d < 0 || !same || len % 3 || (d - lo) % 3) ? -1 : (d - lo) / 3 + 1;
}

// One record per node block (I, J), J <= I: {slot of (3I, 3J), row length of
// 3I, slot of (3J, 3I), row length of 3J}; the transposed block is found by a
// binary search in row 3J, a missing one sets *bad.
__global__ void k_lower_blocks3(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                                const int32_t* __restrict__ lower_ptr, int64_t num_block_rows,
                                int4* __restrict__ blocks, int* __restrict__ bad) {
  const int64_t I = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (I >= num_block_rows) return;
  const int64_t r = 3 * I;
  const int32_t lo = row_ptr[r], len = row_ptr[r + 1] - lo;
  const int32_t base = lower_ptr[I], n = lower_ptr[I + 1] - base;
  for (int32_t t = 0; t < n; ++t) {
    const int32_t l0 = lo + 3 * t;
    const int32_t c = col[l0];
    // the block's three columns are c, c+1, c+2 (l0 + 2 is inside the row: t
    // is at most the diagonal block's position and the row length is a
    // multiple of 3)
    if (c % 3 || col[l0 + 1] != c + 1 || col[l0 + 2] != c + 2) {
      atomicOr(bad, 1);
      blocks[base + t] = make_int4(l0, len, l0, len);
      continue;
    }
    if (t == n - 1) {  // the diagonal block
      blocks[base + t] = make_int4(l0, len, l0, len);
      continue;
    }
    const int64_t rj = c;  // row 3J
    int32_t a = row_ptr[rj], b = row_ptr[rj + 1] - 1, hit = -1;
    while (a <= b) {
      const int32_t m = (a + b) >> 1;
      const int32_t v = col[m];
      if (v == (int32_t)r) {
        hit = m;
        break;
      }
      if (v < (int32_t)r) a = m + 1;
      else b = m - 1;
    }
    const int32_t lenj = row_ptr[rj + 1] - row_ptr[rj];
    if (hit < 0 || hit + 2 >= row_ptr[rj + 1] || col[hit + 1] != (int32_t)r + 1 || col[hit + 2] != (int32_t)r + 2) {
      atomicOr(bad, 1);
      blocks[base + t] = make_int4(l0, len, l0, len);  // harmless diagonal-style record
      continue;
    }
    blocks[base + t] = make_int4(l0, len, hit, lenj);
  }
}

// Strictly-lower part from the upper part, node block by node block (block
// size 3): the 9 entries of a block below the diagonal are 3 rows of 3
// contiguous slots, read from the transposed block's 3 rows of 3 contiguous
// slots; a diagonal block copies its 3 entries below the diagonal.  One
// 16-byte record per block replaces nine 8-byte slot pairs.
__global__ void __launch_bounds__(256) k_mirror_blocks3(const int4* __restrict__ blocks, int64_t n,
                                                        double* __restrict__ values) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += stride) {
    const int4 b = __ldg(blocks + k);
    if (b.z == b.x) {
      const double v10 = values[b.x + 1], v20 = values[b.x + 2], v21 = values[b.x + b.y + 2];
      values[b.x + b.y] = v10;
      values[b.x + 2 * b.y] = v20;
      values[b.x + 2 * b.y + 1] = v21;
      continue;
    }
    double v[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 3; ++a) v[c][a] = values[b.z + c * b.w + a];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) values[b.x + a * b.y + c] = v[c][a];
  }
}

// Cell-to-slot map: block position of dofs1[c,j] inside block row dofs0[c,i].
__global__ void k_build_slotmap(const int32_t* __restrict__ dofs0, const int32_t* __restrict__ dofs1,
                                int64_t num_cells, int k0, int k1, int bs0, int bs1,
                                const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                                int64_t num_rows, uint8_t* __restrict__ pos, unsigned* err) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= num_cells * k0) return;
  const int64_t c = t / k0;
  const int i = (int)(t % k0);
  const int64_t R = dofs0[c * k0 + i];
  const int64_t r = R * bs0;
  if (R < 0 || r + bs0 > num_rows) {
    raise_err(err, DEV_ERR_INDEX);
    return;
  }
  const int32_t lo = row_ptr[r], hi = row_ptr[r + 1];
  for (int j = 0; j < k1; ++j) {
    const int32_t key = dofs1[c * k1 + j] * bs1;
    int32_t a = lo, b = hi;
    while (a < b) {
      const int32_t m = (a + b) >> 1;
      if (col[m] < key) a = m + 1;
      else b = m;
    }
    uint8_t out = 0;
    if (a >= hi || col[a] != key) {
      raise_err(err, DEV_ERR_PATTERN);
    } else {
      const int32_t off = a - lo;
      if (off % bs1) raise_err(err, DEV_ERR_BLOCK);
      const int32_t pb = off / bs1;
      if (pb > 255) raise_err(err, DEV_ERR_ROW_WIDE);
      else out = (uint8_t)pb;
      for (int q = 1; q < bs1; ++q)
        if (a + q >= hi || col[a + q] != key + q) raise_err(err, DEV_ERR_BLOCK);
      for (int q = 1; q < bs0; ++q) {
        const int32_t lq = row_ptr[r + q];
        if (row_ptr[r + q + 1] - lq != hi - lo || col[lq + off] != key) raise_err(err, DEV_ERR_BLOCK);
      }
    }
    pos[t * k1 + j] = out;
  }
}

// Block view of a monolithic pattern: for local scalar row rl of a block form
// placed at (row_offset, col_offset), the first slot of monolithic row
// row_offset + rl whose column is >= col_offset (the block's column segment),
// and that row's diagonal slot.
__global__ void k_view_rows(const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                            const int32_t* __restrict__ diag, int64_t row_offset, int64_t col_offset,
                            int64_t num_local_rows, int32_t* __restrict__ seg, int32_t* __restrict__ vdiag) {
  const int64_t rl = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (rl >= num_local_rows) return;
  const int64_t r = row_offset + rl;
  int32_t a = row_ptr[r], b = row_ptr[r + 1];
  while (a < b) {
    const int32_t m = (a + b) >> 1;
    if (col[m] < col_offset) a = m + 1;
    else b = m;
  }
  seg[rl] = a;
  vdiag[rl] = diag[r];
}

// Cell-to-slot map of a block form through its view: block position of
// dofs1[c,j] inside the column segment of block row dofs0[c,i]; entries of
// excluded dofs (-1) are 0 and never used.
__global__ void k_build_slotmap_view(const int32_t* __restrict__ dofs0, const int32_t* __restrict__ dofs1,
                                     int64_t num_cells, int k0, int k1, int bs0, int bs1,
                                     const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
                                     const int32_t* __restrict__ seg, int64_t row_offset, int64_t col_offset,
                                     uint8_t* __restrict__ pos, unsigned* err) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= num_cells * k0) return;
  const int64_t c = t / k0;
  const int64_t R = dofs0[t];
  if (R < 0) {
    for (int j = 0; j < k1; ++j) pos[t * k1 + j] = 0;
    return;
  }
  const int64_t rl = R * bs0;
  const int32_t lo = seg[rl], hi = row_ptr[row_offset + rl + 1];
  const int32_t L = bs0 > 1 ? seg[rl + 1] - lo : 0;
  for (int j = 0; j < k1; ++j) {
    const int64_t C = dofs1[c * k1 + j];
    uint8_t out = 0;
    if (C >= 0) {
      const int64_t key = col_offset + C * bs1;
      int32_t a = lo, b = hi;
      while (a < b) {
        const int32_t m = (a + b) >> 1;
        if (col[m] < key) a = m + 1;
        else b = m;
      }
      if (a >= hi || col[a] != key) {
        raise_err(err, DEV_ERR_PATTERN);
      } else {
        const int32_t off = a - lo;
        if (off % bs1) raise_err(err, DEV_ERR_BLOCK);
        const int32_t pb = off / bs1;
        if (pb > 255) raise_err(err, DEV_ERR_ROW_WIDE);
        else out = (uint8_t)pb;
        for (int q = 1; q < bs1; ++q)
          if (a + q >= hi || col[a + q] != key + q) raise_err(err, DEV_ERR_BLOCK);
        // the component rows of a block row: equal lengths, same segment layout
        for (int q = 1; q < bs0; ++q) {
          const int32_t sq = seg[rl + q], eq = row_ptr[row_offset + rl + q + 1];
          if (sq - lo != q * L || sq + off >= eq || col[sq + off] != key) raise_err(err, DEV_ERR_BLOCK);
        }
      }
    }
    pos[t * k1 + j] = out;
  }
}

// ---------------------------------------------------------------------------
// Vector assembly (element vector -> atomicAdd), CUDAFormIntegral.cpp:270-357
// ---------------------------------------------------------------------------
struct VecArgs {
  int64_t num_cells;
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  const int32_t* __restrict__ dofs;
  CoefDev f;
  double* __restrict__ b;
  int64_t num_values;
  const uint8_t* __restrict__ skip;  // rows set_bc overwrites in the same launch (fused RHS), else null
};

__device__ __forceinline__ void add_guarded(double* b, int64_t row, int64_t n, double v) {
  if (row >= 0 && row < n) atomicAdd(b + row, v);
}

// The vector and lifting scatters: rows marked in `skip` are left to the
// set_bc part of the fused right-hand-side kernel, which stores them.
__device__ __forceinline__ void add_guarded(double* b, int64_t row, int64_t n, const uint8_t* skip, double v) {
  if (row >= 0 && row < n && !(skip && __ldg(skip + row))) atomicAdd(b + row, v);
}

__device__ __forceinline__ void vec_p1(const VecArgs& a, const int64_t c) {
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  const int4 d = __ldg(reinterpret_cast<const int4*>(a.dofs) + c);
  const int r[4] = {d.x, d.y, d.z, d.w};
  double f[4];
  if (a.f.kind == FE_COEFF_P1) {
    const int4 m = __ldg(reinterpret_cast<const int4*>(a.f.map) + c);
    f[0] = __ldg(a.f.v + m.x);
    f[1] = __ldg(a.f.v + m.y);
    f[2] = __ldg(a.f.v + m.z);
    f[3] = __ldg(a.f.v + m.w);
  } else {
    const double fc = coef_cell(a.f, c);
    f[0] = f[1] = f[2] = f[3] = fc;
  }
  const double s = f[0] + f[1] + f[2] + f[3];
  const double w = g.adet * (1.0 / 120.0);
#pragma unroll
  for (int i = 0; i < 4; ++i) add_guarded(a.b, r[i], a.num_values, a.skip, w * (f[i] + s));
}

__global__ void __launch_bounds__(kBlock) k_vec_p1(const VecArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (c < a.num_cells) vec_p1(a, c);
}

__device__ __forceinline__ void vec_p2(const VecArgs& a, const int64_t c) {
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  const double s = coef_cell(a.f, c) * g.adet;
  const int32_t* d = a.dofs + c * 10;
#pragma unroll
  for (int i = 0; i < 10; ++i) add_guarded(a.b, __ldg(d + i), a.num_values, a.skip, s * p2_basis_integral(i));
}

__global__ void __launch_bounds__(kBlock) k_vec_p2(const VecArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (c < a.num_cells) vec_p2(a, c);
}

// P3 load with a DG0 / constant f: |det J| f int_ref phi_i.  The edge basis
// functions of the equispaced cubic element integrate to exactly zero, so only
// the vertex and face rows receive a contribution.
__device__ __forceinline__ void vec_p3(const VecArgs& a, const int64_t c) {
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  const double s = coef_cell(a.f, c) * g.adet;
  const int32_t* d = a.dofs + c * 20;
#pragma unroll
  for (int i = 0; i < 20; ++i)
    if (i < 4 || i >= 16) add_guarded(a.b, __ldg(d + i), a.num_values, a.skip, s * p3_basis_integral(i));
}

__global__ void __launch_bounds__(kBlock) k_vec_p3(const VecArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (c < a.num_cells) vec_p3(a, c);
}

__device__ __forceinline__ void vec_vp2(const VecArgs& a, const int64_t c) {
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  double f[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) f[q] = (a.f.kind == FE_COEFF_DG0 ? __ldg(a.f.v + 3 * c + q) : a.f.c[q]) * g.adet;
  const int32_t* d = a.dofs + c * 10;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const int64_t R = __ldg(d + i);
    const double w = p2_basis_integral(i);
#pragma unroll
    for (int q = 0; q < 3; ++q) add_guarded(a.b, 3 * R + q, a.num_values, a.skip, f[q] * w);
  }
}

__global__ void __launch_bounds__(kBlock) k_vec_vp2(const VecArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (c < a.num_cells) vec_vp2(a, c);
}

// ---------------------------------------------------------------------------
// Lifting: for cells with a marked trial dof, be = -scale * Ae[:, bc] (g - x0)
// (CUDAFormIntegral.cpp:603-717; rows are not masked, as in the reference)
// ---------------------------------------------------------------------------
struct LiftArgs {
  const int32_t* __restrict__ cells;
  int64_t num_list;
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  const int32_t* __restrict__ dofs0;
  const int32_t* __restrict__ dofs1;
  CoefDev c0, c1;
  const uint8_t* __restrict__ bc1;
  const double* __restrict__ g;
  const double* __restrict__ x0;
  double scale;
  double* __restrict__ b;
  int64_t num_values;
  const uint8_t* __restrict__ skip;  // as VecArgs::skip
};

__device__ __forceinline__ void lift_p1(const LiftArgs& a, const int64_t t) {
  const int64_t c = a.cells[t];
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  double G[4][3];
  p1_grads(g, G);
  const double s = g.adet * (1.0 / 6.0) * coef_mean(a.c0, c);
  const int4 d0 = __ldg(reinterpret_cast<const int4*>(a.dofs0) + c);
  const int4 d1 = __ldg(reinterpret_cast<const int4*>(a.dofs1) + c);
  const int r[4] = {d0.x, d0.y, d0.z, d0.w};
  const int cl[4] = {d1.x, d1.y, d1.z, d1.w};
  double dv[4];
#pragma unroll
  for (int j = 0; j < 4; ++j)
    dv[j] = cl[j] >= 0 && __ldg(a.bc1 + cl[j]) ? (__ldg(a.g + cl[j]) - (a.x0 ? __ldg(a.x0 + cl[j]) : 0.0)) : 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    double acc = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) acc += s * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]) * dv[j];
    add_guarded(a.b, r[i], a.num_values, a.skip, -a.scale * acc);
  }
}

__global__ void __launch_bounds__(kBlock) k_lift_p1(const LiftArgs a) {
  const int64_t t = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (t < a.num_list) lift_p1(a, t);
}

template <int COEF, typename T>
__device__ __forceinline__ void lift_p2(const LiftArgs& a, const int64_t t) {
  const int64_t c = a.cells[t];
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  double Gh[6];
  ghat(g, Gh);
  double dv[10], be[10];
  const int32_t* d0 = a.dofs0 + c * 10;
  const int32_t* d1 = a.dofs1 + c * 10;
#pragma unroll
  for (int j = 0; j < 10; ++j) {
    const int C = __ldg(d1 + j);
    dv[j] = C >= 0 && __ldg(a.bc1 + C) ? (__ldg(a.g + C) - (a.x0 ? __ldg(a.x0 + C) : 0.0)) : 0.0;
    be[j] = 0.0;
  }
  auto emit = [&](int i, int j, double v) {
    be[i] += v * dv[j];
    if (i != j) be[j] += v * dv[i];
  };
  if constexpr (COEF == FE_COEFF_P1) {
    const int4 km = __ldg(reinterpret_cast<const int4*>(a.c0.map) + c);
    const double k[4] = {__ldg(a.c0.v + km.x), __ldg(a.c0.v + km.y), __ldg(a.c0.v + km.z),
                         __ldg(a.c0.v + km.w)};
    T q[24];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int s = 0; s < 6; ++s) q[m * 6 + s] = (T)(k[m] * Gh[s]);
    p2_stiffness_p1coef<T>(q, emit);
  } else {
    const double k = coef_cell(a.c0, c);
    T gq[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
    p2_stiffness_const<T>(gq, emit);
  }
#pragma unroll
  for (int i = 0; i < 10; ++i) add_guarded(a.b, __ldg(d0 + i), a.num_values, a.skip, -a.scale * be[i]);
}

template <int COEF, typename T>
__global__ void __launch_bounds__(kBlock) k_lift_p2(const LiftArgs a) {
  const int64_t t = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (t < a.num_list) lift_p2<COEF, T>(a, t);
}

template <typename T>
__device__ __forceinline__ void lift_p3(const LiftArgs& a, const int64_t t) {
  const int64_t c = a.cells[t];
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  double Gh[6];
  ghat(g, Gh);
  double dv[20], be[20];
  const int32_t* d0 = a.dofs0 + c * 20;
  const int32_t* d1 = a.dofs1 + c * 20;
#pragma unroll
  for (int j = 0; j < 20; ++j) {
    const int C = __ldg(d1 + j);
    dv[j] = C >= 0 && __ldg(a.bc1 + C) ? (__ldg(a.g + C) - (a.x0 ? __ldg(a.x0 + C) : 0.0)) : 0.0;
    be[j] = 0.0;
  }
  const double k = coef_cell(a.c0, c);
  T gq[6];
#pragma unroll
  for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
  p3_stiffness_const<T>(gq, [&](int i, int j, double v) {
    be[i] += v * dv[j];
    if (i != j) be[j] += v * dv[i];
  });
#pragma unroll
  for (int i = 0; i < 20; ++i) add_guarded(a.b, __ldg(d0 + i), a.num_values, a.skip, -a.scale * be[i]);
}

template <typename T>
__global__ void __launch_bounds__(kBlockP3) k_lift_p3(const LiftArgs a) {
  const int64_t t = blockIdx.x * (int64_t)kBlockP3 + threadIdx.x;
  if (t < a.num_list) lift_p3<T>(a, t);
}

template <int K, int COEF>
__device__ __forceinline__ void lift_mass(const LiftArgs& a, const int64_t t) {
  const int64_t c = a.cells[t];
  const double adet = cell_adet(a.x, load_geom(a.geom, c));
  double dv[K], be[K];
  const int32_t* d0 = a.dofs0 + c * K;
  const int32_t* d1 = a.dofs1 + c * K;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    const int C = __ldg(d1 + j);
    dv[j] = C >= 0 && __ldg(a.bc1 + C) ? (__ldg(a.g + C) - (a.x0 ? __ldg(a.x0 + C) : 0.0)) : 0.0;
    be[j] = 0.0;
  }
  mass_element<K, COEF>(a.c0, c, adet, [&](int i, int j, double v) {
    be[i] += v * dv[j];
    if (i != j) be[j] += v * dv[i];
  });
#pragma unroll
  for (int i = 0; i < K; ++i) add_guarded(a.b, __ldg(d0 + i), a.num_values, a.skip, -a.scale * be[i]);
}

template <int K, int COEF>
__global__ void __launch_bounds__(kBlock) k_lift_mass(const LiftArgs a) {
  const int64_t t = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (t < a.num_list) lift_mass<K, COEF>(a, t);
}

template <int COEF>
__device__ __forceinline__ void lift_vmass(const LiftArgs& a, const int64_t t) {
  const int64_t c = a.cells[t];
  const double adet = cell_adet(a.x, load_geom(a.geom, c));
  double dv[30], be[30];
  const int32_t* d0 = a.dofs0 + c * 10;
  const int32_t* d1 = a.dofs1 + c * 10;
#pragma unroll
  for (int j = 0; j < 10; ++j) {
    const int64_t C = __ldg(d1 + j);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int64_t s = 3 * C + q;
      dv[3 * j + q] = C >= 0 && __ldg(a.bc1 + s) ? (__ldg(a.g + s) - (a.x0 ? __ldg(a.x0 + s) : 0.0)) : 0.0;
      be[3 * j + q] = 0.0;
    }
  }
  mass_element<10, COEF>(a.c0, c, adet, [&](int i, int j, double v) {
#pragma unroll
    for (int ca = 0; ca < 3; ++ca) {
      be[3 * i + ca] += v * dv[3 * j + ca];
      if (i != j) be[3 * j + ca] += v * dv[3 * i + ca];
    }
  });
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const int64_t R = __ldg(d0 + i);
#pragma unroll
    for (int q = 0; q < 3; ++q) add_guarded(a.b, 3 * R + q, a.num_values, a.skip, -a.scale * be[3 * i + q]);
  }
}

template <int COEF>
__global__ void __launch_bounds__(kBlock) k_lift_vmass(const LiftArgs a) {
  const int64_t t = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (t < a.num_list) lift_vmass<COEF>(a, t);
}

template <typename T>
__device__ __forceinline__ void lift_vp2(const LiftArgs& a, const int64_t t) {
  const int64_t c = a.cells[t];
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  const double lam = coef_cell(a.c0, c), mu = coef_cell(a.c1, c);
  double dv[30], be[30];
  const int32_t* d0 = a.dofs0 + c * 10;
  const int32_t* d1 = a.dofs1 + c * 10;
#pragma unroll
  for (int j = 0; j < 10; ++j) {
    const int64_t C = __ldg(d1 + j);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int64_t s = 3 * C + q;
      dv[3 * j + q] = C >= 0 && __ldg(a.bc1 + s) ? (__ldg(a.g + s) - (a.x0 ? __ldg(a.x0 + s) : 0.0)) : 0.0;
      be[3 * j + q] = 0.0;
    }
  }
  elasticity_blocks<T>(g, lam, mu, [&](int ca, int cb, int i, int j, double v) {
    be[3 * i + ca] += v * dv[3 * j + cb];
    if (!(ca == cb && i == j)) be[3 * j + cb] += v * dv[3 * i + ca];
  });
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const int64_t R = __ldg(d0 + i);
#pragma unroll
    for (int q = 0; q < 3; ++q) add_guarded(a.b, 3 * R + q, a.num_values, a.skip, -a.scale * be[3 * i + q]);
  }
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_lift_vp2(const LiftArgs a) {
  const int64_t t = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (t < a.num_list) lift_vp2<T>(a, t);
}

// ---------------------------------------------------------------------------
// Diagonal of a bilinear form as a vector (the "part": "diagonal" forms FFCx
// generates, python/test/test_cuda_assembly.py:199-208): b[r] += A_e[r][r]
// over the cells, no BCs.  The element code is the matrix kernels'; the emit
// keeps the diagonal entries only (for FP64 the others are dead code).
// ---------------------------------------------------------------------------
struct DiagArgs {
  int64_t num_cells;
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  const int32_t* __restrict__ dofs;
  CoefDev c0, c1;
  double* __restrict__ b;
  int64_t num_values;
};

__global__ void __launch_bounds__(kBlock) k_diag_p1(const DiagArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (c >= a.num_cells) return;
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  double G[4][3];
  p1_grads(g, G);
  const double s = g.adet * (1.0 / 6.0) * coef_mean(a.c0, c);
  const int4 d = __ldg(reinterpret_cast<const int4*>(a.dofs) + c);
  const int r[4] = {d.x, d.y, d.z, d.w};
#pragma unroll
  for (int i = 0; i < 4; ++i)
    add_guarded(a.b, r[i], a.num_values, s * (G[i][0] * G[i][0] + G[i][1] * G[i][1] + G[i][2] * G[i][2]));
}

template <int COEF, typename T>
__global__ void __launch_bounds__(kBlock) k_diag_p2(const DiagArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (c >= a.num_cells) return;
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  double Gh[6];
  ghat(g, Gh);
  const int32_t* d = a.dofs + c * 10;
  auto emit = [&](int i, int j, double v) {
    if (i == j) add_guarded(a.b, __ldg(d + i), a.num_values, v);
  };
  if constexpr (COEF == FE_COEFF_P1) {
    const int4 km = __ldg(reinterpret_cast<const int4*>(a.c0.map) + c);
    const double k[4] = {__ldg(a.c0.v + km.x), __ldg(a.c0.v + km.y), __ldg(a.c0.v + km.z),
                         __ldg(a.c0.v + km.w)};
    T q[24];
#pragma unroll
    for (int m = 0; m < 4; ++m)
#pragma unroll
      for (int s = 0; s < 6; ++s) q[m * 6 + s] = (T)(k[m] * Gh[s]);
    p2_stiffness_p1coef<T>(q, emit);
  } else {
    const double k = coef_cell(a.c0, c);
    T gq[6];
#pragma unroll
    for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
    p2_stiffness_const<T>(gq, emit);
  }
}

template <typename T>
__global__ void __launch_bounds__(kBlockP3) k_diag_p3(const DiagArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlockP3 + threadIdx.x;
  if (c >= a.num_cells) return;
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  double Gh[6];
  ghat(g, Gh);
  const double k = coef_cell(a.c0, c);
  T gq[6];
#pragma unroll
  for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
  const int32_t* d = a.dofs + c * 20;
  p3_stiffness_const<T>(gq, [&](int i, int j, double v) {
    if (i == j) add_guarded(a.b, __ldg(d + i), a.num_values, v);
  });
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_diag_vp2(const DiagArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (c >= a.num_cells) return;
  CellGeo g;
  cell_geometry(a.x, load_geom(a.geom, c), g);
  const double lam = coef_cell(a.c0, c), mu = coef_cell(a.c1, c);
  const int32_t* d = a.dofs + c * 10;
  elasticity_blocks<T>(g, lam, mu, [&](int ca, int cb, int i, int j, double v) {
    if (ca == cb && i == j) add_guarded(a.b, 3 * (int64_t)__ldg(d + i) + ca, a.num_values, v);
  });
}

template <int K, int COEF>
__global__ void __launch_bounds__(kBlock) k_diag_mass(const DiagArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (c >= a.num_cells) return;
  const double adet = cell_adet(a.x, load_geom(a.geom, c));
  const int32_t* d = a.dofs + c * K;
  mass_element<K, COEF>(a.c0, c, adet, [&](int i, int j, double v) {
    if (i == j) add_guarded(a.b, __ldg(d + i), a.num_values, v);
  });
}

template <int COEF>
__global__ void __launch_bounds__(kBlock) k_diag_vmass(const DiagArgs a) {
  const int64_t c = blockIdx.x * (int64_t)kBlock + threadIdx.x;
  if (c >= a.num_cells) return;
  const double adet = cell_adet(a.x, load_geom(a.geom, c));
  const int32_t* d = a.dofs + c * 10;
  mass_element<10, COEF>(a.c0, c, adet, [&](int i, int j, double v) {
    if (i != j) return;
    const int64_t R = __ldg(d + i);
#pragma unroll
    for (int ca = 0; ca < 3; ++ca) add_guarded(a.b, 3 * R + ca, a.num_values, v);
  });
}

__global__ void k_mark_cells(const int32_t* __restrict__ dofs, int64_t num_cells, int k, int bs,
                             const uint8_t* __restrict__ markers, int32_t* __restrict__ out,
                             unsigned long long* count) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= num_cells) return;
  bool any = false;
  for (int i = 0; i < k && !any; ++i) {
    const int64_t D = dofs[c * k + i];
    if (D < 0) continue;  // outside a restriction
    for (int q = 0; q < bs; ++q) any |= markers[D * bs + q] != 0;
  }
  if (any) out[atomicAdd(count, 1ull)] = (int32_t)c;
}

__global__ void k_set_bc(double* __restrict__ b, int64_t num_values, const int32_t* __restrict__ dofs,
                         int64_t n_bc, const double* __restrict__ g, const double* __restrict__ x0,
                         double scale) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= n_bc) return;
  const int32_t d = dofs[t];
  if (d < 0 || d >= num_values) return;
  b[d] = scale * (g[d] - (x0 ? x0[d] : 0.0));
}

unsigned grid_for(int64_t n, int block) { return (unsigned)((n + block - 1) / block); }

// ---------------------------------------------------------------------------
// Right-hand side: assemble_vector(L) + apply_lifting([a], [bc]) + set_bc(bc)
// (assemble.py:136-166, 287-339, 341-380, three kernels with a context
// synchronise after each in the reference) in two launches without a
// synchronise: the lifting over the cells with a marked trial dof, and one
// kernel whose CTAs take the element vectors of all cells, then the BC dofs.
// Both scatters skip the marked rows and the BC range stores
// b[d] = scale (g[d] - x0[d]) there, so no row is both accumulated and stored
// and the launches need no order; the result equals the three calls (up to
// the order of the FP64 additions into unmarked rows).  The lifting keeps a
// launch of its own: its element tensor needs 70-164 registers per thread,
// which in one kernel would hold the light vector threads (32 registers) to
// its occupancy.
// ---------------------------------------------------------------------------
enum RhsPair { RHS_P1 = 1, RHS_P2 = 2, RHS_P3 = 3, RHS_VP2 = 4 };

struct RhsArgs {
  VecArgs v;
  const int32_t* __restrict__ bc_dofs;
  int64_t n_bc;
  const double* __restrict__ g;
  const double* __restrict__ x0;
  double scale;
  int64_t vec_ctas;
};

template <int PAIR>
__global__ void __launch_bounds__(kBlock) k_rhs_vec_bc(const RhsArgs a) {
  const int64_t blk = blockIdx.x;
  if (blk < a.vec_ctas) {
    const int64_t c = blk * kBlock + threadIdx.x;
    if (c >= a.v.num_cells) return;
    if constexpr (PAIR == RHS_P1) vec_p1(a.v, c);
    else if constexpr (PAIR == RHS_P2) vec_p2(a.v, c);
    else if constexpr (PAIR == RHS_P3) vec_p3(a.v, c);
    else vec_vp2(a.v, c);
    return;
  }
  const int64_t q = (blk - a.vec_ctas) * kBlock + threadIdx.x;
  if (q >= a.n_bc) return;
  const int32_t d = __ldg(a.bc_dofs + q);
  if (d < 0 || d >= a.v.num_values) return;
  a.v.b[d] = a.scale * (__ldg(a.g + d) - (a.x0 ? __ldg(a.x0 + d) : 0.0));
}

}  // namespace

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
void launch_zero(double* v, int64_t n, cudaStream_t s) {
  if (n <= 0) return;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (n / 2 + 255) / 256;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)sms * 8));
  k_zero<<<grid, 256, 0, s>>>(v, n);
  FE_CUDA(cudaGetLastError());
}

namespace {
__global__ void k_gather_diag(const int32_t* __restrict__ rows, int64_t n, const int32_t* __restrict__ diag,
                              int64_t num_rows, int32_t* __restrict__ out) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int32_t r = rows[k];
  out[k] = (r >= 0 && r < num_rows) ? diag[r] : -1;
}
}  // namespace

void launch_zero_diagonal(const fe_sparsity_s& sp, const fe_bc_s* bc, double diagonal, double* values,
                          cudaStream_t s) {
  const int64_t n = sp.nnz;
  if (n <= 0) return;
  if ((reinterpret_cast<uintptr_t>(values) & 15) != 0) {
    launch_zero(values, n, s);
    if (bc) launch_set_diagonal(sp, *bc, diagonal, values, s);
    return;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // 2 blocks of 256 threads per SM: the stores still stream at full bandwidth
  // and work launched beside the matrix call (the right-hand side on another
  // stream) finds room on every SM (P2 n=96 on B200: matrix call 2.44 against
  // 2.45 ms, step 2.65 against 2.72 ms with 8 blocks per SM; 4: 2.49 / 2.71)
  const int64_t blocks = std::max<int64_t>(1, std::min<int64_t>((n / 2 + 255) / 256, (int64_t)sms * 2));
  int64_t chunk = (n + blocks - 1) / blocks;
  chunk += chunk & 1;  // even, so every block's range starts on 16 bytes
  const int64_t grid = (n + chunk - 1) / chunk;
  const int32_t* dslot = nullptr;
  const int32_t* bstart = nullptr;
  if (bc && bc->n_owned) {
    // the BC rows' diagonal slots (ascending: rows ascend) and each block's
    // first one, once per (pattern, launch shape)
    auto& D = bc->diag_slots[sp.id];
    if (!D || D->chunk != chunk || D->grid != grid) {
      D = std::make_unique<fe_bc_s::DiagSlots>();
      DevBuf<int32_t> tmp((size_t)bc->n_owned);
      k_gather_diag<<<(unsigned)((bc->n_owned + 255) / 256), 256, 0, s>>>(bc->rows_sorted.p, bc->n_owned,
                                                                           sp.diag.p, sp.num_rows, tmp.p);
      FE_CUDA(cudaGetLastError());
      std::vector<int32_t> h((size_t)bc->n_owned);
      FE_CUDA(cudaMemcpyAsync(h.data(), tmp.p, h.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
      FE_CUDA(cudaStreamSynchronize(s));
      std::vector<int32_t> slots;
      slots.reserve(h.size());
      for (int32_t d : h)
        if (d >= 0) slots.push_back(d);
      std::sort(slots.begin(), slots.end());
      std::vector<int32_t> starts((size_t)grid + 1);
      for (int64_t b = 0; b <= grid; ++b)
        starts[b] = (int32_t)(std::lower_bound(slots.begin(), slots.end(), (int64_t)std::min(b * chunk, n)) -
                              slots.begin());
      D->slots.alloc(std::max<size_t>(1, slots.size()));
      if (!slots.empty())
        FE_CUDA(cudaMemcpy(D->slots.p, slots.data(), slots.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
      D->starts.alloc(starts.size());
      FE_CUDA(cudaMemcpy(D->starts.p, starts.data(), starts.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
      D->chunk = chunk;
      D->grid = grid;
    }
    dslot = D->slots.p;
    bstart = D->starts.p;
  }
  k_zero_diag<<<(unsigned)grid, 256, 0, s>>>(values, n, chunk, dslot, bstart, diagonal);
  FE_CUDA(cudaGetLastError());
}

void launch_build_slotmap(const fe_form_s& f, cudaStream_t s) {
  const fe_dofmap_s& V0 = *f.V0;
  const fe_dofmap_s& V1 = *f.V1;
  if (is_ifacet_kind(f.kind)) {
    // interior facets: the macro couplings of the two cells of every facet
    const int64_t n = f.num_facets * 2 * V0.k;
    if (n == 0) return;
    k_build_slotmap<<<grid_for(n, 256), 256, 0, s>>>(f.macro0.p, f.macro1.p ? f.macro1.p : f.macro0.p,
                                                     f.num_facets, 2 * V0.k, 2 * V1.k, V0.bs, V1.bs,
                                                     f.sp->row_ptr.p, f.sp->col.p, f.sp->num_rows, f.pos.p,
                                                     device_error_word(f.ctx));
    FE_CUDA(cudaGetLastError());
    return;
  }
  const int64_t n = V0.num_cells * V0.k;
  if (n == 0) return;
  k_build_slotmap<<<grid_for(n, 256), 256, 0, s>>>(V0.dofs.p, V1.dofs.p, V0.num_cells, V0.k, V1.k, V0.bs,
                                                   V1.bs, f.sp->row_ptr.p, f.sp->col.p, f.sp->num_rows,
                                                   f.pos.p, device_error_word(f.ctx));
  FE_CUDA(cudaGetLastError());
}

void launch_build_view(const fe_form_s& f, const fe_sparsity_s& mono, int64_t row_offset, int64_t col_offset,
                       fe_sparsity_s& view, cudaStream_t s) {
  const fe_dofmap_s& V0 = *f.V0;
  const fe_dofmap_s& V1 = *f.V1;
  const int64_t nrows = V0.num_blocks * V0.bs;
  view.row_ptr.alloc(nrows + 1);
  view.diag.alloc(std::max<int64_t>(1, nrows));
  FE_CUDA(cudaMemsetAsync(view.row_ptr.p, 0, (nrows + 1) * sizeof(int32_t), s));
  if (nrows)
    k_view_rows<<<grid_for(nrows, 256), 256, 0, s>>>(mono.row_ptr.p, mono.col.p, mono.diag.p, row_offset, col_offset,
                                                     nrows, view.row_ptr.p, view.diag.p);
  FE_CUDA(cudaGetLastError());
  const int64_t n = V0.num_cells * V0.k;
  if (n)
    k_build_slotmap_view<<<grid_for(n, 256), 256, 0, s>>>(V0.dofs.p, V1.dofs.p, V0.num_cells, V0.k, V1.k, V0.bs, V1.bs,
                                                          mono.row_ptr.p, mono.col.p, view.row_ptr.p, row_offset,
                                                          col_offset, f.pos.p, device_error_word(f.ctx));
  FE_CUDA(cudaGetLastError());
}

void launch_matrix_atomic(const MatLaunch& L, cudaStream_t s) {
  if (L.num_cells == 0) return;
  MatArgs a{};
  a.num_cells = L.num_cells;
  a.x = L.x;
  a.geom = L.geom;
  a.dofs0 = L.dofs0;
  a.dofs1 = L.dofs1;
  a.pos = L.pos;
  a.row_ptr = L.row_ptr;
  a.bc0 = L.bc0;
  a.bc1 = L.bc1;
  a.c0 = to_dev(L.c0);
  a.c1 = to_dev(L.c1);
  a.values = L.values;
  a.upper = L.upper;
  const unsigned grid = grid_for(L.num_cells, kBlock);
  const bool f32 = L.precision == FE_PREC_FP32;
  // tuned launch shape (fe_form_set_launch): cells per CTA and byte-map staging
  const int nt = L.cta_cells ? L.cta_cells : kBlock;
  const bool stage = L.stage != 0;
  switch (L.kind) {
    case FE_FORM_P1_STIFFNESS:
      if (nt == 32) k_mat_p1_atomic<32><<<grid_for(L.num_cells, 32), 32, 0, s>>>(a);
      else if (nt == 64) k_mat_p1_atomic<64><<<grid_for(L.num_cells, 64), 64, 0, s>>>(a);
      else k_mat_p1_atomic<kBlock><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P2_STIFFNESS: {
      auto go = [&](auto coef, auto tv) {
        constexpr int C = decltype(coef)::value;
        using T = typename decltype(tv)::type;
        if (L.coalesced && !a.upper) {
          auto k = stage ? k_mat_p2_coal<C, T, true> : k_mat_p2_coal<C, T, false>;
          k<<<grid_for(L.num_cells, kCoalThreads), kCoalThreads, 0, s>>>(a);
        } else if (nt == 32) {
          if (stage) k_mat_p2_atomic<C, T, 32, true><<<grid_for(L.num_cells, 32), 32, 0, s>>>(a);
          else k_mat_p2_atomic<C, T, 32, false><<<grid_for(L.num_cells, 32), 32, 0, s>>>(a);
        } else if (nt == 64) {
          if (stage) k_mat_p2_atomic<C, T, 64, true><<<grid_for(L.num_cells, 64), 64, 0, s>>>(a);
          else k_mat_p2_atomic<C, T, 64, false><<<grid_for(L.num_cells, 64), 64, 0, s>>>(a);
        } else {
          if (stage) k_mat_p2_atomic<C, T, kBlock, true><<<grid, kBlock, 0, s>>>(a);
          else k_mat_p2_atomic<C, T, kBlock, false><<<grid, kBlock, 0, s>>>(a);
        }
      };
      using P1c = std::integral_constant<int, FE_COEFF_P1>;
      using DGc = std::integral_constant<int, FE_COEFF_DG0>;
      if (a.c0.kind == FE_COEFF_P1) {
        if (f32) go(P1c{}, std::common_type<float>{});
        else go(P1c{}, std::common_type<double>{});
      } else {
        if (f32) go(DGc{}, std::common_type<float>{});
        else go(DGc{}, std::common_type<double>{});
      }
      break;
    }
    case FE_FORM_VP2_ELASTICITY:
      if (L.coalesced && !a.upper) {
        auto k = f32 ? k_mat_vp2_coal<float> : k_mat_vp2_coal<double>;
        k<<<grid_for(L.num_cells, kVCoalThreads), kVCoalThreads, 0, s>>>(a);
      } else if (f32) {
        k_mat_vp2_atomic<float><<<grid, kBlock, 0, s>>>(a);
      } else {
        k_mat_vp2_atomic<double><<<grid, kBlock, 0, s>>>(a);
      }
      break;
    case FE_FORM_P1_MASS:
      if (a.c0.kind == FE_COEFF_P1) k_mat_mass<4, FE_COEFF_P1><<<grid, kBlock, 0, s>>>(a);
      else k_mat_mass<4, FE_COEFF_DG0><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P2_MASS:
      if (a.c0.kind == FE_COEFF_P1) k_mat_mass<10, FE_COEFF_P1><<<grid, kBlock, 0, s>>>(a);
      else k_mat_mass<10, FE_COEFF_DG0><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_VP2_MASS:
      if (a.c0.kind == FE_COEFF_P1) k_mat_vmass<FE_COEFF_P1><<<grid, kBlock, 0, s>>>(a);
      else k_mat_vmass<FE_COEFF_DG0><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P3_STIFFNESS: {
      if (L.coalesced && !a.upper) {
        FE_REQUIRE(!f32, "the coalesced P3 kernel evaluates FP64 element tensors");
        k_mat_p3_coal<<<grid_for(L.num_cells, kP3CoalThreads), kP3CoalThreads, 0, s>>>(a);
        break;
      }
      // one thread per cell: splitting a cell's 210 entries over 2, 4 or 8
      // warps measured the same or slower on B200 (P3 n=48: 1.75-2.12 ms vs
      // 1.79 ms), the reductions themselves bound the kernel
      const unsigned g3 = grid_for(L.num_cells, kBlockP3);
      if (f32) k_mat_p3_atomic<float><<<g3, kBlockP3, 0, s>>>(a);
      else k_mat_p3_atomic<double><<<g3, kBlockP3, 0, s>>>(a);
      break;
    }
    default:
      FE_FAIL(FE_ERR_ARG, "not a bilinear form kind: " + std::to_string(L.kind));
  }
  FE_CUDA(cudaGetLastError());
}

namespace {
// node-block mirror of a block-size-3 pattern; false if the pattern is not
// block-structured or not symmetric
bool build_mirror3(fe_sparsity_s& sp, fe_sparsity_s::Mirror& M, cudaStream_t s) {
  const int64_t NB = sp.num_rows / 3;
  DevBuf<int32_t> cnt(NB);
  k_lower_count3<<<grid_for(NB, 256), 256, 0, s>>>(sp.row_ptr.p, sp.diag.p, NB, cnt.p);
  FE_CUDA(cudaGetLastError());
  std::vector<int32_t> h(NB);
  FE_CUDA(cudaMemcpyAsync(h.data(), cnt.p, NB * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  FE_CUDA(cudaStreamSynchronize(s));
  std::vector<int32_t> lp(NB + 1, 0);
  int64_t tot = 0;
  for (int64_t I = 0; I < NB; ++I) {
    if (h[I] < 0) return false;
    tot += h[I];
    if (tot > INT32_MAX) return false;
    lp[I + 1] = (int32_t)tot;
  }
  M.nblocks = tot;
  M.blocks.alloc(std::max<int64_t>(1, tot));
  DevBuf<int32_t> lower_ptr(NB + 1);
  FE_CUDA(cudaMemcpyAsync(lower_ptr.p, lp.data(), (NB + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  DevBuf<int> bad(1);
  FE_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
  k_lower_blocks3<<<grid_for(NB, 128), 128, 0, s>>>(sp.row_ptr.p, sp.col.p, lower_ptr.p, NB, M.blocks.p, bad.p);
  FE_CUDA(cudaGetLastError());
  int hb = 0;
  FE_CUDA(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  FE_CUDA(cudaStreamSynchronize(s));  // lower_ptr and bad are freed on return
  return hb == 0;
}
}  // namespace

bool ensure_mirror(fe_sparsity_s& sp, cudaStream_t s, int bs) {
  if (sp.mirror && sp.mirror->bs == bs) return sp.mirror->ok;
  auto M = std::make_unique<fe_sparsity_s::Mirror>();
  M->bs = bs;
  const int64_t R = sp.num_rows;
  if (R == 0 || sp.num_rows != sp.num_cols || (bs == 3 && R % 3)) {
    sp.mirror = std::move(M);
    return false;
  }
  if (bs == 3) {
    M->ok = build_mirror3(sp, *M, s);
    if (!M->ok) M->blocks.release();
    sp.mirror = std::move(M);
    return sp.mirror->ok;
  }
  DevBuf<int32_t> cnt(R);
  k_lower_count<<<grid_for(R, 256), 256, 0, s>>>(sp.row_ptr.p, sp.diag.p, R, cnt.p);
  FE_CUDA(cudaGetLastError());
  std::vector<int32_t> h(R);
  FE_CUDA(cudaMemcpyAsync(h.data(), cnt.p, R * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  FE_CUDA(cudaStreamSynchronize(s));
  std::vector<int32_t> lp(R + 1, 0);
  bool ok = true;
  int64_t tot = 0;
  for (int64_t r = 0; r < R; ++r) {
    if (h[r] < 0) ok = false;
    tot += h[r] < 0 ? 0 : h[r];
    if (tot > INT32_MAX) ok = false;
    lp[r + 1] = (int32_t)std::min<int64_t>(tot, INT32_MAX);
  }
  if (ok) {
    M->nlower = tot;
    M->pairs.alloc(std::max<int64_t>(1, tot));
    DevBuf<int32_t> lower_ptr(R + 1);
    FE_CUDA(cudaMemcpyAsync(lower_ptr.p, lp.data(), (R + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    DevBuf<int> bad(1);
    FE_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    k_lower_pairs<<<grid_for(R, 128), 128, 0, s>>>(sp.row_ptr.p, sp.col.p, lower_ptr.p, R, M->pairs.p, bad.p);
    FE_CUDA(cudaGetLastError());
    int hb = 0;
    FE_CUDA(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    FE_CUDA(cudaStreamSynchronize(s));  // lower_ptr and bad are freed on return
    ok = hb == 0;
  }
  M->ok = ok;
  if (!ok) M->pairs.release();
  sp.mirror = std::move(M);
  return ok;
}

void launch_mirror_lower(const fe_sparsity_s& sp, double* values, cudaStream_t s) {
  const auto& M = *sp.mirror;
  if (!M.ok) return;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (M.bs == 3) {
    if (M.nblocks == 0) return;
    const unsigned g3 = (unsigned)std::min<int64_t>((M.nblocks + 255) / 256, (int64_t)sms * 16);
    k_mirror_blocks3<<<g3, 256, 0, s>>>(M.blocks.p, M.nblocks, values);
    FE_CUDA(cudaGetLastError());
    return;
  }
  if (M.nlower == 0) return;
  const unsigned grid =
      (unsigned)std::min<int64_t>((M.nlower + 256 * kMirrorUnroll - 1) / (256 * kMirrorUnroll), (int64_t)sms * 16);
  k_mirror_pairs<<<grid, 256, 0, s>>>(M.pairs.p, M.nlower, values);
  FE_CUDA(cudaGetLastError());
}

void launch_set_diagonal(const fe_sparsity_s& sp, const fe_bc_s& bc, double diagonal, double* values,
                         cudaStream_t s) {
  if (bc.n_owned == 0) return;
  k_set_diagonal<<<grid_for(bc.n_owned, 256), 256, 0, s>>>(bc.dofs.p, bc.n_owned, sp.diag.p, sp.num_rows,
                                                           diagonal, values);
  FE_CUDA(cudaGetLastError());
}

namespace {
VecArgs vec_args(const VecLaunch& L) {
  VecArgs a{};
  a.num_cells = L.num_cells;
  a.x = L.x;
  a.geom = L.geom;
  a.dofs = L.dofs;
  a.f = to_dev(L.f);
  a.b = L.b;
  a.num_values = L.num_values;
  return a;
}

LiftArgs lift_args(const LiftLaunch& L) {
  LiftArgs a{};
  a.cells = L.cells;
  a.num_list = L.num_list;
  a.x = L.x;
  a.geom = L.geom;
  a.dofs0 = L.dofs0;
  a.dofs1 = L.dofs1;
  a.c0 = to_dev(L.c0);
  a.c1 = to_dev(L.c1);
  a.bc1 = L.bc1;
  a.g = L.g;
  a.x0 = L.x0;
  a.scale = L.scale;
  a.b = L.b;
  a.num_values = L.num_values;
  a.skip = L.skip;
  return a;
}
}  // namespace

void launch_vector(const VecLaunch& L, cudaStream_t s) {
  if (L.num_cells == 0) return;
  const VecArgs a = vec_args(L);
  const unsigned grid = grid_for(L.num_cells, kBlock);
  switch (L.kind) {
    case FE_FORM_P1_LOAD:
      k_vec_p1<<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P2_LOAD:
      k_vec_p2<<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_VP2_LOAD:
      k_vec_vp2<<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P3_LOAD:
      k_vec_p3<<<grid, kBlock, 0, s>>>(a);
      break;
    default:
      FE_FAIL(FE_ERR_ARG, "not a linear form kind: " + std::to_string(L.kind));
  }
  FE_CUDA(cudaGetLastError());
}

void launch_lifting(const LiftLaunch& L, cudaStream_t s) {
  if (L.num_list == 0) return;
  const LiftArgs a = lift_args(L);
  const unsigned grid = grid_for(L.num_list, kBlock);
  const bool f32 = L.precision == FE_PREC_FP32;
  switch (L.kind) {
    case FE_FORM_P1_STIFFNESS:
      k_lift_p1<<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P2_STIFFNESS:
      if (a.c0.kind == FE_COEFF_P1) {
        if (f32) k_lift_p2<FE_COEFF_P1, float><<<grid, kBlock, 0, s>>>(a);
        else k_lift_p2<FE_COEFF_P1, double><<<grid, kBlock, 0, s>>>(a);
      } else {
        if (f32) k_lift_p2<FE_COEFF_DG0, float><<<grid, kBlock, 0, s>>>(a);
        else k_lift_p2<FE_COEFF_DG0, double><<<grid, kBlock, 0, s>>>(a);
      }
      break;
    case FE_FORM_VP2_ELASTICITY:
      if (f32) k_lift_vp2<float><<<grid, kBlock, 0, s>>>(a);
      else k_lift_vp2<double><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P1_MASS:
      if (a.c0.kind == FE_COEFF_P1) k_lift_mass<4, FE_COEFF_P1><<<grid, kBlock, 0, s>>>(a);
      else k_lift_mass<4, FE_COEFF_DG0><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P2_MASS:
      if (a.c0.kind == FE_COEFF_P1) k_lift_mass<10, FE_COEFF_P1><<<grid, kBlock, 0, s>>>(a);
      else k_lift_mass<10, FE_COEFF_DG0><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_VP2_MASS:
      if (a.c0.kind == FE_COEFF_P1) k_lift_vmass<FE_COEFF_P1><<<grid, kBlock, 0, s>>>(a);
      else k_lift_vmass<FE_COEFF_DG0><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P3_STIFFNESS: {
      const unsigned g3 = grid_for(L.num_list, kBlockP3);
      if (f32) k_lift_p3<float><<<g3, kBlockP3, 0, s>>>(a);
      else k_lift_p3<double><<<g3, kBlockP3, 0, s>>>(a);
      break;
    }
    default:
      FE_FAIL(FE_ERR_ARG, "lifting needs a bilinear form, got kind " + std::to_string(L.kind));
  }
  FE_CUDA(cudaGetLastError());
}

bool rhs_fused_supported(int vec_kind, int mat_kind) {
  return (vec_kind == FE_FORM_P1_LOAD && mat_kind == FE_FORM_P1_STIFFNESS) ||
         (vec_kind == FE_FORM_P2_LOAD && mat_kind == FE_FORM_P2_STIFFNESS) ||
         (vec_kind == FE_FORM_P3_LOAD && mat_kind == FE_FORM_P3_STIFFNESS) ||
         (vec_kind == FE_FORM_VP2_LOAD && mat_kind == FE_FORM_VP2_ELASTICITY);
}

void launch_rhs_fused(const VecLaunch& V, const LiftLaunch& Lf, const int32_t* bc_dofs, int64_t n_bc,
                      cudaStream_t s) {
  FE_REQUIRE(rhs_fused_supported(V.kind, Lf.kind), "no fused right-hand side for this pair of form kinds");
  // the BC's markers: exactly its dofs (checked when the BC is created)
  LiftLaunch L = Lf;
  L.skip = Lf.bc1;
  launch_lifting(L, s);
  RhsArgs a{};
  a.v = vec_args(V);
  a.v.skip = Lf.bc1;
  a.bc_dofs = bc_dofs;
  a.n_bc = n_bc;
  a.g = Lf.g;
  a.x0 = Lf.x0;
  a.scale = Lf.scale;
  a.vec_ctas = (V.num_cells + kBlock - 1) / kBlock;
  const int64_t total = a.vec_ctas + (n_bc + kBlock - 1) / kBlock;
  if (total == 0) return;
  FE_REQUIRE(total < (int64_t)INT_MAX, "right-hand side too large for one launch");
  const unsigned grid = (unsigned)total;
  switch (V.kind) {
    case FE_FORM_P1_LOAD:
      k_rhs_vec_bc<RHS_P1><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P2_LOAD:
      k_rhs_vec_bc<RHS_P2><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P3_LOAD:
      k_rhs_vec_bc<RHS_P3><<<grid, kBlock, 0, s>>>(a);
      break;
    default:
      k_rhs_vec_bc<RHS_VP2><<<grid, kBlock, 0, s>>>(a);
  }
  FE_CUDA(cudaGetLastError());
}

void launch_diagonal(const MatLaunch& L, double* b, int64_t num_values, cudaStream_t s) {
  if (L.num_cells == 0) return;
  DiagArgs a{};
  a.num_cells = L.num_cells;
  a.x = L.x;
  a.geom = L.geom;
  a.dofs = L.dofs0;
  a.c0 = to_dev(L.c0);
  a.c1 = to_dev(L.c1);
  a.b = b;
  a.num_values = num_values;
  const unsigned grid = grid_for(L.num_cells, kBlock);
  const bool f32 = L.precision == FE_PREC_FP32;
  switch (L.kind) {
    case FE_FORM_P1_STIFFNESS:
      k_diag_p1<<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P2_STIFFNESS:
      if (a.c0.kind == FE_COEFF_P1) {
        if (f32) k_diag_p2<FE_COEFF_P1, float><<<grid, kBlock, 0, s>>>(a);
        else k_diag_p2<FE_COEFF_P1, double><<<grid, kBlock, 0, s>>>(a);
      } else {
        if (f32) k_diag_p2<FE_COEFF_DG0, float><<<grid, kBlock, 0, s>>>(a);
        else k_diag_p2<FE_COEFF_DG0, double><<<grid, kBlock, 0, s>>>(a);
      }
      break;
    case FE_FORM_P3_STIFFNESS: {
      const unsigned g3 = grid_for(L.num_cells, kBlockP3);
      if (f32) k_diag_p3<float><<<g3, kBlockP3, 0, s>>>(a);
      else k_diag_p3<double><<<g3, kBlockP3, 0, s>>>(a);
      break;
    }
    case FE_FORM_VP2_ELASTICITY:
      if (f32) k_diag_vp2<float><<<grid, kBlock, 0, s>>>(a);
      else k_diag_vp2<double><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P1_MASS:
      if (a.c0.kind == FE_COEFF_P1) k_diag_mass<4, FE_COEFF_P1><<<grid, kBlock, 0, s>>>(a);
      else k_diag_mass<4, FE_COEFF_DG0><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_P2_MASS:
      if (a.c0.kind == FE_COEFF_P1) k_diag_mass<10, FE_COEFF_P1><<<grid, kBlock, 0, s>>>(a);
      else k_diag_mass<10, FE_COEFF_DG0><<<grid, kBlock, 0, s>>>(a);
      break;
    case FE_FORM_VP2_MASS:
      if (a.c0.kind == FE_COEFF_P1) k_diag_vmass<FE_COEFF_P1><<<grid, kBlock, 0, s>>>(a);
      else k_diag_vmass<FE_COEFF_DG0><<<grid, kBlock, 0, s>>>(a);
      break;
    default:
      FE_FAIL(FE_ERR_ARG, "the diagonal is offered for the cell bilinear forms (P1/P2/P3 stiffness, P1/P2/vector-P2 mass, "
                          "vector-P2 elasticity), not kind " + std::to_string(L.kind));
  }
  FE_CUDA(cudaGetLastError());
}

void launch_mark_cells(const int32_t* dofs, int64_t num_cells, int k, int bs, const uint8_t* markers,
                       int32_t* out_cells, unsigned long long* out_count, cudaStream_t s) {
  if (num_cells == 0) return;
  k_mark_cells<<<grid_for(num_cells, 256), 256, 0, s>>>(dofs, num_cells, k, bs, markers, out_cells, out_count);
  FE_CUDA(cudaGetLastError());
}

void launch_set_bc(double* b, int64_t num_values, const int32_t* dofs, int64_t n_bc, const double* g,
                   const double* x0, double scale, cudaStream_t s) {
  if (n_bc == 0) return;
  k_set_bc<<<grid_for(n_bc, 256), 256, 0, s>>>(b, num_values, dofs, n_bc, g, x0, scale);
  FE_CUDA(cudaGetLastError());
}

}  // namespace fe
