// Owner-computes matrix assembly ("tile gather") for scalar P1 / P2 forms.
//
// The reference scatters every element entry with an FP64 atomicAdd into
// the CSR values after a separate zero pass (CUDAFormIntegral.cpp:1103-1226,
// CUDAAssembler.cpp:38-56).  On B200 that design is bound by L2 atomic
// throughput and re-reads every value line from HBM.  Here:
//
//   plan (host, once per form + pattern):
//     block rows are sorted along a Morton curve of a point of one of their
//     cells and cut into tiles whose CSR segments fit in shared memory; a
//     tile's cells are all cells touching one of its rows (cells on tile
//     borders are computed by every tile they touch); the incidences
//     (cell, local row i) whose row the tile owns are grouped per chunk of
//     cells and per lane-group (group = local row mod #groups);
//   kernel (one CTA per tile):
//     zero the tile's row segments in shared memory;
//     per chunk: one thread per cell computes the element tensor (symmetric
//     half) into shared memory and stages the cell's slot bytes and column
//     BC mask; then each lane-group walks its incidences in order, lanes
//     j < k adding A_e[i][j] to its row entry -- one group owns a row, so
//     there are no atomics and the summation order is fixed;
//     finally every owned row segment is written once, coalesced (BC rows
//     zero), so there is no zero pass and no read-back of the values.
//   The result is bitwise reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <thread>

#include "fe_element_code.cuh"
#include "fe_internal.h"

namespace fe {

template <int KIND>
struct TileTraits;
template <>
struct TileTraits<FE_FORM_P1_STIFFNESS> {
  static constexpr int K = 4, NU = 10, NUP = 11, CH = 256, NT = 256, LANES = 4;
  static constexpr int ACC = 6144, ROWCAP = 1024;
};
template <>
struct TileTraits<FE_FORM_P2_STIFFNESS> {
  static constexpr int K = 10, NU = 55, NUP = 55, CH = 128, NT = 256, LANES = 10;
  static constexpr int ACC = 12288, ROWCAP = 1024;
};

template <int KIND>
struct TileDerived {
  using Tr = TileTraits<KIND>;
  static constexpr int GPW = 32 / Tr::LANES;           // lane-groups per warp
  static constexpr int NG = (Tr::NT / 32) * GPW;       // lane-groups per CTA
  static constexpr int KK = Tr::K * Tr::K;             // slot bytes per cell
  // shared-memory carve-up (bytes, each part 16-byte aligned)
  static constexpr size_t OFF_ACC = 0;
  static constexpr size_t OFF_AE = OFF_ACC + sizeof(double) * Tr::ACC;
  static constexpr size_t OFF_POS = OFF_AE + sizeof(double) * Tr::CH * Tr::NUP;
  static constexpr size_t OFF_REC = OFF_POS + ((size_t)Tr::CH * KK + 15) / 16 * 16;
  static constexpr size_t OFF_CMASK = OFF_REC + sizeof(uint32_t) * Tr::CH * Tr::K;
  static constexpr size_t OFF_GOFF = OFF_CMASK + sizeof(uint32_t) * Tr::CH;
  static constexpr size_t OFF_SOFF = OFF_GOFF + ((sizeof(int32_t) * (NG + 1) + 15) / 16) * 16;
  static constexpr size_t OFF_GBASE = OFF_SOFF + sizeof(int32_t) * (Tr::ROWCAP + 1);
  static constexpr size_t OFF_LEN = OFF_GBASE + sizeof(int32_t) * Tr::ROWCAP;
  static constexpr size_t OFF_RMASK = OFF_LEN + sizeof(int32_t) * Tr::ROWCAP;
  static constexpr size_t SMEM = OFF_RMASK + Tr::ROWCAP;
};

}  // namespace fe

namespace fe {
namespace {

// ---------------------------------------------------------------------------
// Device side
// ---------------------------------------------------------------------------
struct TileArgs {
  const int32_t* __restrict__ tile_rows_ptr;
  const int32_t* __restrict__ rows;
  const int32_t* __restrict__ row_soff;
  const int32_t* __restrict__ row_tile;
  const int32_t* __restrict__ row_local;
  const int32_t* __restrict__ dofs0;
  const int32_t* __restrict__ tile_cells_ptr;
  const int32_t* __restrict__ cells;
  const int32_t* __restrict__ tile_rec_ptr;
  const uint32_t* __restrict__ recs;
  const int32_t* __restrict__ tile_goff_ptr;
  const int32_t* __restrict__ goff;
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  const int32_t* __restrict__ dofs1;
  const uint8_t* __restrict__ pos;
  const int32_t* __restrict__ row_ptr;
  const uint8_t* __restrict__ bc0;
  const uint8_t* __restrict__ bc1;
  int coef_kind;
  const double* __restrict__ coef;
  const int32_t* __restrict__ coef_map;
  double coef_const;
  int zero;
  double* __restrict__ values;
};

struct TGeo {
  double K[3][3];
  double adet;
};

__device__ __forceinline__ void tgeo(const double* __restrict__ x, int4 v, TGeo& g) {
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

// index of the symmetric entry (i, j) in row-major upper-triangle order
template <int K>
__device__ __forceinline__ int sym_index(int i, int j) {
  const int a = i < j ? i : j, b = i < j ? j : i;
  return a * K - (a * (a - 1)) / 2 + (b - a);
}

// element tensor of cell c (symmetric half): emit(i, j, value) for i <= j,
// in row-major upper-triangle order
template <int KIND, typename T, typename Emit>
__device__ __forceinline__ void element_tensor_emit(const TileArgs& a, int64_t c, Emit&& emit) {
  TGeo g;
  tgeo(a.x, __ldg(reinterpret_cast<const int4*>(a.geom) + c), g);
  if constexpr (KIND == FE_FORM_P1_STIFFNESS) {
    double G[4][3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      G[1][b] = g.K[0][b];
      G[2][b] = g.K[1][b];
      G[3][b] = g.K[2][b];
      G[0][b] = -(g.K[0][b] + g.K[1][b] + g.K[2][b]);
    }
    const double k = a.coef_kind == FE_COEFF_DG0 ? __ldg(a.coef + c) : a.coef_const;
    const double s = g.adet * (1.0 / 6.0) * k;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = i; j < 4; ++j) emit(i, j, s * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]));
  } else {
    const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
    double Gh[6];
#pragma unroll
    for (int s = 0; s < 6; ++s)
      Gh[s] = g.adet * (g.K[pa[s]][0] * g.K[pb[s]][0] + g.K[pa[s]][1] * g.K[pb[s]][1] +
                        g.K[pa[s]][2] * g.K[pb[s]][2]);
    auto emitT = [&](int i, int j, double v) { emit(i, j, v); };
    if (a.coef_kind == FE_COEFF_P1) {
      const int4 km = __ldg(reinterpret_cast<const int4*>(a.coef_map) + c);
      const double k[4] = {__ldg(a.coef + km.x), __ldg(a.coef + km.y), __ldg(a.coef + km.z), __ldg(a.coef + km.w)};
      T q[24];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int s = 0; s < 6; ++s) q[m * 6 + s] = (T)(k[m] * Gh[s]);
      p2_stiffness_p1coef<T>(q, emitT);
    } else {
      const double k = a.coef_kind == FE_COEFF_DG0 ? __ldg(a.coef + c) : a.coef_const;
      T gq[6];
#pragma unroll
      for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
      p2_stiffness_const<T>(gq, emitT);
    }
  }
}

// element tensor of cell c (symmetric half) into ae[0..NU)
template <int KIND, typename T>
__device__ __forceinline__ void element_tensor(const TileArgs& a, int64_t c, double* ae) {
  TGeo g;
  tgeo(a.x, __ldg(reinterpret_cast<const int4*>(a.geom) + c), g);
  if constexpr (KIND == FE_FORM_P1_STIFFNESS) {
    double G[4][3];
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      G[1][b] = g.K[0][b];
      G[2][b] = g.K[1][b];
      G[3][b] = g.K[2][b];
      G[0][b] = -(g.K[0][b] + g.K[1][b] + g.K[2][b]);
    }
    const double k = a.coef_kind == FE_COEFF_DG0 ? __ldg(a.coef + c) : a.coef_const;
    const double s = g.adet * (1.0 / 6.0) * k;
    int e = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = i; j < 4; ++j) ae[e++] = s * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]);
  } else {
    const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
    double Gh[6];
#pragma unroll
    for (int s = 0; s < 6; ++s)
      Gh[s] = g.adet * (g.K[pa[s]][0] * g.K[pb[s]][0] + g.K[pa[s]][1] * g.K[pb[s]][1] +
                        g.K[pa[s]][2] * g.K[pb[s]][2]);
    // unique entry (i <= j) index, row by row
    auto emit = [&](int i, int j, double v) { ae[i * 10 - (i * (i - 1)) / 2 + (j - i)] = v; };
    if (a.coef_kind == FE_COEFF_P1) {
      const int4 km = __ldg(reinterpret_cast<const int4*>(a.coef_map) + c);
      const double k[4] = {__ldg(a.coef + km.x), __ldg(a.coef + km.y), __ldg(a.coef + km.z), __ldg(a.coef + km.w)};
      T q[24];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int s = 0; s < 6; ++s) q[m * 6 + s] = (T)(k[m] * Gh[s]);
      p2_stiffness_p1coef<T>(q, emit);
    } else {
      const double k = a.coef_kind == FE_COEFF_DG0 ? __ldg(a.coef + c) : a.coef_const;
      T gq[6];
#pragma unroll
      for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
      p2_stiffness_const<T>(gq, emit);
    }
  }
}

template <int KIND, typename T>
__global__ void __launch_bounds__(TileTraits<KIND>::NT) k_tile_gather(const TileArgs a) {
  using Tr = TileTraits<KIND>;
  using D = TileDerived<KIND>;
  constexpr int K = Tr::K, NUP = Tr::NUP, CH = Tr::CH, NT = Tr::NT, LANES = Tr::LANES;
  constexpr int NG = D::NG, GPW = D::GPW, KK = D::KK;
  extern __shared__ __align__(16) unsigned char smem[];
  double* acc = reinterpret_cast<double*>(smem + D::OFF_ACC);
  double* s_ae = reinterpret_cast<double*>(smem + D::OFF_AE);
  uint8_t* s_pos = smem + D::OFF_POS;
  uint32_t* s_rec = reinterpret_cast<uint32_t*>(smem + D::OFF_REC);
  uint32_t* s_cmask = reinterpret_cast<uint32_t*>(smem + D::OFF_CMASK);
  int32_t* s_goff = reinterpret_cast<int32_t*>(smem + D::OFF_GOFF);
  int32_t* s_soff = reinterpret_cast<int32_t*>(smem + D::OFF_SOFF);
  int32_t* s_gbase = reinterpret_cast<int32_t*>(smem + D::OFF_GBASE);
  int32_t* s_len = reinterpret_cast<int32_t*>(smem + D::OFF_LEN);
  uint8_t* s_rmask = smem + D::OFF_RMASK;

  const int tid = threadIdx.x;
  const int64_t t = blockIdx.x;
  const int32_t r0 = a.tile_rows_ptr[t], nrows = a.tile_rows_ptr[t + 1] - r0;
  const int32_t c0 = a.tile_cells_ptr[t], ncells = a.tile_cells_ptr[t + 1] - c0;
  const int32_t rec0 = a.tile_rec_ptr[t];
  const int32_t* goff = a.goff + a.tile_goff_ptr[t];

  // owned rows: global base, length, BC flag and (planned) offset in the buffer
  for (int r = tid; r < nrows; r += NT) {
    const int32_t R = a.rows[r0 + r];
    const int32_t lo = a.row_ptr[R];
    s_gbase[r] = lo;
    s_len[r] = a.row_ptr[R + 1] - lo;
    s_rmask[r] = a.bc0 ? a.bc0[R] : 0;
    s_soff[r] = a.row_soff[r0 + r];
  }
  __syncthreads();
  const int32_t stot = nrows ? s_soff[nrows - 1] + s_len[nrows - 1] : 0;
  for (int q = tid; q < stot; q += NT) acc[q] = 0.0;

  const int warp = tid >> 5, lane = tid & 31;
  const int gi = lane / LANES, jl = lane % LANES;
  const bool gvalid = gi < GPW;
  const int g = warp * GPW + gi;

  const int nchunks = (ncells + CH - 1) / CH;
  for (int q = 0; q < nchunks; ++q) {
    const int cbase = q * CH;
    const int nc = min(CH, ncells - cbase);
    __syncthreads();  // previous chunk fully consumed
    // stage records and group offsets of this chunk
    const int32_t* gq = goff + q * (NG + 1);
    const int32_t rfirst = gq[0], rcount = gq[NG] - gq[0];
    for (int u = tid; u <= NG; u += NT) s_goff[u] = gq[u] - rfirst;
    for (int u = tid; u < rcount; u += NT) s_rec[u] = a.recs[rec0 + rfirst + u];
    // slot bytes of the chunk's cells
    if constexpr (KK % 16 == 0) {
      for (int u = tid; u < nc * (KK / 16); u += NT) {
        const int lc = u / (KK / 16), w = u % (KK / 16);
        const int64_t c = a.cells[c0 + cbase + lc];
        reinterpret_cast<uint4*>(s_pos)[u] = __ldg(reinterpret_cast<const uint4*>(a.pos + c * KK) + w);
      }
    } else {
      for (int u = tid; u < nc * (KK / 4); u += NT) {
        const int lc = u / (KK / 4), w = u % (KK / 4);
        const int64_t c = a.cells[c0 + cbase + lc];
        reinterpret_cast<uint32_t*>(s_pos)[u] = __ldg(reinterpret_cast<const uint32_t*>(a.pos + c * KK) + w);
      }
    }
    // element tensors and column BC masks, one thread per cell
    if (tid < nc) {
      const int64_t c = a.cells[c0 + cbase + tid];
      double ae[Tr::NU];
      element_tensor<KIND, T>(a, c, ae);
#pragma unroll
      for (int e = 0; e < Tr::NU; ++e) s_ae[tid * NUP + e] = ae[e];
      uint32_t m = 0;
      if (a.bc1) {
#pragma unroll
        for (int j = 0; j < K; ++j) m |= (a.bc1[__ldg(a.dofs1 + c * K + j)] ? 1u : 0u) << j;
      }
      s_cmask[tid] = m;
    }
    __syncthreads();
    // accumulate: lane-group g owns rows r with r % NG == g
    const int32_t ga = gvalid ? s_goff[g] : 0, gb = gvalid ? s_goff[g + 1] : 0;
    const int mylen = gb - ga;
    const int maxlen = __reduce_max_sync(0xffffffffu, mylen);
    for (int s = 0; s < maxlen; ++s) {
      if (s < mylen && jl < K) {
        const uint32_t rec = s_rec[ga + s];
        const int rl = (int)(rec >> 16), lc = (int)((rec >> 8) & 0xffu), i = (int)(rec & 0xffu);
        if (!s_rmask[rl] && !((s_cmask[lc] >> jl) & 1u)) {
          const int p = s_pos[lc * KK + i * K + jl];
          acc[s_soff[rl] + p] += s_ae[lc * NUP + sym_index<K>(i, jl)];
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  // write every owned row segment once
  const int nwarps = NT / 32;
  for (int r = warp; r < nrows; r += nwarps) {
    const int32_t so = s_soff[r], gb = s_gbase[r], len = s_len[r];
    for (int e = lane; e < len; e += 32) {
      double v = acc[so + e];
      if (!a.zero) v += a.values[gb + e];
      a.values[gb + e] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Shared-memory-atomic tile kernel: same tiles, one thread per tile cell, no
// chunking.  Each cell adds the entries of the rows this tile owns into the
// shared row buffer with FP64 shared atomics (summation order varies, so
// this variant is not bitwise reproducible), then the rows are written once.
// ---------------------------------------------------------------------------
template <int KIND>
struct TileAtomicSmem {
  using Tr = TileTraits<KIND>;
  static constexpr size_t OFF_SOFF = sizeof(double) * Tr::ACC;
  static constexpr size_t OFF_GBASE = OFF_SOFF + sizeof(int32_t) * Tr::ROWCAP;
  static constexpr size_t OFF_LEN = OFF_GBASE + sizeof(int32_t) * Tr::ROWCAP;
  static constexpr size_t OFF_RMASK = OFF_LEN + sizeof(int32_t) * Tr::ROWCAP;
  static constexpr size_t SMEM = OFF_RMASK + Tr::ROWCAP;
};

template <int KIND, typename T>
__global__ void __launch_bounds__(TileTraits<KIND>::NT, 2) k_tile_atomic(const TileArgs a) {
  using Tr = TileTraits<KIND>;
  using S = TileAtomicSmem<KIND>;
  constexpr int K = Tr::K, KK = K * K, NT = Tr::NT;
  extern __shared__ __align__(16) unsigned char smem[];
  double* acc = reinterpret_cast<double*>(smem);
  int32_t* s_soff = reinterpret_cast<int32_t*>(smem + S::OFF_SOFF);
  int32_t* s_gbase = reinterpret_cast<int32_t*>(smem + S::OFF_GBASE);
  int32_t* s_len = reinterpret_cast<int32_t*>(smem + S::OFF_LEN);
  uint8_t* s_rmask = smem + S::OFF_RMASK;

  const int tid = threadIdx.x;
  const int32_t t = blockIdx.x;
  const int32_t r0 = a.tile_rows_ptr[t], nrows = a.tile_rows_ptr[t + 1] - r0;
  const int32_t c0 = a.tile_cells_ptr[t], ncells = a.tile_cells_ptr[t + 1] - c0;
  for (int r = tid; r < nrows; r += NT) {
    const int32_t R = a.rows[r0 + r];
    const int32_t lo = a.row_ptr[R];
    s_gbase[r] = lo;
    s_len[r] = a.row_ptr[R + 1] - lo;
    s_rmask[r] = a.bc0 ? a.bc0[R] : 0;
    s_soff[r] = a.row_soff[r0 + r];
  }
  __syncthreads();
  const int32_t stot = nrows ? s_soff[nrows - 1] + s_len[nrows - 1] : 0;
  for (int q = tid; q < stot; q += NT) acc[q] = 0.0;
  __syncthreads();

  // lanes of a warp take cells 1/32 of the list apart: neighbouring cells
  // share dofs, and same-address shared atomics within a warp serialise
  const int n32 = (ncells + 31) >> 5;
  for (int q = tid; q < n32 * 32; q += NT) {
    const int idx = (q & 31) * n32 + (q >> 5);
    if (idx >= ncells) continue;
    const int64_t c = a.cells[c0 + idx];
    // rows of this cell that the tile owns (and that are not BC rows)
    unsigned own = 0, cmask = 0;
    int soff[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int32_t R = __ldg(a.dofs0 + c * K + i);
      soff[i] = 0;
      if (__ldg(a.row_tile + R) == t) {
        const int32_t rl = __ldg(a.row_local + R);
        if (!s_rmask[rl]) {
          own |= 1u << i;
          soff[i] = s_soff[rl];
        }
      }
      if (a.bc1) cmask |= (a.bc1[__ldg(a.dofs1 + c * K + i)] ? 1u : 0u) << i;
    }
    // slot bytes of the cell
    uint32_t pw[KK / 4];
#pragma unroll
    for (int w = 0; w < KK / 4; ++w) pw[w] = __ldg(reinterpret_cast<const uint32_t*>(a.pos + c * KK) + w);
    auto posb = [&](int i, int j) -> int { return (pw[(i * K + j) >> 2] >> (8 * ((i * K + j) & 3))) & 0xff; };
    element_tensor_emit<KIND, T>(a, c, [&](int i, int j, double v) {
      if (((own >> i) & 1u) && !((cmask >> j) & 1u)) atomicAdd(acc + soff[i] + posb(i, j), v);
      if (i != j && ((own >> j) & 1u) && !((cmask >> i) & 1u)) atomicAdd(acc + soff[j] + posb(j, i), v);
    });
  }
  __syncthreads();
  const int warp = tid >> 5, lane = tid & 31;
  for (int r = warp; r < nrows; r += NT / 32) {
    const int32_t so = s_soff[r], gb = s_gbase[r], len = s_len[r];
    for (int e = lane; e < len; e += 32) {
      double v = acc[so + e];
      if (!a.zero) v += a.values[gb + e];
      a.values[gb + e] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Host plan
// ---------------------------------------------------------------------------
uint64_t spread3(uint64_t v) {  // 21 bits -> every third bit
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffull;
  v = (v | v << 16) & 0x1f0000ff0000ffull;
  v = (v | v << 8) & 0x100f00f00f00f00full;
  v = (v | v << 4) & 0x10c30c30c30c30c3ull;
  v = (v | v << 2) & 0x1249249249249249ull;
  return v;
}

template <typename F>
void par_for(int64_t n, F&& body) {
  unsigned T = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
  if (n < 1024) T = 1;
  std::vector<std::thread> th;
  for (unsigned w = 0; w < T; ++w) th.emplace_back([&, w] { body(n * w / T, n * (w + 1) / T); });
  for (auto& x : th) x.join();
}

template <int KIND>
std::unique_ptr<fe_form_s::TilePlan> build_plan(const fe_form_s& f) {
  using Tr = TileTraits<KIND>;
  using D = TileDerived<KIND>;
  const fe_dofmap_s& V0 = *f.V0;
  const int k = V0.k;
  const int64_t C = V0.num_cells, nR = V0.num_blocks;
  const int32_t* dofs = V0.host.data();
  const std::vector<int32_t>& rp = f.sp->host_row_ptr;
  const std::vector<double>& X = f.mesh->host_x;
  const std::vector<int32_t>& G = f.mesh->host_geom;
  if ((int64_t)rp.size() != nR + 1) FE_FAIL(FE_ERR_ARG, "pattern rows differ from the dofmap");

  // 1. a point per block row: centroid of its lowest-numbered cell
  std::vector<int64_t> first(nR, -1);
  for (int64_t c = C - 1; c >= 0; --c)
    for (int i = 0; i < k; ++i) first[dofs[c * k + i]] = c;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (size_t v = 0; v < X.size() / 3; ++v)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], X[3 * v + d]);
      hi[d] = std::max(hi[d], X[3 * v + d]);
    }
  std::vector<std::pair<uint64_t, int32_t>> key(nR);
  par_for(nR, [&](int64_t a, int64_t b) {
    for (int64_t R = a; R < b; ++R) {
      uint64_t code = 0;
      if (first[R] >= 0) {
        const int64_t c = first[R];
        uint64_t m[3];
        for (int d = 0; d < 3; ++d) {
          double s = 0.0;
          for (int v = 0; v < 4; ++v) s += X[3 * (int64_t)G[4 * c + v] + d];
          const double u = (s * 0.25 - lo[d]) / std::max(hi[d] - lo[d], 1e-300);
          m[d] = (uint64_t)(std::min(std::max(u, 0.0), 1.0) * 2097151.0);
        }
        code = spread3(m[0]) | (spread3(m[1]) << 1) | (spread3(m[2]) << 2);
      }
      key[R] = {code, (int32_t)R};
    }
  });
  std::sort(key.begin(), key.end());

  // 2. greedy tiles along the curve
  std::vector<int32_t> row_tile(nR), row_local(nR), rows(nR), row_soff(nR), tile_rows_ptr(1, 0);
  {
    int64_t acc = 0, cnt = 0;
    for (int64_t q = 0; q < nR; ++q) {
      const int32_t R = key[q].second;
      const int64_t len = rp[R + 1] - rp[R];
      if (len > Tr::ACC) FE_FAIL(FE_ERR_ARG, "a CSR row is longer than the tile buffer");
      if (cnt == Tr::ROWCAP || acc + len > Tr::ACC) {
        tile_rows_ptr.push_back((int32_t)q);
        acc = 0;
        cnt = 0;
      }
      row_tile[R] = (int32_t)tile_rows_ptr.size() - 1;
      row_local[R] = (int32_t)cnt;
      rows[q] = R;
      row_soff[q] = (int32_t)acc;
      acc += len;
      ++cnt;
    }
    tile_rows_ptr.push_back((int32_t)nR);
  }
  const int64_t ntiles = (int64_t)tile_rows_ptr.size() - 1;

  // 3. cells touching each tile (ascending), and incidence counts
  std::vector<int64_t> ccount(ntiles + 1, 0), icount(ntiles + 1, 0);
  auto tiles_of = [&](int64_t c, int32_t* out) {
    int n = 0;
    for (int i = 0; i < k; ++i) {
      const int32_t t = row_tile[dofs[c * k + i]];
      bool seen = false;
      for (int u = 0; u < n; ++u) seen |= out[u] == t;
      if (!seen) out[n++] = t;
    }
    return n;
  };
  for (int64_t c = 0; c < C; ++c) {
    int32_t ts[32];
    const int n = tiles_of(c, ts);
    for (int u = 0; u < n; ++u) ccount[ts[u] + 1]++;
    for (int i = 0; i < k; ++i) icount[row_tile[dofs[c * k + i]] + 1]++;
  }
  for (int64_t t = 0; t < ntiles; ++t) {
    ccount[t + 1] += ccount[t];
    icount[t + 1] += icount[t];
  }
  if (ccount[ntiles] > INT32_MAX || icount[ntiles] > INT32_MAX) FE_FAIL(FE_ERR_ARG, "tile plan too large");
  std::vector<int32_t> cells(ccount[ntiles]);
  {
    std::vector<int64_t> cur(ccount.begin(), ccount.end() - 1);
    for (int64_t c = 0; c < C; ++c) {
      int32_t ts[32];
      const int n = tiles_of(c, ts);
      for (int u = 0; u < n; ++u) cells[cur[ts[u]]++] = (int32_t)c;
    }
  }
  // 4. per tile, per chunk, records grouped by lane-group (row_local % NG)
  std::vector<int64_t> gcount(ntiles + 1, 0);
  for (int64_t t = 0; t < ntiles; ++t) {
    const int64_t nc = ccount[t + 1] - ccount[t];
    gcount[t + 1] = gcount[t] + ((nc + Tr::CH - 1) / Tr::CH) * (D::NG + 1);
  }
  std::vector<uint32_t> recs(icount[ntiles]);
  std::vector<int32_t> goff(gcount[ntiles]);
  par_for(ntiles, [&](int64_t ta, int64_t tb) {
    std::vector<uint32_t> buf;
    std::vector<int32_t> gc(D::NG + 1);
    for (int64_t t = ta; t < tb; ++t) {
      const int64_t cb = ccount[t], nc = ccount[t + 1] - cb;
      int64_t r = icount[t];
      const int64_t rbase = icount[t];
      int32_t* go = goff.data() + gcount[t];
      for (int64_t q = 0; q * Tr::CH < nc; ++q) {
        std::fill(gc.begin(), gc.end(), 0);
        buf.clear();
        const int64_t lc_end = std::min<int64_t>(Tr::CH, nc - q * Tr::CH);
        for (int64_t lc = 0; lc < lc_end; ++lc) {
          const int64_t c = cells[cb + q * Tr::CH + lc];
          for (int i = 0; i < k; ++i) {
            const int32_t R = dofs[c * k + i];
            if (row_tile[R] != t) continue;
            const uint32_t rl = (uint32_t)row_local[R];
            buf.push_back((rl << 16) | ((uint32_t)lc << 8) | (uint32_t)i);
            gc[rl % D::NG + 1]++;
          }
        }
        for (int g = 0; g < D::NG; ++g) gc[g + 1] += gc[g];
        for (int g = 0; g <= D::NG; ++g) go[q * (D::NG + 1) + g] = (int32_t)(r - rbase + gc[g]);
        std::vector<int32_t> cur(gc.begin(), gc.end() - 1);
        for (uint32_t rec : buf) recs[r + cur[(rec >> 16) % D::NG]++] = rec;
        r += (int64_t)buf.size();
      }
    }
  });

  auto P = std::make_unique<fe_form_s::TilePlan>();
  P->ntiles = ntiles;
  P->total_cells = ccount[ntiles];
  auto up32 = [](DevBuf<int32_t>& d, const std::vector<int32_t>& h) {
    d.alloc(std::max<size_t>(1, h.size()));
    if (!h.empty()) FE_CUDA(cudaMemcpy(d.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
  };
  auto up64as32 = [&](DevBuf<int32_t>& d, const std::vector<int64_t>& h) {
    std::vector<int32_t> v(h.begin(), h.end());
    up32(d, v);
  };
  up32(P->tile_rows_ptr, tile_rows_ptr);
  up32(P->rows, rows);
  up32(P->row_soff, row_soff);
  up32(P->row_tile, row_tile);
  up32(P->row_local, row_local);
  up64as32(P->tile_cells_ptr, ccount);
  up32(P->cells, cells);
  up64as32(P->tile_rec_ptr, icount);
  P->recs.alloc(std::max<size_t>(1, recs.size()));
  if (!recs.empty()) FE_CUDA(cudaMemcpy(P->recs.p, recs.data(), recs.size() * 4, cudaMemcpyHostToDevice));
  up64as32(P->tile_goff_ptr, gcount);
  up32(P->goff, goff);
  return P;
}

template <int KIND, typename T>
void launch_tiles(const fe_form_s& f, const fe_form_s::TilePlan& P, double* values, const fe_bc_s* bc0,
                  const fe_bc_s* bc1, bool zero, bool deterministic, cudaStream_t s) {
  TileArgs a{};
  a.tile_rows_ptr = P.tile_rows_ptr.p;
  a.rows = P.rows.p;
  a.row_soff = P.row_soff.p;
  a.row_tile = P.row_tile.p;
  a.row_local = P.row_local.p;
  a.dofs0 = f.V0->dofs.p;
  a.tile_cells_ptr = P.tile_cells_ptr.p;
  a.cells = P.cells.p;
  a.tile_rec_ptr = P.tile_rec_ptr.p;
  a.recs = P.recs.p;
  a.tile_goff_ptr = P.tile_goff_ptr.p;
  a.goff = P.goff.p;
  a.x = f.mesh->x.p;
  a.geom = f.mesh->geom.p;
  a.dofs1 = f.V1->dofs.p;
  a.pos = f.pos.p;
  a.row_ptr = f.sp->row_ptr.p;
  a.bc0 = bc0 ? bc0->markers.p : nullptr;
  a.bc1 = bc1 ? bc1->markers.p : nullptr;
  const Coefficient& k = f.coeff[0];
  a.coef_kind = k.kind < 0 ? FE_COEFF_CONSTANT : k.kind;
  a.coef = k.values;
  a.coef_map = k.map ? k.map->dofs.p : nullptr;
  a.coef_const = k.kind < 0 ? 1.0 : k.constant[0];
  a.zero = zero ? 1 : 0;
  a.values = values;
  if (P.ntiles == 0) return;
  if (deterministic) {
    auto kern = k_tile_gather<KIND, T>;
    constexpr size_t smem = TileDerived<KIND>::SMEM;
    FE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)P.ntiles, TileTraits<KIND>::NT, smem, s>>>(a);
  } else {
    auto kern = k_tile_atomic<KIND, T>;
    constexpr size_t smem = TileAtomicSmem<KIND>::SMEM;
    FE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<(unsigned)P.ntiles, TileTraits<KIND>::NT, smem, s>>>(a);
  }
  FE_CUDA(cudaGetLastError());
}

}  // namespace

void reset_tile_plan(fe_form_s& f) { f.tiles.reset(); }

bool tile_supported(const fe_form_s& f) {
  if (!f.V0 || !f.V1 || f.V0->bs != 1 || f.V1->bs != 1) return false;
  if (f.kind == FE_FORM_P1_STIFFNESS) return f.coeff[0].kind != FE_COEFF_P1;
  return f.kind == FE_FORM_P2_STIFFNESS;
}

void assemble_matrix_tiled(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, bool zero,
                           bool deterministic, cudaStream_t s) {
  if (!f.tiles) {
    f.tiles = (f.kind == FE_FORM_P1_STIFFNESS) ? build_plan<FE_FORM_P1_STIFFNESS>(f)
                                               : build_plan<FE_FORM_P2_STIFFNESS>(f);
  }
  if (f.kind == FE_FORM_P1_STIFFNESS) {
    launch_tiles<FE_FORM_P1_STIFFNESS, double>(f, *f.tiles, values, bc0, bc1, zero, deterministic, s);
  } else if (f.precision == FE_PREC_FP32) {
    launch_tiles<FE_FORM_P2_STIFFNESS, float>(f, *f.tiles, values, bc0, bc1, zero, deterministic, s);
  } else {
    launch_tiles<FE_FORM_P2_STIFFNESS, double>(f, *f.tiles, values, bc0, bc1, zero, deterministic, s);
  }
}

}  // namespace fe
