// Cell-block matrix assembly for scalar P1 / P2 stiffness ("block" variant).
//
// The FP64-atomic scatter issues one uncoalesced L2 reduction per element
// entry; on B200 those run at ~200 G/s, which bounds that kernel.  This
// variant keeps one thread per cell but combines first:
//   plan (host, once per form + pattern):
//     cells are sorted along a Morton curve of their centroids and cut into
//     compact blocks; per block, the sorted list of block rows its cells
//     touch, each row's offset in a shared-memory window, and per cell the
//     window row of each local dof.  Per-cell inputs (geometry dofmap, form
//     dofmaps, slot bytes, coefficient map) are copied in block order so the
//     kernel reads them contiguously;
//   kernel (one CTA per block, after a zero pass over the values):
//     each thread computes its cell's element tensor and adds the entries
//     into the window with shared-memory FP64 atomics; then warps flush the
//     window row by row with reductions to consecutive addresses, skipping
//     entries no cell of the block touched.  Contributions meeting in the
//     window cost one L2 reduction instead of several, and a flush
//     instruction covers a run of consecutive slots.
// Rows/columns of BC dofs are skipped as in the reference
// (CUDAFormIntegral.cpp:1195-1213); set_diagonal follows
// (CUDAAssembler.cpp:131-164).
#include <cuda_runtime.h>

#include <algorithm>
#include <thread>

#include "fe_element_code.cuh"
#include "fe_internal.h"

namespace fe {
namespace {

template <int KIND>
struct BlockTraits;
// WCAP: window slots (8 bytes each); RCAP: touched rows per block; MINB: CTAs per SM to fit
template <>
struct BlockTraits<FE_FORM_P1_STIFFNESS> {
  static constexpr int K = 4, NT = 256, BMAX = 512, WCAP = 3072, RCAP = 512, MINB = 4, VCAP = 512;
};
template <>
struct BlockTraits<FE_FORM_P2_STIFFNESS> {
  static constexpr int K = 10, NT = 128, BMAX = 128, WCAP = 8192, RCAP = 768, MINB = 3, VCAP = 1 << 30;
};

template <int KIND>
struct BlockSmem {
  using Tr = BlockTraits<KIND>;
  static constexpr size_t OFF_SOFF = sizeof(double) * (Tr::WCAP + 2);  // + the spare slot
  static constexpr size_t OFF_GBASE = OFF_SOFF + sizeof(int32_t) * (Tr::RCAP + 1);
  static constexpr size_t OFF_LEN = OFF_GBASE + sizeof(int32_t) * Tr::RCAP;
  static constexpr size_t OFF_RMASK = OFF_LEN + sizeof(int32_t) * Tr::RCAP;
  static constexpr size_t SMEM = OFF_RMASK + Tr::RCAP;
};

struct BlockArgs {
  const int32_t* __restrict__ block_ptr;   // [nblocks+1] into the block-ordered cell arrays
  const int32_t* __restrict__ brow_ptr;    // [nblocks+1] into rows/soff
  const int32_t* __restrict__ rows;        // touched block rows, per block, ascending
  const int32_t* __restrict__ soff;        // window offset of each touched row
  const uint16_t* __restrict__ lrow;       // [cells][K] window row of each local dof
  const int32_t* __restrict__ cell_id;     // original cell id (DG0 coefficients)
  const int4* __restrict__ geom;           // block-ordered geometry dofmap
  const int32_t* __restrict__ dofs0;       // block-ordered
  const int32_t* __restrict__ dofs1;       // block-ordered
  const uint8_t* __restrict__ pos;         // block-ordered slot bytes [cells][K*K]
  const int4* __restrict__ coef_map;       // block-ordered P1 coefficient dofmap
  const double* __restrict__ x;
  const int32_t* __restrict__ row_ptr;
  const uint8_t* __restrict__ bc0;
  const uint8_t* __restrict__ bc1;
  int coef_kind;
  const double* __restrict__ coef;
  double coef_const;
  const double* __restrict__ gbound;       // [nblocks] geometric part of the entry bound
  double term_max;                         // reference-tensor part of the entry bound
  int fx_bits;                             // fixed-point bits S (50..57)
  double* __restrict__ values;
  const int32_t* __restrict__ gvert_ptr;   // P1: [nblocks+1] block geometry nodes
  const double* __restrict__ gx;           // P1: their coordinates, block by block
  const uint16_t* __restrict__ glocal;     // P1: [records][4] block-local node of each vertex
  const int32_t* __restrict__ rec_ptr;     // P1: [nblocks+1] record offsets (lrow, pos, glocal,
                                           // cell_id and dofs1 are indexed by record)
};

__device__ __forceinline__ void block_geom(const double* __restrict__ x, int4 v, double K[3][3], double& adet) {
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
  K[0][0] = c00 * id;
  K[1][0] = c01 * id;
  K[2][0] = c02 * id;
  K[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  K[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  K[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  K[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  K[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  K[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  adet = fabs(det);
}

// coefficient factor of the entry bound of block-ordered cell cb: |k| for a
// cellwise coefficient, sum_m |k_m| for a P1 coefficient
__device__ __forceinline__ double cell_coef_factor(const BlockArgs& a, int64_t cb) {
  if (a.coef_kind == FE_COEFF_P1) {
    const int4 km = __ldg(a.coef_map + cb);
    return fabs(__ldg(a.coef + km.x)) + fabs(__ldg(a.coef + km.y)) + fabs(__ldg(a.coef + km.z)) +
           fabs(__ldg(a.coef + km.w));
  }
  return a.coef_kind == FE_COEFF_DG0 ? fabs(__ldg(a.coef + __ldg(a.cell_id + cb))) : fabs(a.coef_const);
}

// Fixed-point scale of a block.  Every entry of the block lies below bmax <
// 2^ex; it is kept as w = round(v * 2^(S - ex)), |w| < 2^S, S = fx_bits,
// rounded to nearest by one 64-bit conversion.  Quantisation is at most
// 2^(ex - S - 1) per contribution, so a cell whose entries lie 2^kDirect
// below 2^ex would lose precision relative to its own size: such cells add
// their entries with FP64 reductions instead.
struct FixedScale {
  double scale, direct_below;
};

__device__ __forceinline__ FixedScale fixed_scale(double bmax, int fx_bits, int direct_bits) {
  int ex = 0;
  frexp(bmax, &ex);
  const bool ok = bmax > 0.0 && bmax < 1e300;
  FixedScale f;
  f.scale = ok ? ldexp(1.0, fx_bits - ex) : 1.0;
  f.direct_below = ok ? ldexp(1.0, ex - direct_bits) : 0.0;
  return f;
}

__device__ __forceinline__ long long to_fixed(double v, const FixedScale& f) { return __double2ll_rn(v * f.scale); }

// cells whose entry bound lies below 2^(ex - kDirect*) take the FP64 path:
// the P1 bound is the cell's largest entry itself, the P2 one an upper bound
constexpr int kDirectP1 = 8;
constexpr int kDirectP2 = 6;

// element tensor of block-ordered cell cb, entries (i, j, value) for i <= j
// passed to emit, or to emit_direct when an upper bound of the cell's
// |entries| lies below direct_below
template <int KIND, typename T, typename Emit, typename EmitDirect>
__device__ __forceinline__ void cell_entries(const BlockArgs& a, int64_t cb, double direct_below, Emit&& emit,
                                             EmitDirect&& emit_direct) {
  double Km[3][3], adet;
  block_geom(a.x, __ldg(a.geom + cb), Km, adet);
  if constexpr (KIND == FE_FORM_P1_STIFFNESS) {
    double G[4][3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      G[1][d] = Km[0][d];
      G[2][d] = Km[1][d];
      G[3][d] = Km[2][d];
      G[0][d] = -(Km[0][d] + Km[1][d] + Km[2][d]);
    }
    const double k = a.coef_kind == FE_COEFF_DG0 ? __ldg(a.coef + __ldg(a.cell_id + cb)) : a.coef_const;
    const double s = adet * (1.0 / 6.0) * k;
    double g2 = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) g2 = fmax(g2, G[i][0] * G[i][0] + G[i][1] * G[i][1] + G[i][2] * G[i][2]);
    auto run = [&](auto&& e) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = i; j < 4; ++j) e(i, j, s * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]));
    };
    if (!(fabs(s) * g2 < direct_below)) run(emit);
    else run(emit_direct);
  } else {
    const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
    double Gh[6], gsum = 0.0;
#pragma unroll
    for (int s = 0; s < 6; ++s) {
      Gh[s] = adet * (Km[pa[s]][0] * Km[pb[s]][0] + Km[pa[s]][1] * Km[pb[s]][1] + Km[pa[s]][2] * Km[pb[s]][2]);
      gsum += fabs(Gh[s]);
    }
    const bool direct = gsum * cell_coef_factor(a, cb) * a.term_max < direct_below;
    auto emitT = [&](int i, int j, double v) { emit(i, j, v); };
    auto emitD = [&](int i, int j, double v) { emit_direct(i, j, v); };
    if (a.coef_kind == FE_COEFF_P1) {
      const int4 km = __ldg(a.coef_map + cb);
      const double kv[4] = {__ldg(a.coef + km.x), __ldg(a.coef + km.y), __ldg(a.coef + km.z), __ldg(a.coef + km.w)};
      T qv[24];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int s = 0; s < 6; ++s) qv[m * 6 + s] = (T)(kv[m] * Gh[s]);
      if (!direct) p2_stiffness_p1coef<T>(qv, emitT);
      else p2_stiffness_p1coef<T>(qv, emitD);
    } else {
      const double k = a.coef_kind == FE_COEFF_DG0 ? __ldg(a.coef + __ldg(a.cell_id + cb)) : a.coef_const;
      T gq[6];
#pragma unroll
      for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
      if (!direct) p2_stiffness_const<T>(gq, emitT);
      else p2_stiffness_const<T>(gq, emitD);
    }
  }
}

template <int KIND, typename T>
__global__ void __launch_bounds__(BlockTraits<KIND>::NT, BlockTraits<KIND>::MINB) k_block(const BlockArgs a) {
  using Tr = BlockTraits<KIND>;
  using S = BlockSmem<KIND>;
  constexpr int K = Tr::K, KK = K * K, NT = Tr::NT;
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* win = reinterpret_cast<uint32_t*>(smem);  // 2 words per slot
  int32_t* s_soff = reinterpret_cast<int32_t*>(smem + S::OFF_SOFF);
  int32_t* s_gbase = reinterpret_cast<int32_t*>(smem + S::OFF_GBASE);
  int32_t* s_len = reinterpret_cast<int32_t*>(smem + S::OFF_LEN);
  uint8_t* s_rmask = smem + S::OFF_RMASK;

  const int tid = threadIdx.x;
  const int32_t b = blockIdx.x;
  const int32_t r0 = a.brow_ptr[b], nrows = a.brow_ptr[b + 1] - r0;
  const int32_t c0 = a.block_ptr[b], ncells = a.block_ptr[b + 1] - c0;
  for (int r = tid; r < nrows; r += NT) {
    const int32_t R = a.rows[r0 + r];
    const int32_t lo = __ldg(a.row_ptr + R);
    s_gbase[r] = lo;
    s_len[r] = __ldg(a.row_ptr + R + 1) - lo;
    s_soff[r] = a.soff[r0 + r];
    s_rmask[r] = a.bc0 ? a.bc0[R] : 0;
  }
  __shared__ unsigned s_bmax;
  __syncthreads();
  const int32_t wtot = nrows ? s_soff[nrows - 1] + s_len[nrows - 1] : 0;
  for (int q = tid; q < 2 * wtot; q += NT) win[q] = 0u;
  if (tid == 0) s_bmax = 0u;
  __syncthreads();

  // pass 1: bound on every element entry of the block = (geometric bound of
  // the block, from the plan) x (largest coefficient factor of its cells);
  // it fixes the fixed-point scale (non-negative floats order like their bits)
  double kfac = fabs(a.coef_const);
  if (a.coef_kind != FE_COEFF_CONSTANT) {
    for (int q = tid; q < ncells; q += NT)
      atomicMax(&s_bmax, __float_as_uint((float)(cell_coef_factor(a, c0 + q) * 1.0625)));
    __syncthreads();
    kfac = (double)__uint_as_float(s_bmax);
  }
  const double bmax = 1.25 * a.gbound[b] * kfac * a.term_max;
  const FixedScale fs = fixed_scale(bmax, a.fx_bits, kDirectP2);

  // pass 2: entries accumulate as 64-bit fixed-point integers, kept as two
  // 32-bit words so both updates are native shared-memory atomics; integer
  // addition is exact and order-independent, the carry out of the low word
  // is added to the high word exactly once per wrap
  for (int q = tid; q < ncells; q += NT) {
    const int64_t cb = c0 + q;  // block-ordered cell index
    unsigned own = 0, cmask = 0;
    int wbase[K];
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int lr = __ldg(a.lrow + cb * K + i);
      wbase[i] = s_soff[lr];
      own |= (s_rmask[lr] ? 0u : 1u) << i;
      if (a.bc1) cmask |= (a.bc1[__ldg(a.dofs1 + cb * K + i)] ? 1u : 0u) << i;
    }
    uint32_t pw[KK / 4];
#pragma unroll
    for (int w = 0; w < KK / 4; ++w) pw[w] = __ldg(reinterpret_cast<const uint32_t*>(a.pos + cb * KK) + w);
    auto posb = [&](int i, int j) -> int { return (pw[(i * K + j) >> 2] >> (8 * ((i * K + j) & 3))) & 0xff; };
    // branch-free: a contribution to a BC row or column goes to the spare
    // slot WCAP, which is never flushed
    auto add_fixed = [&](int idx, long long w) {
      const uint32_t lo = (uint32_t)(unsigned long long)w;
      const uint32_t hi = (uint32_t)((unsigned long long)w >> 32);
      const uint32_t old = atomicAdd(win + 2 * idx, lo);
      atomicAdd(win + 2 * idx + 1, hi + ((old + lo < old) ? 1u : 0u));
    };
    auto emit = [&](int i, int j, double v) {
      const long long w = to_fixed(v, fs);
      const bool ok_ij = ((own >> i) & 1u) && !((cmask >> j) & 1u);
      add_fixed(ok_ij ? wbase[i] + posb(i, j) : Tr::WCAP, w);
      if (i != j) {
        const bool ok_ji = ((own >> j) & 1u) && !((cmask >> i) & 1u);
        add_fixed(ok_ji ? wbase[j] + posb(j, i) : Tr::WCAP, w);
      }
    };
    // a cell small next to the block's largest entries: FP64 reductions
    // straight into the values
    auto emit_direct = [&](int i, int j, double v) {
      auto lrow = [&](int u) { return (int)__ldg(a.lrow + cb * K + u); };  // rare path: re-read
      if (((own >> i) & 1u) && !((cmask >> j) & 1u)) atomicAdd(a.values + s_gbase[lrow(i)] + posb(i, j), v);
      if (i != j && ((own >> j) & 1u) && !((cmask >> i) & 1u))
        atomicAdd(a.values + s_gbase[lrow(j)] + posb(j, i), v);
    };
    cell_entries<KIND, T>(a, cb, fs.direct_below, emit, emit_direct);
  }
  __syncthreads();
  const double inv = 1.0 / fs.scale;  // exact: a power of two
  // flush: one warp per touched row, lanes over consecutive slots
  const int warp = tid >> 5, lane = tid & 31;
  for (int r = warp; r < nrows; r += NT / 32) {
    const int32_t so = s_soff[r], gb = s_gbase[r], len = s_len[r];
    for (int e = lane; e < len; e += 32) {
      const uint32_t lo = win[2 * (so + e)], hi = win[2 * (so + e) + 1];
      if (lo | hi) {
        // hi * 2^32 + lo, rounded once to double (both halves convert exactly)
        const double v = fma((double)(int32_t)hi, 4294967296.0, (double)lo);
        atomicAdd(a.values + gb + e, v * inv);
      }
    }
  }
}

// P1 specialisation (constant or DG0 coefficient): the same window
// combine, with the per-cell reads vectorised (window rows as one 8-byte
// load, slot bytes as one 16-byte load), BC column masks of square forms
// taken from the window rows instead of global reads, the cells of a warp
// spread over the block (fewer lanes adding into the same window slot at
// once), and a flat flush over the window (a per-slot row table in shared
// memory keeps all lanes busy on 15-slot rows).
// P1 window: a contribution's 64-bit fixed-point value w (|w| < 2^50) is
// kept as two 32-bit shared words (low and high half, two planes); the low
// word's atomic returns its old value, from which the carry into the high
// word is added exactly once per wrap.  (Three carry-free 21-bit fields were
// measured too: the kernel is bound by shared-memory wavefronts, so the third
// atomic per contribution cost more than the carry dependency.)
constexpr int kP1Wcap = BlockTraits<FE_FORM_P1_STIFFNESS>::WCAP;

struct P1Smem {
  using Tr = BlockTraits<FE_FORM_P1_STIFFNESS>;
  static constexpr int PLANE = kP1Wcap + 1;  // + the spare slot
  static constexpr size_t OFF_SOFF = sizeof(uint32_t) * 2 * PLANE + 8;
  static constexpr size_t OFF_GBASE = OFF_SOFF + sizeof(int32_t) * (Tr::RCAP + 1);
  static constexpr size_t OFF_WROW = OFF_GBASE + sizeof(int32_t) * Tr::RCAP;
  static constexpr size_t OFF_RMASK = OFF_WROW + sizeof(uint16_t) * kP1Wcap;
  static constexpr size_t OFF_CMASK = OFF_RMASK + Tr::RCAP;
  static constexpr size_t OFF_X = (OFF_CMASK + Tr::RCAP + 15) / 16 * 16;
  // per window row: window offset | row BC bit 30 | column BC bit 31 (one
  // shared-memory load per local dof instead of three)
  static constexpr size_t OFF_RINFO = OFF_X + sizeof(double) * 3 * Tr::VCAP;
  static constexpr size_t SMEM = OFF_RINFO + sizeof(uint32_t) * Tr::RCAP;
};

__global__ void __launch_bounds__(BlockTraits<FE_FORM_P1_STIFFNESS>::NT, 4) k_block_p1(const BlockArgs a,
                                                                                    int square) {
  using Tr = BlockTraits<FE_FORM_P1_STIFFNESS>;
  using S = P1Smem;
  constexpr int NT = Tr::NT, NW = NT / 32, PLANE = S::PLANE;
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* w0 = reinterpret_cast<uint32_t*>(smem);  // low words
  uint32_t* w1 = w0 + PLANE;                         // high words
  int32_t* s_soff = reinterpret_cast<int32_t*>(smem + S::OFF_SOFF);
  int32_t* s_gbase = reinterpret_cast<int32_t*>(smem + S::OFF_GBASE);
  uint16_t* s_wrow = reinterpret_cast<uint16_t*>(smem + S::OFF_WROW);
  uint8_t* s_rmask = smem + S::OFF_RMASK;
  uint8_t* s_cmask = smem + S::OFF_CMASK;
  double* s_x = reinterpret_cast<double*>(smem + S::OFF_X);
  uint32_t* s_rinfo = reinterpret_cast<uint32_t*>(smem + S::OFF_RINFO);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int32_t b = blockIdx.x;
  const int32_t r0 = a.brow_ptr[b], nrows = a.brow_ptr[b + 1] - r0;
  const int32_t c0 = a.block_ptr[b], ncells = a.block_ptr[b + 1] - c0;
  for (int r = tid; r < nrows; r += NT) {
    const int32_t R = a.rows[r0 + r];
    const int32_t lo = __ldg(a.row_ptr + R), len = __ldg(a.row_ptr + R + 1) - lo;
    const int32_t so = a.soff[r0 + r];
    s_gbase[r] = lo;
    s_soff[r] = so;
    if (r == nrows - 1) s_soff[nrows] = so + len;
    s_rmask[r] = a.bc0 ? a.bc0[R] : 0;
    s_cmask[r] = (square && a.bc1) ? a.bc1[R] : 0;
    s_rinfo[r] = (uint32_t)so | (s_rmask[r] ? 1u << 30 : 0u) | (s_cmask[r] ? 1u << 31 : 0u);
    for (int e = 0; e < len; ++e) s_wrow[so + e] = (uint16_t)r;
  }
  {
    // the block's geometry nodes: one coalesced copy into shared memory
    const int32_t g0 = a.gvert_ptr[b], ng = a.gvert_ptr[b + 1] - g0;
    const double* src = a.gx + 3 * (int64_t)g0;
    for (int q = tid; q < 3 * ng; q += NT) s_x[q] = __ldg(src + q);
  }
  __shared__ unsigned s_bmax;
  if (tid == 0) s_bmax = 0u;
  __syncthreads();
  const int32_t wtot = nrows ? s_soff[nrows] : 0;
  for (int q = tid; q < wtot; q += NT) {
    w0[q] = 0u;
    w1[q] = 0u;
  }
  // records of this block: cell q = lane*span + slot sits at rec0 + slot*32 + lane
  const int span = (ncells + 31) / 32;
  const int32_t rec0 = a.rec_ptr[b];
  if (a.coef_kind != FE_COEFF_CONSTANT) {
    for (int t = tid; t < span * 32; t += NT)
      if ((t & 31) * span + (t >> 5) < ncells)
        atomicMax(&s_bmax, __float_as_uint((float)(cell_coef_factor(a, rec0 + t) * 1.0625)));
  }
  __syncthreads();
  const double kfac = a.coef_kind != FE_COEFF_CONSTANT ? (double)__uint_as_float(s_bmax) : fabs(a.coef_const);
  const double bmax = 1.25 * a.gbound[b] * kfac;
  const FixedScale fs = fixed_scale(bmax, a.fx_bits, kDirectP1);

  // lane l of warp w takes cells l*span + w, l*span + w + NW, ...: the 32
  // cells of one warp instruction lie span cells apart along the curve, and
  // their records are consecutive
  for (int slot = warp; slot < span; slot += NW) {
    const int q = lane * span + slot;
    if (q >= ncells) continue;
    const int64_t cb = rec0 + slot * 32 + lane;
    const uint2 lrw = __ldg(reinterpret_cast<const uint2*>(a.lrow) + cb);
    const int lr[4] = {(int)(lrw.x & 0xffffu), (int)(lrw.x >> 16), (int)(lrw.y & 0xffffu), (int)(lrw.y >> 16)};
    const uint4 pq = __ldg(reinterpret_cast<const uint4*>(a.pos) + cb);
    const uint32_t pw[4] = {pq.x, pq.y, pq.z, pq.w};
    int wbase[4];
    unsigned own = 0, cmask = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t ri = s_rinfo[lr[i]];
      wbase[i] = (int)(ri & 0x3fffffffu);
      own |= (((ri >> 30) & 1u) ^ 1u) << i;
      if (square) cmask |= (ri >> 31) << i;
      else if (a.bc1) cmask |= (a.bc1[__ldg(a.dofs1 + cb * 4 + i)] ? 1u : 0u) << i;
    }
    auto add = [&](int idx, long long w) {
      const uint32_t lo = (uint32_t)(unsigned long long)w;
      const uint32_t hi = (uint32_t)((unsigned long long)w >> 32);
      const uint32_t old = atomicAdd(w0 + idx, lo);
      atomicAdd(w1 + idx, hi + ((old + lo < old) ? 1u : 0u));
    };
    auto emit = [&](int i, int j, double v) {
      const long long w = to_fixed(v, fs);
      const bool ok_ij = ((own >> i) & 1u) && !((cmask >> j) & 1u);
      add(ok_ij ? wbase[i] + (int)((pw[i] >> (8 * j)) & 0xffu) : kP1Wcap, w);
      if (i != j) {
        const bool ok_ji = ((own >> j) & 1u) && !((cmask >> i) & 1u);
        add(ok_ji ? wbase[j] + (int)((pw[j] >> (8 * i)) & 0xffu) : kP1Wcap, w);
      }
    };
    // a cell small next to the block's largest entries: FP64 reductions
    // straight into the values (window slot -> global slot as in the flush)
    auto emit_direct = [&](int i, int j, double v) {
      auto red = [&](int w) {
        const int r = s_wrow[w];
        atomicAdd(a.values + s_gbase[r] + (w - s_soff[r]), v);
      };
      if (((own >> i) & 1u) && !((cmask >> j) & 1u)) red(wbase[i] + (int)((pw[i] >> (8 * j)) & 0xffu));
      if (i != j && ((own >> j) & 1u) && !((cmask >> i) & 1u)) red(wbase[j] + (int)((pw[j] >> (8 * i)) & 0xffu));
    };
    // P1 element from the staged coordinates: grad phi_i = K^T ghat_i,
    // A_ij = k |det J| / 6 grad phi_i . grad phi_j
    const uint2 glw = __ldg(reinterpret_cast<const uint2*>(a.glocal) + cb);
    const int gl[4] = {(int)(glw.x & 0xffffu), (int)(glw.x >> 16), (int)(glw.y & 0xffffu), (int)(glw.y >> 16)};
    double J[3][3];
#pragma unroll
    for (int cc = 0; cc < 3; ++cc)
#pragma unroll
      for (int r = 0; r < 3; ++r) J[r][cc] = s_x[3 * gl[cc + 1] + r] - s_x[3 * gl[0] + r];
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    const double id = 1.0 / det;
    double G[4][3];
    G[1][0] = c00 * id;
    G[1][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
    G[1][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
    G[2][0] = c01 * id;
    G[2][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
    G[2][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
    G[3][0] = c02 * id;
    G[3][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
    G[3][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
#pragma unroll
    for (int d = 0; d < 3; ++d) G[0][d] = -(G[1][d] + G[2][d] + G[3][d]);
    const double kc = a.coef_kind == FE_COEFF_DG0 ? __ldg(a.coef + __ldg(a.cell_id + cb)) : a.coef_const;
    const double sc = fabs(det) * (1.0 / 6.0) * kc;
    double g2 = 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) g2 = fmax(g2, G[i][0] * G[i][0] + G[i][1] * G[i][1] + G[i][2] * G[i][2]);
    if (!(fabs(sc) * g2 < fs.direct_below)) {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = i; j < 4; ++j) emit(i, j, sc * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]));
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = i; j < 4; ++j)
          emit_direct(i, j, sc * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]));
    }
  }
  __syncthreads();
  const double inv = 1.0 / fs.scale;  // exact: a power of two
  // flat flush: consecutive lanes take consecutive window slots
  for (int w = tid; w < wtot; w += NT) {
    const uint32_t lo = w0[w], hi = w1[w];
    if (lo | hi) {
      const int r = s_wrow[w];
      // hi * 2^32 + lo, rounded once to double (both halves convert exactly)
      const double v = fma((double)(int32_t)hi, 4294967296.0, (double)lo);
      atomicAdd(a.values + s_gbase[r] + (w - s_soff[r]), v * inv);
    }
  }
}

uint64_t spread3b(uint64_t v) {
  v &= 0x1fffff;
  v = (v | v << 32) & 0x1f00000000ffffull;
  v = (v | v << 16) & 0x1f0000ff0000ffull;
  v = (v | v << 8) & 0x100f00f00f00f00full;
  v = (v | v << 4) & 0x10c30c30c30c30c3ull;
  v = (v | v << 2) & 0x1249249249249249ull;
  return v;
}

template <int KIND>
std::unique_ptr<fe_form_s::BlockPlan> build_block_plan(const fe_form_s& f) {
  using Tr = BlockTraits<KIND>;
  constexpr int K = Tr::K, KK = K * K;
  const fe_dofmap_s& V0 = *f.V0;
  const fe_dofmap_s& V1 = *f.V1;
  const int64_t C = V0.num_cells;
  const std::vector<int32_t>& rp = f.sp->host_row_ptr;
  const std::vector<double>& X = f.mesh->host_x;
  const std::vector<int32_t>& G = f.mesh->host_geom;

  // a slot collects at most one contribution per cell of its row: with
  // |w| < 2^S per contribution and at most maxcnt of them, S = 62 -
  // ceil(log2(maxcnt + 1)) keeps every slot sum below 2^62 (S <= 57; at least
  // 54 for the 255-cell limit)
  int fx_bits = 57;
  {
    std::vector<int32_t> cnt(V0.num_blocks, 0);
    int32_t maxcnt = 0;
    for (int64_t q = 0; q < C * K; ++q) {
      if (++cnt[V0.host[q]] > 255) FE_FAIL(FE_ERR_ARG, "a dof lies in more than 255 cells (block variant limit)");
      maxcnt = std::max(maxcnt, cnt[V0.host[q]]);
    }
    int bits = 0;
    while ((1 << bits) < maxcnt + 1) ++bits;
    fx_bits = std::min(57, 62 - bits);
  }

  // 1. Morton order of cell centroids
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (size_t v = 0; v < X.size() / 3; ++v)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], X[3 * v + d]);
      hi[d] = std::max(hi[d], X[3 * v + d]);
    }
  std::vector<std::pair<uint64_t, int32_t>> key(C);
  for (int64_t c = 0; c < C; ++c) {
    uint64_t m[3];
    for (int d = 0; d < 3; ++d) {
      double s = 0.0;
      for (int v = 0; v < 4; ++v) s += X[3 * (int64_t)G[4 * c + v] + d];
      const double u = (s * 0.25 - lo[d]) / std::max(hi[d] - lo[d], 1e-300);
      m[d] = (uint64_t)(std::min(std::max(u, 0.0), 1.0) * 2097151.0);
    }
    key[c] = {spread3b(m[0]) | (spread3b(m[1]) << 1) | (spread3b(m[2]) << 2), (int32_t)c};
  }
  std::sort(key.begin(), key.end());

  // 2. blocks: consecutive cells along the curve while the window fits
  std::vector<int32_t> block_ptr(1, 0), brow_ptr(1, 0), rows, soff;
  std::vector<uint16_t> lrow(C * K);
  std::vector<int32_t> mark(V0.num_blocks, -1), local(V0.num_blocks, 0);
  // geometry nodes per block (the P1 kernel stages their coordinates)
  const int64_t nnodes = (int64_t)X.size() / 3;
  std::vector<int32_t> gmark(nnodes, -1), glocal_of(nnodes, 0), gvert_ptr(1, 0), gverts;
  std::vector<uint16_t> glocal(C * 4);
  int64_t q = 0;
  while (q < C) {
    const int32_t bid = (int32_t)block_ptr.size() - 1;
    std::vector<int32_t> brows, bverts;
    int64_t wsize = 0, start = q;
    while (q < C && q - start < Tr::BMAX) {
      const int64_t c = key[q].second;
      int64_t addv = 0;
      for (int v = 0; v < 4; ++v) {
        const int32_t g = G[c * 4 + v];
        bool dup = gmark[g] == bid;
        for (int u = 0; u < v; ++u) dup |= G[c * 4 + u] == g;
        if (!dup) ++addv;
      }
      if (q > start && (int64_t)bverts.size() + addv > Tr::VCAP) break;
      int64_t add = 0, addr = 0;
      for (int i = 0; i < K; ++i) {
        const int32_t R = V0.host[c * K + i];
        if (mark[R] != bid) {
          bool dup = false;
          for (int u = 0; u < i; ++u) dup |= V0.host[c * K + u] == R;
          if (!dup) {
            add += rp[R + 1] - rp[R];
            ++addr;
          }
        }
      }
      if (q > start && (wsize + add > Tr::WCAP || (int64_t)brows.size() + addr > Tr::RCAP)) break;
      if (add > Tr::WCAP || addr > Tr::RCAP) FE_FAIL(FE_ERR_ARG, "a cell's rows exceed the block window");
      for (int i = 0; i < K; ++i) {
        const int32_t R = V0.host[c * K + i];
        if (mark[R] != bid) {
          mark[R] = bid;
          brows.push_back(R);
        }
      }
      for (int v = 0; v < 4; ++v) {
        const int32_t g = G[c * 4 + v];
        if (gmark[g] != bid) {
          gmark[g] = bid;
          glocal_of[g] = (int32_t)bverts.size();
          bverts.push_back(g);
        }
      }
      wsize += add;
      ++q;
    }
    for (int64_t p = start; p < q; ++p) {
      const int64_t c = key[p].second;
      for (int v = 0; v < 4; ++v) glocal[p * 4 + v] = (uint16_t)glocal_of[G[c * 4 + v]];
    }
    gverts.insert(gverts.end(), bverts.begin(), bverts.end());
    gvert_ptr.push_back((int32_t)gverts.size());
    std::sort(brows.begin(), brows.end());
    int32_t off = 0;
    for (size_t u = 0; u < brows.size(); ++u) {
      local[brows[u]] = (int32_t)u;
      rows.push_back(brows[u]);
      soff.push_back(off);
      off += rp[brows[u] + 1] - rp[brows[u]];
    }
    for (int64_t p = start; p < q; ++p) {
      const int64_t c = key[p].second;
      for (int i = 0; i < K; ++i) lrow[p * K + i] = (uint16_t)local[V0.host[c * K + i]];
    }
    block_ptr.push_back((int32_t)q);
    brow_ptr.push_back((int32_t)rows.size());
  }

  // geometric part of the entry bound per block (the kernel multiplies in the
  // coefficient factor and the reference-tensor constant):
  //   P1: |det J|/6 * max_i |grad phi_i|^2;  P2: sum_s |Ghat_s|
  std::vector<double> gbound(block_ptr.size() - 1, 0.0);
  for (size_t b = 0; b + 1 < block_ptr.size(); ++b) {
    double gb = 0.0;
    for (int64_t p = block_ptr[b]; p < block_ptr[b + 1]; ++p) {
      const int64_t c = key[p].second;
      double J[3][3], x0[3];
      for (int r = 0; r < 3; ++r) x0[r] = X[3 * (int64_t)G[4 * c] + r];
      for (int cc = 0; cc < 3; ++cc)
        for (int r = 0; r < 3; ++r) J[r][cc] = X[3 * (int64_t)G[4 * c + cc + 1] + r] - x0[r];
      const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
      const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
      const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
      const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
      const double id = 1.0 / det;
      double Km[3][3];
      Km[0][0] = c00 * id;
      Km[1][0] = c01 * id;
      Km[2][0] = c02 * id;
      Km[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
      Km[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
      Km[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
      Km[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
      Km[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
      Km[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
      const double adet = std::fabs(det);
      double v = 0.0;
      if (KIND == FE_FORM_P1_STIFFNESS) {
        for (int i = 0; i < 4; ++i) {
          double g2 = 0.0;
          for (int d = 0; d < 3; ++d) {
            const double g = (i == 0) ? -(Km[0][d] + Km[1][d] + Km[2][d]) : Km[i - 1][d];
            g2 += g * g;
          }
          v = std::max(v, g2);
        }
        v *= adet / 6.0;
      } else {
        const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
        for (int s = 0; s < 6; ++s)
          v += std::fabs(adet * (Km[pa[s]][0] * Km[pb[s]][0] + Km[pa[s]][1] * Km[pb[s]][1] +
                                 Km[pa[s]][2] * Km[pb[s]][2]));
      }
      gb = std::max(gb, v);
    }
    gbound[b] = gb;
  }

  // 3. per-cell arrays in block order
  std::vector<int32_t> cell_id(C), geom(C * 4), d0(C * K), d1(C * K), cmap;
  std::vector<uint8_t> pos(C * KK);
  std::vector<uint8_t> hpos((size_t)C * KK);
  if (C) FE_CUDA(cudaMemcpy(hpos.data(), f.pos.p, (size_t)C * KK, cudaMemcpyDeviceToHost));
  const Coefficient& kc = f.coeff[0];
  const bool p1coef = kc.kind == FE_COEFF_P1 && kc.map;
  if (p1coef) cmap.resize(C * 4);
  for (int64_t p = 0; p < C; ++p) {
    const int64_t c = key[p].second;
    cell_id[p] = (int32_t)c;
    for (int v = 0; v < 4; ++v) geom[p * 4 + v] = G[c * 4 + v];
    for (int i = 0; i < K; ++i) {
      d0[p * K + i] = V0.host[c * K + i];
      d1[p * K + i] = V1.host[c * K + i];
    }
    std::copy(hpos.begin() + c * KK, hpos.begin() + (c + 1) * KK, pos.begin() + p * KK);
    if (p1coef)
      for (int v = 0; v < 4; ++v) cmap[p * 4 + v] = kc.map->host[c * 4 + v];
  }

  // P1: the kernel's lane l takes the block's cells l*span + slot (32 cells
  // span apart per instruction, so their window rows rarely collide); the
  // per-cell records are stored at slot*32 + lane of the block's padded range
  // so that each of those loads is one coalesced warp access
  std::vector<int32_t> rec_ptr;
  if (KIND == FE_FORM_P1_STIFFNESS) {
    const int64_t nb = (int64_t)block_ptr.size() - 1;
    rec_ptr.assign(nb + 1, 0);
    for (int64_t b = 0; b < nb; ++b) {
      const int64_t n = block_ptr[b + 1] - block_ptr[b], span = (n + 31) / 32;
      rec_ptr[b + 1] = rec_ptr[b] + (int32_t)(span * 32);
    }
    const int64_t NR = rec_ptr[nb];
    std::vector<uint16_t> lrow_r(NR * K, 0), glocal_r(NR * 4, 0);
    std::vector<int32_t> cell_r(NR, 0), d1_r(NR * K, 0);
    std::vector<uint8_t> pos_r(NR * KK, 0);
    for (int64_t b = 0; b < nb; ++b) {
      const int64_t n = block_ptr[b + 1] - block_ptr[b], span = (n + 31) / 32;
      for (int64_t qq = 0; qq < n; ++qq) {
        const int64_t p = block_ptr[b] + qq;
        const int64_t r = rec_ptr[b] + (qq % span) * 32 + qq / span;
        std::copy(lrow.begin() + p * K, lrow.begin() + (p + 1) * K, lrow_r.begin() + r * K);
        std::copy(glocal.begin() + p * 4, glocal.begin() + (p + 1) * 4, glocal_r.begin() + r * 4);
        std::copy(pos.begin() + p * KK, pos.begin() + (p + 1) * KK, pos_r.begin() + r * KK);
        std::copy(d1.begin() + p * K, d1.begin() + (p + 1) * K, d1_r.begin() + r * K);
        cell_r[r] = cell_id[p];
      }
    }
    lrow.swap(lrow_r);
    glocal.swap(glocal_r);
    pos.swap(pos_r);
    d1.swap(d1_r);
    cell_id.swap(cell_r);
  }

  auto P = std::make_unique<fe_form_s::BlockPlan>();
  P->nblocks = (int64_t)block_ptr.size() - 1;
  P->fx_bits = fx_bits;
  P->coef_map_owner = p1coef ? kc.map : nullptr;
  auto up = [](auto& d, const auto& h) {
    using E = typename std::decay_t<decltype(h)>::value_type;
    d.alloc(std::max<size_t>(1, h.size()));
    if (!h.empty()) FE_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(E), cudaMemcpyHostToDevice));
  };
  up(P->block_ptr, block_ptr);
  up(P->brow_ptr, brow_ptr);
  up(P->rows, rows);
  up(P->soff, soff);
  up(P->lrow, lrow);
  up(P->cell_id, cell_id);
  up(P->geom, geom);
  up(P->dofs0, d0);
  up(P->dofs1, d1);
  up(P->pos, pos);
  if (p1coef) up(P->coef_map, cmap);
  up(P->gbound, gbound);
  if (KIND == FE_FORM_P1_STIFFNESS) {
    std::vector<double> gx(gverts.size() * 3);
    for (size_t u = 0; u < gverts.size(); ++u)
      for (int d = 0; d < 3; ++d) gx[3 * u + d] = X[3 * (int64_t)gverts[u] + d];
    up(P->gvert_ptr, gvert_ptr);
    up(P->gx, gx);
    up(P->glocal, glocal);
    up(P->rec_ptr, rec_ptr);
  }
  return P;
}

template <int KIND, typename T>
void launch_block(const fe_form_s& f, const fe_form_s::BlockPlan& P, double* values, const fe_bc_s* bc0,
                  const fe_bc_s* bc1, cudaStream_t s) {
  BlockArgs a{};
  a.block_ptr = P.block_ptr.p;
  a.brow_ptr = P.brow_ptr.p;
  a.rows = P.rows.p;
  a.soff = P.soff.p;
  a.lrow = P.lrow.p;
  a.cell_id = P.cell_id.p;
  a.geom = reinterpret_cast<const int4*>(P.geom.p);
  a.dofs0 = P.dofs0.p;
  a.dofs1 = P.dofs1.p;
  a.pos = P.pos.p;
  a.coef_map = reinterpret_cast<const int4*>(P.coef_map.p);
  a.x = f.mesh->x.p;
  a.row_ptr = f.sp->row_ptr.p;
  a.bc0 = bc0 ? bc0->markers.p : nullptr;
  a.bc1 = bc1 ? bc1->markers.p : nullptr;
  const Coefficient& k = f.coeff[0];
  a.coef_kind = k.kind < 0 ? FE_COEFF_CONSTANT : k.kind;
  a.coef = k.values;
  a.coef_const = k.kind < 0 ? 1.0 : k.constant[0];
  a.gbound = P.gbound.p;
  a.fx_bits = P.fx_bits;
  if (KIND == FE_FORM_P1_STIFFNESS) a.term_max = 1.0;
  else a.term_max = (a.coef_kind == FE_COEFF_P1) ? kP2P1CoefTermMax : kP2ConstTermMax;
  a.values = values;
  a.gvert_ptr = P.gvert_ptr.p;
  a.gx = P.gx.p;
  a.glocal = P.glocal.p;
  a.rec_ptr = P.rec_ptr.p;
  if (P.nblocks == 0) return;
  if constexpr (KIND == FE_FORM_P1_STIFFNESS) {
    constexpr size_t smem = P1Smem::SMEM;
    FE_CUDA(cudaFuncSetAttribute(k_block_p1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_block_p1<<<(unsigned)P.nblocks, BlockTraits<KIND>::NT, smem, s>>>(a, f.V0 == f.V1 ? 1 : 0);
    FE_CUDA(cudaGetLastError());
    return;
  }
  auto kern = k_block<KIND, T>;
  constexpr size_t smem = BlockSmem<KIND>::SMEM;
  FE_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)P.nblocks, BlockTraits<KIND>::NT, smem, s>>>(a);
  FE_CUDA(cudaGetLastError());
}

}  // namespace

void reset_block_plan(fe_form_s& f) { f.blocks.reset(); }

bool block_supported(const fe_form_s& f) { return tile_supported(f); }

void assemble_matrix_block(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, bool zero,
                           double diagonal, cudaStream_t s) {
  const Coefficient& kc = f.coeff[0];
  const fe_dofmap_s* want_map = (kc.kind == FE_COEFF_P1) ? kc.map : nullptr;
  if (f.blocks && f.blocks->coef_map_owner != want_map) f.blocks.reset();  // coefficient space changed
  if (!f.blocks)
    f.blocks = (f.kind == FE_FORM_P1_STIFFNESS) ? build_block_plan<FE_FORM_P1_STIFFNESS>(f)
                                                : build_block_plan<FE_FORM_P2_STIFFNESS>(f);
  // BC rows take no window flush and no direct reduction: their diagonal is
  // written with the zero pass
  if (zero) launch_zero_diagonal(*f.sp, bc0, diagonal, values, s);
  if (f.kind == FE_FORM_P1_STIFFNESS)
    launch_block<FE_FORM_P1_STIFFNESS, double>(f, *f.blocks, values, bc0, bc1, s);
  else if (f.precision == FE_PREC_FP32)
    launch_block<FE_FORM_P2_STIFFNESS, float>(f, *f.blocks, values, bc0, bc1, s);
  else
    launch_block<FE_FORM_P2_STIFFNESS, double>(f, *f.blocks, values, bc0, bc1, s);
  if (!zero && bc0) launch_set_diagonal(*f.sp, *bc0, diagonal, values, s);
}

}  // namespace fe
