// Batched assembly: many coefficient instances of one bilinear form on one
// mesh and one sparsity pattern, written into as many caller-owned CSR value
// arrays.
//
// The reference assembles one form instance per call (python/cudolfinx/
// assemble.py:52-110, one launch of CUDAFormIntegral.cpp:1103-1226 per
// matrix); it has no batch path.  For a cellwise-constant (DG0) coefficient k
// the element matrix of instance s is k_s(c) * A_c, with A_c the element
// matrix of the unit coefficient, so
//     A_s[slot] = sum over the slot's element entries (c, e) of k_s(c) * A_c[e].
// The batch computes A_c once per call, in FP32 (geometry, Jacobian,
// determinant and inverse in FP64; each diagonal entry is minus the FP64 sum
// of its row's FP32 off-diagonal entries, so element rows sum to zero as the
// exact ones do), and then forms every instance's values with FP64
// accumulation in one persistent launch:
//   k_batch_elem_*  unit-coefficient element tensors E[c][i*K+j]     } once per
//   k_batch_fill    rec[r] = {E of record r, cell of record r}, records } mesh and
//                   in slot order (the sorted-slot plan of fe_gather.cu)  } pattern
//   k_batch_fused   one persistent cooperative launch per call: k_s(c)
//                   (FP64, one array per instance) -> kp[c][s] (FP32), a
//                   tiled transpose (the batch's pack_coefficients); a grid
//                   barrier; then the gather, one warp per (8 slots x 32*IPL
//                   instances):
//                   lane = instance while summing a slot's records (the
//                   coefficient row kp[c][..] is one coalesced load), lane =
//                   slot while storing (a staging tile in shared memory turns
//                   the result so each instance's 8 slots go out as one
//                   64-byte store, four instances per instruction).  BC rows/columns and the BC diagonal are
//                   applied in the store.
// Every instance's slot sum runs in the plan's fixed record order, so the
// result is bitwise reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <type_traits>

#include "fe_element_code.cuh"
#include "fe_internal.h"

namespace fe {
namespace {

constexpr int kMaxBatchLaunch = 384;  // instances per launch: the pointer tables travel as kernel
                                       // parameters (< 4 KB); a multiple of 128 keeps chunks aligned
constexpr int kSlotsPerItem = 8;  // slots per gather work item

unsigned nblocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// slot-sorted record: unit element-tensor entry (FP32 value, held as double)
// and its cell
struct alignas(16) BatchRec {
  double ae;
  int32_t cell;
  int32_t pad;
};

// ---- plan ----------------------------------------------------------------
__global__ void k_plan_records(const int32_t* __restrict__ contrib, int64_t nrec, int64_t num_cells,
                               int32_t* __restrict__ rec_cell, uint8_t* __restrict__ rec_entry) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  const int64_t id = contrib[r];  // entry * num_cells + cell
  const int64_t e = id / num_cells;
  rec_cell[r] = (int32_t)(id - e * num_cells);
  rec_entry[r] = (uint8_t)e;
}

__global__ void k_plan_slot_row(const int32_t* __restrict__ row_ptr, int64_t num_rows, int32_t* __restrict__ slot_row) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= num_rows) return;
  for (int32_t s = row_ptr[r]; s < row_ptr[r + 1]; ++s) slot_row[s] = (int32_t)r;
}

// ---- unit-coefficient element tensors (FP32 out, FP64 geometry) ----------
struct ElemArgs {
  int64_t num_cells;
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  double* __restrict__ E;
};

struct Geo {
  double K[3][3];
  double adet;
};

__device__ __forceinline__ void geometry(const double* __restrict__ x, const int32_t* __restrict__ geom, int64_t c,
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

__global__ void k_batch_elem_p1(const ElemArgs a) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= a.num_cells) return;
  Geo g;
  geometry(a.x, a.geom, c, g);
  double G[4][3];
#pragma unroll
  for (int b = 0; b < 3; ++b) {
    G[1][b] = g.K[0][b];
    G[2][b] = g.K[1][b];
    G[3][b] = g.K[2][b];
    G[0][b] = -(g.K[0][b] + g.K[1][b] + g.K[2][b]);
  }
  // FP32 off-diagonal entries; each diagonal entry is minus the FP64 sum of
  // its row's off-diagonal entries, so every element row sums to zero exactly
  const double s = g.adet * (1.0 / 6.0);
  double v[16];
  double rs[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = i + 1; j < 4; ++j) {
      const double e = (double)(float)(s * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]));
      v[i * 4 + j] = e;
      v[j * 4 + i] = e;
      rs[i] += e;
      rs[j] += e;
    }
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i * 5] = -rs[i];
  double2* out = reinterpret_cast<double2*>(a.E + c * 16);
#pragma unroll
  for (int q = 0; q < 8; ++q) out[q] = make_double2(v[2 * q], v[2 * q + 1]);
}

__global__ void k_batch_elem_p2(const ElemArgs a) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= a.num_cells) return;
  Geo g;
  geometry(a.x, a.geom, c, g);
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
  float gq[6];
#pragma unroll
  for (int s = 0; s < 6; ++s)
    gq[s] = (float)(g.adet * (g.K[pa[s]][0] * g.K[pb[s]][0] + g.K[pa[s]][1] * g.K[pb[s]][1] +
                              g.K[pa[s]][2] * g.K[pb[s]][2]));
  double* __restrict__ E = a.E + c * 100;
  p2_stiffness_const<float>(gq, [&](int i, int j, double v) {
    E[i * 10 + j] = v;
    if (i != j) E[j * 10 + i] = v;
  });
}

__global__ void k_batch_fill(const int32_t* __restrict__ rec_cell, const uint8_t* __restrict__ rec_entry,
                             int64_t nrec, int KK, const double* __restrict__ E, BatchRec* __restrict__ rec) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  const int32_t c = rec_cell[r];
  rec[r] = BatchRec{__ldg(E + (int64_t)c * KK + rec_entry[r]), c, 0};
}

// ---- persistent gather ---------------------------------------------------
struct GatherArgs {
  int64_t nnz;
  int num_inst;        // instances in this launch
  int col0;            // kp column of the launch's first instance
  int64_t ld;          // kp row stride (floats)
  int64_t num_items;   // slot groups * instance chunks
  int num_chunks;
  const int32_t* seg;
  const BatchRec* rec;
  const float* kp;
  const int32_t* slot_row;
  const int32_t* col;
  const uint8_t* bc0;
  const uint8_t* bc1;
  double diagonal;
  int zero;
  double* values[kMaxBatchLaunch];
};

template <int IPL>
struct GatherCfg {
  static constexpr int CHUNK = 32 * IPL;        // instances per work item
  static constexpr int WARPS = 8;
  static constexpr int TSTRIDE = CHUNK + 1;     // doubles per staged slot
  static constexpr int MIN_BLOCKS = 3;          // 24 resident warps per SM
  static constexpr size_t WARP_SMEM = kSlotsPerItem * TSTRIDE * sizeof(double) + 32 * sizeof(BatchRec);
  static constexpr size_t SMEM = WARPS * WARP_SMEM;
};

constexpr unsigned kFull = 0xffffffffu;
constexpr int kLoadBatch = 8;  // coefficient loads in flight per warp

template <int IPL>
struct KVec;
template <>
struct KVec<1> {
  using T = float;
  static __device__ __forceinline__ double at(const float& v, int) { return (double)v; }
};
template <>
struct KVec<2> {
  using T = float2;
  static __device__ __forceinline__ double at(const float2& v, int t) { return (double)(t ? v.y : v.x); }
};
template <>
struct KVec<4> {
  using T = float4;
  static __device__ __forceinline__ double at(const float4& v, int t) {
    return (double)(t == 0 ? v.x : t == 1 ? v.y : t == 2 ? v.z : v.w);
  }
};

// One warp per work item (kSlotsPerItem consecutive slots x CHUNK instances;
// lane l holds instances l*IPL .. l*IPL+IPL-1 of the chunk).  The item's
// records are a contiguous range, read 32 at a time with one coalesced load
// into a per-warp buffer and broadcast from there, so the coefficient loads
// (one coalesced CHUNK-wide row segment per record) do not wait on a record
// load and kLoadBatch of them are in flight.  Staged results use column
// (i % IPL) * 32 + i / IPL for instance i, so the per-lane writes are
// conflict-free.
// kp loads: through the read-only path when kp was written by an earlier
// launch, at L2 (ld.global.cg) when this launch wrote it before its grid
// barrier (loading those lines through L1 measured no faster: 2.91 ms per
// 256-instance call either way)
template <bool WRITTEN_HERE, typename KV>
__device__ __forceinline__ KV load_kp(const KV* p) {
  if constexpr (WRITTEN_HERE) return __ldcg(p);
  else return __ldg(p);
}

template <int IPL, bool WRITTEN_HERE>
__device__ __forceinline__ void gather_items(const GatherArgs& a, unsigned char* smem_raw) {
  using Cfg = GatherCfg<IPL>;
  using KV = typename KVec<IPL>::T;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned char* wbase = smem_raw + wid * Cfg::WARP_SMEM;
  BatchRec* __restrict__ R = reinterpret_cast<BatchRec*>(wbase);
  double* __restrict__ T = reinterpret_cast<double*>(wbase + 32 * sizeof(BatchRec));
  const int64_t nw = (int64_t)gridDim.x * Cfg::WARPS;
  for (int64_t item = blockIdx.x * (int64_t)Cfg::WARPS + wid; item < a.num_items; item += nw) {
    const uint32_t g32 = (uint32_t)item / (uint32_t)a.num_chunks;  // items < 2^31 (host check)
    const int64_t g = g32;
    const int ioff = (int)((uint32_t)item - g32 * (uint32_t)a.num_chunks) * Cfg::CHUNK;
    const int64_t s0 = g * kSlotsPerItem;
    const int ns = (int)min((int64_t)kSlotsPerItem, a.nnz - s0);
    const KV* __restrict__ kb = reinterpret_cast<const KV*>(a.kp + a.col0 + ioff + lane * IPL);
    const int64_t ldv = a.ld / IPL;
    // lane l < ns holds the end of slot l's record list
    const int32_t my_end = lane < ns ? __ldg(a.seg + s0 + lane + 1) : INT32_MAX;
    const int32_t R0 = __ldg(a.seg + s0);
    const int32_t R1 = __shfl_sync(kFull, my_end, ns - 1);
    int j = 0;
    int32_t cur_end = __shfl_sync(kFull, my_end, 0);
    double acc[IPL];
#pragma unroll
    for (int t = 0; t < IPL; ++t) acc[t] = 0.0;
    auto flush = [&]() {
#pragma unroll
      for (int t = 0; t < IPL; ++t) {
        T[j * Cfg::TSTRIDE + t * 32 + lane] = acc[t];
        acc[t] = 0.0;
      }
      ++j;
    };
    auto consume = [&](int32_t rr, double ae, const KV& kv) {
      while (rr >= cur_end) {  // the current slot is complete
        flush();
        cur_end = __shfl_sync(kFull, my_end, j);
      }
#pragma unroll
      for (int t = 0; t < IPL; ++t) acc[t] = fma(ae, KVec<IPL>::at(kv, t), acc[t]);
    };
    for (int32_t base = R0; base < R1; base += 32) {
      const int cnt = min(32, R1 - base);
      __syncwarp();
      if (lane < cnt) R[lane] = a.rec[base + lane];
      __syncwarp();
      int q0 = 0;
      for (; q0 + kLoadBatch <= cnt; q0 += kLoadBatch) {
        KV kv[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) kv[u] = load_kp<WRITTEN_HERE>(kb + (int64_t)R[q0 + u].cell * ldv);
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) consume(base + q0 + u, R[q0 + u].ae, kv[u]);
      }
      if (q0 < cnt) {
        KV kv[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u)
          if (q0 + u < cnt) kv[u] = load_kp<WRITTEN_HERE>(kb + (int64_t)R[q0 + u].cell * ldv);
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u)
          if (q0 + u < cnt) consume(base + q0 + u, R[q0 + u].ae, kv[u]);
      }
    }
    while (j < ns) flush();  // the last slot (and any slot without records)
    __syncwarp();
    // store: lane = pair of consecutive slots (2p, 2p+1) of the item for one
    // instance; kSub lane groups take successive instances, so one store
    // instruction writes kSub instances' kSlotsPerItem consecutive values
    constexpr int kPairs = kSlotsPerItem / 2;
    constexpr int kSub = 32 / kPairs;
    const int p = lane % kPairs, sub = lane / kPairs;
    const int sa = 2 * p;
    if (sa < ns) {
      const int64_t slot = s0 + sa;
      const bool two = sa + 1 < ns;
      bool mask[2] = {false, false}, diag[2] = {false, false};
      if (a.bc0 || a.bc1) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (h == 0 || two) {
            const int32_t row = __ldg(a.slot_row + slot + h), cl = __ldg(a.col + slot + h);
            const bool rm = a.bc0 && a.bc0[row];
            mask[h] = rm || (a.bc1 && a.bc1[cl]);
            diag[h] = rm && row == cl;
          }
        }
      }
      const int nin = min(Cfg::CHUNK, a.num_inst - ioff);
      for (int i = sub; i < nin; i += kSub) {
        double* __restrict__ out = a.values[ioff + i] + slot;
        const int c = (i % IPL) * 32 + i / IPL;
        double v0 = a.zero ? 0.0 : out[0];
        double v1 = (a.zero || !two) ? 0.0 : out[1];
        if (!mask[0]) v0 += T[sa * Cfg::TSTRIDE + c];
        if (two && !mask[1]) v1 += T[(sa + 1) * Cfg::TSTRIDE + c];
        if (diag[0]) v0 = a.diagonal;
        if (diag[1]) v1 = a.diagonal;
        if (two && ((reinterpret_cast<uintptr_t>(out) & 15) == 0)) {
          *reinterpret_cast<double2*>(out) = make_double2(v0, v1);
        } else {
          out[0] = v0;
          if (two) out[1] = v1;
        }
      }
    }
    __syncwarp();
  }
}

// One persistent launch per batch of instances: phase 1 packs the instances'
// coefficients into kp (32 cells x 32 instances per tile, the transpose of
// a plain pack kernel), a grid barrier, phase 2 gathers (gather_items).  Launched
// cooperatively, so every block is resident and the barrier completes; its
// wait is still bounded: a block that waits too long sets DEV_ERR_BARRIER in
// the error word and returns.
struct FusedArgs {
  int64_t num_cells;
  int64_t pack_cols;    // kp columns this launch writes (its instances + trailing zero padding)
  const double* coef[kMaxBatchLaunch];
  float* kp;            // the packed coefficients the gather reads (g.kp)
  unsigned* barrier;    // zeroed before the launch
  unsigned* err;
  GatherArgs g;
};

constexpr long long kBarrierSpins = 1ll << 26;  // x ~100 ns: a few seconds

template <int IPL>
__global__ void __launch_bounds__(32 * GatherCfg<IPL>::WARPS, GatherCfg<IPL>::MIN_BLOCKS)
    k_batch_fused(const __grid_constant__ FusedArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float(*t)[33] = reinterpret_cast<float(*)[33]>(smem_raw);  // 32 x 33 floats of the gather buffers
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int64_t tiles_c = (a.num_cells + 31) / 32, tiles_s = (a.pack_cols + 31) / 32;
  for (int64_t tile = blockIdx.x; tile < tiles_c * tiles_s; tile += gridDim.x) {
    const int64_t c0 = (tile % tiles_c) * 32;
    const int s0 = (int)(tile / tiles_c) * 32;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int sl = ty + 8 * j, si = s0 + sl;
      const int64_t c = c0 + tx;
      t[sl][tx] = (si < a.g.num_inst && c < a.num_cells) ? (float)__ldg(a.coef[si] + c) : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int cl = ty + 8 * j;
      const int64_t c = c0 + cl;
      if (c < a.num_cells && s0 + tx < a.pack_cols) a.kp[c * a.g.ld + a.g.col0 + s0 + tx] = t[tx][cl];
    }
  }
  // grid barrier
  __shared__ int abort_flag;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(a.barrier, 1u);
    long long spins = 0;
    while (*(volatile unsigned*)a.barrier < gridDim.x && spins < kBarrierSpins) {
      __nanosleep(100);
      ++spins;
    }
    abort_flag = spins >= kBarrierSpins;
    if (abort_flag) atomicOr(a.err, DEV_ERR_BARRIER);
    __threadfence();
  }
  __syncthreads();
  if (abort_flag) return;
  gather_items<IPL, true>(a.g, smem_raw);
}

template <int IPL>
void launch_fused(FusedArgs& fa, int num_sms, cudaStream_t s) {
  using Cfg = GatherCfg<IPL>;
  // per device and cheap: set on every launch rather than cached
  FE_CUDA(cudaFuncSetAttribute(k_batch_fused<IPL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::SMEM));
  int per_sm = 0;
  FE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_fused<IPL>, 32 * Cfg::WARPS, Cfg::SMEM));
  const int64_t want = std::max<int64_t>((fa.g.num_items + Cfg::WARPS - 1) / Cfg::WARPS,
                                         ((fa.num_cells + 31) / 32) * ((fa.pack_cols + 31) / 32));
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)num_sms * std::max(1, per_sm)));
  FE_CUDA(cudaMemsetAsync(fa.barrier, 0, sizeof(unsigned), s));
  void* args[] = {&fa};
  FE_CUDA(cudaLaunchCooperativeKernel((const void*)k_batch_fused<IPL>, dim3((unsigned)grid), dim3(32 * Cfg::WARPS),
                                      args, Cfg::SMEM, s));
}

}  // namespace

bool batch_supported(const fe_form_s& f) {
  return (f.kind == FE_FORM_P1_STIFFNESS || f.kind == FE_FORM_P2_STIFFNESS) && f.V0 && f.V0->bs == 1;
}

void reset_batch_plan(fe_form_s& f) { f.batch.reset(); }

void assemble_matrix_batch(fe_form_s& f, int num_instances, const double* const* coefficients,
                           double* const* values, const fe_bc_s* bc0, const fe_bc_s* bc1, double diagonal,
                           bool zero, cudaStream_t s) {
  FE_REQUIRE(batch_supported(f), "batched assembly supports P1/P2 stiffness with a DG0 coefficient only");
  FE_REQUIRE(num_instances >= 0, "negative instance count");
  if (bc0) FE_REQUIRE(bc0->n_owned == bc0->n_bc, "batched assembly needs every BC dof owned");
  if (num_instances == 0) return;
  FE_REQUIRE(coefficients && values, "null coefficient or value table");
  const int64_t C = f.mesh->num_cells;
  const int64_t nnz = f.sp->nnz;
  for (int i = 0; i < num_instances; ++i) {
    FE_REQUIRE(coefficients[i] || C == 0, "null coefficient array");
    FE_REQUIRE(values[i] || nnz == 0, "null value array");
  }
  const int K = f.V0->k;
  const int KK = K * K;
  if (!f.batch) {
    ensure_gather_plan(f, s);
    auto B = std::make_unique<fe_form_s::BatchPlan>();
    B->num_records = f.gather->num_contrib;
    B->KK = KK;
    B->rec_cell.alloc(std::max<int64_t>(1, B->num_records));
    B->rec_entry.alloc(std::max<int64_t>(1, B->num_records));
    B->slot_row.alloc(std::max<int64_t>(1, nnz));
    B->E.alloc(std::max<int64_t>(1, C * KK));
    B->rec.alloc(std::max<int64_t>(1, B->num_records));
    if (B->num_records) {
      k_plan_records<<<nblocks(B->num_records, 256), 256, 0, s>>>(f.gather->contrib.p, B->num_records, C,
                                                                  B->rec_cell.p, B->rec_entry.p);
      FE_CUDA(cudaGetLastError());
    }
    if (f.sp->num_rows) {
      k_plan_slot_row<<<nblocks(f.sp->num_rows, 256), 256, 0, s>>>(f.sp->row_ptr.p, f.sp->num_rows, B->slot_row.p);
      FE_CUDA(cudaGetLastError());
    }
    f.batch = std::move(B);
  }
  auto& B = *f.batch;
  // packed coefficients: one row of ld floats per cell, resized on demand
  const int ipl = num_instances > 64 ? 4 : (num_instances > 32 ? 2 : 1);
  const int chunk = 32 * ipl;
  const int64_t ld = ((int64_t)num_instances + chunk - 1) / chunk * chunk;
  if (B.kp_ld != ld || !B.kp.p) {
    B.kp.alloc(std::max<int64_t>(1, C * ld));
    B.kp_ld = ld;
  }
  // the unit-coefficient element tensors and the slot-sorted records depend
  // only on the mesh (immutable once created) and the plan: built on the
  // first call
  if (C && !B.rec_valid) {
    ElemArgs ea{C, f.mesh->x.p, f.mesh->geom.p, B.E.p};
    if (f.kind == FE_FORM_P1_STIFFNESS) k_batch_elem_p1<<<nblocks(C, 128), 128, 0, s>>>(ea);
    else k_batch_elem_p2<<<nblocks(C, 128), 128, 0, s>>>(ea);
    FE_CUDA(cudaGetLastError());
    k_batch_fill<<<nblocks(B.num_records, 256), 256, 0, s>>>(B.rec_cell.p, B.rec_entry.p, B.num_records, KK, B.E.p,
                                                             reinterpret_cast<BatchRec*>(B.rec.p));
    FE_CUDA(cudaGetLastError());
    B.rec_valid = true;
  }
  if (!B.barrier.p) B.barrier.alloc(1);
  for (int i0 = 0; i0 < num_instances; i0 += kMaxBatchLaunch) {
    FusedArgs fa{};
    fa.num_cells = C;
    fa.kp = B.kp.p;
    fa.barrier = B.barrier.p;
    fa.err = device_error_word(f.ctx);
    GatherArgs& ga = fa.g;
    ga.nnz = nnz;
    ga.num_inst = std::min(kMaxBatchLaunch, num_instances - i0);
    // the last launch also zeroes the padding columns up to ld
    fa.pack_cols = (i0 + kMaxBatchLaunch >= num_instances) ? ld - i0 : ga.num_inst;
    for (int i = 0; i < ga.num_inst; ++i) fa.coef[i] = coefficients[i0 + i];
    ga.col0 = i0;
    ga.ld = ld;
    ga.num_chunks = (ga.num_inst + chunk - 1) / chunk;
    ga.num_items = nnz ? ((nnz + kSlotsPerItem - 1) / kSlotsPerItem) * ga.num_chunks : 0;
    FE_REQUIRE(ga.num_items < INT32_MAX, "batch too large for one gather launch");
    ga.seg = f.gather->seg.p;
    ga.rec = reinterpret_cast<const BatchRec*>(B.rec.p);
    ga.kp = B.kp.p;
    ga.slot_row = B.slot_row.p;
    ga.col = f.sp->col.p;
    ga.bc0 = bc0 ? bc0->markers.p : nullptr;
    ga.bc1 = bc1 ? bc1->markers.p : nullptr;
    ga.diagonal = diagonal;
    ga.zero = zero ? 1 : 0;
    for (int i = 0; i < ga.num_inst; ++i) ga.values[i] = values[i0 + i];
    if (!C && !nnz) continue;
    if (ipl == 4) launch_fused<4>(fa, f.ctx->num_sms, s);
    else if (ipl == 2) launch_fused<2>(fa, f.ctx->num_sms, s);
    else launch_fused<1>(fa, f.ctx->num_sms, s);
  }
}

}  // namespace fe
