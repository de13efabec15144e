// Row-gather matrix assembly for P1 stiffness.
//
// One warp per CSR row: the lanes take the row's incidences (cell c, local
// vertex i) from an inverse dofmap built once, each lane recomputes the
// (cheap) P1 geometry of its cell and adds row i of the element matrix into a
// per-warp shared row buffer at the cell's slot bytes; then the warp writes
// the row segment once, coalesced.  There are no global atomics and no zero
// pass: every CSR value is written exactly once per assembly.  Rows of BC
// dofs are written as zeros (set_diagonal runs afterwards, as in the
// reference, CUDAAssembler.cpp:131-164); columns of BC dofs are skipped
// (CUDAFormIntegral.cpp:1195-1213).
#include <cuda_runtime.h>

#include "fe_internal.h"

namespace fe {
namespace {

constexpr int kWarps = 8;       // warps per CTA
constexpr int kRowBuf = 64;     // doubles per warp row buffer (longest supported row)

struct RowArgs {
  int64_t num_rows;
  const int32_t* __restrict__ inc_ptr;
  const int32_t* __restrict__ inc;  // c*4 + i
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  const int32_t* __restrict__ dofs1;
  const uint32_t* __restrict__ pos;  // 4 slot bytes per (cell, i)
  const int32_t* __restrict__ row_ptr;
  const uint8_t* __restrict__ bc0;
  const uint8_t* __restrict__ bc1;
  int coef_kind;
  const double* __restrict__ coef;
  double coef_const;
  int zero;
  double* __restrict__ values;
};

__global__ void __launch_bounds__(kWarps * 32) k_row_p1(const RowArgs a) {
  __shared__ double buf[kWarps][kRowBuf];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* rb = buf[warp];
  const int64_t nwarps = (int64_t)gridDim.x * kWarps;
  for (int64_t R = blockIdx.x * (int64_t)kWarps + warp; R < a.num_rows; R += nwarps) {
    const int32_t lo = __ldg(a.row_ptr + R);
    const int L = __ldg(a.row_ptr + R + 1) - lo;  // <= kRowBuf (checked when the plan is built)
    for (int l = lane; l < L; l += 32) rb[l] = 0.0;
    __syncwarp();
    const bool rmask = a.bc0 && a.bc0[R];
    if (!rmask) {
      const int32_t i0 = __ldg(a.inc_ptr + R), n = __ldg(a.inc_ptr + R + 1) - i0;
      for (int t = lane; t < n; t += 32) {
        const int32_t e = __ldg(a.inc + i0 + t);
        const int64_t c = e >> 2;
        const int i = e & 3;
        const int4 v = __ldg(reinterpret_cast<const int4*>(a.geom) + c);
        const int vv[4] = {v.x, v.y, v.z, v.w};
        double X[4][3];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int d = 0; d < 3; ++d) X[q][d] = __ldg(a.x + 3 * (int64_t)vv[q] + d);
        double J[3][3];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc)
#pragma unroll
          for (int r = 0; r < 3; ++r) J[r][cc] = X[cc + 1][r] - X[0][r];
        const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
        const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
        const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
        const double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
        const double id = 1.0 / det;
        double K[3][3];
        K[0][0] = c00 * id;
        K[1][0] = c01 * id;
        K[2][0] = c02 * id;
        K[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
        K[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
        K[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
        K[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
        K[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
        K[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
        double G[4][3];
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          G[1][b] = K[0][b];
          G[2][b] = K[1][b];
          G[3][b] = K[2][b];
          G[0][b] = -(K[0][b] + K[1][b] + K[2][b]);
        }
        const double k = a.coef_kind == FE_COEFF_DG0 ? __ldg(a.coef + c) : a.coef_const;
        const double s = fabs(det) * (1.0 / 6.0) * k;
        double gi[3];
#pragma unroll
        for (int b = 0; b < 3; ++b) gi[b] = (i == 0) ? G[0][b] : (i == 1 ? G[1][b] : (i == 2 ? G[2][b] : G[3][b]));
        const uint32_t pw = __ldg(a.pos + c * 4 + i);
        unsigned cm = 0;
        if (a.bc1) {
          const int4 d1 = __ldg(reinterpret_cast<const int4*>(a.dofs1) + c);
          cm = (a.bc1[d1.x] ? 1u : 0u) | (a.bc1[d1.y] ? 2u : 0u) | (a.bc1[d1.z] ? 4u : 0u) | (a.bc1[d1.w] ? 8u : 0u);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if ((cm >> j) & 1u) continue;
          const double val = s * (gi[0] * G[j][0] + gi[1] * G[j][1] + gi[2] * G[j][2]);
          atomicAdd(rb + ((pw >> (8 * j)) & 0xffu), val);
        }
      }
    }
    __syncwarp();
    for (int l = lane; l < L; l += 32) {
      double val = rb[l];
      if (!a.zero) val += a.values[lo + l];
      a.values[lo + l] = val;
    }
    __syncwarp();
  }
}

}  // namespace

bool rowgather_supported(const fe_form_s& f) {
  return f.kind == FE_FORM_P1_STIFFNESS && f.V0 && f.V1 && f.V0->bs == 1 && f.V1->bs == 1 &&
         f.coeff[0].kind != FE_COEFF_P1;
}

void reset_row_plan(fe_form_s& f) { f.rows.reset(); }

void assemble_matrix_rowgather(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, bool zero,
                               cudaStream_t s) {
  const fe_dofmap_s& V0 = *f.V0;
  if (!f.rows) {
    // inverse dofmap: per block row the incidences (cell*4 + i), ascending
    const int64_t C = V0.num_cells, nR = V0.num_blocks;
    const std::vector<int32_t>& rp = f.sp->host_row_ptr;
    for (int64_t R = 0; R < nR; ++R)
      if (rp[R + 1] - rp[R] > kRowBuf)
        FE_FAIL(FE_ERR_ARG, "row-gather supports rows of at most " + std::to_string(kRowBuf) + " entries");
    if (C * 4 > INT32_MAX) FE_FAIL(FE_ERR_ARG, "too many cells for the row-gather plan");
    std::vector<int32_t> ptr(nR + 1, 0), inc(C * 4);
    for (int64_t q = 0; q < C * 4; ++q) ptr[V0.host[q] + 1]++;
    for (int64_t R = 0; R < nR; ++R) ptr[R + 1] += ptr[R];
    std::vector<int32_t> cur(ptr.begin(), ptr.end() - 1);
    for (int64_t q = 0; q < C * 4; ++q) inc[cur[V0.host[q]]++] = (int32_t)q;  // q = c*4 + i
    auto P = std::make_unique<fe_form_s::RowPlan>();
    P->inc_ptr.alloc(ptr.size());
    P->inc.alloc(std::max<size_t>(1, inc.size()));
    FE_CUDA(cudaMemcpy(P->inc_ptr.p, ptr.data(), ptr.size() * 4, cudaMemcpyHostToDevice));
    if (!inc.empty()) FE_CUDA(cudaMemcpy(P->inc.p, inc.data(), inc.size() * 4, cudaMemcpyHostToDevice));
    f.rows = std::move(P);
  }
  RowArgs a{};
  a.num_rows = V0.num_blocks;
  a.inc_ptr = f.rows->inc_ptr.p;
  a.inc = f.rows->inc.p;
  a.x = f.mesh->x.p;
  a.geom = f.mesh->geom.p;
  a.dofs1 = f.V1->dofs.p;
  a.pos = reinterpret_cast<const uint32_t*>(f.pos.p);
  a.row_ptr = f.sp->row_ptr.p;
  a.bc0 = bc0 ? bc0->markers.p : nullptr;
  a.bc1 = bc1 ? bc1->markers.p : nullptr;
  const Coefficient& k = f.coeff[0];
  a.coef_kind = k.kind < 0 ? FE_COEFF_CONSTANT : k.kind;
  a.coef = k.values;
  a.coef_const = k.kind < 0 ? 1.0 : k.constant[0];
  a.zero = zero ? 1 : 0;
  a.values = values;
  if (a.num_rows == 0) return;
  const int64_t blocks_needed = (a.num_rows + kWarps - 1) / kWarps;
  const unsigned grid = (unsigned)std::min<int64_t>(blocks_needed, (int64_t)f.ctx->num_sms * 16);
  k_row_p1<<<grid, kWarps * 32, 0, s>>>(a);
  FE_CUDA(cudaGetLastError());
}

}  // namespace fe
