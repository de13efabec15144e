// Grouped matrix assembly for P2 stiffness ("grouped" variant).
//
// The FP64-atomic scatter (fe_kernels.cu) issues one L2 reduction per
// element entry: 100 per P2 cell, 531 M for the 5.3 M-cell benchmark mesh,
// and the L2 reduction units (about 200-230 G entries/s on B200) bound it.
// Neighbouring cells share most of their couplings: within 48 cells that are
// close in space only about half of the 4800 entries land in distinct CSR
// slots.  This variant sums them on the SM first:
//   plan (host, once per form + pattern, from the dofmap only): the cells,
//     in the mesh's own order (meshes are ordered for locality -- DOLFINx
//     reorders its cells so -- so consecutive cells are neighbours), cut into
//     groups of 48; per group a group-local numbering of its dofs (first
//     appearance) and the "template": the group's distinct (row, column)
//     pairs in row-major order, each with the list of (cell, upper-triangle
//     entry) contributions.  Groups with the same local structure share one
//     template (the structured unit-cube meshes have one), and a template
//     does not depend on the global dof numbering.  A mesh whose groups repeat
//     no structure (more than 4096 templates) keeps the atomic scatter;
//   kernel (one CTA per group, after a zero pass): each thread computes one
//   cell's element tensor into shared memory (upper triangle, FP64); then the
//   threads walk the template's distinct entries, sum each one's
//   contributions in a fixed order and issue one reduction per distinct slot
//   (consecutive threads take consecutive columns of a row), with BC rows
//   and columns skipped as in the reference (CUDAFormIntegral.cpp:1195-1213).
// The slot of a distinct entry is row_ptr[row] + the byte map of its first
// contribution, so the plan adds no per-entry slot data.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <unordered_map>

#include "fe_element_code.cuh"
#include "fe_internal.h"

namespace fe {
namespace {

constexpr int kK = 10;                 // P2 dofs per cell
constexpr int kKK = kK * kK;
constexpr int kNU = kK * (kK + 1) / 2;  // upper-triangle entries
constexpr int kG = 48;                  // cells per group
constexpr int kThreads = 64;
constexpr int kMaxLocal = 255;          // group-local dofs (8-bit indices)

__host__ __device__ constexpr int upper_index(int i, int j) { return i * (2 * kK - i + 1) / 2 + (j - i); }

struct GroupArgs {
  int64_t num_cells;
  const int32_t* __restrict__ tmpl_of;    // [groups] template id
  const int4* __restrict__ tmeta;         // per template: entry offset, entries, contribution offset, first offset
  const int32_t* __restrict__ tnd;        // per template: group-local dofs
  const uint2* __restrict__ ent;          // {r | c << 8 | count << 16, start | pos index << 16}
  const uint16_t* __restrict__ contrib;   // cell << 9 | upper entry
  const uint16_t* __restrict__ first;     // group-local dof -> cell << 4 | local dof
  const double* __restrict__ x;
  const int32_t* __restrict__ geom;
  const int32_t* __restrict__ dofs;
  const uint8_t* __restrict__ pos;
  const int32_t* __restrict__ row_ptr;
  const uint8_t* __restrict__ bc0;
  const uint8_t* __restrict__ bc1;
  int coef_kind;
  const double* __restrict__ coef;
  const int32_t* __restrict__ coef_map;
  double coef_const;
  double* __restrict__ values;
};

__device__ __forceinline__ void geometry(const double* __restrict__ x, int4 v, double Gh[6]) {
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
  const double adet = fabs(det);
  const int pa[6] = {0, 1, 2, 0, 0, 1}, pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int s = 0; s < 6; ++s)
    Gh[s] = adet * (K[pa[s]][0] * K[pb[s]][0] + K[pa[s]][1] * K[pb[s]][1] + K[pa[s]][2] * K[pb[s]][2]);
}

template <typename T, int COEF>
__global__ void __launch_bounds__(kThreads, 7) k_mat_p2_grouped(const GroupArgs a) {
  __shared__ double Eu[kG * kNU];
  __shared__ __align__(16) uint8_t spos[kG * kKK];
  __shared__ int32_t sdof[kG * kK];
  __shared__ int32_t srp[kMaxLocal + 1];
  __shared__ uint8_t smask[kMaxLocal + 1];  // bit 0: BC row, bit 1: BC column
  const int tid = threadIdx.x;
  const int64_t g = blockIdx.x;
  const int64_t c0 = g * kG;
  const int64_t left = a.num_cells - c0;
  const int nc = left < kG ? (int)left : kG;
  const int tm = __ldg(a.tmpl_of + g);
  const int4 meta = __ldg(a.tmeta + tm);
  const int nd = __ldg(a.tnd + tm);
  // stage the group's dofs and byte maps
  for (int t = tid; t < nc * kK; t += kThreads) {
    const int q = t / kK;
    sdof[t] = __ldg(a.dofs + (c0 + q) * kK + (t - q * kK));
  }
  for (int t = tid; t < nc * (kKK / 4); t += kThreads) {
    // the group's byte maps are contiguous: 48 * 100 bytes from a 16-byte boundary
    reinterpret_cast<uint32_t*>(spos)[t] = __ldg(reinterpret_cast<const uint32_t*>(a.pos + c0 * kKK) + t);
  }
  __syncthreads();
  for (int r = tid; r < nd; r += kThreads) {
    const uint16_t code = __ldg(a.first + meta.w + r);
    const int d = sdof[(code >> 4) * kK + (code & 15)];
    srp[r] = __ldg(a.row_ptr + d);
    smask[r] = (uint8_t)((a.bc0 && a.bc0[d] ? 1 : 0) | (a.bc1 && a.bc1[d] ? 2 : 0));
  }
  if (tid < nc) {
    const int64_t cell = c0 + tid;
    double Gh[6];
    geometry(a.x, __ldg(reinterpret_cast<const int4*>(a.geom) + cell), Gh);
    double* E = Eu + tid * kNU;
    auto emit = [&](int i, int j, double v) { E[upper_index(i, j)] = v; };
    if constexpr (COEF == FE_COEFF_P1) {
      const int4 km = __ldg(reinterpret_cast<const int4*>(a.coef_map) + cell);
      const double k[4] = {__ldg(a.coef + km.x), __ldg(a.coef + km.y), __ldg(a.coef + km.z), __ldg(a.coef + km.w)};
      T q[24];
#pragma unroll
      for (int m = 0; m < 4; ++m)
#pragma unroll
        for (int s = 0; s < 6; ++s) q[m * 6 + s] = (T)(k[m] * Gh[s]);
      p2_stiffness_p1coef<T>(q, emit);
    } else {
      const double k = COEF == FE_COEFF_DG0 ? __ldg(a.coef + cell) : a.coef_const;
      T gq[6];
#pragma unroll
      for (int s = 0; s < 6; ++s) gq[s] = (T)(k * Gh[s]);
      p2_stiffness_const<T>(gq, emit);
    }
  }
  __syncthreads();
  // one reduction per distinct (row, column) of the group
  for (int e = tid; e < meta.y; e += kThreads) {
    const uint2 rec = __ldg(a.ent + meta.x + e);
    const int r = rec.x & 0xff, c = (rec.x >> 8) & 0xff, cnt = rec.x >> 16;
    if ((smask[r] & 1) | (smask[c] & 2)) continue;
    const int start = rec.y & 0xffff, pidx = rec.y >> 16;
    double s = 0.0;
    for (int k = 0; k < cnt; ++k) {
      const uint16_t code = __ldg(a.contrib + meta.z + start + k);
      s += Eu[(code >> 9) * kNU + (code & 511)];
    }
    atomicAdd(a.values + srp[r] + spos[pidx], s);
  }
}

}  // namespace

bool grouped_supported(const fe_form_s& f) {
  return f.kind == FE_FORM_P2_STIFFNESS && f.V0 == f.V1 && !f.V0->excluded && f.V0->k == kK && f.V0->bs == 1 &&
         f.sp && !f.sp->parent;
}

void reset_group_plan(fe_form_s& f) { f.groups.reset(); }

namespace {

struct Template {
  std::vector<uint2> ent;
  std::vector<uint16_t> contrib;
  std::vector<uint16_t> first;
};

std::unique_ptr<fe_form_s::GroupPlan> build_group_plan(const fe_form_s& f) {
  const int64_t C = f.mesh->num_cells;
  const std::vector<int32_t>& D = f.V0->host;
  auto P = std::make_unique<fe_form_s::GroupPlan>();
  // 2. groups and their templates
  const int64_t ngroups = (C + kG - 1) / kG;
  std::vector<int32_t> tmpl_of(ngroups);
  std::unordered_map<std::string, int32_t> index;
  std::vector<Template> T;
  std::vector<int32_t> stamp(f.V0->num_blocks, -1), lid(f.V0->num_blocks, 0);
  std::string sig;
  struct Item {
    uint32_t rc;
    uint16_t code, pidx;
  };
  std::vector<Item> items;
  for (int64_t g = 0; g < ngroups; ++g) {
    const int64_t c0 = g * kG;
    const int nc = (int)std::min<int64_t>(kG, C - c0);
    // group-local numbering by first appearance; the signature is the
    // group-local dof of every (cell, local dof)
    sig.assign(1, (char)nc);
    int nd = 0;
    std::vector<uint16_t> first;
    for (int q = 0; q < nc; ++q)
      for (int i = 0; i < kK; ++i) {
        const int32_t d = D[(c0 + q) * kK + i];
        if (stamp[d] != (int32_t)g) {
          stamp[d] = (int32_t)g;
          if (nd >= kMaxLocal) return nullptr;  // too many dofs for 8-bit local indices
          lid[d] = nd++;
          first.push_back((uint16_t)(q << 4 | i));
        }
        sig.push_back((char)(uint8_t)lid[d]);
      }
    auto it = index.find(sig);
    if (it != index.end()) {
      tmpl_of[g] = it->second;
      continue;
    }
    // a new template: the group's entries sorted by (row, column), runs of
    // equal pairs summed in cell order
    items.clear();
    for (int q = 0; q < nc; ++q)
      for (int i = 0; i < kK; ++i)
        for (int j = 0; j < kK; ++j) {
          const int r = (uint8_t)sig[1 + q * kK + i], c = (uint8_t)sig[1 + q * kK + j];
          const int u = i <= j ? upper_index(i, j) : upper_index(j, i);
          items.push_back(Item{(uint32_t)(r << 8 | c), (uint16_t)(q << 9 | u), (uint16_t)(q * kKK + i * kK + j)});
        }
    std::stable_sort(items.begin(), items.end(), [](const Item& A, const Item& B) { return A.rc < B.rc; });
    Template t;
    t.first = std::move(first);
    for (size_t s = 0; s < items.size();) {
      size_t e = s;
      while (e < items.size() && items[e].rc == items[s].rc) ++e;
      const uint32_t r = items[s].rc >> 8, c = items[s].rc & 0xff;
      t.ent.push_back(make_uint2(r | c << 8 | (uint32_t)(e - s) << 16,
                                 (uint32_t)t.contrib.size() | (uint32_t)items[s].pidx << 16));
      for (size_t k = s; k < e; ++k) t.contrib.push_back(items[k].code);
      s = e;
    }
    const int32_t id = (int32_t)T.size();
    T.push_back(std::move(t));
    index.emplace(sig, id);
    tmpl_of[g] = id;
    // a mesh without repeated local structure gains nothing from shared
    // templates: leave it to the atomic scatter
    if (T.size() > 4096) return nullptr;
  }
  // 3. device arrays
  std::vector<int4> meta(T.size());
  std::vector<int32_t> nds(T.size());
  std::vector<uint2> ent;
  std::vector<uint16_t> contrib, firsts;
  for (size_t t = 0; t < T.size(); ++t) {
    meta[t] = make_int4((int)ent.size(), (int)T[t].ent.size(), (int)contrib.size(), (int)firsts.size());
    nds[t] = (int32_t)T[t].first.size();
    ent.insert(ent.end(), T[t].ent.begin(), T[t].ent.end());
    contrib.insert(contrib.end(), T[t].contrib.begin(), T[t].contrib.end());
    firsts.insert(firsts.end(), T[t].first.begin(), T[t].first.end());
  }
  auto up = [](auto& d, const auto& h) {
    using E = typename std::decay_t<decltype(h)>::value_type;
    d.alloc(std::max<size_t>(1, h.size()));
    if (!h.empty()) FE_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(E), cudaMemcpyHostToDevice));
  };
  P->ngroups = ngroups;
  P->ntemplates = (int64_t)T.size();
  up(P->tmpl_of, tmpl_of);
  up(P->tmeta, meta);
  up(P->tnd, nds);
  up(P->ent, ent);
  up(P->contrib, contrib);
  up(P->first, firsts);
  return P;
}

}  // namespace

bool assemble_matrix_grouped(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, bool zero,
                             cudaStream_t s) {
  if (!grouped_supported(f)) return false;
  if (!f.groups) {
    f.groups = build_group_plan(f);
    if (!f.groups) {
      f.group_plan_failed = true;
      return false;
    }
  }
  if (zero) launch_zero(values, f.sp->nnz, s);
  const fe_form_s::GroupPlan& P = *f.groups;
  if (P.ngroups == 0) return true;
  GroupArgs a{};
  a.num_cells = f.mesh->num_cells;
  a.tmpl_of = P.tmpl_of.p;
  a.tmeta = P.tmeta.p;
  a.tnd = P.tnd.p;
  a.ent = P.ent.p;
  a.contrib = P.contrib.p;
  a.first = P.first.p;
  a.x = f.mesh->x.p;
  a.geom = f.mesh->geom.p;
  a.dofs = f.V0->dofs.p;
  a.pos = f.pos.p;
  a.row_ptr = f.sp->row_ptr.p;
  a.bc0 = bc0 ? bc0->markers.p : nullptr;
  a.bc1 = bc1 ? bc1->markers.p : nullptr;
  const Coefficient& k = f.coeff[0];
  a.coef_kind = k.kind < 0 ? FE_COEFF_CONSTANT : k.kind;
  a.coef = k.values;
  a.coef_map = k.map ? k.map->dofs.p : nullptr;
  a.coef_const = k.kind < 0 ? 1.0 : k.constant[0];
  a.values = values;
  const unsigned grid = (unsigned)P.ngroups;
  const bool fp32 = f.precision == FE_PREC_FP32;
  if (a.coef_kind == FE_COEFF_P1) {
    if (fp32) k_mat_p2_grouped<float, FE_COEFF_P1><<<grid, kThreads, 0, s>>>(a);
    else k_mat_p2_grouped<double, FE_COEFF_P1><<<grid, kThreads, 0, s>>>(a);
  } else if (a.coef_kind == FE_COEFF_DG0) {
    if (fp32) k_mat_p2_grouped<float, FE_COEFF_DG0><<<grid, kThreads, 0, s>>>(a);
    else k_mat_p2_grouped<double, FE_COEFF_DG0><<<grid, kThreads, 0, s>>>(a);
  } else {
    if (fp32) k_mat_p2_grouped<float, FE_COEFF_CONSTANT><<<grid, kThreads, 0, s>>>(a);
    else k_mat_p2_grouped<double, FE_COEFF_CONSTANT><<<grid, kThreads, 0, s>>>(a);
  }
  FE_CUDA(cudaGetLastError());
  return true;
}

}  // namespace fe
