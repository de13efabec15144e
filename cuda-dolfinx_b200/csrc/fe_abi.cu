// C ABI of the assembly engine (declared in include/cudolfinx_b200.h).
//
// Host-side counterpart of the reference's C++ orchestration
// (cpp/cudolfinx/fem/CUDAAssembler.h, CUDAForm.h, CUDADirichletBC.h,
// mesh/CUDAMesh.h, la/CUDAMatrix.cpp) and of its nanobind functions
// (python/cudolfinx/wrappers/fem.cpp:74-383).  Differences by design:
//  * everything is enqueued on the caller's stream, no per-kernel sync;
//  * coefficients are uploaded once and gathered inside the element kernels
//    (no pack_coefficients pass, no re-upload on every assemble call);
//  * the CSR column search is done once per (form, pattern) into a byte map.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>

#include "fe_internal.h"

namespace fe {

namespace {
thread_local std::string g_last_error;
std::atomic<uint64_t> g_next_id{1};

template <typename F>
int guard(F&& body) {
  try {
    body();
    return FE_OK;
  } catch (const Error& e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return FE_ERR_ARG;
  }
}

struct DeviceScope {
  explicit DeviceScope(fe_context ctx) {
    if (!ctx) FE_FAIL(FE_ERR_ARG, "null context");
    FE_CUDA(cudaSetDevice(ctx->device));
  }
};

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Re-raise the status of a nested C-ABI call inside a guard (its message is
// already the thread's last error).
void rethrow_status(int status) {
  if (status != FE_OK) throw Error(status, g_last_error);
}

std::string decode_device_error(unsigned w) {
  std::string s;
  if (w & DEV_ERR_PATTERN) s += " [cell coupling missing from the CSR pattern]";
  if (w & DEV_ERR_ROW_WIDE) s += " [block row wider than 255 block columns]";
  if (w & DEV_ERR_BLOCK) s += " [CSR rows of a block row are not block-structured]";
  if (w & DEV_ERR_INDEX) s += " [index out of range]";
  if (w & DEV_ERR_FACET) s += " [the two sides of an interior facet are different triangles]";
  if (w & DEV_ERR_BARRIER) s += " [a grid barrier timed out]";
  return s;
}

// Reads and clears the error word; throws if a kernel reported an error.
void check_device_errors(fe_context ctx, cudaStream_t s, int code) {
  unsigned w = 0;
  FE_CUDA(cudaMemcpyAsync(&w, ctx->err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  FE_CUDA(cudaStreamSynchronize(s));
  if (w) {
    FE_CUDA(cudaMemsetAsync(ctx->err.p, 0, sizeof(unsigned), s));
    FE_CUDA(cudaStreamSynchronize(s));
    FE_FAIL(code, "device error word 0x" + std::to_string(w) + decode_device_error(w));
  }
}

int form_rank(int kind) {
  switch (kind) {
    case FE_FORM_P1_STIFFNESS:
    case FE_FORM_P2_STIFFNESS:
    case FE_FORM_P1_MASS:
    case FE_FORM_P2_MASS:
    case FE_FORM_VP2_MASS:
    case FE_FORM_VP2_ELASTICITY:
    case FE_FORM_P1_FACET_MASS:
    case FE_FORM_P2_FACET_MASS:
    case FE_FORM_P3_STIFFNESS:
    case FE_FORM_DG0_JUMP:
    case FE_FORM_DG1_JUMP:
      return 2;
    case FE_FORM_P1_LOAD:
    case FE_FORM_P2_LOAD:
    case FE_FORM_VP2_LOAD:
    case FE_FORM_P1_FACET_LOAD:
    case FE_FORM_P2_FACET_LOAD:
    case FE_FORM_VP2_FACET_LOAD:
    case FE_FORM_P3_LOAD:
    case FE_FORM_DG0_AVG_LOAD:
    case FE_FORM_DG1_AVG_LOAD:
      return 1;
    case FE_FORM_INTEGRAL:
    case FE_FORM_P1_ENERGY:
    case FE_FORM_P2_ENERGY:
    case FE_FORM_FACET_INTEGRAL:
    case FE_FORM_JUMP_NORM:
      return 0;
    default:
      return -1;
  }
}

// expected (dofs per cell, block size) of the form's spaces
void form_space(int kind, int& k, int& bs) {
  switch (kind) {
    case FE_FORM_P1_STIFFNESS:
    case FE_FORM_P1_MASS:
    case FE_FORM_P1_LOAD:
    case FE_FORM_P1_FACET_MASS:
    case FE_FORM_P1_FACET_LOAD:
      k = 4, bs = 1;
      return;
    case FE_FORM_P2_STIFFNESS:
    case FE_FORM_P2_MASS:
    case FE_FORM_P2_LOAD:
    case FE_FORM_P2_FACET_MASS:
    case FE_FORM_P2_FACET_LOAD:
      k = 10, bs = 1;
      return;
    case FE_FORM_P3_STIFFNESS:
    case FE_FORM_P3_LOAD:
      k = 20, bs = 1;
      return;
    case FE_FORM_DG0_JUMP:
    case FE_FORM_DG0_AVG_LOAD:
      k = 1, bs = 1;
      return;
    case FE_FORM_DG1_JUMP:
    case FE_FORM_DG1_AVG_LOAD:
      k = 4, bs = 1;
      return;
    default:
      k = 10, bs = 3;
      return;
  }
}

int64_t scalar_size(const fe_dofmap_s* d) { return d->num_blocks * d->bs; }

template <typename T>
void upload(DevBuf<T>& dst, const T* src, size_t n) {
  dst.alloc(n);
  if (n) FE_CUDA(cudaMemcpy(dst.p, src, n * sizeof(T), cudaMemcpyHostToDevice));
}

fe_bc_s::CellList& lift_cells(fe_bc_s& bc, const fe_dofmap_s& V, cudaStream_t s) {
  auto it = bc.lift_cells.find(V.id);
  if (it != bc.lift_cells.end()) return *it->second;
  auto L = std::make_unique<fe_bc_s::CellList>();
  L->cells.alloc(std::max<int64_t>(1, V.num_cells));
  DevBuf<unsigned long long> cnt(1);
  FE_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), s));
  launch_mark_cells(V.dofs.p, V.num_cells, V.k, V.bs, bc.markers.p, L->cells.p, cnt.p, s);
  unsigned long long h = 0;
  FE_CUDA(cudaMemcpyAsync(&h, cnt.p, sizeof(h), cudaMemcpyDeviceToHost, s));
  FE_CUDA(cudaStreamSynchronize(s));
  L->count = (int64_t)h;
  auto& ref = *L;
  bc.lift_cells.emplace(V.id, std::move(L));
  return ref;
}

}  // namespace

[[noreturn]] void fail(int code, const std::string& msg, const char* file, int line) {
  throw Error(code, msg + " (at " + file + ":" + std::to_string(line) + ")");
}

void check_cuda(cudaError_t e, const char* what, const char* file, int line) {
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    int code = (e == cudaErrorMemoryAllocation) ? FE_ERR_NOMEM : FE_ERR_CUDA;
    fail(code, std::string(what) + " failed with " + cudaGetErrorString(e), file, line);
  }
}

unsigned* device_error_word(fe_context ctx) { return ctx->err.p; }

void set_last_error(const std::string& msg) { g_last_error = msg; }

}  // namespace fe

using namespace fe;

extern "C" {

const char* fe_last_error(void) { return g_last_error.c_str(); }

const char* fe_version(void) { return "cudolfinx_b200 0.1.0 (sm_100a)"; }

int fe_context_create(int device, fe_context* out) {
  return guard([&] {
    FE_REQUIRE(out, "null output pointer");
    int n = 0;
    FE_CUDA(cudaGetDeviceCount(&n));
    FE_REQUIRE(device >= 0 && device < n, "no CUDA device " + std::to_string(device));
    FE_CUDA(cudaSetDevice(device));
    int major = 0, minor = 0;
    FE_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
    FE_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
    if (major != 10 || minor != 0)
      FE_FAIL(FE_ERR_CUDA, "this library is built for sm_100a (B200); device " + std::to_string(device) +
                               " is sm_" + std::to_string(major) + std::to_string(minor));
    auto ctx = std::make_unique<fe_context_s>();
    ctx->device = device;
    FE_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
    ctx->err.alloc(1);
    FE_CUDA(cudaMemset(ctx->err.p, 0, sizeof(unsigned)));
    *out = ctx.release();
  });
}

int fe_context_destroy(fe_context ctx) {
  return guard([&] {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    delete ctx;
  });
}

int fe_context_synchronize(fe_context ctx) {
  return guard([&] {
    DeviceScope d(ctx);
    FE_CUDA(cudaDeviceSynchronize());
    check_device_errors(ctx, nullptr, FE_ERR_DEVICE);
  });
}

int fe_mesh_create(fe_context ctx, const double* coords, int64_t num_nodes, const int32_t* geom_dofmap,
                   int64_t num_cells, int nodes_per_cell, fe_mesh* out) {
  return guard([&] {
    DeviceScope d(ctx);
    FE_REQUIRE(out, "null output pointer");
    FE_REQUIRE(nodes_per_cell == 4, "only affine tetrahedra (4 nodes per cell) are supported");
    FE_REQUIRE(num_nodes >= 0 && num_cells >= 0, "negative size");
    FE_REQUIRE((coords || !num_nodes) && (geom_dofmap || !num_cells), "null input array");
    for (int64_t q = 0; q < num_cells * 4; ++q)
      if (geom_dofmap[q] < 0 || geom_dofmap[q] >= num_nodes)
        FE_FAIL(FE_ERR_ARG, "geometry dofmap entry out of range at " + std::to_string(q));
    auto m = std::make_unique<fe_mesh_s>();
    m->ctx = ctx;
    m->num_nodes = num_nodes;
    m->num_cells = num_cells;
    upload(m->x, coords, (size_t)num_nodes * 3);
    upload(m->geom, geom_dofmap, (size_t)num_cells * 4);
    m->host_x.assign(coords, coords + num_nodes * 3);
    m->host_geom.assign(geom_dofmap, geom_dofmap + num_cells * 4);
    *out = m.release();
  });
}

int fe_mesh_destroy(fe_mesh m) {
  return guard([&] { delete m; });
}

int fe_dofmap_create(fe_context ctx, const int32_t* cell_dofs, int64_t num_cells, int dofs_per_cell, int bs,
                     int64_t num_blocks, fe_dofmap* out) {
  return guard([&] {
    DeviceScope d(ctx);
    FE_REQUIRE(out, "null output pointer");
    FE_REQUIRE(dofs_per_cell > 0 && dofs_per_cell <= 32, "dofs_per_cell must be in 1..32");
    FE_REQUIRE(bs >= 1 && bs <= 3, "block size must be 1..3");
    FE_REQUIRE(num_cells >= 0 && num_blocks >= 0, "negative size");
    FE_REQUIRE(num_blocks * bs <= INT32_MAX, "too many dofs for int32 indices");
    FE_REQUIRE(cell_dofs || !num_cells, "null dofmap");
    const int64_t n = num_cells * dofs_per_cell;
    for (int64_t q = 0; q < n; ++q)
      if (cell_dofs[q] < 0 || cell_dofs[q] >= num_blocks)
        FE_FAIL(FE_ERR_ARG, "dofmap entry out of range at " + std::to_string(q));
    auto m = std::make_unique<fe_dofmap_s>();
    m->ctx = ctx;
    m->num_cells = num_cells;
    m->num_blocks = num_blocks;
    m->k = dofs_per_cell;
    m->bs = bs;
    m->host.assign(cell_dofs, cell_dofs + n);
    upload(m->dofs, cell_dofs, (size_t)n);
    m->id = g_next_id++;
    *out = m.release();
  });
}

int fe_dofmap_create_restricted(fe_context ctx, const int32_t* cell_dofs, int64_t num_cells, int dofs_per_cell,
                                int bs, int64_t num_blocks, fe_dofmap* out) {
  return guard([&] {
    DeviceScope d(ctx);
    FE_REQUIRE(out, "null output pointer");
    FE_REQUIRE(dofs_per_cell > 0 && dofs_per_cell <= 32, "dofs_per_cell must be in 1..32");
    FE_REQUIRE(bs >= 1 && bs <= 3, "block size must be 1..3");
    FE_REQUIRE(num_cells >= 0 && num_blocks >= 0, "negative size");
    FE_REQUIRE(num_blocks * bs <= INT32_MAX, "too many dofs for int32 indices");
    FE_REQUIRE(cell_dofs || !num_cells, "null dofmap");
    const int64_t n = num_cells * dofs_per_cell;
    bool excluded = false;
    for (int64_t q = 0; q < n; ++q) {
      if (cell_dofs[q] < -1 || cell_dofs[q] >= num_blocks)
        FE_FAIL(FE_ERR_ARG, "restricted dofmap entry out of range at " + std::to_string(q));
      excluded |= cell_dofs[q] == -1;
    }
    auto m = std::make_unique<fe_dofmap_s>();
    m->ctx = ctx;
    m->num_cells = num_cells;
    m->num_blocks = num_blocks;
    m->k = dofs_per_cell;
    m->bs = bs;
    m->excluded = excluded;
    m->host.assign(cell_dofs, cell_dofs + n);
    upload(m->dofs, cell_dofs, (size_t)n);
    m->id = g_next_id++;
    *out = m.release();
  });
}

int fe_dofmap_destroy(fe_dofmap d) {
  return guard([&] { delete d; });
}

int fe_sparsity_build(fe_dofmap rows, fe_dofmap cols, fe_sparsity* out) {
  return guard([&] {
    FE_REQUIRE(rows && cols && out, "null argument");
    FE_REQUIRE(rows->ctx == cols->ctx, "dofmaps belong to different contexts");
    FE_REQUIRE(rows->num_cells == cols->num_cells, "dofmaps cover different cell counts");
    DeviceScope d(rows->ctx);
    std::vector<int64_t> bptr;
    std::vector<int32_t> bcol, row_ptr, col, diag;
    build_block_pattern(rows->host.data(), cols->host.data(), rows->num_cells, rows->k, cols->k, rows->num_blocks,
                        cols->num_blocks, bptr, bcol);
    unroll_pattern(bptr, bcol, rows->bs, cols->bs, row_ptr, col, diag);
    auto s = std::make_unique<fe_sparsity_s>();
    s->ctx = rows->ctx;
    s->num_rows = scalar_size(rows);
    s->num_cols = scalar_size(cols);
    s->nnz = (int64_t)col.size();
    upload(s->row_ptr, row_ptr.data(), row_ptr.size());
    upload(s->col, col.data(), col.size());
    upload(s->diag, diag.data(), diag.size());
    s->host_row_ptr = std::move(row_ptr);
    s->id = g_next_id++;
    *out = s.release();
  });
}

int fe_sparsity_build_block(fe_context ctx, int num_parts, const fe_dofmap* rows, const fe_dofmap* cols,
                            const int64_t* row_offsets, const int64_t* col_offsets, int64_t num_rows,
                            int64_t num_cols, fe_sparsity* out) {
  return guard([&] {
    FE_REQUIRE(ctx && out, "null argument");
    FE_REQUIRE(num_parts >= 0 && (num_parts == 0 || (rows && cols && row_offsets && col_offsets)), "null part table");
    DeviceScope d(ctx);
    std::vector<SystemPart> parts;
    for (int p = 0; p < num_parts; ++p) {
      FE_REQUIRE(rows[p] && cols[p], "null dofmap in part " + std::to_string(p));
      FE_REQUIRE(rows[p]->ctx == ctx && cols[p]->ctx == ctx, "part " + std::to_string(p) + " belongs to another context");
      parts.push_back(SystemPart{rows[p], cols[p], row_offsets[p], col_offsets[p]});
    }
    std::vector<int32_t> row_ptr, col, diag;
    build_system_pattern(parts, num_rows, num_cols, row_ptr, col, diag);
    auto sp = std::make_unique<fe_sparsity_s>();
    sp->ctx = ctx;
    sp->num_rows = num_rows;
    sp->num_cols = num_cols;
    sp->nnz = (int64_t)col.size();
    upload(sp->row_ptr, row_ptr.data(), row_ptr.size());
    upload(sp->col, col.data(), col.size());
    upload(sp->diag, diag.data(), diag.size());
    sp->host_row_ptr = std::move(row_ptr);
    sp->id = g_next_id++;
    *out = sp.release();
  });
}

int fe_sparsity_build_forms(int num_forms, const fe_form* forms, fe_sparsity* out) {
  return guard([&] {
    FE_REQUIRE(out && num_forms > 0 && forms, "need at least one form");
    const fe_form f0 = forms[0];
    FE_REQUIRE(f0 && f0->rank == 2, "the forms must be bilinear");
    DeviceScope d(f0->ctx);
    std::vector<std::unique_ptr<fe_dofmap_s>> macro;  // host-only macro dofmaps of interior-facet forms
    std::vector<SystemPart> parts;
    for (int q = 0; q < num_forms; ++q) {
      const fe_form f = forms[q];
      FE_REQUIRE(f && f->rank == 2 && f->ctx == f0->ctx, "form " + std::to_string(q) + " is not a bilinear form of "
                                                          "the same context");
      FE_REQUIRE(f->V0->num_blocks == f0->V0->num_blocks && f->V0->bs == f0->V0->bs &&
                     f->V1->num_blocks == f0->V1->num_blocks && f->V1->bs == f0->V1->bs,
                 "form " + std::to_string(q) + " acts on spaces of other sizes");
      if (!is_ifacet_kind(f->kind)) {
        parts.push_back(SystemPart{f->V0, f->V1, 0, 0});
        continue;
      }
      FE_REQUIRE(f->facets_set, "form " + std::to_string(q) + ": set the interior facets first");
      const int64_t F = f->num_facets;
      fe_dofmap_s* side[2];
      for (int t = 0; t < 2; ++t) {
        const fe_dofmap_s* V = t == 0 ? f->V0 : f->V1;
        auto m = std::make_unique<fe_dofmap_s>();
        m->num_cells = F;
        m->k = 2 * V->k;
        m->bs = V->bs;
        m->num_blocks = V->num_blocks;
        m->host.resize((size_t)F * m->k);
        for (int64_t e = 0; e < F; ++e)
          for (int i = 0; i < V->k; ++i) {
            m->host[e * m->k + i] = V->host[(int64_t)f->host_facets[4 * e] * V->k + i];
            m->host[e * m->k + V->k + i] = V->host[(int64_t)f->host_facets[4 * e + 2] * V->k + i];
          }
        side[t] = m.get();
        macro.push_back(std::move(m));
      }
      parts.push_back(SystemPart{side[0], side[1], 0, 0});
    }
    std::vector<int32_t> row_ptr, col, diag;
    build_system_pattern(parts, scalar_size(f0->V0), scalar_size(f0->V1), row_ptr, col, diag);
    auto sp = std::make_unique<fe_sparsity_s>();
    sp->ctx = f0->ctx;
    sp->num_rows = scalar_size(f0->V0);
    sp->num_cols = scalar_size(f0->V1);
    sp->nnz = (int64_t)col.size();
    upload(sp->row_ptr, row_ptr.data(), row_ptr.size());
    upload(sp->col, col.data(), col.size());
    upload(sp->diag, diag.data(), diag.size());
    sp->host_row_ptr = std::move(row_ptr);
    sp->id = g_next_id++;
    *out = sp.release();
  });
}

int fe_sparsity_build_device(fe_dofmap rows, fe_dofmap cols, void* stream, fe_sparsity* out) {
  return guard([&] {
    FE_REQUIRE(rows && cols && out, "null argument");
    FE_REQUIRE(rows->ctx == cols->ctx, "dofmaps belong to different contexts");
    FE_REQUIRE(rows->num_cells == cols->num_cells, "dofmaps cover different cell counts");
    DeviceScope d(rows->ctx);
    auto s = std::make_unique<fe_sparsity_s>();
    s->ctx = rows->ctx;
    build_pattern_device(*rows, *cols, as_stream(stream), *s);
    s->id = g_next_id++;
    *out = s.release();
  });
}

int fe_pattern_build_host(const int32_t* dofs0, const int32_t* dofs1, int64_t num_cells, int k0, int k1, int bs0,
                          int bs1, int64_t num_blocks0, int64_t num_blocks1, int64_t* nnz, int32_t** row_ptr_out,
                          int32_t** col_out) {
  return guard([&] {
    FE_REQUIRE(dofs0 && dofs1 && nnz && row_ptr_out && col_out, "null argument");
    FE_REQUIRE(num_cells >= 0 && k0 > 0 && k1 > 0 && bs0 >= 1 && bs1 >= 1, "invalid sizes");
    std::vector<int64_t> bptr;
    std::vector<int32_t> bcol, row_ptr, col, diag;
    build_block_pattern(dofs0, dofs1, num_cells, k0, k1, num_blocks0, num_blocks1, bptr, bcol);
    unroll_pattern(bptr, bcol, bs0, bs1, row_ptr, col, diag);
    auto* rp = static_cast<int32_t*>(std::malloc(row_ptr.size() * sizeof(int32_t)));
    auto* cl = static_cast<int32_t*>(std::malloc(std::max<size_t>(1, col.size()) * sizeof(int32_t)));
    if (!rp || !cl) {
      std::free(rp);
      std::free(cl);
      FE_FAIL(FE_ERR_NOMEM, "host allocation failed");
    }
    std::memcpy(rp, row_ptr.data(), row_ptr.size() * sizeof(int32_t));
    if (!col.empty()) std::memcpy(cl, col.data(), col.size() * sizeof(int32_t));
    *nnz = (int64_t)col.size();
    *row_ptr_out = rp;
    *col_out = cl;
  });
}

void fe_free_host(void* p) { std::free(p); }

int fe_sparsity_create(fe_context ctx, const int32_t* row_ptr, const int32_t* col, int64_t num_rows,
                       int64_t num_cols, fe_sparsity* out) {
  return guard([&] {
    DeviceScope d(ctx);
    FE_REQUIRE(out && row_ptr && num_rows >= 0 && num_cols >= 0, "invalid argument");
    FE_REQUIRE(row_ptr[0] == 0, "row_ptr[0] must be 0");
    const int64_t nnz = row_ptr[num_rows];
    FE_REQUIRE(col || nnz == 0, "null column array");
    std::vector<int32_t> diag(num_rows, -1);
    for (int64_t r = 0; r < num_rows; ++r) {
      FE_REQUIRE(row_ptr[r + 1] >= row_ptr[r], "row_ptr not monotone at row " + std::to_string(r));
      for (int64_t q = row_ptr[r]; q < row_ptr[r + 1]; ++q) {
        FE_REQUIRE(col[q] >= 0 && col[q] < num_cols, "column out of range at " + std::to_string(q));
        FE_REQUIRE(q == row_ptr[r] || col[q] > col[q - 1], "columns not sorted/unique in row " + std::to_string(r));
        if (col[q] == r) diag[r] = (int32_t)q;
      }
    }
    auto s = std::make_unique<fe_sparsity_s>();
    s->ctx = ctx;
    s->num_rows = num_rows;
    s->num_cols = num_cols;
    s->nnz = nnz;
    upload(s->row_ptr, row_ptr, (size_t)num_rows + 1);
    upload(s->col, col, (size_t)nnz);
    upload(s->diag, diag.data(), diag.size());
    s->host_row_ptr.assign(row_ptr, row_ptr + num_rows + 1);
    s->id = g_next_id++;
    *out = s.release();
  });
}

int fe_sparsity_info(fe_sparsity s, int64_t* num_rows, int64_t* num_cols, int64_t* nnz) {
  return guard([&] {
    FE_REQUIRE(s, "null sparsity");
    if (num_rows) *num_rows = s->num_rows;
    if (num_cols) *num_cols = s->num_cols;
    if (nnz) *nnz = s->nnz;
  });
}

int fe_sparsity_copy_to_host(fe_sparsity s, int32_t* row_ptr, int32_t* col) {
  return guard([&] {
    FE_REQUIRE(s, "null sparsity");
    DeviceScope d(s->ctx);
    if (row_ptr)
      FE_CUDA(cudaMemcpy(row_ptr, s->row_ptr.p, (s->num_rows + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (col && s->nnz) FE_CUDA(cudaMemcpy(col, s->col.p, s->nnz * sizeof(int32_t), cudaMemcpyDeviceToHost));
  });
}

int fe_sparsity_device_arrays(fe_sparsity s, const int32_t** row_ptr, const int32_t** col) {
  return guard([&] {
    FE_REQUIRE(s, "null sparsity");
    if (row_ptr) *row_ptr = s->row_ptr.p;
    if (col) *col = s->col.p;
  });
}

int fe_sparsity_destroy(fe_sparsity s) {
  return guard([&] { delete s; });
}

int fe_form_create(fe_context ctx, int form_kind, fe_mesh mesh, fe_dofmap test, fe_dofmap trial, fe_form* out) {
  return guard([&] {
    DeviceScope d(ctx);
    const int rank = form_rank(form_kind);
    FE_REQUIRE(rank >= 0, "unknown form kind " + std::to_string(form_kind));
    FE_REQUIRE(out && mesh && (test || rank == 0), "null argument");
    FE_REQUIRE((rank == 2) == (trial != nullptr), "bilinear forms need a trial dofmap, others none");
    FE_REQUIRE(rank > 0 || test == nullptr, "functionals take no test dofmap");
    int k = 0, bs = 0;
    form_space(form_kind, k, bs);
    for (fe_dofmap V : {test, trial}) {
      if (!V) continue;
      FE_REQUIRE(V->k == k && V->bs == bs, "dofmap has " + std::to_string(V->k) + " dofs/cell bs " +
                                               std::to_string(V->bs) + "; form kind " + std::to_string(form_kind) +
                                               " needs " + std::to_string(k) + " bs " + std::to_string(bs));
      FE_REQUIRE(V->num_cells == mesh->num_cells, "dofmap and mesh cell counts differ");
      FE_REQUIRE(!V->excluded || !is_facet_kind(form_kind), "exterior-facet forms take unrestricted dofmaps");
      FE_REQUIRE(!V->excluded || !is_ifacet_kind(form_kind), "interior-facet forms take unrestricted dofmaps");
    }
    auto f = std::make_unique<fe_form_s>();
    f->ctx = ctx;
    f->kind = form_kind;
    f->rank = rank;
    f->mesh = mesh;
    f->V0 = test;
    f->V1 = trial;
    *out = f.release();
  });
}

int fe_form_set_coefficient(fe_form f, int index, int coeff_kind, fe_dofmap cmap, const double* values, int64_t n,
                            int values_on_device, void* stream) {
  return guard([&] {
    FE_REQUIRE(f, "null form");
    FE_REQUIRE(!f->ffcx, "FFCx forms take their coefficients through fe_form_set_coefficient_field");
    DeviceScope d(f->ctx);
    const int ncoef =
        (f->kind == FE_FORM_VP2_ELASTICITY || f->kind == FE_FORM_P1_ENERGY || f->kind == FE_FORM_P2_ENERGY) ? 2 : 1;
    FE_REQUIRE(index >= 0 && index < ncoef, "coefficient index out of range");
    FE_REQUIRE(values, "null values");
    const int ncomp = (f->kind == FE_FORM_VP2_LOAD || f->kind == FE_FORM_VP2_FACET_LOAD) ? 3 : 1;
    Coefficient& c = f->coeff[index];
    const int64_t C = f->mesh->num_cells;
    if (coeff_kind == FE_COEFF_CONSTANT) {
      FE_REQUIRE(!values_on_device, "constant coefficients are passed in host memory");
      FE_REQUIRE(n == ncomp, "constant coefficient needs " + std::to_string(ncomp) + " value(s)");
      for (int q = 0; q < ncomp; ++q) c.constant[q] = values[q];
      c.kind = FE_COEFF_CONSTANT;
      c.values = nullptr;
      c.map = nullptr;
      return;
    }
    if (coeff_kind == FE_COEFF_DG0) {
      FE_REQUIRE(n == C * ncomp, "DG0 coefficient needs num_cells*" + std::to_string(ncomp) + " values");
    } else if (coeff_kind == FE_COEFF_P1) {
      FE_REQUIRE(cmap && cmap->k == 4 && cmap->bs == 1 && cmap->num_cells == C && !cmap->excluded,
                 "P1 coefficient needs an unrestricted P1 dofmap");
      FE_REQUIRE(n >= cmap->num_blocks, "P1 coefficient has fewer values than dofs");
      FE_REQUIRE(f->kind == FE_FORM_P2_STIFFNESS || f->kind == FE_FORM_P1_STIFFNESS || f->kind == FE_FORM_P1_LOAD ||
                     f->kind == FE_FORM_P1_MASS ||
                     f->kind == FE_FORM_P2_MASS || f->kind == FE_FORM_VP2_MASS ||
                     f->kind == FE_FORM_P1_FACET_LOAD || f->kind == FE_FORM_P2_FACET_LOAD ||
                     f->kind == FE_FORM_INTEGRAL || f->kind == FE_FORM_FACET_INTEGRAL ||
                     f->kind == FE_FORM_JUMP_NORM || (f->kind == FE_FORM_P1_ENERGY && index == 1),
                 "P1 coefficients are supported by P1/P2 stiffness, mass, P1 load, facet load and functional forms");
    } else if (coeff_kind == FE_COEFF_P2) {
      FE_REQUIRE(f->kind == FE_FORM_P2_ENERGY && index == 1, "P2 coefficients are the u of FE_FORM_P2_ENERGY");
      FE_REQUIRE(cmap && cmap->k == 10 && cmap->bs == 1 && cmap->num_cells == C && !cmap->excluded,
                 "P2 coefficient needs an unrestricted P2 dofmap");
      FE_REQUIRE(n >= cmap->num_blocks, "P2 coefficient has fewer values than dofs");
    } else {
      FE_FAIL(FE_ERR_ARG, "unknown coefficient kind " + std::to_string(coeff_kind));
    }
    if (f->kind == FE_FORM_VP2_ELASTICITY || f->kind == FE_FORM_P2_LOAD ||
        f->kind == FE_FORM_VP2_LOAD || f->kind == FE_FORM_P1_FACET_MASS || f->kind == FE_FORM_P2_FACET_MASS ||
        f->kind == FE_FORM_VP2_FACET_LOAD || f->kind == FE_FORM_P3_STIFFNESS || f->kind == FE_FORM_P3_LOAD ||
        is_ifacet_kind(f->kind))
      FE_REQUIRE(coeff_kind != FE_COEFF_P1, "this form takes constant or DG0 coefficients");
    if ((f->kind == FE_FORM_P1_ENERGY || f->kind == FE_FORM_P2_ENERGY) && index == 1)
      FE_REQUIRE(coeff_kind == (f->kind == FE_FORM_P1_ENERGY ? FE_COEFF_P1 : FE_COEFF_P2),
                 "u of an energy functional is a P1 / P2 field");
    c.kind = coeff_kind;
    c.map = (coeff_kind == FE_COEFF_P1 || coeff_kind == FE_COEFF_P2) ? cmap : nullptr;
    c.n = n;
    if (values_on_device) {
      c.own.release();
      c.values = values;
    } else {
      if (c.own.n != (size_t)n) c.own.alloc(n);
      FE_CUDA(cudaMemcpyAsync(c.own.p, values, n * sizeof(double), cudaMemcpyHostToDevice, as_stream(stream)));
      c.values = c.own.p;
    }
  });
}

int fe_form_set_facets(fe_form f, const int32_t* pairs, int64_t num_facets) {
  return guard([&] {
    FE_REQUIRE(f, "null form");
    FE_REQUIRE(is_facet_kind(f->kind) || f->kind == FE_FORM_FACET_INTEGRAL, "not an exterior-facet form");
    FE_REQUIRE(num_facets >= 0 && (pairs || num_facets == 0), "invalid facet list");
    DeviceScope d(f->ctx);
    const int64_t C = f->mesh->num_cells;
    for (int64_t q = 0; q < num_facets; ++q)
      if (pairs[2 * q] < 0 || pairs[2 * q] >= C || pairs[2 * q + 1] < 0 || pairs[2 * q + 1] > 3)
        FE_FAIL(FE_ERR_ARG, "facet " + std::to_string(q) + " is not a (cell, local facet 0..3) pair of the mesh");
    upload(f->facets, pairs, (size_t)(2 * num_facets));
    f->num_facets = num_facets;
    f->facets_set = true;
  });
}

int fe_form_set_interior_facets(fe_form f, const int32_t* quads, int64_t num_facets) {
  return guard([&] {
    FE_REQUIRE(f, "null form");
    FE_REQUIRE(is_ifacet_kind(f->kind) || f->kind == FE_FORM_JUMP_NORM, "not an interior-facet form");
    FE_REQUIRE(num_facets >= 0 && (quads || num_facets == 0), "invalid facet list");
    DeviceScope d(f->ctx);
    const int64_t C = f->mesh->num_cells;
    const std::vector<int32_t>& G = f->mesh->host_geom;
    for (int64_t q = 0; q < num_facets; ++q) {
      const int32_t c0 = quads[4 * q], l0 = quads[4 * q + 1], c1 = quads[4 * q + 2], l1 = quads[4 * q + 3];
      if (c0 < 0 || c0 >= C || c1 < 0 || c1 >= C || l0 < 0 || l0 > 3 || l1 < 0 || l1 > 3 || c0 == c1)
        FE_FAIL(FE_ERR_ARG, "interior facet " + std::to_string(q) + " is not a (cell, facet, cell, facet) quadruple "
                            "of two different cells of the mesh");
      // the two local facets must be the same triangle
      for (int t = 0; t < 4; ++t) {
        if (t == l0) continue;
        bool found = false;
        for (int u = 0; u < 4; ++u)
          if (u != l1 && G[4 * (int64_t)c1 + u] == G[4 * (int64_t)c0 + t]) found = true;
        if (!found)
          FE_FAIL(FE_ERR_ARG, "interior facet " + std::to_string(q) + ": the two local facets are different triangles");
      }
    }
    f->host_facets.assign(quads, quads + 4 * num_facets);
    upload(f->facets, quads, (size_t)(4 * num_facets));
    f->num_facets = num_facets;
    f->facets_set = true;
    // macro dofmaps: cell0's dofs then cell1's, per facet
    for (int side = 0; side < 2; ++side) {
      const fe_dofmap_s* V = side == 0 ? f->V0 : f->V1;
      fe::DevBuf<int32_t>& dst = side == 0 ? f->macro0 : f->macro1;
      if (!V || (side == 1 && f->V1 == f->V0)) {
        dst.release();
        continue;
      }
      const int k = V->k;
      std::vector<int32_t> m((size_t)num_facets * 2 * k);
      for (int64_t q = 0; q < num_facets; ++q)
        for (int i = 0; i < k; ++i) {
          m[q * 2 * k + i] = V->host[(int64_t)quads[4 * q] * k + i];
          m[q * 2 * k + k + i] = V->host[(int64_t)quads[4 * q + 2] * k + i];
        }
      upload(dst, m.data(), m.size());
    }
    if (f->ffcx) ffcx_set_interior_permutations(*f);
    f->sp = nullptr;  // the byte map depends on the facets: bind again
    f->view.reset();
  });
}

int fe_form_set_launch(fe_form f, int cells_per_cta, int stage) {
  return guard([&] {
    FE_REQUIRE(f, "null form");
    FE_REQUIRE(cells_per_cta == 0 || cells_per_cta == 32 || cells_per_cta == 64 || cells_per_cta == 128,
               "cells per CTA must be 0 (default), 32, 64 or 128");
    FE_REQUIRE(stage == 0 || stage == 1, "stage must be 0 or 1");
    f->launch_cells = cells_per_cta;
    f->launch_stage = stage;
  });
}

int fe_form_set_precision(fe_form f, int precision) {
  return guard([&] {
    FE_REQUIRE(f, "null form");
    FE_REQUIRE(precision == FE_PREC_FP64 || precision == FE_PREC_FP32, "unknown precision");
    FE_REQUIRE(precision == FE_PREC_FP64 || f->kind == FE_FORM_P2_STIFFNESS || f->kind == FE_FORM_P3_STIFFNESS ||
                   f->kind == FE_FORM_VP2_ELASTICITY,
               "FP32 element tensors are offered for P2 / P3 stiffness and vector-P2 elasticity");
    f->precision = precision;
  });
}

int fe_form_bind_sparsity(fe_form f, fe_sparsity s, void* stream) {
  return guard([&] {
    FE_REQUIRE(f && s, "null argument");
    FE_REQUIRE(f->rank == 2, "only bilinear forms bind a matrix pattern");
    FE_REQUIRE(s->ctx == f->ctx, "pattern belongs to another context");
    FE_REQUIRE(!f->V0->excluded && !f->V1->excluded,
               "forms on restricted dofmaps bind to a block pattern (fe_form_bind_sparsity_block)");
    FE_REQUIRE(!s->parent, "a block view cannot be bound directly");
    FE_REQUIRE(s->num_rows == scalar_size(f->V0) && s->num_cols == scalar_size(f->V1),
               "pattern shape does not match the form's spaces");
    FE_REQUIRE(!is_ifacet_kind(f->kind) || f->facets_set,
               "set the interior facets first (fe_form_set_interior_facets)");
    DeviceScope d(f->ctx);
    cudaStream_t st = as_stream(stream);
    const size_t bytes = is_ifacet_kind(f->kind)
                             ? (size_t)f->num_facets * (2 * f->V0->k) * (2 * f->V1->k)
                             : (size_t)f->mesh->num_cells * f->V0->k * f->V1->k;
    f->pos.alloc((bytes + 15) / 16 * 16 + 16);
    FE_CUDA(cudaMemsetAsync(f->pos.p, 0, f->pos.bytes(), st));
    f->sp = s;
    f->view.reset();
    reset_gather_plan(*f);
    try {
      launch_build_slotmap(*f, st);
      check_device_errors(f->ctx, st, FE_ERR_PATTERN);
    } catch (...) {
      f->sp = nullptr;  // the byte map is incomplete: the form stays unbound
      throw;
    }
  });
}

int fe_form_bind_sparsity_block(fe_form f, fe_sparsity s, int64_t row_offset, int64_t col_offset, void* stream) {
  return guard([&] {
    FE_REQUIRE(f && s, "null argument");
    FE_REQUIRE(f->rank == 2, "only bilinear forms bind a matrix pattern");
    FE_REQUIRE(s->ctx == f->ctx, "pattern belongs to another context");
    FE_REQUIRE(!s->parent, "bind to the monolithic pattern, not to a view");
    FE_REQUIRE(!is_ifacet_kind(f->kind), "interior-facet forms bind with fe_form_bind_sparsity");
    FE_REQUIRE(row_offset >= 0 && col_offset >= 0 && row_offset + scalar_size(f->V0) <= s->num_rows &&
                   col_offset + scalar_size(f->V1) <= s->num_cols,
               "the form's block does not fit the pattern at these offsets");
    DeviceScope d(f->ctx);
    cudaStream_t st = as_stream(stream);
    const size_t bytes = (size_t)f->mesh->num_cells * f->V0->k * f->V1->k;
    f->pos.alloc((bytes + 15) / 16 * 16 + 16);
    FE_CUDA(cudaMemsetAsync(f->pos.p, 0, f->pos.bytes(), st));
    auto v = std::make_unique<fe_sparsity_s>();
    v->ctx = f->ctx;
    v->num_rows = scalar_size(f->V0);
    v->num_cols = scalar_size(f->V1);
    v->nnz = s->nnz;
    v->parent = s;
    v->id = g_next_id++;
    f->sp = nullptr;
    f->view.reset();
    reset_gather_plan(*f);
    launch_build_view(*f, *s, row_offset, col_offset, *v, st);
    check_device_errors(f->ctx, st, FE_ERR_PATTERN);  // the form stays unbound on a missing coupling
    f->view = std::move(v);
    f->sp = f->view.get();
  });
}

int fe_form_destroy(fe_form f) {
  return guard([&] { delete f; });
}

int fe_form_create_ffcx(fe_context ctx, fe_mesh mesh, fe_dofmap test, fe_dofmap trial, int integral_type,
                        const char* tabulate_name, const char* tabulate_body, int num_coefficients,
                        const int* coefficient_sizes, int num_constants, const char* cachedir, fe_form* out) {
  return guard([&] {
    DeviceScope d(ctx);
    FE_REQUIRE(out && mesh, "null argument");
    FE_REQUIRE(test || !trial, "a trial dofmap needs a test dofmap");
    for (fe_dofmap V : {test, trial}) {
      if (!V) continue;
      FE_REQUIRE(V->ctx == ctx && V->num_cells == mesh->num_cells, "dofmap and mesh cell counts differ");
      FE_REQUIRE(!V->excluded || integral_type == FE_INTEGRAL_CELL,
                 "facet integrals take unrestricted dofmaps");
    }
    auto f = std::make_unique<fe_form_s>();
    f->ctx = ctx;
    f->rank = (test ? 1 : 0) + (trial ? 1 : 0);
    f->mesh = mesh;
    f->V0 = test;
    f->V1 = trial;
    ffcx_create(*f, integral_type, tabulate_name, tabulate_body, num_coefficients, coefficient_sizes, num_constants,
                cachedir);
    *out = f.release();
  });
}

int fe_form_set_coefficient_field(fe_form f, int index, fe_dofmap cmap, const double* values, int64_t n,
                                  int values_on_device, void* stream) {
  return guard([&] {
    FE_REQUIRE(f && f->ffcx, "not a form built from an FFCx body");
    DeviceScope d(f->ctx);
    ffcx_set_coefficient(*f, index, cmap, values, n, values_on_device != 0, as_stream(stream));
  });
}

int fe_form_set_constants(fe_form f, const double* values, int n, void* stream) {
  return guard([&] {
    FE_REQUIRE(f && f->ffcx, "not a form built from an FFCx body");
    DeviceScope d(f->ctx);
    ffcx_set_constants(*f, values, n, as_stream(stream));
  });
}

int fe_bc_create(fe_context ctx, int64_t num_dofs, const uint8_t* markers, const int32_t* dofs, int64_t n_bc,
                 int64_t n_owned, const double* g, fe_bc* out) {
  return guard([&] {
    DeviceScope d(ctx);
    FE_REQUIRE(out && num_dofs >= 0 && n_bc >= 0 && n_owned >= 0 && n_owned <= n_bc, "invalid argument");
    FE_REQUIRE(markers && g && (dofs || !n_bc), "null input array");
    std::vector<uint8_t> listed((size_t)num_dofs, 0);
    int64_t distinct = 0, marked = 0;
    for (int64_t q = 0; q < n_bc; ++q) {
      FE_REQUIRE(dofs[q] >= 0 && dofs[q] < num_dofs, "BC dof out of range at " + std::to_string(q));
      FE_REQUIRE(markers[dofs[q]], "BC dof " + std::to_string(dofs[q]) + " is not marked");
      distinct += !listed[dofs[q]];
      listed[dofs[q]] = 1;
    }
    for (int64_t d = 0; d < num_dofs; ++d) marked += markers[d] != 0;
    auto bc = std::make_unique<fe_bc_s>();
    bc->markers_are_dofs = distinct == n_bc && marked == n_bc;
    {
      std::vector<int32_t> owned(dofs, dofs + n_owned);
      std::sort(owned.begin(), owned.end());
      upload(bc->rows_sorted, owned.data(), owned.size());
    }
    bc->ctx = ctx;
    bc->num_dofs = num_dofs;
    bc->n_bc = n_bc;
    bc->n_owned = n_owned;
    upload(bc->markers, markers, (size_t)num_dofs);
    upload(bc->dofs, dofs, (size_t)n_bc);
    upload(bc->g, g, (size_t)num_dofs);
    *out = bc.release();
  });
}

int fe_bc_update(fe_bc bc, const double* g, void* stream) {
  return guard([&] {
    FE_REQUIRE(bc && g, "null argument");
    DeviceScope d(bc->ctx);
    FE_CUDA(cudaMemcpyAsync(bc->g.p, g, bc->num_dofs * sizeof(double), cudaMemcpyHostToDevice, as_stream(stream)));
  });
}

int fe_bc_destroy(fe_bc bc) {
  return guard([&] { delete bc; });
}

}  // extern "C"

namespace fe {
// deterministic sorted-slot variant (fe_gather.cu)
void assemble_matrix_gather(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, double diagonal,
                            bool zero, cudaStream_t s);
}  // namespace fe

extern "C" {

int fe_assemble_matrix(fe_form a, double* values, fe_bc bc0, fe_bc bc1, double diagonal, unsigned flags,
                       void* stream) {
  return guard([&] {
    FE_REQUIRE(a, "null form");
    FE_REQUIRE(a->rank == 2, "assemble_matrix needs a bilinear form");
    FE_REQUIRE(a->sp, "bind a sparsity pattern first (fe_form_bind_sparsity)");
    FE_REQUIRE(values || a->sp->nnz == 0, "null values array");
    DeviceScope d(a->ctx);
    for (int q = 0; q < 2; ++q) {
      const int need = (a->kind == FE_FORM_VP2_ELASTICITY) ? 2 : (a->kind == FE_FORM_P2_STIFFNESS ? 1 : 0);
      if (q < need) FE_REQUIRE(a->coeff[q].kind >= 0, "coefficient " + std::to_string(q) + " is not set");
    }
    if (bc0) FE_REQUIRE(bc0->num_dofs == a->sp->num_rows, "bc0 size differs from the number of rows");
    if (bc1) FE_REQUIRE(bc1->num_dofs == a->sp->num_cols, "bc1 size differs from the number of columns");
    cudaStream_t st = as_stream(stream);
    const bool zero = (flags & FE_ASM_ZERO) != 0;
    const bool view = a->sp->parent != nullptr;
    if (view)
      FE_REQUIRE(!(flags & (FE_ASM_DETERMINISTIC | FE_ASM_SORTED_SLOT | FE_ASM_TILE | FE_ASM_ROW_GATHER |
                            FE_ASM_BLOCK)),
                 "a form bound to a block pattern assembles with the atomic scatter only");
    if (a->ffcx) {
      FE_REQUIRE(!(flags & (FE_ASM_DETERMINISTIC | FE_ASM_SORTED_SLOT | FE_ASM_TILE | FE_ASM_ROW_GATHER |
                            FE_ASM_BLOCK)),
                 "forms built from FFCx bodies assemble with the atomic scatter only");
      if (zero) launch_zero(values, a->sp->nnz, st);
      ffcx_assemble_matrix(*a, values, bc0, bc1, st);
      if (bc0) launch_set_diagonal(*a->sp, *bc0, diagonal, values, st);
      return;
    }
    if (is_ifacet_kind(a->kind)) {
      FE_REQUIRE(!(flags & (FE_ASM_DETERMINISTIC | FE_ASM_SORTED_SLOT | FE_ASM_TILE | FE_ASM_ROW_GATHER |
                            FE_ASM_BLOCK)),
                 "interior-facet forms assemble with the atomic scatter only");
      if (zero) launch_zero(values, a->sp->nnz, st);
      assemble_matrix_ifacets(*a, values, bc0, bc1, st);
      if (bc0) launch_set_diagonal(*a->sp, *bc0, diagonal, values, st);
      return;
    }
    if (is_facet_kind(a->kind)) {
      FE_REQUIRE(!(flags & (FE_ASM_DETERMINISTIC | FE_ASM_SORTED_SLOT | FE_ASM_TILE | FE_ASM_ROW_GATHER |
                            FE_ASM_BLOCK)),
                 "exterior-facet forms assemble with the atomic scatter only");
      FE_REQUIRE(a->V0 == a->V1, "exterior-facet mass forms need the same test and trial dofmap");
      if (zero) launch_zero(values, a->sp->nnz, st);
      assemble_matrix_facets(*a, values, bc0, bc1, st);
      if (bc0) launch_set_diagonal(*a->sp, *bc0, diagonal, values, st);
      return;
    }
    if (flags & FE_ASM_SORTED_SLOT) {
      assemble_matrix_gather(*a, values, bc0, bc1, diagonal, zero, st);
      return;
    }
    if (flags & FE_ASM_COALESCED)
      FE_REQUIRE(a->kind == FE_FORM_P2_STIFFNESS || a->kind == FE_FORM_VP2_ELASTICITY ||
                     (a->kind == FE_FORM_P3_STIFFNESS && a->precision == FE_PREC_FP64),
                 "the coalesced variant supports P2 stiffness, vector-P2 elasticity and FP64 P3 stiffness");
    if (flags & FE_ASM_GROUPED) {
      FE_REQUIRE(grouped_supported(*a), "the grouped variant supports P2 stiffness on an unrestricted pattern");
      if (assemble_matrix_grouped(*a, values, bc0, bc1, zero, st)) {
        if (bc0) launch_set_diagonal(*a->sp, *bc0, diagonal, values, st);
        return;
      }
      // no repeated group structure in this mesh: the atomic scatter below
    }
    if (flags & FE_ASM_DETERMINISTIC) {
      if (tile_supported(*a)) {
        assemble_matrix_tiled(*a, values, bc0, bc1, zero, true, st);
        if (bc0) launch_set_diagonal(*a->sp, *bc0, diagonal, values, st);
      } else {
        assemble_matrix_gather(*a, values, bc0, bc1, diagonal, zero, st);
      }
      return;
    }
    if (flags & FE_ASM_TILE) {
      FE_REQUIRE(tile_supported(*a), "the tile variant supports P1/P2 stiffness only");
      assemble_matrix_tiled(*a, values, bc0, bc1, zero, false, st);
      if (bc0) launch_set_diagonal(*a->sp, *bc0, diagonal, values, st);
      return;
    }
    if (flags & FE_ASM_ROW_GATHER) {
      FE_REQUIRE(rowgather_supported(*a), "the row-gather variant supports P1 stiffness only");
      assemble_matrix_rowgather(*a, values, bc0, bc1, zero, st);
      if (bc0) launch_set_diagonal(*a->sp, *bc0, diagonal, values, st);
      return;
    }
    // default: the block variant for P1 meshes above ~1M cells (measured faster
    // on B200 at 12.6M cells: 0.54 vs 0.73 ms), the FP64-atomic scatter otherwise
    // (for P2 stiffness with warp-coalesced reductions, below)
    const bool auto_block = !(flags & FE_ASM_ATOMIC) && !view && a->kind == FE_FORM_P1_STIFFNESS &&
                            a->mesh->num_cells >= (int64_t(1) << 20);
    const bool want_block = (flags & FE_ASM_BLOCK) || auto_block;
    if (flags & FE_ASM_BLOCK) FE_REQUIRE(block_supported(*a), "the block variant supports P1/P2 stiffness only");
    if (want_block && block_supported(*a)) {
      assemble_matrix_block(*a, values, bc0, bc1, zero, diagonal, st);
      return;
    }
    // every built-in bilinear form is symmetric: on a symmetric pattern with
    // the same BCs on rows and columns, P1, P3 and vector-P2 elasticity
    // reduce each unique entry once into the upper triangle and a gather pass
    // fills the lower triangle from it (on B200, vector P2 n=64: 7.6 ms
    // instead of about 12 ms; P3 n=48: 1.79 instead of 2.23 ms; P1 n=128 on
    // the atomic path: 0.73 instead of 0.85 ms; P1 n=32: equal).  For P2 the
    // pass costs what the halved reductions save (n=96: 2.80 ms either way),
    // so it keeps both reductions, as does FE_ASM_FULL_SCATTER for every form.
    // P2 stiffness, vector-P2 elasticity and FP64 P3 stiffness by default
    // with warp-coalesced reductions (measured on B200 at P2 n=96: 2.44 ms per
    // matrix call against 2.81 ms for the thread-per-cell reductions, which
    // FE_ASM_ATOMIC keeps; P3 n=48: 1.30 against 1.78 ms for the upper mode)
    const bool coalesced = (flags & FE_ASM_COALESCED) ||
                           (!(flags & FE_ASM_ATOMIC) && !view &&
                            (a->kind == FE_FORM_P2_STIFFNESS || a->kind == FE_FORM_VP2_ELASTICITY ||
                             (a->kind == FE_FORM_P3_STIFFNESS && a->precision == FE_PREC_FP64)));
    const bool upper = !coalesced && zero && !view && !(flags & FE_ASM_FULL_SCATTER) &&
                       (a->kind == FE_FORM_VP2_ELASTICITY || a->kind == FE_FORM_P3_STIFFNESS ||
                        a->kind == FE_FORM_P1_STIFFNESS || a->kind == FE_FORM_P1_MASS ||
                        a->kind == FE_FORM_VP2_MASS) && a->V0 == a->V1 &&
                       bc0 == bc1 && ensure_mirror(*a->sp, st, a->V0->bs);
    // the element scatters skip BC rows: their diagonal is written with the
    // zero pass (plain patterns; a block view's row table is not the values')
    const bool zero_diag = zero && !view;
    if (zero_diag) launch_zero_diagonal(*a->sp, bc0, diagonal, values, st);
    else if (zero) launch_zero(values, a->sp->nnz, st);
    MatLaunch L{};
    L.kind = a->kind;
    L.precision = a->precision;
    L.num_cells = a->mesh->num_cells;
    L.x = a->mesh->x.p;
    L.geom = a->mesh->geom.p;
    L.dofs0 = a->V0->dofs.p;
    L.dofs1 = a->V1->dofs.p;
    L.k0 = a->V0->k;
    L.k1 = a->V1->k;
    L.bs = a->V0->bs;
    L.pos = a->pos.p;
    L.row_ptr = a->sp->row_ptr.p;
    L.bc0 = bc0 ? bc0->markers.p : nullptr;
    L.bc1 = bc1 ? bc1->markers.p : nullptr;
    L.c0 = &a->coeff[0];
    L.c1 = &a->coeff[1];
    L.values = values;
    L.upper = upper ? 1 : 0;
    L.cta_cells = a->launch_cells;
    L.stage = a->launch_stage;
    L.coalesced = coalesced ? 1 : 0;
    launch_matrix_atomic(L, st);
    if (upper) launch_mirror_lower(*a->sp, values, st);
    if (bc0 && !zero_diag) launch_set_diagonal(*a->sp, *bc0, diagonal, values, st);
  });
}

int fe_assemble_matrix_batch(fe_form a, int num_instances, const double* const* coefficients,
                             double* const* values, fe_bc bc0, fe_bc bc1, double diagonal, unsigned flags,
                             void* stream) {
  return guard([&] {
    FE_REQUIRE(a, "null form");
    FE_REQUIRE(a->rank == 2, "assemble_matrix_batch needs a bilinear form");
    FE_REQUIRE(a->sp, "bind a sparsity pattern first (fe_form_bind_sparsity)");
    FE_REQUIRE(!a->sp->parent, "batched assembly does not take block-bound forms");
    if (bc0) FE_REQUIRE(bc0->num_dofs == a->sp->num_rows, "bc0 size differs from the number of rows");
    if (bc1) FE_REQUIRE(bc1->num_dofs == a->sp->num_cols, "bc1 size differs from the number of columns");
    DeviceScope d(a->ctx);
    assemble_matrix_batch(*a, num_instances, coefficients, values, bc0, bc1, diagonal, (flags & FE_ASM_ZERO) != 0,
                          as_stream(stream));
  });
}

int fe_assemble_scalar(fe_form M, double* result, void* stream) {
  return guard([&] {
    FE_REQUIRE(M && result, "null argument");
    if (M->ffcx) {
      FE_REQUIRE(M->rank == 0, "assemble_scalar needs a functional");
      DeviceScope d(M->ctx);
      *result = ffcx_assemble_scalar(*M, as_stream(stream));
      return;
    }
    FE_REQUIRE(M->rank == 0 && is_scalar_kind(M->kind), "assemble_scalar needs a functional");
    if (M->kind == FE_FORM_INTEGRAL || M->kind == FE_FORM_FACET_INTEGRAL || M->kind == FE_FORM_JUMP_NORM)
      FE_REQUIRE(M->coeff[0].kind >= 0, "coefficient 0 is not set");
    if (M->kind == FE_FORM_JUMP_NORM)
      FE_REQUIRE(M->facets_set, "set the interior facets first (fe_form_set_interior_facets)");
    if (M->kind == FE_FORM_P1_ENERGY || M->kind == FE_FORM_P2_ENERGY)
      FE_REQUIRE(M->coeff[1].kind >= 0, "coefficient 1 (u) is not set");
    DeviceScope d(M->ctx);
    *result = assemble_scalar(*M, as_stream(stream));
  });
}

int fe_zero_entries(double* values, int64_t n, void* stream) {
  return guard([&] {
    FE_REQUIRE(n >= 0 && (values || n == 0), "invalid argument");
    launch_zero(values, n, as_stream(stream));
  });
}

int fe_assemble_vector(fe_form Lf, double* b, unsigned flags, void* stream) {
  return guard([&] {
    FE_REQUIRE(Lf, "null form");
    FE_REQUIRE(Lf->rank == 1, "assemble_vector needs a linear form");
    FE_REQUIRE(b || scalar_size(Lf->V0) == 0, "null vector");
    if (Lf->ffcx) {
      DeviceScope d(Lf->ctx);
      cudaStream_t st = as_stream(stream);
      if (flags & FE_ASM_ZERO) launch_zero(b, scalar_size(Lf->V0), st);
      ffcx_assemble_vector(*Lf, b, st);
      return;
    }
    FE_REQUIRE(Lf->coeff[0].kind >= 0, "coefficient 0 (f) is not set");
    DeviceScope d(Lf->ctx);
    cudaStream_t st = as_stream(stream);
    const int64_t n = scalar_size(Lf->V0);
    if (flags & FE_ASM_ZERO) launch_zero(b, n, st);
    if (is_facet_kind(Lf->kind)) {
      assemble_vector_facets(*Lf, b, n, st);
      return;
    }
    if (is_ifacet_kind(Lf->kind)) {
      FE_REQUIRE(Lf->facets_set, "set the interior facets first (fe_form_set_interior_facets)");
      assemble_vector_ifacets(*Lf, b, n, st);
      return;
    }
    VecLaunch L{};
    L.kind = Lf->kind;
    L.num_cells = Lf->mesh->num_cells;
    L.x = Lf->mesh->x.p;
    L.geom = Lf->mesh->geom.p;
    L.dofs = Lf->V0->dofs.p;
    L.k = Lf->V0->k;
    L.bs = Lf->V0->bs;
    L.f = &Lf->coeff[0];
    L.b = b;
    L.num_values = n;
    launch_vector(L, st);
  });
}

int fe_assemble_diagonal(fe_form a, double* b, unsigned flags, void* stream) {
  return guard([&] {
    FE_REQUIRE(a, "null form");
    FE_REQUIRE(a->rank == 2, "the diagonal is taken of a bilinear form");
    FE_REQUIRE(!a->ffcx, "the diagonal of an FFCx form is a linear form of its own (FFCx's \"part\": \"diagonal\")");
    FE_REQUIRE(a->V0 && a->V1 && a->V0->num_blocks == a->V1->num_blocks && a->V0->bs == a->V1->bs &&
                   a->V0->k == a->V1->k,
               "the diagonal needs the same test and trial space");
    FE_REQUIRE(b || scalar_size(a->V0) == 0, "null vector");
    const int need = (a->kind == FE_FORM_VP2_ELASTICITY) ? 2 : (a->kind == FE_FORM_P2_STIFFNESS ? 1 : 0);
    for (int q = 0; q < need; ++q) FE_REQUIRE(a->coeff[q].kind >= 0, "coefficient not set");
    DeviceScope d(a->ctx);
    cudaStream_t st = as_stream(stream);
    const int64_t n = scalar_size(a->V0);
    if (flags & FE_ASM_ZERO) launch_zero(b, n, st);
    MatLaunch L{};
    L.kind = a->kind;
    L.precision = a->precision;
    L.num_cells = a->mesh->num_cells;
    L.x = a->mesh->x.p;
    L.geom = a->mesh->geom.p;
    L.dofs0 = a->V0->dofs.p;
    L.dofs1 = a->V1->dofs.p;
    L.k0 = a->V0->k;
    L.k1 = a->V1->k;
    L.bs = a->V0->bs;
    L.c0 = &a->coeff[0];
    L.c1 = &a->coeff[1];
    launch_diagonal(L, b, n, st);
  });
}

int fe_apply_lifting(double* b, int num_forms, const fe_form* a, const fe_bc* bc1, const double* const* x0,
                     double scale, void* stream) {
  return guard([&] {
    FE_REQUIRE(num_forms >= 0 && (a || !num_forms), "invalid argument");
    for (int i = 0; i < num_forms; ++i)
      FE_REQUIRE(b || !a[i] || scalar_size(a[i]->V0) == 0, "null vector");
    cudaStream_t st = as_stream(stream);
    for (int i = 0; i < num_forms; ++i) {
      fe_form f = a[i];
      FE_REQUIRE(f && f->rank == 2, "apply_lifting needs bilinear forms");
      fe_bc bc = bc1 ? bc1[i] : nullptr;
      if (!bc) continue;
      DeviceScope d(f->ctx);
      FE_REQUIRE(bc->num_dofs == scalar_size(f->V1), "bc size differs from the trial space size");
      if (f->ffcx) {
        ffcx_lifting(*f, *bc, x0 ? x0[i] : nullptr, scale, b, st);
        continue;
      }
      if (is_facet_kind(f->kind)) {
        lifting_facets(*f, *bc, x0 ? x0[i] : nullptr, scale, b, scalar_size(f->V0), st);
        continue;
      }
      if (is_ifacet_kind(f->kind)) {
        FE_REQUIRE(f->facets_set, "set the interior facets first (fe_form_set_interior_facets)");
        lifting_ifacets(*f, *bc, x0 ? x0[i] : nullptr, scale, b, scalar_size(f->V0), st);
        continue;
      }
      const int need = (f->kind == FE_FORM_VP2_ELASTICITY) ? 2 : (f->kind == FE_FORM_P2_STIFFNESS ? 1 : 0);
      for (int q = 0; q < need; ++q) FE_REQUIRE(f->coeff[q].kind >= 0, "coefficient not set");
      auto& cells = lift_cells(*bc, *f->V1, st);
      LiftLaunch L{};
      L.kind = f->kind;
      L.precision = f->precision;
      L.cells = cells.cells.p;
      L.num_list = cells.count;
      L.x = f->mesh->x.p;
      L.geom = f->mesh->geom.p;
      L.dofs0 = f->V0->dofs.p;
      L.dofs1 = f->V1->dofs.p;
      L.k0 = f->V0->k;
      L.k1 = f->V1->k;
      L.bs = f->V0->bs;
      L.c0 = &f->coeff[0];
      L.c1 = &f->coeff[1];
      L.bc1 = bc->markers.p;
      L.g = bc->g.p;
      L.x0 = x0 ? x0[i] : nullptr;
      L.scale = scale;
      L.b = b;
      L.num_values = scalar_size(f->V0);
      launch_lifting(L, st);
    }
  });
}

int fe_interpolate(fe_dofmap target, double* u1, fe_dofmap source, const double* u0, const double* matrix,
                   void* stream) {
  return guard([&] {
    FE_REQUIRE(target && source && matrix, "null argument");
    FE_REQUIRE(target->ctx == source->ctx, "dofmaps belong to different contexts");
    FE_REQUIRE(target->num_cells == source->num_cells, "the spaces are on different meshes (cell counts differ)");
    FE_REQUIRE(target->bs == source->bs, "interpolation maps between spaces of the same block size");
    FE_REQUIRE(!source->excluded, "the source space must be unrestricted");
    FE_REQUIRE((u1 || !target->num_blocks) && (u0 || !source->num_blocks), "null coefficient array");
    DeviceScope d(target->ctx);
    interpolate(*target, u1, *source, u0, matrix, as_stream(stream));
  });
}

int fe_assemble_rhs(fe_form Lf, fe_form a, fe_bc bc, double* b, const double* x0, double scale, unsigned flags,
                    void* stream) {
  return guard([&] {
    FE_REQUIRE(Lf && a, "null form");
    FE_REQUIRE(Lf->rank == 1 && a->rank == 2, "assemble_rhs takes a linear and a bilinear form");
    FE_REQUIRE(Lf->ctx == a->ctx && (!bc || bc->ctx == a->ctx), "the forms and the BC belong to different contexts");
    FE_REQUIRE(scalar_size(Lf->V0) == scalar_size(a->V0) && scalar_size(a->V0) == scalar_size(a->V1),
               "assemble_rhs needs one space for the vector, the test and the trial space");
    FE_REQUIRE(!bc || bc->num_dofs == scalar_size(a->V1), "bc size differs from the trial space size");
    const int64_t n = scalar_size(Lf->V0);
    FE_REQUIRE(b || n == 0, "null vector");
    const bool fused = bc && bc->markers_are_dofs && !Lf->ffcx && !a->ffcx && Lf->mesh == a->mesh &&
                       Lf->V0->dofs.p == a->V0->dofs.p && a->V0->dofs.p == a->V1->dofs.p &&
                       rhs_fused_supported(Lf->kind, a->kind) && Lf->coeff[0].kind >= 0;
    if (!fused) {
      // the same result through the three calls
      rethrow_status(fe_assemble_vector(Lf, b, flags & FE_ASM_ZERO, stream));
      if (bc) {
        const double* xs[1] = {x0};
        rethrow_status(fe_apply_lifting(b, 1, &a, &bc, x0 ? xs : nullptr, scale, stream));
        rethrow_status(fe_set_bc(b, n, bc, x0, scale, stream));
      }
      return;
    }
    const int need = (a->kind == FE_FORM_VP2_ELASTICITY) ? 2 : (a->kind == FE_FORM_P2_STIFFNESS ? 1 : 0);
    for (int q = 0; q < need; ++q) FE_REQUIRE(a->coeff[q].kind >= 0, "coefficient not set");
    DeviceScope d(a->ctx);
    cudaStream_t st = as_stream(stream);
    if (flags & FE_ASM_ZERO) launch_zero(b, n, st);
    auto& cells = lift_cells(*bc, *a->V1, st);
    VecLaunch V{};
    V.kind = Lf->kind;
    V.num_cells = Lf->mesh->num_cells;
    V.x = Lf->mesh->x.p;
    V.geom = Lf->mesh->geom.p;
    V.dofs = Lf->V0->dofs.p;
    V.k = Lf->V0->k;
    V.bs = Lf->V0->bs;
    V.f = &Lf->coeff[0];
    V.b = b;
    V.num_values = n;
    LiftLaunch L{};
    L.kind = a->kind;
    L.precision = a->precision;
    L.cells = cells.cells.p;
    L.num_list = cells.count;
    L.x = a->mesh->x.p;
    L.geom = a->mesh->geom.p;
    L.dofs0 = a->V0->dofs.p;
    L.dofs1 = a->V1->dofs.p;
    L.k0 = a->V0->k;
    L.k1 = a->V1->k;
    L.bs = a->V0->bs;
    L.c0 = &a->coeff[0];
    L.c1 = &a->coeff[1];
    L.bc1 = bc->markers.p;
    L.g = bc->g.p;
    L.x0 = x0;
    L.scale = scale;
    L.b = b;
    L.num_values = n;
    launch_rhs_fused(V, L, bc->dofs.p, bc->n_bc, st);
  });
}

int fe_set_bc(double* b, int64_t num_values, fe_bc bc, const double* x0, double scale, void* stream) {
  return guard([&] {
    FE_REQUIRE(bc, "null bc");
    FE_REQUIRE(b || num_values == 0, "null vector");
    DeviceScope d(bc->ctx);
    launch_set_bc(b, num_values, bc->dofs.p, bc->n_bc, bc->g.p, x0, scale, as_stream(stream));
  });
}

}  // extern "C"
