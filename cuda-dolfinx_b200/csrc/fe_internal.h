// Internal declarations shared by the host ABI (fe_abi.cu), the host sparsity
// builder (fe_sparsity.cpp) and the kernels (fe_kernels.cu, fe_pcg.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cudolfinx_b200.h"

namespace fe {

// Error carrying an fe_status code; caught at the ABI boundary and turned into
// a status + thread-local message.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(int code, const std::string& msg, const char* file, int line);
void set_last_error(const std::string& msg);
void check_cuda(cudaError_t e, const char* what, const char* file, int line);

#define FE_FAIL(code, msg) ::fe::fail((code), (msg), __FILE__, __LINE__)
#define FE_CUDA(call) ::fe::check_cuda((call), #call, __FILE__, __LINE__)
#define FE_REQUIRE(cond, msg)                  \
  do {                                         \
    if (!(cond)) FE_FAIL(FE_ERR_ARG, (msg));   \
  } while (0)

// Device error word bits (set with atomicOr by kernels; never a trap).
enum DeviceError : unsigned {
  DEV_ERR_PATTERN = 1u,    // a cell coupling was not found in the CSR row
  DEV_ERR_ROW_WIDE = 2u,   // a block row has more than 255 block columns
  DEV_ERR_BLOCK = 4u,      // the CSR rows of one block row differ
  DEV_ERR_INDEX = 8u,      // an index outside its array
  DEV_ERR_FACET = 16u,     // the two local facets of an interior facet are not the same triangle
  DEV_ERR_BARRIER = 32u    // a grid barrier was not reached by every block in time
};

// RAII device buffer.
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) {
      cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
      if (e != cudaSuccess) {
        p = nullptr;
        n = 0;
        (void)cudaGetLastError();
        throw Error(FE_ERR_NOMEM, std::string("cudaMalloc of ") + std::to_string(count * sizeof(T)) +
                                      " bytes failed: " + cudaGetErrorString(e));
      }
    }
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

}  // namespace fe

struct fe_context_s {
  int device = 0;
  int num_sms = 0;
  fe::DevBuf<unsigned> err;  // device error word
  // stream-ordered scratch of the solvers (fe_pcg.cu): a pool of this
  // context's own that keeps up to a quarter of the device memory cached
  // between calls, instead of the default pool, which returns its memory at
  // every synchronise and maps it again on the next solve
  cudaMemPool_t scratch_pool = nullptr;
  ~fe_context_s() {
    if (scratch_pool) (void)cudaMemPoolDestroy(scratch_pool);
  }
};

struct fe_mesh_s {
  fe_context ctx = nullptr;
  int64_t num_nodes = 0, num_cells = 0;
  int nodes_per_cell = 4;
  fe::DevBuf<double> x;      // [num_nodes*3]
  fe::DevBuf<int32_t> geom;  // [num_cells*4]
  std::vector<double> host_x;      // host copies (tile planning)
  std::vector<int32_t> host_geom;
};

struct fe_dofmap_s {
  fe_context ctx = nullptr;
  int64_t num_cells = 0, num_blocks = 0;
  int k = 0, bs = 1;
  fe::DevBuf<int32_t> dofs;      // [num_cells*k] block dofs
  std::vector<int32_t> host;     // host copy (sparsity build)
  uint64_t id = 0;               // unique id for caches
  bool excluded = false;         // some entries are -1: dofs outside a restriction
  fe::DevBuf<int32_t> owner;     // [num_blocks] lowest cell*k + i listing each dof (interpolation), on first use
};

struct fe_sparsity_s {
  fe_context ctx = nullptr;
  int64_t num_rows = 0, num_cols = 0, nnz = 0;
  fe::DevBuf<int32_t> row_ptr;   // [num_rows+1]
  fe::DevBuf<int32_t> col;       // [nnz]
  fe::DevBuf<int32_t> diag;      // [num_rows] slot of (r, r) or -1
  std::vector<int32_t> host_row_ptr;  // host copy (tile planning)
  uint64_t id = 0;
  // transpose map of the strictly lower triangle (symmetric patterns): one
  // {lower slot, slot of its transpose} pair per strictly-lower slot, in slot
  // order; built on first use
  struct Mirror {
    fe::DevBuf<int2> pairs;         // [lower slots]
    int64_t nlower = 0;
    // block size 3 (vector P2): one record per node block on or below the
    // block diagonal, {lower base, lower row length, upper base, upper row
    // length}; a diagonal block has upper base == lower base
    int bs = 1;
    fe::DevBuf<int4> blocks;
    int64_t nblocks = 0;
    bool ok = false;                // pattern symmetric with every diagonal present
  };
  std::unique_ptr<Mirror> mirror;
  // block view (fe_form_bind_sparsity_block): the rows of one block form
  // inside a monolithic pattern.  row_ptr[r] is then the first slot of the
  // block's column segment in monolithic row offset + r (nnz = the monolithic
  // count, so zeroing covers the whole value array), diag[r] the slot of the
  // monolithic diagonal entry of that row; col is empty.
  fe_sparsity parent = nullptr;
};

struct fe_bc_s {
  fe_context ctx = nullptr;
  int64_t num_dofs = 0, n_bc = 0, n_owned = 0;
  bool markers_are_dofs = false;  // the marked dofs are exactly the listed ones, each listed once
  fe::DevBuf<int32_t> rows_sorted;  // the n_owned owned dofs in ascending order
  // per pattern id: the owned rows' diagonal slots (ascending) and, per block
  // of the zero-with-diagonal pass, its first slot index; built on first use
  struct DiagSlots {
    fe::DevBuf<int32_t> slots, starts;
    int64_t chunk = 0, grid = 0;
  };
  mutable std::map<uint64_t, std::unique_ptr<DiagSlots>> diag_slots;  // a cache: filled on const use
  fe::DevBuf<uint8_t> markers;   // [num_dofs]
  fe::DevBuf<int32_t> dofs;      // [n_bc], owned first
  fe::DevBuf<double> g;          // [num_dofs]
  // cells with a marked dof, per dofmap id (lifting); built on first use
  struct CellList {
    fe::DevBuf<int32_t> cells;
    int64_t count = 0;
  };
  std::map<uint64_t, std::unique_ptr<CellList>> lift_cells;
};

namespace fe {
struct Coefficient {
  int kind = -1;                 // fe_coeff_kind, -1 = unset
  fe_dofmap map = nullptr;       // P1 dofmap
  const double* values = nullptr;  // device pointer (own or caller's)
  DevBuf<double> own;            // storage when uploaded from host
  int64_t n = 0;
  double constant[3] = {1.0, 1.0, 1.0};
};
}  // namespace fe

struct fe_form_s {
  fe_context ctx = nullptr;
  int kind = 0, rank = 0;
  int precision = FE_PREC_FP64;
  int launch_cells = 0;  // atomic scatter launch shape (fe_form_set_launch)
  int launch_stage = 1;
  fe_mesh mesh = nullptr;
  fe_dofmap V0 = nullptr, V1 = nullptr;
  fe::Coefficient coeff[2];
  fe_sparsity sp = nullptr;
  std::unique_ptr<fe_sparsity_s> view;  // block view that sp points to (fe_form_bind_sparsity_block)
  fe::DevBuf<uint8_t> pos;       // [num_cells * k0 * k1] block column positions (padded to 16 B)
  fe::DevBuf<int32_t> facets;    // exterior-facet forms: [num_facets][2] (cell, local facet);
                                 // interior-facet forms: [num_facets][4] (cell0, facet0, cell1, facet1)
  int64_t num_facets = 0;
  std::vector<int32_t> host_facets;        // interior-facet forms: host copy (pattern construction)
  bool facets_set = false;                 // fe_form_set_facets / fe_form_set_interior_facets was called
  fe::DevBuf<int32_t> macro0, macro1;      // interior-facet forms: [num_facets][2k] test / trial dofs
                                           // of the two cells (cell0's, then cell1's)
  fe::DevBuf<double> scalar_partial;  // functionals: per-block partial sums + the result
  // deterministic sorted-slot plan (fe_gather.cu); built on first use
  struct Gather;
  std::unique_ptr<Gather> gather;
  // owner-computes tile plan (fe_tile.cu); built on first use
  struct TilePlan;
  std::unique_ptr<TilePlan> tiles;
  // row-gather plan (fe_rowgather.cu): inverse dofmap; built on first use
  struct RowPlan;
  std::unique_ptr<RowPlan> rows;
  // cell-block plan (fe_block.cu); built on first use
  struct BlockPlan;
  std::unique_ptr<BlockPlan> blocks;
  // batched-instance plan (fe_batch.cu); built on first use
  struct BatchPlan;
  std::unique_ptr<BatchPlan> batch;
  // form integral given as an FFCx tabulate_tensor body (fe_ffcx.cu)
  struct Ffcx;
  std::unique_ptr<Ffcx> ffcx;
  // grouped-summation plan (fe_group.cu); built on first use
  struct GroupPlan;
  std::unique_ptr<GroupPlan> groups;

  bool group_plan_failed = false;  // the mesh has no repeated group structure
  fe_form_s();
  ~fe_form_s();
};

namespace fe {
struct FfcxLibrary;
// internal kinds of forms built from FFCx tabulate_tensor bodies (fe_ffcx.cu)
constexpr int FE_FORM_FFCX_CELL = 41;
constexpr int FE_FORM_FFCX_EXTERIOR = 42;
constexpr int FE_FORM_FFCX_INTERIOR = 43;
inline bool is_ffcx_kind(int kind) { return kind >= FE_FORM_FFCX_CELL && kind <= FE_FORM_FFCX_INTERIOR; }
}  // namespace fe

struct fe_form_s::Ffcx {
  int integral_type = FE_INTEGRAL_CELL;
  std::string name;                    // the tabulate_tensor function name
  std::string body;                    // its body, as FFCx generated it
  std::vector<int> offsets;            // coefficient q: values [offsets[q], offsets[q+1]) of a cell
  int W = 0;                           // coefficient values per cell
  int num_constants = 0;
  std::vector<double> host_consts;
  fe::DevBuf<double> consts;
  struct Field {
    fe_dofmap map = nullptr;           // the coefficient's space
    const double* values = nullptr;    // device values (own or the caller's)
    fe::DevBuf<double> own;
  };
  std::vector<std::unique_ptr<Field>> fields;
  fe::DevBuf<double> packed;           // [cells][W], packed on every assembly call
  fe::DevBuf<uint8_t> perms;           // interior facets: [facets][2] quadrature permutations
  fe::DevBuf<double> partial;          // functionals: block partial sums + the result
  std::shared_ptr<fe::FfcxLibrary> lib;
};

// Plans owned by a form (defined here so every translation unit can destroy them)
struct fe_form_s::Gather {
  fe::DevBuf<int32_t> seg;      // [nnz+1] start of each slot's contribution list
  fe::DevBuf<int32_t> contrib;  // [num_contrib] sorted contribution ids
  fe::DevBuf<double> E;         // [num_contrib] element tensors, entry-major
  int64_t num_contrib = 0;
  int K = 0;                    // scalar dofs per cell (k*bs)
};

struct fe_form_s::TilePlan {
  int64_t ntiles = 0;
  fe::DevBuf<int32_t> tile_rows_ptr;  // [ntiles+1] into rows
  fe::DevBuf<int32_t> rows;           // owned block rows, tile by tile
  fe::DevBuf<int32_t> row_soff;       // offset of each owned row's segment in the tile buffer
  fe::DevBuf<int32_t> row_tile;       // [block rows] owning tile of each row
  fe::DevBuf<int32_t> row_local;      // [block rows] index of the row inside its tile
  fe::DevBuf<int32_t> tile_cells_ptr; // [ntiles+1] into cells
  fe::DevBuf<int32_t> cells;          // cells touching each tile (ascending within a tile)
  fe::DevBuf<int32_t> tile_rec_ptr;   // [ntiles+1] into recs
  fe::DevBuf<uint32_t> recs;          // (row_local << 16) | (lc << 8) | i
  fe::DevBuf<int32_t> tile_goff_ptr;  // [ntiles+1] into goff
  fe::DevBuf<int32_t> goff;           // per chunk: NG+1 offsets relative to the tile's first record
  int64_t total_cells = 0;            // sum of tile cell lists (>= num_cells: border cells repeat)
};

struct fe_form_s::RowPlan {
  fe::DevBuf<int32_t> inc_ptr;        // [block rows + 1]
  fe::DevBuf<int32_t> inc;            // incidences cell*k + i, grouped by row
};

struct fe_form_s::BlockPlan {
  int64_t nblocks = 0;
  const fe_dofmap_s* coef_map_owner = nullptr;  // P1 coefficient dofmap the plan copied
  fe::DevBuf<int32_t> block_ptr;      // [nblocks+1] cell ranges (block order)
  fe::DevBuf<int32_t> brow_ptr;       // [nblocks+1] into rows/soff
  fe::DevBuf<int32_t> rows;           // touched block rows per block (ascending)
  fe::DevBuf<int32_t> soff;           // window offset of each touched row
  fe::DevBuf<uint16_t> lrow;          // [cells][k] window row of each local dof
  fe::DevBuf<int32_t> cell_id;        // block order -> original cell
  fe::DevBuf<int32_t> geom;           // [cells][4] geometry dofmap, block order
  fe::DevBuf<int32_t> dofs0, dofs1;   // [cells][k] form dofmaps, block order
  fe::DevBuf<uint8_t> pos;            // [cells][k*k] slot bytes, block order
  fe::DevBuf<int32_t> coef_map;       // [cells][4] P1 coefficient dofmap, block order
  fe::DevBuf<double> gbound;          // [nblocks] geometric part of the element-entry bound
  int fx_bits = 50;                   // fixed-point bits S of the block bound: slot sums of up to
                                      // max cells-per-dof contributions of |w| < 2^S fit in 63 bits
  fe::DevBuf<int32_t> gvert_ptr;      // [nblocks+1] into gx: each block's geometry nodes
  fe::DevBuf<double> gx;              // [block nodes][3] coordinates, block by block
  fe::DevBuf<uint16_t> glocal;        // [cells][4] block-local geometry node of each cell vertex
  fe::DevBuf<int32_t> rec_ptr;        // P1: [nblocks+1] per-cell records of each block, padded to
                                      // whole warps and stored in the kernel's lane order
};

struct fe_form_s::GroupPlan {
  int64_t ngroups = 0, ntemplates = 0;
  fe::DevBuf<int32_t> tmpl_of;        // [groups] template of each group
  fe::DevBuf<int4> tmeta;             // per template: entry offset, entry count, contribution offset,
                                      // first-dof offset
  fe::DevBuf<int32_t> tnd;            // per template: group-local dofs
  fe::DevBuf<uint2> ent;              // distinct (row, column) entries of all templates
  fe::DevBuf<uint16_t> contrib;       // their (cell, upper entry) contributions
  fe::DevBuf<uint16_t> first;         // group-local dof -> (cell, local dof) of its first appearance
};

struct fe_form_s::BatchPlan {
  int64_t num_records = 0;            // num_cells * K * K
  int KK = 0;                         // element entries per cell
  fe::DevBuf<int32_t> rec_cell;       // [records] cell of each slot-sorted record
  fe::DevBuf<uint8_t> rec_entry;      // [records] local entry i*K+j of each record
  fe::DevBuf<int32_t> slot_row;       // [nnz] CSR row of each slot
  fe::DevBuf<double> E;               // [cells][KK] unit-coefficient element tensors (FP32 values)
  fe::DevBuf<double2> rec;            // [records] {entry value, cell} (16 B each)
  bool rec_valid = false;             // E and rec built (they depend on the mesh and the plan only)
  fe::DevBuf<unsigned> barrier;       // grid-barrier counter of the fused launch
  fe::DevBuf<float> kp;               // [cells][ld] packed instance coefficients (FP32)
  int64_t kp_ld = 0;
};

namespace fe {

// ---- host sparsity (fe_sparsity.cpp) ----
void build_block_pattern(const int32_t* dofs0, const int32_t* dofs1, int64_t num_cells, int k0, int k1,
                         int64_t nblock_rows, int64_t nblock_cols, std::vector<int64_t>& bptr,
                         std::vector<int32_t>& bcol);
void unroll_pattern(const std::vector<int64_t>& bptr, const std::vector<int32_t>& bcol, int bs0, int bs1,
                    std::vector<int32_t>& row_ptr, std::vector<int32_t>& col, std::vector<int32_t>& diag);
// one coupling of a block system: the cell couplings of (rows, cols) placed
// at scalar offsets of the monolithic matrix; -1 entries are skipped
struct SystemPart {
  const fe_dofmap_s* rows;
  const fe_dofmap_s* cols;
  int64_t row_offset, col_offset;
};
// monolithic scalar pattern: the union of the parts' unrolled couplings, each
// row's columns sorted and unique (DOLFINx's block SparsityPattern, block
// size 1, as create_cuda_matrix_block builds it)
void build_system_pattern(const std::vector<SystemPart>& parts, int64_t num_rows, int64_t num_cols,
                          std::vector<int32_t>& row_ptr, std::vector<int32_t>& col, std::vector<int32_t>& diag);

// ---- kernels (fe_kernels.cu) ----
struct MatLaunch {
  int kind, precision;
  int64_t num_cells;
  const double* x;
  const int32_t* geom;
  const int32_t* dofs0;
  const int32_t* dofs1;
  int k0, k1, bs;
  const uint8_t* pos;
  const int32_t* row_ptr;
  const uint8_t* bc0;
  const uint8_t* bc1;
  const Coefficient* c0;
  const Coefficient* c1;
  double* values;
  int upper = 0;  // reduce only into the upper triangle and the diagonal
  int cta_cells = 0;  // cells per CTA of the P1 / P2 atomic kernels (0: 128)
  int stage = 1;      // P2 atomic kernel: stage the byte maps in shared memory
  int coalesced = 0;  // P2: reductions issued per warp, row by row (k_mat_p2_coal)
};
void launch_zero(double* v, int64_t n, cudaStream_t s);
// values = 0, then values[diag slot of each owned bc row] = diagonal, in one
// launch (for scatters that skip BC rows); bc may be null (zero only)
void launch_zero_diagonal(const fe_sparsity_s& sp, const fe_bc_s* bc, double diagonal, double* values,
                          cudaStream_t s);
// symmetric-pattern transpose map (built once per pattern); false if the
// pattern is not symmetric or lacks a diagonal entry
bool ensure_mirror(fe_sparsity_s& sp, cudaStream_t s, int bs = 1);
// values[lower slot] = values[its transpose] for every strictly-lower slot
void launch_mirror_lower(const fe_sparsity_s& sp, double* values, cudaStream_t s);
void launch_build_slotmap(const fe_form_s& f, cudaStream_t s);
// block view of a monolithic pattern for form f at the given scalar offsets:
// fills view.row_ptr (segment starts), view.diag and f.pos
void launch_build_view(const fe_form_s& f, const fe_sparsity_s& mono, int64_t row_offset, int64_t col_offset,
                       fe_sparsity_s& view, cudaStream_t s);
void launch_matrix_atomic(const MatLaunch& a, cudaStream_t s);
// diagonal of a cell bilinear form into b (no BCs)
void launch_diagonal(const MatLaunch& a, double* b, int64_t num_values, cudaStream_t s);
void launch_set_diagonal(const fe_sparsity_s& sp, const fe_bc_s& bc, double diagonal, double* values,
                         cudaStream_t s);

struct VecLaunch {
  int kind;
  int64_t num_cells;
  const double* x;
  const int32_t* geom;
  const int32_t* dofs;
  int k, bs;
  const Coefficient* f;
  double* b;
  int64_t num_values;
};
void launch_vector(const VecLaunch& a, cudaStream_t s);

struct LiftLaunch {
  int kind, precision;
  const int32_t* cells;   // cells with a marked trial dof
  int64_t num_list;
  const double* x;
  const int32_t* geom;
  const int32_t* dofs0;
  const int32_t* dofs1;
  int k0, k1, bs;
  const Coefficient* c0;
  const Coefficient* c1;
  const uint8_t* bc1;
  const double* g;
  const double* x0;
  double scale;
  double* b;
  int64_t num_values;
  const uint8_t* skip = nullptr;  // rows left out of the scatter (stored by set_bc in the same pass)
};
void launch_lifting(const LiftLaunch& a, cudaStream_t s);
void launch_mark_cells(const int32_t* dofs, int64_t num_cells, int k, int bs, const uint8_t* markers,
                       int32_t* out_cells, unsigned long long* out_count, cudaStream_t s);
void launch_set_bc(double* b, int64_t num_values, const int32_t* dofs, int64_t n_bc, const double* g,
                   const double* x0, double scale, cudaStream_t s);
// assemble_vector + apply_lifting + set_bc in two launches (lifting; vector
// and set_bc) for the pairs
// (P1 load, P1 stiffness), (P2 load, P2 stiffness), (P3 load, P3 stiffness),
// (vector-P2 load, elasticity); the lifting launch's bc1 markers are the rows
// the scatters skip and bc_dofs the rows the kernel stores.
bool rhs_fused_supported(int vec_kind, int mat_kind);
void launch_rhs_fused(const VecLaunch& v, const LiftLaunch& l, const int32_t* bc_dofs, int64_t n_bc,
                      cudaStream_t s);

// same-map interpolation u1 = I u0 (fe_interp.cu); im is the host
// [target.k][source.k] matrix; one owner cell per target dof
void interpolate(fe_dofmap_s& target, double* u1, const fe_dofmap_s& source, const double* u0, const double* im,
                 cudaStream_t s);

// error word of the current context's kernels
unsigned* device_error_word(fe_context ctx);

// drops the deterministic plans of a form (fe_gather.cu, fe_tile.cu)
void reset_gather_plan(fe_form_s& f);
void reset_tile_plan(fe_form_s& f);

// owner-computes tile assembly (fe_tile.cu): true if the form kind has a tile kernel
bool tile_supported(const fe_form_s& f);
void assemble_matrix_tiled(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, bool zero,
                           bool deterministic, cudaStream_t s);

// grouped assembly (fe_group.cu) for P2 stiffness: false when the form or its
// mesh does not take it (the caller falls back to the atomic scatter)
bool grouped_supported(const fe_form_s& f);
void reset_group_plan(fe_form_s& f);
bool assemble_matrix_grouped(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, bool zero,
                             cudaStream_t s);

// cell-block assembly (fe_block.cu) for P1/P2 stiffness
bool block_supported(const fe_form_s& f);
void reset_block_plan(fe_form_s& f);
void assemble_matrix_block(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, bool zero,
                           double diagonal, cudaStream_t s);

// exterior-facet forms (fe_facet.cu)
bool is_facet_kind(int kind);
// interior-facet (dS) forms of discontinuous spaces (fe_ifacet.cu)
bool is_ifacet_kind(int kind);
void assemble_matrix_ifacets(const fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1,
                             cudaStream_t s);
void assemble_vector_ifacets(const fe_form_s& f, double* b, int64_t num_values, cudaStream_t s);
void lifting_ifacets(const fe_form_s& f, const fe_bc_s& bc, const double* x0, double scale, double* b,
                     int64_t num_values, cudaStream_t s);
void assemble_matrix_facets(const fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1,
                            cudaStream_t s);
void assemble_vector_facets(const fe_form_s& f, double* b, int64_t num_values, cudaStream_t s);
void lifting_facets(const fe_form_s& f, const fe_bc_s& bc, const double* x0, double scale, double* b,
                    int64_t num_values, cudaStream_t s);

// forms from FFCx tabulate_tensor bodies (fe_ffcx.cu): NVRTC compilation of the
// body inside the engine's skeletons, packed coefficients, constants
void ffcx_create(fe_form_s& f, int integral_type, const char* name, const char* body, int num_coefficients,
                 const int* coefficient_sizes, int num_constants, const char* cachedir);
void ffcx_set_coefficient(fe_form_s& f, int index, fe_dofmap map, const double* values, int64_t n,
                          bool on_device, cudaStream_t s);
void ffcx_set_constants(fe_form_s& f, const double* values, int n, cudaStream_t s);
void ffcx_set_interior_permutations(fe_form_s& f);
void ffcx_assemble_matrix(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, cudaStream_t s);
void ffcx_assemble_vector(fe_form_s& f, double* b, cudaStream_t s);
void ffcx_lifting(fe_form_s& f, const fe_bc_s& bc, const double* x0, double scale, double* b, cudaStream_t s);
double ffcx_assemble_scalar(fe_form_s& f, cudaStream_t s);

// functionals (fe_scalar.cu)
bool is_scalar_kind(int kind);
double assemble_scalar(fe_form_s& f, cudaStream_t s);

// device pattern build (fe_sparsity_dev.cu): fills num_rows/num_cols/nnz,
// row_ptr, col, diag and host_row_ptr of `sp`
void build_pattern_device(const fe_dofmap_s& rows, const fe_dofmap_s& cols, cudaStream_t s, fe_sparsity_s& sp);

// sorted-slot plan (fe_gather.cu): per CSR slot the ordered list of element
// entries that land there; built on first use
void ensure_gather_plan(fe_form_s& f, cudaStream_t s);

// batched assembly of many DG0-coefficient instances on one mesh and pattern
// (fe_batch.cu)
bool batch_supported(const fe_form_s& f);
void reset_batch_plan(fe_form_s& f);
void assemble_matrix_batch(fe_form_s& f, int num_instances, const double* const* coefficients,
                           double* const* values, const fe_bc_s* bc0, const fe_bc_s* bc1, double diagonal,
                           bool zero, cudaStream_t s);

// row-gather assembly (fe_rowgather.cu) for P1 stiffness
bool rowgather_supported(const fe_form_s& f);
void reset_row_plan(fe_form_s& f);
void assemble_matrix_rowgather(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, bool zero,
                               cudaStream_t s);

}  // namespace fe
