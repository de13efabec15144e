/* cudolfinx_b200.h -- C ABI of the B200 finite-element assembly engine.
 *
 * Drop-in boundary for the cudolfinx assembly path.  Every entry point returns
 * an int status (FE_OK = 0); on failure fe_last_error() gives a thread-local
 * message naming the failing call and source location, the same information
 * the reference puts in its std::runtime_error (e.g.
 * cpp/cudolfinx/fem/CUDAFormIntegral.h:961-975) which nanobind turns into a
 * Python RuntimeError.
 *
 * Conventions
 *  - Sizes are int64_t, indices int32_t (the reference's dofmaps and CSR are
 *    int32: cpp/cudolfinx/fem/CUDADofMap.cpp:199-236, la/CUDASeqMatrix.cpp:101-198).
 *  - Pointers documented "host" are read during the call; "device" pointers
 *    must be device memory of the context's GPU.  CSR value arrays and vectors
 *    are caller-owned device memory (PETSc lends its AIJCUSPARSE / VECCUDA
 *    arrays in the reference: la/CUDASeqMatrix.cpp:435-457,
 *    la/CUDAVector.cpp:348-365).
 *  - `stream` is a cudaStream_t passed as void* (NULL = the legacy default
 *    stream).  Work is enqueued asynchronously; nothing synchronises unless
 *    documented.  The reference launches on the NULL stream and calls
 *    cuCtxSynchronize after each kernel (CUDAFormIntegral.cpp:2354-2361).
 */
#ifndef CUDOLFINX_B200_H
#define CUDOLFINX_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum fe_status {
  FE_OK = 0,
  FE_ERR_ARG = 1,       /* invalid argument / size mismatch            */
  FE_ERR_CUDA = 2,      /* a CUDA runtime call or kernel failed         */
  FE_ERR_PATTERN = 3,   /* an element coupling is missing from the CSR  */
  FE_ERR_NOMEM = 4,     /* device allocation refused                    */
  FE_ERR_DEVICE = 5,    /* a kernel reported an error word (no trap)    */
  FE_ERR_NOT_CONVERGED = 6
};

typedef struct fe_context_s* fe_context;
typedef struct fe_mesh_s* fe_mesh;
typedef struct fe_dofmap_s* fe_dofmap;
typedef struct fe_sparsity_s* fe_sparsity;
typedef struct fe_bc_s* fe_bc;
typedef struct fe_form_s* fe_form;

/* Built-in forms (element tensors written from the mathematics; replaces the
 * FFCx tabulate_tensor bodies wrapped by python/cudolfinx/jit.py:61-114). */
enum fe_form_kind {
  FE_FORM_P1_STIFFNESS = 1,    /* k*inner(grad u, grad v)*dx, P1;   coeff 0 = k (constant / DG0 / P1;
                                  a P1 k enters through its cell mean, exact)      */
  FE_FORM_P2_STIFFNESS = 2,    /* k*inner(grad u, grad v)*dx, P2;   coeff 0 = k    */
  FE_FORM_VP2_ELASTICITY = 3,  /* 2mu eps(u):eps(v) + lam div u div v, vector P2;
                                  coeff 0 = lam, coeff 1 = mu                       */
  FE_FORM_P1_MASS = 9,         /* c*u*v*dx, P1;      coeff 0 = c (constant / DG0 / P1) */
  FE_FORM_P2_MASS = 10,        /* c*u*v*dx, P2;      coeff 0 = c (constant / DG0 / P1) */
  FE_FORM_VP2_MASS = 20,       /* rho*inner(u, v)*dx, vector P2; coeff 0 = rho (constant / DG0 / P1) */
  FE_FORM_P1_LOAD = 11,        /* f*v*dx, P1;        coeff 0 = f                    */
  FE_FORM_P2_LOAD = 12,        /* f*v*dx, P2;        coeff 0 = f                    */
  FE_FORM_VP2_LOAD = 13,       /* inner(f, v)*dx, vector P2; coeff 0 = f (3 comps)  */
  /* P3 Lagrange on equispaced points (20 dofs per cell: vertices, two per
   * edge, one per face) */
  FE_FORM_P3_STIFFNESS = 6,    /* k*inner(grad u, grad v)*dx, P3;   coeff 0 = k (constant / DG0) */
  FE_FORM_P3_LOAD = 17,        /* f*v*dx, P3;        coeff 0 = f (constant / DG0)   */
  /* exterior-facet (ds) forms over the facets given by fe_form_set_facets
   * (CUDAFormIntegral.cpp:361-447 vector, :1667-1793 matrix, :721-837 lifting) */
  FE_FORM_P1_FACET_MASS = 4,   /* alpha*u*v*ds, P1;  coeff 0 = alpha (constant / DG0 of the facet's cell) */
  FE_FORM_P2_FACET_MASS = 5,   /* alpha*u*v*ds, P2;  coeff 0 = alpha                 */
  FE_FORM_P1_FACET_LOAD = 14,  /* g*v*ds, P1;        coeff 0 = g (constant / DG0 / P1) */
  FE_FORM_P2_FACET_LOAD = 15,  /* g*v*ds, P2;        coeff 0 = g (constant / DG0 / P1) */
  FE_FORM_VP2_FACET_LOAD = 16, /* inner(t, v)*ds, vector P2; coeff 0 = t (3 comps)   */
  /* interior-facet (dS) forms of discontinuous spaces over the facets given by
   * fe_form_set_interior_facets (CUDAFormIntegral.cpp:451-522 vector,
   * :1988-2103 matrix); jump(u) = u(cell0) - u(cell1), avg(v) = (v(cell0) +
   * v(cell1))/2; a DG0 coefficient enters as the average of the two cells */
  FE_FORM_DG0_JUMP = 7,        /* alpha*jump(u)*jump(v)*dS, DG0 (1 dof/cell); coeff 0 = alpha */
  FE_FORM_DG1_JUMP = 8,        /* the same on DG1 (4 dofs/cell, one per vertex)  */
  FE_FORM_DG0_AVG_LOAD = 18,   /* g*avg(v)*dS, DG0;  coeff 0 = g (constant / DG0) */
  FE_FORM_DG1_AVG_LOAD = 19,   /* g*avg(v)*dS, DG1                                */
  /* functionals (rank 0, fe_assemble_scalar; CUDAFormIntegral.cpp:66-266) */
  FE_FORM_INTEGRAL = 31,       /* int f dx;          coeff 0 = f (constant / DG0 / P1) */
  FE_FORM_P1_ENERGY = 32,      /* int k |grad u|^2 dx; coeff 0 = k (constant / DG0),
                                  coeff 1 = u (P1, through its P1 dofmap)           */
  FE_FORM_P2_ENERGY = 33,      /* as P1_ENERGY with u a P2 field (FE_COEFF_P2)      */
  FE_FORM_FACET_INTEGRAL = 34, /* int g ds over fe_form_set_facets; coeff 0 = g     */
  FE_FORM_JUMP_NORM = 35       /* int jump(u)^2 dS over fe_form_set_interior_facets;
                                  coeff 0 = u: DG0 (FE_COEFF_DG0) or DG1 / P1 through
                                  its 4-dof dofmap (FE_COEFF_P1)                    */
};

/* Coefficient representations (CUDAFormCoefficients.h:352-365 packs these
 * per cell; here the element kernels gather them directly). */
enum fe_coeff_kind {
  FE_COEFF_CONSTANT = 0, /* one value (or 3 for a vector load) for all cells */
  FE_COEFF_DG0 = 1,      /* one value per cell (3 per cell for a vector load) */
  FE_COEFF_P1 = 2,       /* vertex values through a P1 dofmap                 */
  FE_COEFF_P2 = 3        /* P2 node values through a P2 dofmap (energy functional) */
};

/* Element-tensor precision of a matrix form. */
enum fe_precision {
  FE_PREC_FP64 = 0, /* FP64 throughout (parity path)                                   */
  FE_PREC_FP32 = 1  /* FP64 geometry, FP32 element-tensor contraction, FP64 accumulation */
};

/* Flags of fe_assemble_matrix.  Without a variant flag the default runs: the
 * block variant for P1 stiffness on meshes of >= 2^20 cells, the coalesced
 * variant for P2 stiffness, vector-P2 elasticity and FP64 P3 stiffness, the
 * FP64-atomic scatter otherwise (the fastest measured on B200 for each case). */
#define FE_ASM_ZERO 1u            /* overwrite instead of accumulating (assemble.py:52 zero=True)   */
#define FE_ASM_DETERMINISTIC 2u   /* bitwise reproducible: ordered tile gather (P1/P2), else sorted-slot */
#define FE_ASM_ATOMIC 4u          /* FP64-atomic scatter through the slot map (zero pass first); for
                                     P1 (stiffness, mass), P3 and vector-P2 (elasticity, mass) forms on a symmetric pattern with equal
                                     row/column BCs (and FE_ASM_ZERO) each unique entry is reduced
                                     once into the upper triangle and a pass copies it to the lower
                                     triangle                                                        */
#define FE_ASM_SORTED_SLOT 8u     /* global sorted-slot segmented reduction (reproducible)          */
#define FE_ASM_TILE 16u           /* owner-computes row tiles, shared-memory accumulation (P1/P2)   */
#define FE_ASM_ROW_GATHER 32u     /* one warp per CSR row over the row's cells (P1)                 */
#define FE_ASM_BLOCK 64u          /* Morton cell blocks combined in shared memory, then coalesced
                                     reductions (P1/P2)                                              */
#define FE_ASM_FULL_SCATTER 128u  /* atomic scatter into both triangles, as the reference does      */
#define FE_ASM_GROUPED 256u       /* P2 stiffness: consecutive cells in groups of 48, each group's element
                                     entries summed per distinct CSR slot in shared memory, then one
                                     reduction per slot (falls back to the atomic scatter when the
                                     mesh's groups share no structure)                                */
#define FE_ASM_COALESCED 512u     /* P2 stiffness, vector-P2 elasticity, FP64 P3 stiffness (the default
                                     for each): the warp's reductions issued row by row (consecutive
                                     lanes on one cell's CSR row, so an instruction's reductions
                                     share L2 sectors); FE_ASM_ATOMIC keeps one thread's reductions
                                     per cell                                                       */

/* ---- errors / context --------------------------------------------------- */
const char* fe_last_error(void);
const char* fe_version(void);

/* Replaces CUDA::Context (cpp/cudolfinx/common/CUDA.cpp:28-52) and
 * cudolfinx.context.get_cuda_context (python/cudolfinx/context.py:29-35). */
int fe_context_create(int device, fe_context* out);
int fe_context_destroy(fe_context ctx);
/* Blocks until all work of the context's GPU is done; returns the first
 * pending device error word (see FE_ERR_DEVICE). */
int fe_context_synchronize(fe_context ctx);

/* ---- mesh / dofmaps ------------------------------------------------------ */
/* Replaces CUDAMesh (cpp/cudolfinx/mesh/CUDAMesh.h:41-163): 3 FP64 coordinates
 * per node (host) and the affine-tet geometry dofmap int32[num_cells*4] (host). */
int fe_mesh_create(fe_context ctx, const double* coords, int64_t num_nodes,
                   const int32_t* geom_dofmap, int64_t num_cells, int nodes_per_cell,
                   fe_mesh* out);
int fe_mesh_destroy(fe_mesh m);

/* Replaces CUDADofMap (cpp/cudolfinx/fem/CUDADofMap.cpp:199-236).  Cell dofs
 * are BLOCK dofs int32[num_cells*dofs_per_cell] (host); scalar dof = block*bs + comp
 * is derived in the kernels instead of storing the unrolled map. */
int fe_dofmap_create(fe_context ctx, const int32_t* cell_dofs, int64_t num_cells,
                     int dofs_per_cell, int bs, int64_t num_blocks, fe_dofmap* out);
/* A restricted dofmap (CUDADofMap::update with a restriction map,
 * cpp/cudolfinx/fem/CUDADofMap.cpp:199-236, set by CUDAForm::set_restriction,
 * cpp/cudolfinx/fem/CUDAForm.h:201-232): entries are block dofs of the
 * restricted numbering 0..num_blocks-1, or -1 for a cell dof outside the
 * restriction, which then takes no matrix, vector or lifting entry.  Forms on
 * such dofmaps bind with fe_form_bind_sparsity_block and assemble with the
 * atomic scatter; exterior-facet forms and coefficients take unrestricted
 * dofmaps. */
int fe_dofmap_create_restricted(fe_context ctx, const int32_t* cell_dofs, int64_t num_cells,
                                int dofs_per_cell, int bs, int64_t num_blocks, fe_dofmap* out);
int fe_dofmap_destroy(fe_dofmap d);

/* ---- sparsity ------------------------------------------------------------ */
/* Replaces create_cuda_matrix (cpp/cudolfinx/fem/petsc.h:31-37 ->
 * la/petsc.cpp:14-151): the DOLFINx SparsityPattern of a cell integral (sorted
 * unique block columns per block row) unrolled to scalar AIJ exactly as
 * la/petsc.cpp:45-65 does.  Built on the host from the dofmaps. */
int fe_sparsity_build(fe_dofmap rows, fe_dofmap cols, fe_sparsity* out);
/* The same pattern built on the device (radix sort + unique of the cell
 * couplings, then the same unroll), bit-exact with fe_sparsity_build; for
 * callers that create many meshes.  Synchronises `stream`. */
int fe_sparsity_build_device(fe_dofmap rows, fe_dofmap cols, void* stream, fe_sparsity* out);
/* The pattern of a sum of bilinear forms on the same spaces, as DOLFINx's
 * create_sparsity_pattern builds it for a form with several integrals: the
 * union of the cell couplings of cell and exterior-facet forms and of the
 * couplings of both cells of every facet of interior-facet forms
 * (cpp/cudolfinx/fem/utils.h:61-83 inserts the same macro-cell dofs).
 * Built on the host. */
int fe_sparsity_build_forms(int num_forms, const fe_form* forms, fe_sparsity* out);
/* Replaces create_cuda_matrix_block (cpp/cudolfinx/fem/petsc.h:39-107): the
 * monolithic scalar pattern of a block form.  Part p contributes the cell
 * couplings of (rows[p], cols[p]) unrolled and shifted to scalar row
 * row_offsets[p] and column col_offsets[p] (the offsets of BlockCUDAForm,
 * python/cudolfinx/form.py:127-160); -1 entries of restricted dofmaps couple
 * nothing.  Columns are sorted and unique per row (DOLFINx's block
 * SparsityPattern at block size 1).  Built on the host. */
int fe_sparsity_build_block(fe_context ctx, int num_parts, const fe_dofmap* rows, const fe_dofmap* cols,
                            const int64_t* row_offsets, const int64_t* col_offsets, int64_t num_rows,
                            int64_t num_cols, fe_sparsity* out);
/* Adopt an existing pattern (e.g. the arrays of a PETSc AIJ matrix); host arrays. */
int fe_sparsity_create(fe_context ctx, const int32_t* row_ptr, const int32_t* col,
                       int64_t num_rows, int64_t num_cols, fe_sparsity* out);
int fe_sparsity_info(fe_sparsity s, int64_t* num_rows, int64_t* num_cols, int64_t* nnz);
/* Copy the pattern to host arrays of num_rows+1 and nnz entries. */
int fe_sparsity_copy_to_host(fe_sparsity s, int32_t* row_ptr, int32_t* col);
/* Host-only construction of the same pattern, without a GPU (e.g. to create
 * the PETSc AIJ matrix that the device values are later written into).  The
 * arrays are allocated by the library and released with fe_free_host. */
int fe_pattern_build_host(const int32_t* dofs0, const int32_t* dofs1, int64_t num_cells, int k0, int k1,
                          int bs0, int bs1, int64_t num_blocks0, int64_t num_blocks1, int64_t* nnz,
                          int32_t** row_ptr, int32_t** col);
void fe_free_host(void* p);
/* Device pointers of the pattern (owned by the sparsity object). */
int fe_sparsity_device_arrays(fe_sparsity s, const int32_t** row_ptr, const int32_t** col);
int fe_sparsity_destroy(fe_sparsity s);

/* ---- forms ------------------------------------------------------------- */
/* Replaces CUDAForm (cpp/cudolfinx/fem/CUDAForm.h:40-147) for the built-in
 * forms.  `trial` is NULL for linear forms. */
int fe_form_create(fe_context ctx, int form_kind, fe_mesh mesh, fe_dofmap test,
                   fe_dofmap trial, fe_form* out);
/* Upload coefficient `index` (replaces CUDAForm::to_device + pack_coefficients,
 * CUDAForm.h:195-199, CUDAAssembler.h:177-283).  `values` is host memory when
 * values_on_device == 0 (copied on `stream`), else device memory that the form
 * reads in place during later assembly calls.  P1 coefficients need the P1
 * dofmap `cmap`; n is the number of values. */
int fe_form_set_coefficient(fe_form f, int index, int coeff_kind, fe_dofmap cmap,
                            const double* values, int64_t n, int values_on_device,
                            void* stream);
int fe_form_set_precision(fe_form f, int precision);
/* Launch shape of the atomic scatter for P1 / P2 stiffness (no counterpart in
 * the reference, which takes max_threads_per_block / min_blocks_per_multiprocessor
 * in CUDAForm::compile, python/cudolfinx/form.py:66-71): cells per CTA (32, 64
 * or 128; 0 = the default 128) and, for P2, whether the CTA stages its cells'
 * byte maps in shared memory (1, the default) or each thread reads its own (0).
 * Small meshes fill more SMs with smaller CTAs; cudolfinx.VariantTuner picks
 * the pair per size class. */
int fe_form_set_launch(fe_form f, int cells_per_cta, int stage);
/* Integration domain of an exterior-facet form (facet kinds and
 * FE_FORM_FACET_INTEGRAL): num_facets (cell, local
 * facet) pairs, int32[2*num_facets] host array; local facet f is the facet
 * opposite vertex f of the cell (the pairs DOLFINx packs for the reference's
 * active_mesh_entities, CUDAFormIntegral.cpp:361-447). */
int fe_form_set_facets(fe_form f, const int32_t* cell_facet_pairs, int64_t num_facets);
/* Integration domain of an interior-facet form (FE_FORM_DG*_JUMP,
 * FE_FORM_DG*_AVG_LOAD, FE_FORM_JUMP_NORM): num_facets quadruples (cell0,
 * local facet0, cell1, local facet1), host int32, where the two local facets
 * are the same triangle (the interior-facet entities DOLFINx packs for the
 * reference, CUDAFormIntegral.cpp:451-522).  The element tensors couple the
 * dofs of both cells.  A facet whose two sides differ is reported as
 * FE_ERR_DEVICE by the next synchronising call and contributes nothing. */
int fe_form_set_interior_facets(fe_form f, const int32_t* quads, int64_t num_facets);
/* Bind the matrix pattern and build the cell-to-slot map once (the reference's
 * unused lookup-table prototype, CUDAFormIntegral.cpp:1230-1407, made the
 * default).  Fails with FE_ERR_PATTERN if a cell coupling is missing. */
int fe_form_bind_sparsity(fe_form f, fe_sparsity s, void* stream);
/* Bind form (i, j) of a block form to a monolithic pattern with its rows at
 * scalar row_offset and its columns at col_offset (set_restriction offsets,
 * cpp/cudolfinx/fem/CUDAForm.h:201-232).  fe_assemble_matrix then adds the
 * block into the monolithic value array: FE_ASM_ZERO zeroes all of it, owned
 * BC rows of bc0 get the diagonal on the monolithic diagonal; the atomic
 * scatter only (assemble_matrix_block, python/cudolfinx/assemble.py:112-134,
 * calls it per block with zero=False).  Fails with FE_ERR_PATTERN if a
 * coupling is missing from the pattern. */
int fe_form_bind_sparsity_block(fe_form f, fe_sparsity s, int64_t row_offset, int64_t col_offset,
                                void* stream);
int fe_form_destroy(fe_form f);

/* ---- forms from FFCx tabulate_tensor bodies ------------------------------ */
/* Integral types (ufcx / DOLFINx IntegralType). */
enum fe_integral_type {
  FE_INTEGRAL_CELL = 0,
  FE_INTEGRAL_EXTERIOR_FACET = 1,
  FE_INTEGRAL_INTERIOR_FACET = 2
};
/* Replaces CUDAForm_float64 + CUDAForm::compile for one integral of a form
 * (python/cudolfinx/form.py:26-71, jit.py:15-114; kernel source
 * cpp/cudolfinx/fem/CUDAFormIntegral.cpp:2366-2469, NVRTC compile and cache
 * :2472-2558).  `tabulate_body` is the body (between the outer braces) of an
 * FFCx tabulate_tensor_integral_* function -- what jit.py extracts from the
 * generated C file -- and `tabulate_name` its name (a C identifier).  The body
 * reads A, w, c, coordinate_dofs, entity_local_index and quadrature_permutation
 * with FFCx's meaning and adds into A.  The rank is 2 with a trial dofmap, 1
 * with a test dofmap only, 0 with neither (a functional).  Coefficient q of
 * the form has coefficient_sizes[q] values per cell (its element's dofs times
 * block size); the form has num_constants constant values.  The body is
 * compiled here, for the device's architecture, inside the engine's assembly
 * skeletons; the compiled code is cached per process and, when `cachedir` is
 * not NULL, in that directory (keyed on a hash of the whole generated source).
 * A body NVRTC rejects gives FE_ERR_ARG with the compiler log.  Facet integrals
 * take their facets from fe_form_set_facets / fe_form_set_interior_facets;
 * matrices bind a pattern with fe_form_bind_sparsity (cell and exterior-facet
 * integrals: also fe_form_bind_sparsity_block) and assemble with the atomic
 * scatter through fe_assemble_matrix, fe_assemble_vector, fe_apply_lifting and
 * fe_assemble_scalar. */
int fe_form_create_ffcx(fe_context ctx, fe_mesh mesh, fe_dofmap test, fe_dofmap trial, int integral_type,
                        const char* tabulate_name, const char* tabulate_body, int num_coefficients,
                        const int* coefficient_sizes, int num_constants, const char* cachedir,
                        fe_form* out);
/* Coefficient `index` of an FFCx form: a function on the space of dofmap
 * `cmap` (k*bs values per cell, which must equal the coefficient's size),
 * `values` its num_blocks*bs dof values (host, copied on `stream`, or device
 * memory read in place when values_on_device != 0).  The values are packed
 * per cell before every assembly call, as pack_coefficients does
 * (cpp/cudolfinx/fem/CUDAAssembler.cpp:59-96). */
int fe_form_set_coefficient_field(fe_form f, int index, fe_dofmap cmap, const double* values, int64_t n,
                                  int values_on_device, void* stream);
/* The CUDA C++ translation unit fe_form_create_ffcx compiles for an integral
 * with these sizes (test / trial dofs per cell k0 / k1 and block sizes; unused
 * for lower ranks), without compiling it and without a GPU: for inspecting the
 * generated kernels (the reference keeps its generated sources in its cache
 * directory).  Writes at most capacity-1 characters and a terminating NUL to
 * `out` (may be NULL) and the full length to *length. */
int fe_ffcx_source(int integral_type, int rank, int k0, int bs0, int k1, int bs1, int num_coefficients,
                   const int* coefficient_sizes, const char* tabulate_name, const char* tabulate_body, char* out,
                   int64_t capacity, int64_t* length);
/* The constant values of an FFCx form (host; replaces CUDAFormConstants,
 * cpp/cudolfinx/fem/CUDAFormConstants.h:36-70, 123-145). */
int fe_form_set_constants(fe_form f, const double* values, int n, void* stream);

/* ---- Dirichlet BCs ------------------------------------------------------- */
/* Replaces CUDADirichletBC (cpp/cudolfinx/fem/CUDADirichletBC.h:56-194):
 * markers u8[num_dofs] (scalar dofs), dof list int32[n_bc] with the n_owned
 * owned dofs first, and full-length values g f64[num_dofs]; host arrays. */
int fe_bc_create(fe_context ctx, int64_t num_dofs, const uint8_t* markers,
                 const int32_t* dofs, int64_t n_bc, int64_t n_owned, const double* g,
                 fe_bc* out);
/* Replaces CUDADirichletBC::update (CUDADirichletBC.h:255-261). */
int fe_bc_update(fe_bc bc, const double* g, void* stream);
int fe_bc_destroy(fe_bc bc);

/* ---- assembly ----------------------------------------------------------- */
/* Replaces zero_matrix_entries + assemble_matrix_on_device + set_diagonal
 * (python/cudolfinx/wrappers/fem.cpp:212-252, CUDAAssembler.h:681-740,
 * CUDAAssembler.cpp:131-164).  values: device f64[nnz] of the bound pattern.
 * BC rows/cols of bc0/bc1 (may be NULL) receive no element contributions and
 * owned bc0 rows get `diagonal` on the diagonal when the form is square. */
int fe_assemble_matrix(fe_form a, double* values, fe_bc bc0, fe_bc bc1, double diagonal,
                       unsigned flags, void* stream);
/* Batched matrix assembly; no counterpart in the reference, whose
 * assemble_matrix (python/cudolfinx/assemble.py:52-110) takes one form
 * instance per call.  Assembles `num_instances` instances of the P1 or P2
 * stiffness form `a` that differ only in a DG0 coefficient:
 * coefficients[i] (device f64[num_cells]) is instance i's k, values[i]
 * (device f64[nnz] of a's bound pattern) receives instance i's CSR values.
 * Both tables are host arrays of device pointers.  Element tensors are FP32,
 * slot sums FP64 in a fixed order (bitwise reproducible).  BC handling and
 * FE_ASM_ZERO as fe_assemble_matrix; other flags are ignored.  The form's own
 * coefficient is not used. */
int fe_assemble_matrix_batch(fe_form a, int num_instances, const double* const* coefficients,
                             double* const* values, fe_bc bc0, fe_bc bc1, double diagonal,
                             unsigned flags, void* stream);
/* Replaces assemble_scalar_on_device (python/cudolfinx/assemble.py:204-226):
 * the value of a functional (FE_FORM_INTEGRAL, *_ENERGY, FE_FORM_FACET_INTEGRAL)
 * into *result (host).  The sum runs in a fixed order, so the value is
 * bitwise reproducible on a given GPU (the reference adds per-thread partials
 * with atomicAdd).  Synchronises `stream`. */
int fe_assemble_scalar(fe_form M, double* result, void* stream);
/* Replaces zero_matrix_entries / zero_vector_entries (wrappers/fem.cpp:212-222,
 * 256-266; kernel CUDAAssembler.cpp:38-56): values[0..n) = 0 on `stream`. */
int fe_zero_entries(double* values, int64_t n, void* stream);
/* Replaces zero_vector_entries + assemble_vector_on_device
 * (wrappers/fem.cpp:254-289, CUDAAssembler.h:367-424). b: device f64. */
int fe_assemble_vector(fe_form L, double* b, unsigned flags, void* stream);
/* Replaces apply_lifting_on_device (wrappers/fem.cpp:327-355,
 * CUDAAssembler.h:562-603): b -= scale * A_i (g_i - x0_i) for each form a[i]
 * on the columns of bc1[i]; x0 may be NULL or hold NULL entries. */
int fe_apply_lifting(double* b, int num_forms, const fe_form* a, const fe_bc* bc1,
                     const double* const* x0, double scale, void* stream);
/* The diagonal of a cell bilinear form (P1 / P2 / P3 stiffness, vector-P2
 * elasticity) as a vector, b[r] += A_e[r][r] over the cells with no BCs: what
 * the reference assembles from a form compiled with the FFCx option
 * "part": "diagonal" (python/test/test_cuda_assembly.py:199-208), e.g. for a
 * Jacobi preconditioner.  FE_ASM_ZERO zeroes b first. */
int fe_assemble_diagonal(fe_form a, double* b, unsigned flags, void* stream);
/* The right-hand side of a linear system in one call: b = [0 with
 * FE_ASM_ZERO] + L - scale * A (g - x0) on the BC columns, then
 * b[d] = scale * (g[d] - x0[d]) on the BC dofs.  Replaces the sequence
 * assemble_vector_on_device + apply_lifting_on_device([a], [bc]) +
 * set_bc_on_device (wrappers/fem.cpp:291-309, 327-383; assemble.py:136-166, 287-339,
 * 341-380), which the reference runs as three kernels with a synchronise
 * after each.  Two launches with no order between them (the lifting; the
 * element vectors with set_bc) when L and a are a (P1 load, P1 stiffness),
 * (P2 load, P2 stiffness), (P3 load, P3 stiffness) or (vector-P2 load,
 * elasticity) pair on one space and the BC's markers are its dof list: the
 * scatters skip the BC rows that set_bc stores.  Other forms (FFCx, facet,
 * restricted) take the three calls, with the same result.  bc may be NULL (b = L).  x0 may be
 * NULL.  Entries outside the BC rows equal the three calls' up to the order of
 * FP64 additions; the BC rows are equal. */
int fe_assemble_rhs(fe_form L, fe_form a, fe_bc bc, double* b, const double* x0, double scale,
                    unsigned flags, void* stream);
/* Replaces set_bc_on_device (wrappers/fem.cpp:357-383, CUDAAssembler.h:443-529):
 * b[d] = scale * (g[d] - x0[d]) for the BC dofs; x0 may be NULL. */
int fe_set_bc(double* b, int64_t num_values, fe_bc bc, const double* x0, double scale,
              void* stream);

/* ---- interpolation ------------------------------------------------------- */
/* Replaces CUDACoefficient::interpolate (cpp/cudolfinx/fem/CUDACoefficient.h:64-83
 * -> interpolate_same_map, cpp/cudolfinx/fem/CUDAInterpolate.cu): u1 = I u0 for
 * two spaces on the same mesh and reference map.  `matrix` (host, row-major
 * target.k x source.k) is the interpolation operator: the target element's
 * nodes evaluated in the source element's basis (create_interpolation_operator).
 * u0 / u1 are device arrays of num_blocks*bs values; block spaces interpolate
 * component by component.  Each target dof is computed once, from the lowest
 * (cell, local dof) that lists it (the reference lets the last writer win);
 * dofs listed by no cell keep their values. */
int fe_interpolate(fe_dofmap target, double* u1, fe_dofmap source, const double* u0, const double* matrix,
                   void* stream);

/* ---- solver (the reference hands A, b to PETSc KSP cg + jacobi:
 * python/examples/poisson.py:116-125) ------------------------------------ */
/* Jacobi-preconditioned CG on device.  x is the initial guess and the result
 * (device f64[n]).  Stops when ||r||_2 <= rtol*||b||_2 or after max_iter; then
 * *iterations and *rel_residual are written (host) and the call synchronises
 * the stream.  Returns FE_ERR_NOT_CONVERGED if max_iter was reached. */
int fe_pcg_solve(fe_sparsity s, const double* values, const double* b, double* x, double rtol,
                 int max_iter, int* iterations, double* rel_residual, void* stream);

/* Mixed-precision Jacobi-PCG (no counterpart in the reference; the served
 * requests of cudolfinx.serve use it).  Inner PCG iterations read an FP32 copy
 * of the values -- with block_size 3 (vector P2 patterns) in a 3x3
 * block-column layout, one column index per block -- and stop at inner_rtol
 * relative to their right-hand side; an FP64 refinement loop recomputes
 * r = b - A x from the FP64 values and adds the inner solutions until
 * |r| <= rtol |b|, so the result meets rtol in FP64.  max_iter bounds the
 * inner iterations in total; *iterations receives them, *refinements the
 * outer steps.  Allocates its scratch with cudaMallocAsync on `stream` and
 * synchronises it.  Returns FE_ERR_NOT_CONVERGED when max_iter is reached and
 * FE_ERR_ARG when block_size is 3 and the pattern is not block-structured. */
int fe_pcg_solve_mixed(fe_sparsity s, const double* values, const double* b, double* x, double rtol,
                       double inner_rtol, int max_iter, int block_size, int* iterations, int* refinements,
                       double* rel_residual, void* stream);

/* Allocation-free variant of fe_pcg_solve (no counterpart in the reference).
 * For callers that cannot allocate device memory while they solve: an
 * application whose device memory is already reserved by its own pool
 * allocator (a framework caching allocator, a PETSc / Kokkos arena sized to
 * the card), or a latency-critical loop that must not enter the CUDA
 * allocator.  Same arguments and status codes as fe_pcg_solve, and on one
 * GPU bitwise the same results (same kernels, same launch shapes), but the
 * solver's scratch vectors live in one file-scope device array of 10.5 MB
 * (5 vectors of 262,144 doubles plus reduction slots), which every GPU that
 * loads the library holds until the process exits; it calls no cudaMalloc /
 * cudaFree.
 *  - Matrices with more than 262,144 rows are rejected with FE_ERR_ARG.
 *  - The first call on a device looks up the array's device address (once per
 *    device, with that device current) and keeps it; make that first call
 *    before any stream capture, and do not reset the device
 *    (cudaDeviceReset) while the library is loaded, which would leave the
 *    kept address stale.
 *  - Every call shares the one array and re-initialises all of it that it
 *    reads; calls that overlap on the GPU (other streams, other threads) race
 *    on it and must be serialised by the caller. */
int fe_pcg_solve_noalloc(fe_sparsity s, const double* values, const double* b, double* x, double rtol,
                         int max_iter, int* iterations, double* rel_residual, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CUDOLFINX_B200_H */
