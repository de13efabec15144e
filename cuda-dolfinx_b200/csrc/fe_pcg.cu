// On-device Jacobi-preconditioned conjugate gradients.
//
// The reference hands the assembled CUDA matrix/vector to PETSc
// (KSP "cg" + PC "jacobi", python/examples/poisson.py:116-125).  Here the
// solver runs on the engine's own CSR arrays:
//   * SpMV with a sub-warp per row (width from the mean row length) fused
//     with the p.Ap dot product;
//   * x/r/z update fused with the r.z and r.r dot products;
//   * dot products reduce per block into fixed slots, then one block sums the
//     slots in a fixed order, so the iteration is bitwise reproducible;
//   * alpha/beta and the stopping test live on the device: every kernel
//     returns immediately once `done` is set, so the host enqueues iterations
//     in batches and synchronises once per batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <mutex>
#include <vector>

#include "fe_internal.h"

namespace fe {
namespace {

constexpr int kThreads = 256;

struct Scalars {
  double rz, rz_new, pAp, rr, bb, alpha, beta, tol2;
  int iter, max_iter, done, pad;
};

__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = (threadIdx.x < blockDim.x / 32) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

// y_r = sum_s A_rs x_s for the row handled by this SUB-lane group.  Called by
// all 32 lanes of a warp together (the shuffles name the full warp); a group
// whose row is past the end passes active = false and contributes nothing.
template <int SUB>
__device__ __forceinline__ double row_dot(const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                                          const double* __restrict__ val, const double* __restrict__ x, int64_t r,
                                          bool active, int lane) {
  double acc = 0.0;
  const int32_t lo = active ? __ldg(rp + r) : 0, hi = active ? __ldg(rp + r + 1) : 0;
  for (int32_t s = lo + lane; s < hi; s += SUB) acc += __ldg(val + s) * __ldg(x + __ldg(col + s));
#pragma unroll
  for (int o = SUB / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, SUB);
  return acc;
}

// Row loop with a trip count that is uniform across each warp: warp w handles
// rows [w*32/SUB, w*32/SUB + 32/SUB) + k*stride.
template <int SUB, typename F>
__device__ __forceinline__ void for_rows(int64_t n, F&& body) {
  constexpr int kGroups = 32 / SUB;
  const int64_t warp = (blockIdx.x * (int64_t)kThreads + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
  const int sub = (threadIdx.x & 31) / SUB;
  for (int64_t base = warp * kGroups; base < n; base += nwarps * kGroups) {
    const int64_t row = base + sub;
    body(row, row < n);
  }
}

template <int SUB>
__global__ void __launch_bounds__(kThreads) k_init(int64_t n, const int32_t* __restrict__ rp,
                                                   const int32_t* __restrict__ col, const double* __restrict__ val,
                                                   const int32_t* __restrict__ diag, const double* __restrict__ b,
                                                   const double* __restrict__ x, double* __restrict__ r,
                                                   double* __restrict__ z, double* __restrict__ p,
                                                   double* __restrict__ dinv, double* __restrict__ part) {
  __shared__ double sh[32];
  const int lane = threadIdx.x % SUB;
  double rz = 0.0, rr = 0.0, bb = 0.0;
  for_rows<SUB>(n, [&](int64_t row, bool active) {
    const double ax = row_dot<SUB>(rp, col, val, x, row, active, lane);
    if (active && lane == 0) {
      const int32_t ds = diag[row];
      const double d = ds >= 0 ? val[ds] : 1.0;
      const double di = d != 0.0 ? 1.0 / d : 1.0;
      const double rv = b[row] - ax;
      const double zv = di * rv;
      dinv[row] = di;
      r[row] = rv;
      z[row] = zv;
      p[row] = zv;
      rz += rv * zv;
      rr += rv * rv;
      bb += b[row] * b[row];
    }
  });
  rz = block_sum(rz, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = rz;
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = rr;
  bb = block_sum(bb, sh);
  if (threadIdx.x == 0) part[2 * gridDim.x + blockIdx.x] = bb;
}

// sums `nparts` partial arrays of length m in a fixed order; stage selects the scalar update
__global__ void k_reduce(const double* __restrict__ part, int m, int stage, Scalars* sc) {
  __shared__ double sh[32];
  __shared__ double res[3];
  if (stage != 0 && sc->done) return;
  const int nparts = stage == 1 ? 1 : (stage == 0 ? 3 : 2);
  for (int q = 0; q < nparts; ++q) {
    double v = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) v += part[q * m + i];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) res[q] = v;
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  if (stage == 0) {  // init: rz, rr, bb
    sc->rz = res[0];
    sc->rr = res[1];
    sc->bb = res[2];
    sc->iter = 0;
    sc->done = (res[1] <= sc->tol2 * res[2]) || res[2] == 0.0 || sc->max_iter <= 0;
  } else if (stage == 1) {  // alpha
    sc->pAp = res[0];
    if (res[0] == 0.0) sc->done = 1;
    else sc->alpha = sc->rz / res[0];
  } else {  // beta: rz_new, rr
    sc->rz_new = res[0];
    sc->rr = res[1];
    sc->beta = res[0] / sc->rz;
    sc->rz = res[0];
    sc->iter += 1;
    if (res[1] <= sc->tol2 * sc->bb || sc->iter >= sc->max_iter) sc->done = 1;
  }
}

template <int SUB>
__global__ void __launch_bounds__(kThreads) k_spmv(int64_t n, const int32_t* __restrict__ rp,
                                                   const int32_t* __restrict__ col, const double* __restrict__ val,
                                                   const double* __restrict__ p, double* __restrict__ Ap,
                                                   double* __restrict__ part, const Scalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  const int lane = threadIdx.x % SUB;
  double pap = 0.0;
  for_rows<SUB>(n, [&](int64_t row, bool active) {
    const double y = row_dot<SUB>(rp, col, val, p, row, active, lane);
    if (active && lane == 0) {
      Ap[row] = y;
      pap += p[row] * y;
    }
  });
  pap = block_sum(pap, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = pap;
}

__global__ void __launch_bounds__(kThreads) k_update(int64_t n, double* __restrict__ x, double* __restrict__ r,
                                                     double* __restrict__ z, const double* __restrict__ p,
                                                     const double* __restrict__ Ap, const double* __restrict__ dinv,
                                                     double* __restrict__ part, const Scalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  const double alpha = sc->alpha;
  double rz = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    x[i] += alpha * p[i];
    const double rv = r[i] - alpha * Ap[i];
    r[i] = rv;
    const double zv = dinv[i] * rv;
    z[i] = zv;
    rz += rv * zv;
    rr += rv * rv;
  }
  rz = block_sum(rz, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = rz;
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = rr;
}

__global__ void __launch_bounds__(kThreads) k_update_p(int64_t n, const double* __restrict__ z,
                                                       double* __restrict__ p, const Scalars* sc) {
  if (sc->done) return;
  const double beta = sc->beta;
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads)
    p[i] = z[i] + beta * p[i];
}

// cudaMallocAsync'd buffers freed with cudaFreeAsync on the same stream when
// the scope ends, normally or by an exception.
cudaMemPool_t scratch_pool(fe_context_s& ctx) {
  static std::mutex m;  // solver calls on several host threads share the context
  std::lock_guard<std::mutex> lock(m);
  if (!ctx.scratch_pool) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = ctx.device;
    cudaMemPool_t pool = nullptr;
    FE_CUDA(cudaMemPoolCreate(&pool, &props));
    size_t free_b = 0, total_b = 0;
    FE_CUDA(cudaMemGetInfo(&free_b, &total_b));
    uint64_t keep = total_b / 4;
    FE_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    ctx.scratch_pool = pool;
  }
  return ctx.scratch_pool;
}

struct StreamScratch {
  cudaStream_t s;
  cudaMemPool_t pool;
  std::vector<void*> ptrs;
  StreamScratch(cudaStream_t st, cudaMemPool_t p) : s(st), pool(p) {}
  StreamScratch(const StreamScratch&) = delete;
  StreamScratch& operator=(const StreamScratch&) = delete;
  template <typename T>
  T* get(int64_t count) {
    void* q = nullptr;
    FE_CUDA(cudaMallocFromPoolAsync(&q, (size_t)std::max<int64_t>(count, 1) * sizeof(T), pool, s));
    ptrs.push_back(q);
    return static_cast<T*>(q);
  }
  void release() {
    while (!ptrs.empty()) {
      void* q = ptrs.back();
      ptrs.pop_back();
      FE_CUDA(cudaFreeAsync(q, s));
    }
  }
  ~StreamScratch() {
    for (void* q : ptrs) (void)cudaFreeAsync(q, s);
    if (!ptrs.empty()) (void)cudaGetLastError();
  }
};

template <int SUB>
void run(const fe_sparsity_s& A, const double* val, const double* b, double* x, double rtol, int max_iter,
         int* iterations, double* rel_res, cudaStream_t s) {
  const int64_t n = A.num_rows;
  // the row kernels (k_init, k_spmv: 32 registers) wait on dependent loads
  // (row bounds -> columns and values -> gathered entries): they run 8 CTAs
  // per SM, the vector updates (40 registers) 4; each reduction sums the
  // partials of the launch that wrote them
  const unsigned grid = (unsigned)(A.ctx->num_sms * 4);
  const unsigned grid_rows = (unsigned)(A.ctx->num_sms * 8);
  // stream-ordered scratch, released on every exit path (a launch or
  // synchronisation error inside the loop throws)
  StreamScratch buf(s, scratch_pool(*A.ctx));
  double* r = buf.get<double>(n);
  double* z = buf.get<double>(n);
  double* p = buf.get<double>(n);
  double* Ap = buf.get<double>(n);
  double* dinv = buf.get<double>(n);
  double* part = buf.get<double>(3 * (int64_t)grid_rows);
  Scalars* sc = buf.get<Scalars>(1);
  Scalars h{};
  h.tol2 = rtol * rtol;
  h.max_iter = max_iter;
  FE_CUDA(cudaMemcpyAsync(sc, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  k_init<SUB><<<grid_rows, kThreads, 0, s>>>(n, A.row_ptr.p, A.col.p, val, A.diag.p, b, x, r, z, p, dinv, part);
  k_reduce<<<1, 1024, 0, s>>>(part, grid_rows, 0, sc);
  FE_CUDA(cudaGetLastError());
  const int batch = 16;
  for (int it = 0;; it += batch) {
    for (int q = 0; q < batch; ++q) {
      k_spmv<SUB><<<grid_rows, kThreads, 0, s>>>(n, A.row_ptr.p, A.col.p, val, p, Ap, part, sc);
      k_reduce<<<1, 1024, 0, s>>>(part, grid_rows, 1, sc);
      k_update<<<grid, kThreads, 0, s>>>(n, x, r, z, p, Ap, dinv, part, sc);
      k_reduce<<<1, 1024, 0, s>>>(part, grid, 2, sc);
      k_update_p<<<grid, kThreads, 0, s>>>(n, z, p, sc);
    }
    FE_CUDA(cudaGetLastError());
    FE_CUDA(cudaMemcpyAsync(&h, sc, sizeof(h), cudaMemcpyDeviceToHost, s));
    FE_CUDA(cudaStreamSynchronize(s));
    if (h.done || it >= max_iter) break;
  }
  buf.release();
  *iterations = h.iter;
  *rel_res = h.bb > 0 ? sqrt(h.rr / h.bb) : 0.0;
}

}  // namespace

int pcg_solve(const fe_sparsity_s& A, const double* val, const double* b, double* x, double rtol, int max_iter,
              int* iterations, double* rel_res, cudaStream_t s) {
  FE_REQUIRE(A.num_rows == A.num_cols, "PCG needs a square matrix");
  const double mean = A.num_rows ? (double)A.nnz / (double)A.num_rows : 0.0;
  if (mean <= 6) run<4>(A, val, b, x, rtol, max_iter, iterations, rel_res, s);
  else if (mean <= 14) run<8>(A, val, b, x, rtol, max_iter, iterations, rel_res, s);
  else if (mean <= 40) run<16>(A, val, b, x, rtol, max_iter, iterations, rel_res, s);
  else run<32>(A, val, b, x, rtol, max_iter, iterations, rel_res, s);
  return *iterations;
}

}  // namespace fe

extern "C" int fe_pcg_solve(fe_sparsity s, const double* values, const double* b, double* x, double rtol,
                            int max_iter, int* iterations, double* rel_residual, void* stream) {
  int it = 0;
  double res = 0.0;
  int status = FE_OK;
  try {
    if (!s || !values || !b || !x) FE_FAIL(FE_ERR_ARG, "null argument");
    FE_CUDA(cudaSetDevice(s->ctx->device));
    fe::pcg_solve(*s, values, b, x, rtol, max_iter, &it, &res, reinterpret_cast<cudaStream_t>(stream));
    if (iterations) *iterations = it;
    if (rel_residual) *rel_residual = res;
    if (!(res <= rtol)) status = FE_ERR_NOT_CONVERGED;
  } catch (const fe::Error& e) {
    fe::set_last_error(e.what());
    return e.code;
  }
  if (status != FE_OK) fe::set_last_error("PCG stopped after " + std::to_string(it) + " iterations at relative residual " +
                                          std::to_string(res));
  return status;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the solver.
//
// Some callers cannot allocate device memory while they solve: an embedding
// application whose device memory is already handed to its own pool (a
// framework caching allocator, or a PETSc / Kokkos arena sized to the card)
// can have cudaMalloc fail or steal its budget, and a latency-critical loop
// must not enter the CUDA allocator, which may synchronise the device.
// fe_pcg_solve_noalloc gives them the same solver with its scratch vectors in
// a fixed file-scope device array instead of cudaMallocAsync.
// ---------------------------------------------------------------------------
namespace fe {
namespace {

constexpr int64_t kNoAllocMaxRows = int64_t(1) << 18;  // 262,144 rows
constexpr int kNoAllocMaxGrid = 2048;                   // reduction slots per dot product
constexpr int64_t kNoAllocScalarWords = 16;            // room for one Scalars record (in doubles)
static_assert(sizeof(Scalars) <= kNoAllocScalarWords * sizeof(double), "Scalars record does not fit");

// r, z, p, Ap, dinv (kNoAllocMaxRows each), 3 x kNoAllocMaxGrid partial sums, one Scalars record:
// 5 * 262,144 * 8 B + 3 * 2048 * 8 B + 128 B = 10.5 MB held by every device that loads the library.
static __device__ __align__(256) double g_pcg_scratch[5 * kNoAllocMaxRows + 3 * kNoAllocMaxGrid +
                                                      kNoAllocScalarWords];

// Device address of g_pcg_scratch, looked up once per device (with that device current).
constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

double* scratch_address(int device) {
  if (device < 0 || device >= kMaxDevices) FE_FAIL(FE_ERR_ARG, "device ordinal out of range for the scratch table");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_ptr[device]) {
    void* p = nullptr;
    FE_CUDA(cudaGetSymbolAddress(&p, g_pcg_scratch));
    g_scratch_ptr[device] = static_cast<double*>(p);
  }
  return g_scratch_ptr[device];
}

template <int SUB>
void run_noalloc(const fe_sparsity_s& A, const double* val, const double* b, double* x, double rtol, int max_iter,
                 int* iterations, double* rel_res, double* scratch, cudaStream_t s) {
  const int64_t n = A.num_rows;
  // the launch shapes of fe_pcg_solve (8 CTAs per SM for the row kernels, 4
  // for the vector updates), so the partial sums are grouped identically and
  // the two solvers give bitwise-equal results on the same GPU
  const unsigned grid = (unsigned)std::min(A.ctx->num_sms * 4, kNoAllocMaxGrid);
  const unsigned grid_rows = (unsigned)std::min(A.ctx->num_sms * 8, kNoAllocMaxGrid);
  double* r = scratch;
  double* z = r + kNoAllocMaxRows;
  double* p = z + kNoAllocMaxRows;
  double* Ap = p + kNoAllocMaxRows;
  double* dinv = Ap + kNoAllocMaxRows;
  double* part = dinv + kNoAllocMaxRows;
  Scalars* sc = reinterpret_cast<Scalars*>(part + 3 * kNoAllocMaxGrid);
  // Every scratch word a kernel reads is written earlier in the same call:
  // k_init writes r, z, p, dinv for all n rows, k_spmv writes Ap before
  // k_update reads it, partial sums are written before each reduction, and
  // the Scalars record is re-initialised here.
  Scalars h{};
  h.tol2 = rtol * rtol;
  h.max_iter = max_iter;
  FE_CUDA(cudaMemcpyAsync(sc, &h, sizeof(h), cudaMemcpyHostToDevice, s));
  k_init<SUB><<<grid_rows, kThreads, 0, s>>>(n, A.row_ptr.p, A.col.p, val, A.diag.p, b, x, r, z, p, dinv, part);
  k_reduce<<<1, 1024, 0, s>>>(part, grid_rows, 0, sc);
  FE_CUDA(cudaGetLastError());
  const int batch = 16;
  for (int it = 0;; it += batch) {
    for (int q = 0; q < batch; ++q) {
      k_spmv<SUB><<<grid_rows, kThreads, 0, s>>>(n, A.row_ptr.p, A.col.p, val, p, Ap, part, sc);
      k_reduce<<<1, 1024, 0, s>>>(part, grid_rows, 1, sc);
      k_update<<<grid, kThreads, 0, s>>>(n, x, r, z, p, Ap, dinv, part, sc);
      k_reduce<<<1, 1024, 0, s>>>(part, grid, 2, sc);
      k_update_p<<<grid, kThreads, 0, s>>>(n, z, p, sc);
    }
    FE_CUDA(cudaGetLastError());
    FE_CUDA(cudaMemcpyAsync(&h, sc, sizeof(h), cudaMemcpyDeviceToHost, s));
    FE_CUDA(cudaStreamSynchronize(s));
    if (h.done || it >= max_iter) break;
  }
  *iterations = h.iter;
  *rel_res = h.bb > 0 ? sqrt(h.rr / h.bb) : 0.0;
}

}  // namespace
}  // namespace fe

extern "C" int fe_pcg_solve_noalloc(fe_sparsity s, const double* values, const double* b, double* x, double rtol,
                                    int max_iter, int* iterations, double* rel_residual, void* stream) {
  int it = 0;
  double res = 0.0;
  try {
    if (!s || !values || !b || !x) FE_FAIL(FE_ERR_ARG, "null argument");
    if (s->num_rows != s->num_cols) FE_FAIL(FE_ERR_ARG, "PCG needs a square matrix");
    if (s->num_rows > fe::kNoAllocMaxRows)
      FE_FAIL(FE_ERR_ARG, "fe_pcg_solve_noalloc supports at most " + std::to_string(fe::kNoAllocMaxRows) +
                              " rows (its static scratch size); the matrix has " + std::to_string(s->num_rows) +
                              " rows: use fe_pcg_solve");
    FE_CUDA(cudaSetDevice(s->ctx->device));
    double* scratch = fe::scratch_address(s->ctx->device);
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const double mean = s->num_rows ? (double)s->nnz / (double)s->num_rows : 0.0;
    if (mean <= 6) fe::run_noalloc<4>(*s, values, b, x, rtol, max_iter, &it, &res, scratch, st);
    else if (mean <= 14) fe::run_noalloc<8>(*s, values, b, x, rtol, max_iter, &it, &res, scratch, st);
    else if (mean <= 40) fe::run_noalloc<16>(*s, values, b, x, rtol, max_iter, &it, &res, scratch, st);
    else fe::run_noalloc<32>(*s, values, b, x, rtol, max_iter, &it, &res, scratch, st);
    if (iterations) *iterations = it;
    if (rel_residual) *rel_residual = res;
  } catch (const fe::Error& e) {
    fe::set_last_error(e.what());
    return e.code;
  }
  if (!(res <= rtol)) {
    fe::set_last_error("PCG stopped after " + std::to_string(it) + " iterations at relative residual " +
                       std::to_string(res));
    return FE_ERR_NOT_CONVERGED;
  }
  return FE_OK;
}

// ---------------------------------------------------------------------------
// Mixed-precision solve (served requests): inner Jacobi-PCG iterations read an
// FP32 copy of the matrix values -- for block-size-3 patterns (vector P2) in a
// 3x3 block-column layout, one column index per block, about 4.4 bytes per
// nonzero instead of the 12 of FP64 CSR -- and an FP64 refinement loop
// recomputes r = b - A x with the FP64 values until |r| <= rtol |b|.  The
// inner solves start from d = 0 and stop at inner_rtol relative to their
// right-hand side; x += d after each.
// ---------------------------------------------------------------------------
namespace fe {
namespace {

template <int SUB>
__global__ void __launch_bounds__(kThreads) k_spmv32(int64_t n, const int32_t* __restrict__ rp,
                                                     const int32_t* __restrict__ col, const float* __restrict__ val,
                                                     const double* __restrict__ p, double* __restrict__ Ap,
                                                     double* __restrict__ part, const Scalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  const int lane = threadIdx.x % SUB;
  double pap = 0.0;
  for_rows<SUB>(n, [&](int64_t row, bool active) {
    double acc = 0.0;
    const int32_t lo = active ? __ldg(rp + row) : 0, hi = active ? __ldg(rp + row + 1) : 0;
    for (int32_t s = lo + lane; s < hi; s += SUB) acc += (double)__ldg(val + s) * __ldg(p + __ldg(col + s));
#pragma unroll
    for (int o = SUB / 2; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o, SUB);
    if (active && lane == 0) {
      Ap[row] = acc;
      pap += p[row] * acc;
    }
  });
  pap = block_sum(pap, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = pap;
}

// block rows of a block-size-3 pattern: block k of block row R covers rows
// 3R..3R+2 and columns 3C..3C+2 (C = bcol[k]), its 9 values row-major
template <int SUB>
__global__ void __launch_bounds__(kThreads) k_spmv_b3(int64_t nb, const int32_t* __restrict__ brp,
                                                      const int32_t* __restrict__ bcol, const float* __restrict__ bval,
                                                      const double* __restrict__ p, double* __restrict__ Ap,
                                                      double* __restrict__ part, const Scalars* sc) {
  __shared__ double sh[32];
  if (sc->done) return;
  const int lane = threadIdx.x % SUB;
  double pap = 0.0;
  for_rows<SUB>(nb, [&](int64_t R, bool active) {
    double y0 = 0.0, y1 = 0.0, y2 = 0.0;
    const int32_t lo = active ? __ldg(brp + R) : 0, hi = active ? __ldg(brp + R + 1) : 0;
    for (int32_t k = lo + lane; k < hi; k += SUB) {
      const int64_t c3 = 3 * (int64_t)__ldg(bcol + k);
      const double x0 = __ldg(p + c3), x1 = __ldg(p + c3 + 1), x2 = __ldg(p + c3 + 2);
      const float* v = bval + 9 * (int64_t)k;
      y0 += (double)__ldg(v + 0) * x0 + (double)__ldg(v + 1) * x1 + (double)__ldg(v + 2) * x2;
      y1 += (double)__ldg(v + 3) * x0 + (double)__ldg(v + 4) * x1 + (double)__ldg(v + 5) * x2;
      y2 += (double)__ldg(v + 6) * x0 + (double)__ldg(v + 7) * x1 + (double)__ldg(v + 8) * x2;
    }
#pragma unroll
    for (int o = SUB / 2; o > 0; o >>= 1) {
      y0 += __shfl_down_sync(0xffffffffu, y0, o, SUB);
      y1 += __shfl_down_sync(0xffffffffu, y1, o, SUB);
      y2 += __shfl_down_sync(0xffffffffu, y2, o, SUB);
    }
    if (active && lane == 0) {
      Ap[3 * R] = y0;
      Ap[3 * R + 1] = y1;
      Ap[3 * R + 2] = y2;
      pap += p[3 * R] * y0 + p[3 * R + 1] * y1 + p[3 * R + 2] * y2;
    }
  });
  pap = block_sum(pap, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = pap;
}

// block layout of a block-size-3 pattern (checked: the three rows of a block
// row list the same columns, in triples 3C, 3C+1, 3C+2)
__global__ void k_b3_layout(int64_t nb, const int32_t* __restrict__ rp, const int32_t* __restrict__ col,
                            int32_t* __restrict__ brp, int32_t* __restrict__ bcol, unsigned* err) {
  const int64_t R = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (R >= nb) return;
  const int32_t s0 = rp[3 * R], len = rp[3 * R + 1] - s0;
  brp[R] = s0 / 9;
  if (R == nb - 1) brp[nb] = rp[3 * nb] / 9;
  if (len % 3 || rp[3 * R + 2] - rp[3 * R + 1] != len || rp[3 * R + 3] - rp[3 * R + 2] != len || s0 % 9) {
    atomicOr(err, DEV_ERR_BLOCK);
    return;
  }
  for (int32_t k = 0; k < len / 3; ++k) {
    const int32_t c = col[s0 + 3 * k];
    bool ok = c % 3 == 0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) ok &= col[s0 + a * len + 3 * k + b] == c + b;
    if (!ok) atomicOr(err, DEV_ERR_BLOCK);
    bcol[s0 / 9 + k] = c / 3;
  }
}

__global__ void k_to_b3(int64_t nb, const int32_t* __restrict__ rp, const int32_t* __restrict__ brp,
                        const double* __restrict__ val, float* __restrict__ bval) {
  const int64_t R = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (R >= nb) return;
  const int32_t b0 = brp[R], m = brp[R + 1] - b0;
  for (int a = 0; a < 3; ++a) {
    const double* src = val + rp[3 * R + a];
    for (int32_t k = 0; k < m; ++k)
      for (int b = 0; b < 3; ++b) bval[9 * (int64_t)(b0 + k) + 3 * a + b] = (float)src[3 * k + b];
  }
}

__global__ void k_to_f32(int64_t n, const double* __restrict__ v, float* __restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    w[i] = (float)v[i];
}

// inner start: r is the right-hand side, d = 0, z = p = dinv r; partial r.z, r.r, r.r
__global__ void __launch_bounds__(kThreads) k_init_zero(int64_t n, const double* __restrict__ r,
                                                        const double* __restrict__ dinv, double* __restrict__ z,
                                                        double* __restrict__ p, double* __restrict__ d,
                                                        double* __restrict__ part) {
  __shared__ double sh[32];
  double rz = 0.0, rr = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    const double rv = r[i], zv = dinv[i] * rv;
    z[i] = zv;
    p[i] = zv;
    d[i] = 0.0;
    rz += rv * zv;
    rr += rv * rv;
  }
  rz = block_sum(rz, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = rz;
  rr = block_sum(rr, sh);
  if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = rr;
  if (threadIdx.x == 0) part[2 * gridDim.x + blockIdx.x] = rr;  // the "b.b" of the inner system
}

__global__ void k_axpy(int64_t n, const double* __restrict__ d, double* __restrict__ x) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += d[i];
}

int sub_for(double mean) { return mean <= 6 ? 4 : (mean <= 14 ? 8 : (mean <= 40 ? 16 : 32)); }

template <typename F>
void launch_sub(int sub, F&& f) {
  switch (sub) {
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 8: f(std::integral_constant<int, 8>{}); break;
    case 16: f(std::integral_constant<int, 16>{}); break;
    default: f(std::integral_constant<int, 32>{}); break;
  }
}

}  // namespace

int pcg_solve_mixed(const fe_sparsity_s& A, const double* val, const double* b, double* x, double rtol,
                    double inner_rtol, int max_iter, int block_size, int* iterations, int* refinements,
                    double* rel_res, cudaStream_t s) {
  FE_REQUIRE(A.num_rows == A.num_cols, "PCG needs a square matrix");
  FE_REQUIRE(block_size == 1 || block_size == 3, "block size must be 1 or 3");
  FE_REQUIRE(block_size == 1 || A.num_rows % 3 == 0, "the pattern does not have block size 3");
  FE_REQUIRE(inner_rtol > 0.0 && inner_rtol < 1.0, "inner_rtol must lie in (0, 1)");
  const int64_t n = A.num_rows, nnz = A.nnz, nb = n / 3;
  const unsigned grid = (unsigned)(A.ctx->num_sms * 4);
  const unsigned grid_rows = (unsigned)(A.ctx->num_sms * 8);
  StreamScratch buf(s, scratch_pool(*A.ctx));
  double* r = buf.get<double>(n);
  double* z = buf.get<double>(n);
  double* p = buf.get<double>(n);
  double* Ap = buf.get<double>(n);
  double* dinv = buf.get<double>(n);
  double* d = buf.get<double>(n);
  double* part = buf.get<double>(3 * (int64_t)grid_rows);
  Scalars* sco = buf.get<Scalars>(1);
  Scalars* sci = buf.get<Scalars>(1);
  float* v32 = buf.get<float>(nnz);
  int32_t* brp = nullptr;
  int32_t* bcol = nullptr;
  if (block_size == 3) {
    brp = buf.get<int32_t>(nb + 1);
    bcol = buf.get<int32_t>(std::max<int64_t>(1, nnz / 9));
    if (nb) {
      // the layout is checked before anything reads it
      k_b3_layout<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(nb, A.row_ptr.p, A.col.p, brp, bcol, A.ctx->err.p);
      FE_CUDA(cudaGetLastError());
      unsigned w = 0;
      FE_CUDA(cudaMemcpyAsync(&w, A.ctx->err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
      FE_CUDA(cudaStreamSynchronize(s));
      if (w & DEV_ERR_BLOCK) {
        FE_CUDA(cudaMemsetAsync(A.ctx->err.p, 0, sizeof(unsigned), s));
        FE_CUDA(cudaStreamSynchronize(s));
        FE_FAIL(FE_ERR_ARG, "the pattern is not block-structured with block size 3");
      }
      k_to_b3<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(nb, A.row_ptr.p, brp, val, v32);
    }
  } else if (nnz) {
    k_to_f32<<<grid, kThreads, 0, s>>>(nnz, val, v32);
  }
  FE_CUDA(cudaGetLastError());
  const int sub64 = sub_for(n ? (double)nnz / (double)n : 0.0);
  const int sub32 = block_size == 3 ? sub_for(nb ? (double)nnz / 9.0 / (double)nb : 0.0) : sub64;
  int inner_total = 0, outer = 0;
  Scalars ho{}, hi{};
  for (;; ++outer) {
    // r = b - A x in FP64 (also dinv from the FP64 diagonal); stop at rtol
    Scalars h0{};
    h0.tol2 = rtol * rtol;
    h0.max_iter = 1;
    FE_CUDA(cudaMemcpyAsync(sco, &h0, sizeof(h0), cudaMemcpyHostToDevice, s));
    launch_sub(sub64, [&](auto S) {
      k_init<decltype(S)::value><<<grid_rows, kThreads, 0, s>>>(n, A.row_ptr.p, A.col.p, val, A.diag.p, b, x, r, z,
                                                                p, dinv, part);
    });
    k_reduce<<<1, 1024, 0, s>>>(part, grid_rows, 0, sco);
    FE_CUDA(cudaGetLastError());
    FE_CUDA(cudaMemcpyAsync(&ho, sco, sizeof(ho), cudaMemcpyDeviceToHost, s));
    FE_CUDA(cudaStreamSynchronize(s));
    if (ho.rr <= rtol * rtol * ho.bb || ho.bb == 0.0 || inner_total >= max_iter) break;
    // inner FP32 solve of A d = r from d = 0
    Scalars h1{};
    h1.tol2 = inner_rtol * inner_rtol;
    h1.max_iter = max_iter - inner_total;
    FE_CUDA(cudaMemcpyAsync(sci, &h1, sizeof(h1), cudaMemcpyHostToDevice, s));
    k_init_zero<<<grid, kThreads, 0, s>>>(n, r, dinv, z, p, d, part);
    k_reduce<<<1, 1024, 0, s>>>(part, grid, 0, sci);
    FE_CUDA(cudaGetLastError());
    const unsigned gsp = grid_rows;
    for (int it = 0;; it += 16) {
      for (int q = 0; q < 16; ++q) {
        if (block_size == 3) {
          launch_sub(sub32, [&](auto S) {
            k_spmv_b3<decltype(S)::value><<<gsp, kThreads, 0, s>>>(nb, brp, bcol, v32, p, Ap, part, sci);
          });
        } else {
          launch_sub(sub32, [&](auto S) {
            k_spmv32<decltype(S)::value><<<gsp, kThreads, 0, s>>>(n, A.row_ptr.p, A.col.p, v32, p, Ap, part, sci);
          });
        }
        k_reduce<<<1, 1024, 0, s>>>(part, gsp, 1, sci);
        k_update<<<grid, kThreads, 0, s>>>(n, d, r, z, p, Ap, dinv, part, sci);
        k_reduce<<<1, 1024, 0, s>>>(part, grid, 2, sci);
        k_update_p<<<grid, kThreads, 0, s>>>(n, z, p, sci);
      }
      FE_CUDA(cudaGetLastError());
      FE_CUDA(cudaMemcpyAsync(&hi, sci, sizeof(hi), cudaMemcpyDeviceToHost, s));
      FE_CUDA(cudaStreamSynchronize(s));
      if (hi.done) break;
    }
    inner_total += hi.iter;
    k_axpy<<<grid, kThreads, 0, s>>>(n, d, x);
    FE_CUDA(cudaGetLastError());
    if (hi.iter == 0) break;  // no progress possible
  }
  buf.release();
  if (iterations) *iterations = inner_total;
  if (refinements) *refinements = outer;
  if (rel_res) *rel_res = ho.bb > 0 ? sqrt(ho.rr / ho.bb) : 0.0;
  return inner_total;
}

}  // namespace fe

extern "C" int fe_pcg_solve_mixed(fe_sparsity s, const double* values, const double* b, double* x, double rtol,
                                  double inner_rtol, int max_iter, int block_size, int* iterations,
                                  int* refinements, double* rel_residual, void* stream) {
  int it = 0, ref = 0;
  double res = 0.0;
  try {
    if (!s || !values || !b || !x) FE_FAIL(FE_ERR_ARG, "null argument");
    FE_CUDA(cudaSetDevice(s->ctx->device));
    const cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    fe::pcg_solve_mixed(*s, values, b, x, rtol, inner_rtol, max_iter, block_size, &it, &ref, &res, st);
    if (iterations) *iterations = it;
    if (refinements) *refinements = ref;
    if (rel_residual) *rel_residual = res;
  } catch (const fe::Error& e) {
    fe::set_last_error(e.what());
    return e.code;
  }
  if (!(res <= rtol)) {
    fe::set_last_error("mixed-precision PCG stopped after " + std::to_string(it) + " inner iterations and " +
                       std::to_string(ref) + " refinements at relative residual " + std::to_string(res));
    return FE_ERR_NOT_CONVERGED;
  }
  return FE_OK;
}
