// Forms given as FFCx tabulate_tensor bodies, compiled at run time for sm_100a.
//
// The reference accepts any UFL form: FFCx generates C code for each
// integral, python/cudolfinx/jit.py:15-59 extracts the body of every
// tabulate_tensor_integral_* function, jit.py:61-114 puts a CUDA signature in
// front of it, and CUDAFormIntegral.cpp:2366-2469 pastes it into string
// templates of the assembly kernels that NVRTC compiles to PTX, cached on disk
// by the integral's name alone (CUDAFormIntegral.cpp:2472-2558).
//
// Here the body keeps the FFCx signature
//     A, w, c, coordinate_dofs, entity_local_index, quadrature_permutation
// and becomes a __device__ __forceinline__ function of a generated
// translation unit that also holds this engine's own skeletons: one thread per
// integration entity (cell, exterior facet, interior facet), the element
// tensor in registers / local memory, rows and columns of BC dofs and of dofs
// outside a restriction skipped, the scatter through the byte map of the
// bound pattern (no column search), FP64 atomics; a vector, a lifting and a
// functional kernel with a fixed-order sum.  NVRTC compiles the unit to a
// cubin for the device's architecture (sm_100a on B200); cubins are cached in
// memory and, with a cache directory, on disk, keyed on a hash of the whole
// generated source and the options (so two forms whose bodies differ never
// share a kernel), and loaded with cudaLibraryLoadData.
//
// Data the bodies read, as DOLFINx packs it for FFCx:
//   w                 coefficient values of the entity's cell: coefficient q
//                     occupies [offset_q, offset_q + size_q), its element dofs
//                     node-major with the block components interleaved
//                     (dof*bs + comp); packed once per assembly call from the
//                     coefficient arrays through their dofmaps.  Interior
//                     facets: per coefficient the values of cell 0, then of
//                     cell 1 (offsets doubled).
//   c                 the form's constants.
//   coordinate_dofs   the 4 vertices x 3 coordinates of the cell (interior
//                     facets: cell 0's, then cell 1's).
//   entity_local_index  the local facet (exterior), both local facets (interior).
//   quadrature_permutation  interior facets: per side the facet's
//                     (rotations, reflection) code 2*rot + ref relative to its
//                     lowest-numbered global vertex, the code DOLFINx computes
//                     for triangle facets and FFCx's permuted tables expect.
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "fe_internal.h"

namespace fe {

// One compiled translation unit (the kernels of one form integral).
struct FfcxLibrary {
  int device = 0;
  cudaLibrary_t lib = nullptr;
  cudaKernel_t mat = nullptr, vec = nullptr, lift = nullptr, scalar = nullptr, scalar_sum = nullptr;
  std::vector<char> cubin;  // kept to fill other cache directories
  ~FfcxLibrary() {
    if (lib) (void)cudaLibraryUnload(lib);
  }
};

namespace {

constexpr int kThreads = 128;
constexpr int kScalarBlocks = 1024;  // fixed grid of the functional: a fixed summation order

// Kernel argument record.  The generated source declares the same struct
// (kArgsDecl); both sides are compiled for 64-bit targets with natural
// alignment, so the layouts agree.
struct FfcxArgs {
  long long num_entities;
  const int* entities;          // exterior: [n][2] (cell, facet); interior: [n][4]
  const unsigned char* perms;   // interior: [n][2] quadrature permutation of each side
  const double* x;              // [nodes][3]
  const int* geom;              // [cells][4]
  const int* dofs0;             // [cells][K0] (interior: macro [n][2*K0])
  const int* dofs1;
  const unsigned char* pos;     // byte map: [cells][K0][K1] or [facets][2K0][2K1]
  const int* row_ptr;
  const unsigned char* bc0;
  const unsigned char* bc1;
  const double* w;              // packed coefficients [cells][W]
  const double* c;              // constants
  double* out;                  // CSR values / vector
  const double* g;              // lifting: BC values
  const double* x0;
  double scale;
  double* partial;              // functional: [kScalarBlocks] + result
};

const char* kArgsDecl = R"(
struct FfcxArgs {
  long long num_entities;
  const int* entities;
  const unsigned char* perms;
  const double* x;
  const int* geom;
  const int* dofs0;
  const int* dofs1;
  const unsigned char* pos;
  const int* row_ptr;
  const unsigned char* bc0;
  const unsigned char* bc1;
  const double* w;
  const double* c;
  double* out;
  const double* g;
  const double* x0;
  double scale;
  double* partial;
};
)";

// The skeletons.  Placeholders @X@ are replaced by the form's sizes.
const char* kSkeleton = R"(
#define IT @IT@
#define RANK @RANK@
#define K0 @K0@
#define BS0 @BS0@
#define K1 @K1@
#define BS1 @BS1@
#define NS @NS@
#define W @W@
#define NCOEF @NCOEF@
#define NK0 (NS * K0)
#define NK1 (NS * K1)
#define NA @NA@
#define NTHREADS @NT@
#define NSBLOCKS @NSB@
static __device__ const int kCoefOffset[NCOEF + 1] = {@COFF@};

// geometry, coefficients and local facets of entity e
__device__ __forceinline__ void ffcx_entity(const FfcxArgs& a, long long e, int cell[2], int eli[2],
                                            unsigned char perm[2], double* cd, double* wl) {
  if (IT == 0) {
    cell[0] = (int)e;
    eli[0] = 0;
  } else if (IT == 1) {
    cell[0] = __ldg(a.entities + 2 * e);
    eli[0] = __ldg(a.entities + 2 * e + 1);
  } else {
    cell[0] = __ldg(a.entities + 4 * e);
    eli[0] = __ldg(a.entities + 4 * e + 1);
    cell[1] = __ldg(a.entities + 4 * e + 2);
    eli[1] = __ldg(a.entities + 4 * e + 3);
    perm[0] = __ldg(a.perms + 2 * e);
    perm[1] = __ldg(a.perms + 2 * e + 1);
  }
  for (int s = 0; s < NS; ++s) {
    const int4 v = __ldg(reinterpret_cast<const int4*>(a.geom) + cell[s]);
    const int vv[4] = {v.x, v.y, v.z, v.w};
    for (int q = 0; q < 4; ++q)
      for (int d = 0; d < 3; ++d) cd[s * 12 + q * 3 + d] = __ldg(a.x + 3 * (long long)vv[q] + d);
  }
  if (NS == 2) {
    // interior facets: per coefficient cell 0's values, then cell 1's
    for (int q = 0; q < NCOEF; ++q) {
      const int o = kCoefOffset[q], n = kCoefOffset[q + 1] - o;
      for (int s = 0; s < 2; ++s)
        for (int t = 0; t < n; ++t) wl[2 * o + s * n + t] = __ldg(a.w + (long long)cell[s] * W + o + t);
    }
  }
}

__device__ __forceinline__ int ffcx_dof0(const FfcxArgs& a, long long e, const int cell[2], int i) {
  return NS == 2 ? __ldg(a.dofs0 + e * NK0 + i) : __ldg(a.dofs0 + (long long)cell[0] * K0 + i);
}
__device__ __forceinline__ int ffcx_dof1(const FfcxArgs& a, long long e, const int cell[2], int j) {
  return NS == 2 ? __ldg(a.dofs1 + e * NK1 + j) : __ldg(a.dofs1 + (long long)cell[0] * K1 + j);
}

#if RANK == 2
extern "C" __global__ void __launch_bounds__(NTHREADS) fe_ffcx_mat(const FfcxArgs a) {
  for (long long e = blockIdx.x * (long long)NTHREADS + threadIdx.x; e < a.num_entities;
       e += (long long)gridDim.x * NTHREADS) {
    int cell[2] = {0, 0}, eli[2] = {0, 0};
    unsigned char perm[2] = {0, 0};
    double cd[NS * 12];
    double wl[NS == 2 ? 2 * W + 1 : 1];
    ffcx_entity(a, e, cell, eli, perm, cd, wl);
    double A[NA];
    for (int q = 0; q < NA; ++q) A[q] = 0.0;
    TABULATE(A, NS == 2 ? wl : a.w + (long long)cell[0] * W, a.c, cd, eli, perm);
    const unsigned char* pe = a.pos + (NS == 2 ? e : (long long)cell[0]) * (NK0 * NK1);
    for (int i = 0; i < NK0; ++i) {
      const int d0 = ffcx_dof0(a, e, cell, i);
      if (d0 < 0) continue;
      for (int al = 0; al < BS0; ++al) {
        const long long r = (long long)d0 * BS0 + al;
        if (a.bc0 && a.bc0[r]) continue;
        const int rp = __ldg(a.row_ptr + r);
        for (int j = 0; j < NK1; ++j) {
          const int d1 = ffcx_dof1(a, e, cell, j);
          if (d1 < 0) continue;
          const int p = pe[i * NK1 + j];
          for (int be = 0; be < BS1; ++be) {
            if (a.bc1 && a.bc1[(long long)d1 * BS1 + be]) continue;
            atomicAdd(a.out + rp + BS1 * p + be, A[(i * BS0 + al) * (NK1 * BS1) + j * BS1 + be]);
          }
        }
      }
    }
  }
}

// b[row] -= scale * sum over BC columns of A[row][col] (g - x0)[col], for the
// entities with a BC column (CUDAFormIntegral.cpp:647-715), every row
extern "C" __global__ void __launch_bounds__(NTHREADS) fe_ffcx_lift(const FfcxArgs a) {
  for (long long e = blockIdx.x * (long long)NTHREADS + threadIdx.x; e < a.num_entities;
       e += (long long)gridDim.x * NTHREADS) {
    int cell[2] = {0, 0};
    {
      if (IT == 1) cell[0] = __ldg(a.entities + 2 * e);
      else if (IT == 0) cell[0] = (int)e;
    }
    bool any = false;
    for (int j = 0; j < NK1 && !any; ++j) {
      const int d1 = ffcx_dof1(a, e, cell, j);
      if (d1 < 0) continue;
      for (int be = 0; be < BS1; ++be) any |= a.bc1[(long long)d1 * BS1 + be] != 0;
    }
    if (!any) continue;
    int eli[2] = {0, 0};
    unsigned char perm[2] = {0, 0};
    double cd[NS * 12];
    double wl[NS == 2 ? 2 * W + 1 : 1];
    ffcx_entity(a, e, cell, eli, perm, cd, wl);
    double A[NA];
    for (int q = 0; q < NA; ++q) A[q] = 0.0;
    TABULATE(A, NS == 2 ? wl : a.w + (long long)cell[0] * W, a.c, cd, eli, perm);
    for (int i = 0; i < NK0; ++i) {
      const int d0 = ffcx_dof0(a, e, cell, i);
      if (d0 < 0) continue;
      for (int al = 0; al < BS0; ++al) {
        double s = 0.0;
        for (int j = 0; j < NK1; ++j) {
          const int d1 = ffcx_dof1(a, e, cell, j);
          if (d1 < 0) continue;
          for (int be = 0; be < BS1; ++be) {
            const long long cc = (long long)d1 * BS1 + be;
            if (!a.bc1[cc]) continue;
            s += A[(i * BS0 + al) * (NK1 * BS1) + j * BS1 + be] * (a.g[cc] - (a.x0 ? a.x0[cc] : 0.0));
          }
        }
        if (s != 0.0) atomicAdd(a.out + (long long)d0 * BS0 + al, -a.scale * s);
      }
    }
  }
}
#endif

#if RANK == 1
extern "C" __global__ void __launch_bounds__(NTHREADS) fe_ffcx_vec(const FfcxArgs a) {
  for (long long e = blockIdx.x * (long long)NTHREADS + threadIdx.x; e < a.num_entities;
       e += (long long)gridDim.x * NTHREADS) {
    int cell[2] = {0, 0}, eli[2] = {0, 0};
    unsigned char perm[2] = {0, 0};
    double cd[NS * 12];
    double wl[NS == 2 ? 2 * W + 1 : 1];
    ffcx_entity(a, e, cell, eli, perm, cd, wl);
    double A[NA];
    for (int q = 0; q < NA; ++q) A[q] = 0.0;
    TABULATE(A, NS == 2 ? wl : a.w + (long long)cell[0] * W, a.c, cd, eli, perm);
    for (int i = 0; i < NK0; ++i) {
      const int d0 = ffcx_dof0(a, e, cell, i);
      if (d0 < 0) continue;
      for (int al = 0; al < BS0; ++al) atomicAdd(a.out + (long long)d0 * BS0 + al, A[i * BS0 + al]);
    }
  }
}
#endif

#if RANK == 0
// per block: its threads' entity sums in a fixed order, then a fixed tree
extern "C" __global__ void __launch_bounds__(NTHREADS) fe_ffcx_scalar(const FfcxArgs a) {
  __shared__ double sh[NTHREADS];
  double acc = 0.0;
  for (long long e = blockIdx.x * (long long)NTHREADS + threadIdx.x; e < a.num_entities;
       e += (long long)gridDim.x * NTHREADS) {
    int cell[2] = {0, 0}, eli[2] = {0, 0};
    unsigned char perm[2] = {0, 0};
    double cd[NS * 12];
    double wl[NS == 2 ? 2 * W + 1 : 1];
    ffcx_entity(a, e, cell, eli, perm, cd, wl);
    double A[1] = {0.0};
    TABULATE(A, NS == 2 ? wl : a.w + (long long)cell[0] * W, a.c, cd, eli, perm);
    acc += A[0];
  }
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int h = NTHREADS / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.partial[blockIdx.x] = sh[0];
}

// the block partials summed in index order into partial[NSBLOCKS]
extern "C" __global__ void fe_ffcx_scalar_sum(const FfcxArgs a, int nblocks) {
  __shared__ double sh[NTHREADS];
  double acc = 0.0;
  for (int q = threadIdx.x; q < nblocks; q += NTHREADS) acc += a.partial[q];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int h = NTHREADS / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) sh[threadIdx.x] += sh[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.partial[NSBLOCKS] = sh[0];
}
#endif
)";

const char* kPreamble = R"(
#define restrict __restrict__
typedef unsigned char uint8_t;
typedef unsigned int uint32_t;
typedef int int32_t;
typedef long long int64_t;
typedef double ufc_scalar_t;
)";

void replace_all(std::string& s, const std::string& from, const std::string& to) {
  size_t p = 0;
  while ((p = s.find(from, p)) != std::string::npos) {
    s.replace(p, from.size(), to);
    p += to.size();
  }
}

bool valid_identifier(const std::string& s) {
  if (s.empty() || !(isalpha((unsigned char)s[0]) || s[0] == '_')) return false;
  for (char ch : s)
    if (!(isalnum((unsigned char)ch) || ch == '_')) return false;
  return true;
}

std::string generate_source(int itype, int rank, int k0, int bs0, int k1, int bs1, const std::vector<int>& offsets,
                            const std::string& name, const std::string& body) {
  const int ns = itype == FE_INTEGRAL_INTERIOR_FACET ? 2 : 1;
  if (rank < 1) k0 = bs0 = 1;
  if (rank < 2) k1 = bs1 = 1;
  int na = 1;
  if (rank == 1) na = ns * k0 * bs0;
  if (rank == 2) na = ns * k0 * bs0 * ns * k1 * bs1;
  std::string sk = kSkeleton;
  replace_all(sk, "@IT@", std::to_string(itype));
  replace_all(sk, "@RANK@", std::to_string(rank));
  replace_all(sk, "@K0@", std::to_string(k0));
  replace_all(sk, "@BS0@", std::to_string(bs0));
  replace_all(sk, "@K1@", std::to_string(k1));
  replace_all(sk, "@BS1@", std::to_string(bs1));
  replace_all(sk, "@NS@", std::to_string(ns));
  replace_all(sk, "@W@", std::to_string(offsets.back()));
  replace_all(sk, "@NCOEF@", std::to_string(offsets.size() - 1));
  replace_all(sk, "@NA@", std::to_string(na));
  replace_all(sk, "@NT@", std::to_string(kThreads));
  replace_all(sk, "@NSB@", std::to_string(kScalarBlocks));
  std::string off;
  for (size_t q = 0; q < offsets.size(); ++q) off += (q ? ", " : "") + std::to_string(offsets[q]);
  replace_all(sk, "@COFF@", off);
  std::ostringstream src;
  src << kPreamble << "\n"
      << "static __device__ __forceinline__ void " << name << "(double* restrict A, const double* restrict w,\n"
      << "    const double* restrict c, const double* restrict coordinate_dofs,\n"
      << "    const int* restrict entity_local_index, const uint8_t* restrict quadrature_permutation)\n{\n"
      << body << "\n}\n"
      << kArgsDecl << "\n#define TABULATE " << name << "\n"
      << sk;
  return src.str();
}

std::string generate_source(const fe_form_s& f) {
  const fe_form_s::Ffcx& X = *f.ffcx;
  return generate_source(X.integral_type, f.rank, f.rank >= 1 ? f.V0->k : 1, f.rank >= 1 ? f.V0->bs : 1,
                         f.rank == 2 ? f.V1->k : 1, f.rank == 2 ? f.V1->bs : 1, X.offsets, X.name, X.body);
}

std::string hex64(uint64_t v) {
  char b[17];
  std::snprintf(b, sizeof(b), "%016llx", (unsigned long long)v);
  return b;
}

// FNV-1a: a stable 64-bit key of the source (std::hash is not stable across runs)
uint64_t fnv1a(const std::string& s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char ch : s) {
    h ^= ch;
    h *= 1099511628211ull;
  }
  return h;
}

std::vector<char> nvrtc_compile(const std::string& src, const std::string& name, const std::string& arch) {
  nvrtcProgram prog;
  nvrtcResult r = nvrtcCreateProgram(&prog, src.c_str(), (name + ".cu").c_str(), 0, nullptr, nullptr);
  if (r != NVRTC_SUCCESS) FE_FAIL(FE_ERR_ARG, std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(r));
  const std::string archopt = "-arch=" + arch;
  const char* opts[] = {archopt.c_str(), "-std=c++17", "-lineinfo"};
  r = nvrtcCompileProgram(prog, 3, opts);
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  std::string log(log_size, '\0');
  if (log_size) nvrtcGetProgramLog(prog, &log[0]);
  if (r != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    FE_FAIL(FE_ERR_ARG, "NVRTC could not compile the tabulate_tensor body of '" + name + "' (" +
                            nvrtcGetErrorString(r) + "):\n" + log);
  }
  size_t n = 0;
  r = nvrtcGetCUBINSize(prog, &n);
  std::vector<char> cubin(n);
  if (r == NVRTC_SUCCESS) r = nvrtcGetCUBIN(prog, cubin.data());
  nvrtcDestroyProgram(&prog);
  if (r != NVRTC_SUCCESS) FE_FAIL(FE_ERR_ARG, std::string("nvrtcGetCUBIN: ") + nvrtcGetErrorString(r));
  return cubin;
}

std::mutex g_lib_mutex;
std::map<std::string, std::shared_ptr<FfcxLibrary>> g_libs;  // key: device/hash

std::shared_ptr<FfcxLibrary> load_library(int device, int rank, const std::string& src, const std::string& name,
                                          const std::string& cachedir) {
  int major = 0, minor = 0;
  FE_CUDA(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device));
  FE_CUDA(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device));
  // the "a" targets (sm_90a, sm_100a) expose the full instruction set of the part
  const std::string arch = "sm_" + std::to_string(major * 10 + minor) + (major >= 9 ? "a" : "");
  const std::string key_src = src + "\n// " + arch;
  const std::string hash = hex64(fnv1a(key_src));
  const std::string key = std::to_string(device) + "/" + hash;
  std::lock_guard<std::mutex> lock(g_lib_mutex);
  const std::string stem = cachedir.empty() ? std::string() : cachedir + "/" + name + "_" + hash;
  auto write_cache = [&](const std::vector<char>& bin) {
    if (stem.empty()) return;
    std::ofstream(stem + ".cu", std::ios::binary) << key_src;
    std::ofstream(stem + ".cubin", std::ios::binary).write(bin.data(), (std::streamsize)bin.size());
  };
  auto it = g_libs.find(key);
  if (it != g_libs.end()) {
    // loaded already in this process: still fill a cache directory that lacks it
    if (!stem.empty() && !std::ifstream(stem + ".cubin", std::ios::binary)) write_cache(it->second->cubin);
    return it->second;
  }
  std::vector<char> cubin;
  if (!stem.empty()) {
    // a cached cubin is used only if its recorded source is this source
    std::ifstream fs(stem + ".cu", std::ios::binary), fb(stem + ".cubin", std::ios::binary);
    if (fs && fb) {
      std::string cached((std::istreambuf_iterator<char>(fs)), std::istreambuf_iterator<char>());
      if (cached == key_src) cubin.assign(std::istreambuf_iterator<char>(fb), std::istreambuf_iterator<char>());
    }
  }
  if (cubin.empty()) {
    cubin = nvrtc_compile(src, name, arch);
    write_cache(cubin);
  }
  auto L = std::make_shared<FfcxLibrary>();
  L->device = device;
  L->cubin = cubin;
  FE_CUDA(cudaLibraryLoadData(&L->lib, L->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
  if (rank == 2) {
    FE_CUDA(cudaLibraryGetKernel(&L->mat, L->lib, "fe_ffcx_mat"));
    FE_CUDA(cudaLibraryGetKernel(&L->lift, L->lib, "fe_ffcx_lift"));
  } else if (rank == 1) {
    FE_CUDA(cudaLibraryGetKernel(&L->vec, L->lib, "fe_ffcx_vec"));
  } else {
    FE_CUDA(cudaLibraryGetKernel(&L->scalar, L->lib, "fe_ffcx_scalar"));
    FE_CUDA(cudaLibraryGetKernel(&L->scalar_sum, L->lib, "fe_ffcx_scalar_sum"));
  }
  g_libs[key] = L;
  return L;
}

__global__ void k_pack_field(const int32_t* __restrict__ map, int k, int bs, const double* __restrict__ vals,
                             double* __restrict__ packed, int64_t num_cells, int W, int offset) {
  const int64_t n = num_cells * k * bs;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = t / (k * bs);
    const int r = (int)(t - c * k * bs);
    const int i = r / bs, a = r - i * bs;
    packed[c * W + offset + r] = __ldg(vals + (int64_t)__ldg(map + c * k + i) * bs + a);
  }
}

unsigned grid_for(int64_t n) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + kThreads - 1) / kThreads, 148 * 64));
}

int64_t num_entities(const fe_form_s& f) {
  return f.ffcx->integral_type == FE_INTEGRAL_CELL ? f.mesh->num_cells : f.num_facets;
}

// packs every coefficient into [cells][W] (the reference's pack_coefficients,
// CUDAAssembler.cpp:59-96, once per assembly call)
void pack(fe_form_s& f, cudaStream_t s) {
  fe_form_s::Ffcx& X = *f.ffcx;
  const int64_t C = f.mesh->num_cells;
  if (X.W == 0 || C == 0) return;
  if (X.packed.n < (size_t)(C * X.W)) X.packed.alloc((size_t)(C * X.W));
  for (size_t q = 0; q + 1 < X.offsets.size(); ++q) {
    const fe_form_s::Ffcx::Field& F = *X.fields[q];
    if (!F.map) FE_FAIL(FE_ERR_ARG, "coefficient " + std::to_string(q) + " is not set");
    const int64_t n = C * F.map->k * F.map->bs;
    k_pack_field<<<grid_for(n), kThreads, 0, s>>>(F.map->dofs.p, F.map->k, F.map->bs, F.values, X.packed.p, C, X.W,
                                                  X.offsets[q]);
    FE_CUDA(cudaGetLastError());
  }
}

FfcxArgs base_args(fe_form_s& f) {
  FfcxArgs a{};
  const fe_form_s::Ffcx& X = *f.ffcx;
  a.num_entities = num_entities(f);
  a.entities = f.facets.p;
  a.perms = X.perms.p;
  a.x = f.mesh->x.p;
  a.geom = f.mesh->geom.p;
  if (f.rank >= 1) a.dofs0 = X.integral_type == FE_INTEGRAL_INTERIOR_FACET ? f.macro0.p : f.V0->dofs.p;
  if (f.rank == 2) {
    a.dofs1 = X.integral_type == FE_INTEGRAL_INTERIOR_FACET ? (f.macro1.p ? f.macro1.p : f.macro0.p) : f.V1->dofs.p;
  }
  a.w = X.packed.p;
  a.c = X.consts.p;
  return a;
}

void launch(cudaKernel_t k, unsigned grid, FfcxArgs& a, cudaStream_t s) {
  void* args[] = {&a};
  FE_CUDA(cudaLaunchKernel((const void*)k, dim3(grid), dim3(kThreads), args, 0, s));
}

void require_ready(const fe_form_s& f) {
  const fe_form_s::Ffcx& X = *f.ffcx;
  if (X.integral_type != FE_INTEGRAL_CELL && !f.facets_set)
    FE_FAIL(FE_ERR_ARG, "set the integration facets of the facet integral first");
  if ((int)X.host_consts.size() != X.num_constants)
    FE_FAIL(FE_ERR_ARG, "the form's " + std::to_string(X.num_constants) + " constant(s) are not set");
}

}  // namespace

void ffcx_create(fe_form_s& f, int integral_type, const char* name, const char* body, int num_coefficients,
                 const int* coefficient_sizes, int num_constants, const char* cachedir) {
  FE_REQUIRE(integral_type >= FE_INTEGRAL_CELL && integral_type <= FE_INTEGRAL_INTERIOR_FACET,
             "unknown integral type " + std::to_string(integral_type));
  FE_REQUIRE(name && valid_identifier(name), "the tabulate_tensor name must be a C identifier");
  FE_REQUIRE(body, "null tabulate_tensor body");
  FE_REQUIRE(num_coefficients >= 0 && (coefficient_sizes || num_coefficients == 0) && num_constants >= 0,
             "invalid coefficient / constant counts");
  auto X = std::make_unique<fe_form_s::Ffcx>();
  X->integral_type = integral_type;
  X->name = name;
  X->body = body;
  X->offsets.push_back(0);
  for (int q = 0; q < num_coefficients; ++q) {
    FE_REQUIRE(coefficient_sizes[q] > 0, "coefficient sizes must be positive");
    X->offsets.push_back(X->offsets.back() + coefficient_sizes[q]);
  }
  X->W = X->offsets.back();
  for (int q = 0; q < num_coefficients; ++q) X->fields.push_back(std::make_unique<fe_form_s::Ffcx::Field>());
  X->num_constants = num_constants;
  f.ffcx = std::move(X);
  f.kind = integral_type == FE_INTEGRAL_CELL ? FE_FORM_FFCX_CELL
                                             : (integral_type == FE_INTEGRAL_EXTERIOR_FACET ? FE_FORM_FFCX_EXTERIOR
                                                                                            : FE_FORM_FFCX_INTERIOR);
  const std::string src = generate_source(f);
  f.ffcx->lib = load_library(f.ctx->device, f.rank, src, name, cachedir ? cachedir : "");
}

void ffcx_set_coefficient(fe_form_s& f, int index, fe_dofmap map, const double* values, int64_t n,
                          bool on_device, cudaStream_t s) {
  fe_form_s::Ffcx& X = *f.ffcx;
  FE_REQUIRE(index >= 0 && index + 1 < (int)X.offsets.size(), "coefficient index out of range");
  FE_REQUIRE(map && values, "null argument");
  FE_REQUIRE(map->ctx == f.ctx && map->num_cells == f.mesh->num_cells && !map->excluded,
             "a coefficient needs an unrestricted dofmap of the form's mesh");
  const int size = X.offsets[index + 1] - X.offsets[index];
  FE_REQUIRE(map->k * map->bs == size, "coefficient " + std::to_string(index) + " has " + std::to_string(size) +
                                           " values per cell; the dofmap gives " +
                                           std::to_string(map->k * map->bs));
  FE_REQUIRE(n >= map->num_blocks * map->bs, "fewer coefficient values than the dofmap's dofs");
  fe_form_s::Ffcx::Field& F = *X.fields[index];
  F.map = map;
  if (on_device) {
    F.own.release();
    F.values = values;
  } else {
    if (F.own.n < (size_t)n) F.own.alloc((size_t)n);
    FE_CUDA(cudaMemcpyAsync(F.own.p, values, n * sizeof(double), cudaMemcpyHostToDevice, s));
    F.values = F.own.p;
  }
}

void ffcx_set_constants(fe_form_s& f, const double* values, int n, cudaStream_t s) {
  fe_form_s::Ffcx& X = *f.ffcx;
  FE_REQUIRE(n == X.num_constants, "the form has " + std::to_string(X.num_constants) + " constant value(s)");
  FE_REQUIRE(values || n == 0, "null constants");
  X.host_consts.assign(values, values + n);
  if (n) {
    if (X.consts.n < (size_t)n) X.consts.alloc((size_t)n);
    FE_CUDA(cudaMemcpyAsync(X.consts.p, X.host_consts.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
  }
}

void ffcx_set_interior_permutations(fe_form_s& f) {
  // per side: facet f of a tetrahedron has the local vertices {0,1,2,3} \ {f}
  // in increasing order; rot = position of the lowest global vertex, ref = 1
  // when the vertex after it (cyclically) is numbered above the one before it
  const std::vector<int32_t>& G = f.mesh->host_geom;
  const int64_t F = f.num_facets;
  std::vector<uint8_t> perm((size_t)std::max<int64_t>(1, 2 * F), 0);
  for (int64_t e = 0; e < F; ++e)
    for (int s = 0; s < 2; ++s) {
      const int32_t c = f.host_facets[4 * e + 2 * s], lf = f.host_facets[4 * e + 2 * s + 1];
      int64_t v[3];
      int m = 0;
      for (int t = 0; t < 4; ++t)
        if (t != lf) v[m++] = G[4 * (int64_t)c + t];
      int rot = 0;
      for (int t = 1; t < 3; ++t)
        if (v[t] < v[rot]) rot = t;
      const int64_t pre = v[(rot + 2) % 3], post = v[(rot + 1) % 3];
      const int ref = post > pre ? 1 : 0;
      perm[2 * e + s] = (uint8_t)(2 * rot + ref);
    }
  fe_form_s::Ffcx& X = *f.ffcx;
  X.perms.alloc(perm.size());
  FE_CUDA(cudaMemcpy(X.perms.p, perm.data(), perm.size(), cudaMemcpyHostToDevice));
}

void ffcx_assemble_matrix(fe_form_s& f, double* values, const fe_bc_s* bc0, const fe_bc_s* bc1, cudaStream_t s) {
  require_ready(f);
  pack(f, s);
  FfcxArgs a = base_args(f);
  if (!a.num_entities) return;
  a.pos = f.pos.p;
  a.row_ptr = f.sp->row_ptr.p;
  a.bc0 = bc0 ? bc0->markers.p : nullptr;
  a.bc1 = bc1 ? bc1->markers.p : nullptr;
  a.out = values;
  launch(f.ffcx->lib->mat, grid_for(a.num_entities), a, s);
}

void ffcx_assemble_vector(fe_form_s& f, double* b, cudaStream_t s) {
  require_ready(f);
  pack(f, s);
  FfcxArgs a = base_args(f);
  if (!a.num_entities) return;
  a.out = b;
  launch(f.ffcx->lib->vec, grid_for(a.num_entities), a, s);
}

void ffcx_lifting(fe_form_s& f, const fe_bc_s& bc, const double* x0, double scale, double* b, cudaStream_t s) {
  require_ready(f);
  pack(f, s);
  FfcxArgs a = base_args(f);
  if (!a.num_entities) return;
  a.bc1 = bc.markers.p;
  a.g = bc.g.p;
  a.x0 = x0;
  a.scale = scale;
  a.out = b;
  launch(f.ffcx->lib->lift, grid_for(a.num_entities), a, s);
}

double ffcx_assemble_scalar(fe_form_s& f, cudaStream_t s) {
  require_ready(f);
  pack(f, s);
  fe_form_s::Ffcx& X = *f.ffcx;
  if (X.partial.n < (size_t)kScalarBlocks + 1) X.partial.alloc(kScalarBlocks + 1);
  FfcxArgs a = base_args(f);
  a.partial = X.partial.p;
  const unsigned grid = (unsigned)std::min<int64_t>(kScalarBlocks, std::max<int64_t>(
                                                                       1, (a.num_entities + kThreads - 1) / kThreads));
  launch(X.lib->scalar, grid, a, s);
  int nb = (int)grid;
  void* args[] = {&a, &nb};
  FE_CUDA(cudaLaunchKernel((const void*)X.lib->scalar_sum, dim3(1), dim3(kThreads), args, 0, s));
  double r = 0.0;
  FE_CUDA(cudaMemcpyAsync(&r, X.partial.p + kScalarBlocks, sizeof(double), cudaMemcpyDeviceToHost, s));
  FE_CUDA(cudaStreamSynchronize(s));
  return r;
}

}  // namespace fe

extern "C" int fe_ffcx_source(int integral_type, int rank, int k0, int bs0, int k1, int bs1, int num_coefficients,
                              const int* coefficient_sizes, const char* tabulate_name, const char* tabulate_body,
                              char* out, int64_t capacity, int64_t* length) {
  try {
    FE_REQUIRE(integral_type >= FE_INTEGRAL_CELL && integral_type <= FE_INTEGRAL_INTERIOR_FACET,
               "unknown integral type");
    FE_REQUIRE(rank >= 0 && rank <= 2, "rank must be 0, 1 or 2");
    FE_REQUIRE(tabulate_name && fe::valid_identifier(tabulate_name), "the tabulate_tensor name must be a C identifier");
    FE_REQUIRE(tabulate_body, "null tabulate_tensor body");
    FE_REQUIRE(num_coefficients >= 0 && (coefficient_sizes || !num_coefficients), "invalid coefficients");
    FE_REQUIRE(rank < 1 || (k0 > 0 && bs0 > 0), "invalid test element size");
    FE_REQUIRE(rank < 2 || (k1 > 0 && bs1 > 0), "invalid trial element size");
    std::vector<int> offsets{0};
    for (int q = 0; q < num_coefficients; ++q) offsets.push_back(offsets.back() + coefficient_sizes[q]);
    const std::string src = fe::generate_source(integral_type, rank, k0, bs0, k1, bs1, offsets, tabulate_name,
                                                tabulate_body);
    if (length) *length = (int64_t)src.size();
    if (out && capacity > 0) {
      const size_t n = std::min<size_t>(src.size(), (size_t)capacity - 1);
      std::memcpy(out, src.data(), n);
      out[n] = '\0';
    }
  } catch (const fe::Error& e) {
    fe::set_last_error(e.what());
    return e.code;
  }
  return FE_OK;
}
