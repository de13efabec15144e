// Host construction of the CSR pattern of a cell-integral bilinear form.
//
// Equivalent of DOLFINx's SparsityPattern for a cell integral (every pair of
// dofs of a cell couples; each row keeps its columns sorted and unique) as the
// reference builds it in create_cuda_matrix (cpp/cudolfinx/fem/petsc.h:31-37),
// followed by the scalar unroll of la/petsc.cpp:38-65: block row R with block
// columns C_0 < C_1 < ... becomes scalar rows bs0*R + a (a < bs0), each with
// columns bs1*C_t + b in (t, b) order.
//
// Method: a row -> cells inverse map (counting sort), then per block row a
// marker sweep over the dofs of its cells, in parallel over row ranges.
#include <algorithm>
#include <thread>

#include "fe_internal.h"

namespace fe {

namespace {
template <typename F>
void parallel_for(int64_t n, F&& body) {
  unsigned T = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
  if (n < 4096) T = 1;
  std::vector<std::thread> th;
  for (unsigned t = 0; t < T; ++t) {
    int64_t lo = n * t / T, hi = n * (t + 1) / T;
    th.emplace_back([&body, lo, hi, t] { body(lo, hi, t); });
  }
  for (auto& x : th) x.join();
}
}  // namespace

void build_block_pattern(const int32_t* dofs0, const int32_t* dofs1, int64_t num_cells, int k0, int k1,
                         int64_t nR, int64_t nC, std::vector<int64_t>& bptr, std::vector<int32_t>& bcol) {
  std::vector<int64_t> cptr(nR + 1, 0);
  for (int64_t q = 0; q < num_cells * k0; ++q) {
    int32_t r = dofs0[q];
    if (r < 0 || r >= nR) FE_FAIL(FE_ERR_ARG, "row dofmap entry out of range: " + std::to_string(r));
    cptr[r + 1]++;
  }
  for (int64_t q = 0; q < num_cells * k1; ++q) {
    int32_t c = dofs1[q];
    if (c < 0 || c >= nC) FE_FAIL(FE_ERR_ARG, "column dofmap entry out of range: " + std::to_string(c));
  }
  for (int64_t r = 0; r < nR; ++r) cptr[r + 1] += cptr[r];
  std::vector<int32_t> rcells(cptr[nR]);
  {
    std::vector<int64_t> cur(cptr.begin(), cptr.end() - 1);
    for (int64_t c = 0; c < num_cells; ++c)
      for (int i = 0; i < k0; ++i) rcells[cur[dofs0[c * k0 + i]]++] = (int32_t)c;
  }
  std::vector<int64_t> len(nR, 0);
  parallel_for(nR, [&](int64_t lo, int64_t hi, unsigned) {
    std::vector<int32_t> mark(nC, -1);
    for (int64_t r = lo; r < hi; ++r) {
      int64_t cnt = 0;
      for (int64_t q = cptr[r]; q < cptr[r + 1]; ++q) {
        const int32_t* d = dofs1 + (int64_t)rcells[q] * k1;
        for (int j = 0; j < k1; ++j)
          if (mark[d[j]] != (int32_t)r) {
            mark[d[j]] = (int32_t)r;
            ++cnt;
          }
      }
      len[r] = cnt;
    }
  });
  bptr.assign(nR + 1, 0);
  for (int64_t r = 0; r < nR; ++r) bptr[r + 1] = bptr[r] + len[r];
  bcol.resize(bptr[nR]);
  parallel_for(nR, [&](int64_t lo, int64_t hi, unsigned) {
    std::vector<int32_t> mark(nC, -1);
    for (int64_t r = lo; r < hi; ++r) {
      int64_t o = bptr[r];
      for (int64_t q = cptr[r]; q < cptr[r + 1]; ++q) {
        const int32_t* d = dofs1 + (int64_t)rcells[q] * k1;
        for (int j = 0; j < k1; ++j)
          if (mark[d[j]] != (int32_t)r) {
            mark[d[j]] = (int32_t)r;
            bcol[o++] = d[j];
          }
      }
      std::sort(bcol.begin() + bptr[r], bcol.begin() + bptr[r + 1]);
    }
  });
}

void unroll_pattern(const std::vector<int64_t>& bptr, const std::vector<int32_t>& bcol, int bs0, int bs1,
                    std::vector<int32_t>& row_ptr, std::vector<int32_t>& col, std::vector<int32_t>& diag) {
  const int64_t nR = (int64_t)bptr.size() - 1;
  const int64_t nnz = bptr[nR] * bs0 * bs1;
  if (nnz > INT32_MAX) FE_FAIL(FE_ERR_ARG, "pattern has " + std::to_string(nnz) + " entries (> int32)");
  row_ptr.assign(nR * bs0 + 1, 0);
  for (int64_t R = 0; R < nR; ++R) {
    int64_t L = (bptr[R + 1] - bptr[R]) * bs1;
    for (int a = 0; a < bs0; ++a) row_ptr[R * bs0 + a + 1] = (int32_t)(row_ptr[R * bs0 + a] + L);
  }
  col.resize(nnz);
  diag.assign(nR * bs0, -1);
  parallel_for(nR, [&](int64_t lo, int64_t hi, unsigned) {
    for (int64_t R = lo; R < hi; ++R) {
      for (int a = 0; a < bs0; ++a) {
        int64_t r = R * bs0 + a;
        int64_t o = row_ptr[r];
        for (int64_t t = bptr[R]; t < bptr[R + 1]; ++t)
          for (int b = 0; b < bs1; ++b) {
            int32_t c = bcol[t] * bs1 + b;
            if (c == r) diag[r] = (int32_t)o;
            col[o++] = c;
          }
      }
    }
  });
}

}  // namespace fe
