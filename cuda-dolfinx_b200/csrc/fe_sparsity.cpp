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

namespace {
// block pattern of one dofmap pair; with skip_excluded, -1 entries (dofs
// outside a restriction) take part in no coupling
void block_pattern_impl(const int32_t* dofs0, const int32_t* dofs1, int64_t num_cells, int k0, int k1, int64_t nR,
                        int64_t nC, bool skip_excluded, std::vector<int64_t>& bptr, std::vector<int32_t>& bcol) {
  std::vector<int64_t> cptr(nR + 1, 0);
  for (int64_t q = 0; q < num_cells * k0; ++q) {
    int32_t r = dofs0[q];
    if (skip_excluded && r == -1) continue;
    if (r < 0 || r >= nR) FE_FAIL(FE_ERR_ARG, "row dofmap entry out of range: " + std::to_string(r));
    cptr[r + 1]++;
  }
  for (int64_t q = 0; q < num_cells * k1; ++q) {
    int32_t c = dofs1[q];
    if (skip_excluded && c == -1) continue;
    if (c < 0 || c >= nC) FE_FAIL(FE_ERR_ARG, "column dofmap entry out of range: " + std::to_string(c));
  }
  for (int64_t r = 0; r < nR; ++r) cptr[r + 1] += cptr[r];
  std::vector<int32_t> rcells(cptr[nR]);
  {
    std::vector<int64_t> cur(cptr.begin(), cptr.end() - 1);
    for (int64_t c = 0; c < num_cells; ++c)
      for (int i = 0; i < k0; ++i) {
        const int32_t r = dofs0[c * k0 + i];
        if (r >= 0) rcells[cur[r]++] = (int32_t)c;
      }
  }
  std::vector<int64_t> len(nR, 0);
  parallel_for(nR, [&](int64_t lo, int64_t hi, unsigned) {
    std::vector<int32_t> mark(nC, -1);
    for (int64_t r = lo; r < hi; ++r) {
      int64_t cnt = 0;
      for (int64_t q = cptr[r]; q < cptr[r + 1]; ++q) {
        const int32_t* d = dofs1 + (int64_t)rcells[q] * k1;
        for (int j = 0; j < k1; ++j)
          if (d[j] >= 0 && mark[d[j]] != (int32_t)r) {
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
          if (d[j] >= 0 && mark[d[j]] != (int32_t)r) {
            mark[d[j]] = (int32_t)r;
            bcol[o++] = d[j];
          }
      }
      std::sort(bcol.begin() + bptr[r], bcol.begin() + bptr[r + 1]);
    }
  });
}
}  // namespace

void build_block_pattern(const int32_t* dofs0, const int32_t* dofs1, int64_t num_cells, int k0, int k1,
                         int64_t nR, int64_t nC, std::vector<int64_t>& bptr, std::vector<int32_t>& bcol) {
  block_pattern_impl(dofs0, dofs1, num_cells, k0, k1, nR, nC, false, bptr, bcol);
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

void build_system_pattern(const std::vector<SystemPart>& parts, int64_t num_rows, int64_t num_cols,
                          std::vector<int32_t>& row_ptr, std::vector<int32_t>& col, std::vector<int32_t>& diag) {
  if (num_rows < 0 || num_cols < 0 || num_rows > INT32_MAX || num_cols > INT32_MAX)
    FE_FAIL(FE_ERR_ARG, "matrix size out of range");
  struct Block {
    std::vector<int64_t> bptr;
    std::vector<int32_t> bcol;
  };
  std::vector<Block> B(parts.size());
  std::vector<int64_t> cnt(num_rows + 1, 0);
  for (size_t p = 0; p < parts.size(); ++p) {
    const SystemPart& P = parts[p];
    const fe_dofmap_s& R = *P.rows;
    const fe_dofmap_s& C = *P.cols;
    if (R.num_cells != C.num_cells) FE_FAIL(FE_ERR_ARG, "part " + std::to_string(p) + ": dofmaps cover different cells");
    if (P.row_offset < 0 || P.row_offset + R.num_blocks * R.bs > num_rows || P.col_offset < 0 ||
        P.col_offset + C.num_blocks * C.bs > num_cols)
      FE_FAIL(FE_ERR_ARG, "part " + std::to_string(p) + " does not fit the matrix at its offsets");
    block_pattern_impl(R.host.data(), C.host.data(), R.num_cells, R.k, C.k, R.num_blocks, C.num_blocks, true,
                       B[p].bptr, B[p].bcol);
    for (int64_t r = 0; r < R.num_blocks; ++r) {
      const int64_t L = (B[p].bptr[r + 1] - B[p].bptr[r]) * C.bs;
      for (int a = 0; a < R.bs; ++a) cnt[P.row_offset + r * R.bs + a + 1] += L;
    }
  }
  for (int64_t r = 0; r < num_rows; ++r) cnt[r + 1] += cnt[r];
  // every part's unrolled columns per row, then sorted and made unique (parts
  // that share rows and columns add up in the same entries)
  std::vector<int32_t> tmp(cnt[num_rows]);
  {
    std::vector<int64_t> cur(cnt.begin(), cnt.end() - 1);
    for (size_t p = 0; p < parts.size(); ++p) {
      const SystemPart& P = parts[p];
      const int bs0 = P.rows->bs, bs1 = P.cols->bs;
      for (int64_t R = 0; R < P.rows->num_blocks; ++R)
        for (int a = 0; a < bs0; ++a) {
          const int64_t r = P.row_offset + R * bs0 + a;
          for (int64_t t = B[p].bptr[R]; t < B[p].bptr[R + 1]; ++t)
            for (int b = 0; b < bs1; ++b) tmp[cur[r]++] = (int32_t)(P.col_offset + (int64_t)B[p].bcol[t] * bs1 + b);
        }
    }
  }
  std::vector<int64_t> len(num_rows, 0);
  parallel_for(num_rows, [&](int64_t lo, int64_t hi, unsigned) {
    for (int64_t r = lo; r < hi; ++r) {
      auto b = tmp.begin() + cnt[r], e = tmp.begin() + cnt[r + 1];
      std::sort(b, e);
      len[r] = std::unique(b, e) - b;
    }
  });
  int64_t nnz = 0;
  for (int64_t r = 0; r < num_rows; ++r) nnz += len[r];
  if (nnz > INT32_MAX) FE_FAIL(FE_ERR_ARG, "pattern has " + std::to_string(nnz) + " entries (> int32)");
  row_ptr.assign(num_rows + 1, 0);
  for (int64_t r = 0; r < num_rows; ++r) row_ptr[r + 1] = (int32_t)(row_ptr[r] + len[r]);
  col.resize(nnz);
  diag.assign(num_rows, -1);
  parallel_for(num_rows, [&](int64_t lo, int64_t hi, unsigned) {
    for (int64_t r = lo; r < hi; ++r) {
      int64_t o = row_ptr[r];
      for (int64_t t = 0; t < len[r]; ++t) {
        const int32_t c = tmp[cnt[r] + t];
        if (c == r) diag[r] = (int32_t)o;
        col[o++] = c;
      }
    }
  });
}

}  // namespace fe
