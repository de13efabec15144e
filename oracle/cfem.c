/* C restatement of the cudolfinx assembly path (TEST INFRASTRUCTURE ONLY).
 *
 * This is the checker and the timed CPU baseline ("port" kind), never the
 * product: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * --impl reference legs load it.  Parity status: unpinned against DOLFINx
 * (the reference and DOLFINx cannot run here); pinned to the closed-form
 * checks in tests/test_oracle.py and to the numpy oracle.
 *
 * Algorithm (reference file:line, paths relative to the cuda-dolfinx tree):
 *   matrix  : per cell tabulate Ae, skip BC rows/cols, locate each column in
 *             its CSR row by binary search and add
 *             (cpp/cudolfinx/fem/CUDAFormIntegral.cpp:1154-1224,
 *              binary_search :2572-2602), then set the diagonal of owned BC
 *             rows (cpp/cudolfinx/fem/CUDAAssembler.cpp:131-164).  This is also
 *             the structure of DOLFINx's CPU assemble_matrix + MatSetValues.
 *   vector  : per cell element vector added into b
 *             (cpp/cudolfinx/fem/CUDAFormIntegral.cpp:309-355).
 *   lifting : b -= scale*Ae[:,bc](g - x0)[bc] for cells with a BC column
 *             (cpp/cudolfinx/fem/CUDAFormIntegral.cpp:647-715).
 *   set_bc  : b[d] = scale*(g[d]-x0[d]) (cpp/cudolfinx/fem/CUDAAssembler.cpp:115-124).
 *
 * Threading follows DOLFINx's ghosted MPI assembly: each thread owns a range
 * of block rows and assembles every cell touching them, inserting only its
 * own rows (no atomics; shared cells are recomputed).
 *
 * Element kinds: 1 = P1 Poisson (k DG0 or 1), 2 = P2 Poisson (k P1 field),
 * 3 = vector P2 elasticity (lam, mu DG0), 4 = equispaced P3 Poisson (k DG0).
 * Reference tensors are passed in by cfem_set_tables() / cfem_set_tables_p3()
 * from the exact rational tables of fem_oracle.py.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static double R2w[4][3][3][10][10]; /* int lambda_m d_a phi_i d_b phi_j */
static double R2[3][3][10][10];     /* int d_a phi_i d_b phi_j          */
static double W2[10];               /* int phi_i                         */
static double R3[3][3][20][20];     /* int d_a psi_i d_b psi_j (P3)      */
static double W3[20];               /* int psi_i (P3)                    */

void cfem_set_tables(const double* r2w, const double* r2, const double* w2)
{
  memcpy(R2w, r2w, sizeof(R2w));
  memcpy(R2, r2, sizeof(R2));
  memcpy(W2, w2, sizeof(W2));
}

void cfem_set_tables_p3(const double* r3, const double* w3)
{
  memcpy(R3, r3, sizeof(R3));
  memcpy(W3, w3, sizeof(W3));
}

/* ---------------- geometry ---------------- */
static inline void cell_geom(const double* coords, const int32_t* v, double K[3][3], double* adet)
{
  double x0[3], J[3][3];
  for (int r = 0; r < 3; ++r) x0[r] = coords[3 * (int64_t)v[0] + r];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) J[r][c] = coords[3 * (int64_t)v[c + 1] + r] - x0[r];
  double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
  double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
  double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
  double det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
  double id = 1.0 / det;
  K[0][0] = c00 * id;
  K[1][0] = c01 * id;
  K[2][0] = c02 * id;
  K[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
  K[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
  K[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
  K[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
  K[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
  K[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
  *adet = fabs(det);
}

static const double P1G[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};

/* Ae is k0 x k1 row-major (k0 = k1 = 4, 10, 20 or 30) */
static void tabulate(int kind, const double* coords, const int32_t* v, int64_t c,
                     const double* coeff0, const double* coeff1, double* Ae)
{
  double K[3][3], adet;
  cell_geom(coords, v, K, &adet);
  if (kind == 1) {
    double G[4][3];
    for (int i = 0; i < 4; ++i)
      for (int b = 0; b < 3; ++b)
        G[i][b] = P1G[i][0] * K[0][b] + P1G[i][1] * K[1][b] + P1G[i][2] * K[2][b];
    double s = adet / 6.0 * (coeff0 ? coeff0[c] : 1.0);
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j)
        Ae[i * 4 + j] = s * (G[i][0] * G[j][0] + G[i][1] * G[j][1] + G[i][2] * G[j][2]);
  } else if (kind == 2) {
    double Gh[3][3];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        Gh[a][b] = adet * (K[a][0] * K[b][0] + K[a][1] * K[b][1] + K[a][2] * K[b][2]);
    double km[4];
    for (int m = 0; m < 4; ++m) km[m] = coeff0[v[m]];
    for (int i = 0; i < 100; ++i) Ae[i] = 0.0;
    for (int m = 0; m < 4; ++m)
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
          double w = km[m] * Gh[a][b];
          const double* R = &R2w[m][a][b][0][0];
          for (int e = 0; e < 100; ++e) Ae[e] += w * R[e];
        }
  } else if (kind == 4) {
    double s = coeff0 ? coeff0[c] : 1.0;
    for (int i = 0; i < 400; ++i) Ae[i] = 0.0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double w = s * adet * (K[a][0] * K[b][0] + K[a][1] * K[b][1] + K[a][2] * K[b][2]);
        const double* R = &R3[a][b][0][0];
        for (int e = 0; e < 400; ++e) Ae[e] += w * R[e];
      }
  } else {
    static __thread double D[3][3][100];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double* Dab = D[a][b];
        for (int e = 0; e < 100; ++e) Dab[e] = 0.0;
        for (int p = 0; p < 3; ++p)
          for (int q = 0; q < 3; ++q) {
            double w = adet * K[p][a] * K[q][b];
            const double* R = &R2[p][q][0][0];
            for (int e = 0; e < 100; ++e) Dab[e] += w * R[e];
          }
      }
    double lam = coeff0[c], mu = coeff1[c];
    for (int i = 0; i < 10; ++i)
      for (int a = 0; a < 3; ++a)
        for (int j = 0; j < 10; ++j)
          for (int b = 0; b < 3; ++b) {
            int e = i * 10 + j;
            double S = (a == b) ? (D[0][0][e] + D[1][1][e] + D[2][2][e]) : 0.0;
            Ae[(3 * i + a) * 30 + 3 * j + b] = mu * (S + D[b][a][e]) + lam * D[a][b][e];
          }
  }
}

/* be has k0 entries */
static void tabulate_vec(int kind, const double* coords, const int32_t* v, int64_t c,
                         const double* f, double* be)
{
  double K[3][3], adet;
  cell_geom(coords, v, K, &adet);
  if (kind == 1) {
    double s = f[v[0]] + f[v[1]] + f[v[2]] + f[v[3]];
    for (int i = 0; i < 4; ++i) be[i] = adet / 120.0 * (f[v[i]] + s);
  } else if (kind == 2) {
    for (int i = 0; i < 10; ++i) be[i] = f[c] * adet * W2[i];
  } else if (kind == 4) {
    for (int i = 0; i < 20; ++i) be[i] = f[c] * adet * W3[i];
  } else {
    for (int i = 0; i < 10; ++i)
      for (int a = 0; a < 3; ++a) be[3 * i + a] = f[3 * c + a] * adet * W2[i];
  }
}

static inline int kdofs(int kind) { return kind == 1 ? 4 : (kind == 4 ? 20 : 10); }

/* ---------------- row-owning partition ---------------- */
typedef struct {
  int nthreads;
  int64_t* row_lo; /* block-row range [row_lo[t], row_lo[t+1]) */
  int64_t** cells; /* cells touching the range */
  int64_t* ncells;
} plan_t;

void* cfem_plan_create(int nthreads, const int32_t* dofs, int64_t ncells, int k, int64_t nblocks)
{
  plan_t* p = (plan_t*)calloc(1, sizeof(plan_t));
  p->nthreads = nthreads;
  p->row_lo = (int64_t*)malloc(sizeof(int64_t) * (nthreads + 1));
  for (int t = 0; t <= nthreads; ++t) p->row_lo[t] = nblocks * t / nthreads;
  p->cells = (int64_t**)calloc(nthreads, sizeof(int64_t*));
  p->ncells = (int64_t*)calloc(nthreads, sizeof(int64_t));
  int64_t* count = (int64_t*)calloc(nthreads, sizeof(int64_t));
  int* owner = (int*)malloc(sizeof(int) * (size_t)(nblocks > 0 ? nblocks : 1));
  for (int t = 0; t < nthreads; ++t)
    for (int64_t r = p->row_lo[t]; r < p->row_lo[t + 1]; ++r) owner[r] = t;
  char* seen = (char*)malloc(nthreads);
  for (int pass = 0; pass < 2; ++pass) {
    for (int t = 0; t < nthreads; ++t) {
      if (pass == 1) p->cells[t] = (int64_t*)malloc(sizeof(int64_t) * (count[t] ? count[t] : 1));
      count[t] = 0;
    }
    for (int64_t c = 0; c < ncells; ++c) {
      memset(seen, 0, nthreads);
      for (int i = 0; i < k; ++i) {
        int t = owner[dofs[c * k + i]];
        if (!seen[t]) {
          seen[t] = 1;
          if (pass == 1) p->cells[t][count[t]] = c;
          count[t]++;
        }
      }
    }
  }
  for (int t = 0; t < nthreads; ++t) p->ncells[t] = count[t];
  free(seen);
  free(owner);
  free(count);
  return p;
}

void cfem_plan_destroy(void* vp)
{
  plan_t* p = (plan_t*)vp;
  if (!p) return;
  for (int t = 0; t < p->nthreads; ++t) free(p->cells[t]);
  free(p->cells);
  free(p->ncells);
  free(p->row_lo);
  free(p);
}

int64_t cfem_plan_total_cells(void* vp)
{
  plan_t* p = (plan_t*)vp;
  int64_t s = 0;
  for (int t = 0; t < p->nthreads; ++t) s += p->ncells[t];
  return s;
}

/* ---------------- jobs ---------------- */
typedef struct {
  plan_t* plan;
  int t, kind, bs, op;
  const double *coords, *coeff0, *coeff1, *f, *g, *x0;
  const int32_t *cells, *dofs, *row_ptr, *col, *bc_dofs;
  const uint8_t* markers;
  double *values, *b;
  double diagonal, scale;
  int64_t n_bc;
  /* bound mode: accumulate the per-entry parity bound (fem_oracle.py
   * matrix_bound / vector_bound / lifting_bound) instead of the values */
  int bound;
  double rtol, frel;
} job_t;

static inline double absmax(const double* a, int n)
{
  double m = 0.0;
  for (int i = 0; i < n; ++i) m = fmax(m, fabs(a[i]));
  return m;
}

static inline int64_t find_col(const int32_t* row_ptr, const int32_t* col, int64_t row, int32_t c)
{
  int64_t lo = row_ptr[row], hi = row_ptr[row + 1];
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (col[mid] < c) lo = mid + 1;
    else hi = mid;
  }
  return (lo < row_ptr[row + 1] && col[lo] == c) ? lo : -1;
}

static void* run_job(void* arg)
{
  job_t* J = (job_t*)arg;
  plan_t* P = J->plan;
  const int k = kdofs(J->kind), bs = J->bs, ks = k * bs;
  const int64_t rlo = P->row_lo[J->t] * bs, rhi = P->row_lo[J->t + 1] * bs;
  double Ae[900], be[30];
  int64_t rows[30];
  int32_t colsx[30];
  const int64_t* my = P->cells[J->t];
  const int64_t nmy = P->ncells[J->t];
  if (J->op == 0) { /* matrix */
    for (int64_t r = rlo; r < rhi; ++r)
      for (int64_t s = J->row_ptr[r]; s < J->row_ptr[r + 1]; ++s) J->values[s] = 0.0;
    for (int64_t q = 0; q < nmy; ++q) {
      int64_t c = my[q];
      tabulate(J->kind, J->coords, J->cells + 4 * c, c, J->coeff0, J->coeff1, Ae);
      for (int i = 0; i < k; ++i)
        for (int a = 0; a < bs; ++a) {
          rows[i * bs + a] = (int64_t)J->dofs[c * k + i] * bs + a;
          colsx[i * bs + a] = J->dofs[c * k + i] * bs + a;
        }
      if (J->bound) {
        const double f = J->frel * absmax(Ae, ks * ks);
        for (int e = 0; e < ks * ks; ++e) Ae[e] = J->rtol * fabs(Ae[e]) + f;
      }
      for (int ii = 0; ii < ks; ++ii) {
        int64_t r = rows[ii];
        if (r < rlo || r >= rhi || J->markers[r]) continue;
        for (int jj = 0; jj < ks; ++jj) {
          if (J->markers[colsx[jj]]) continue;
          int64_t s = find_col(J->row_ptr, J->col, r, colsx[jj]);
          if (s >= 0) J->values[s] += Ae[ii * ks + jj];
        }
      }
    }
    /* the diagonal of BC rows is written, not summed: bound 0 */
    if (!J->bound)
      for (int64_t q = 0; q < J->n_bc; ++q) {
        int64_t r = J->bc_dofs[q];
        if (r < rlo || r >= rhi) continue;
        int64_t s = find_col(J->row_ptr, J->col, r, (int32_t)r);
        if (s >= 0) J->values[s] = J->diagonal;
      }
  } else if (J->op == 1) { /* vector */
    for (int64_t r = rlo; r < rhi; ++r) J->b[r] = 0.0;
    for (int64_t q = 0; q < nmy; ++q) {
      int64_t c = my[q];
      tabulate_vec(J->kind, J->coords, J->cells + 4 * c, c, J->f, be);
      if (J->bound) {
        const double f = J->frel * absmax(be, ks);
        for (int e = 0; e < ks; ++e) be[e] = J->rtol * fabs(be[e]) + f;
      }
      for (int i = 0; i < k; ++i)
        for (int a = 0; a < bs; ++a) {
          int64_t r = (int64_t)J->dofs[c * k + i] * bs + a;
          if (r >= rlo && r < rhi) J->b[r] += be[i * bs + a];
        }
    }
  } else { /* lifting */
    for (int64_t q = 0; q < nmy; ++q) {
      int64_t c = my[q];
      int any = 0;
      for (int i = 0; i < k && !any; ++i)
        for (int a = 0; a < bs; ++a)
          if (J->markers[(int64_t)J->dofs[c * k + i] * bs + a]) any = 1;
      if (!any) continue;
      tabulate(J->kind, J->coords, J->cells + 4 * c, c, J->coeff0, J->coeff1, Ae);
      double d[30];
      for (int j = 0; j < k; ++j)
        for (int b = 0; b < bs; ++b) {
          int64_t cc = (int64_t)J->dofs[c * k + j] * bs + b;
          d[j * bs + b] = J->markers[cc] ? (J->g[cc] - (J->x0 ? J->x0[cc] : 0.0)) : 0.0;
        }
      double fl = 0.0;
      if (J->bound) {
        double dsum = 0.0;
        for (int jj = 0; jj < ks; ++jj) {
          d[jj] = fabs(d[jj]);
          dsum += d[jj];
        }
        fl = J->frel * absmax(Ae, ks * ks) * dsum;
      }
      for (int ii = 0; ii < ks; ++ii) {
        int64_t r = (int64_t)J->dofs[c * k + ii / bs] * bs + ii % bs;
        if (r < rlo || r >= rhi) continue;
        double s = 0.0;
        if (J->bound) {
          for (int jj = 0; jj < ks; ++jj) s += fabs(Ae[ii * ks + jj]) * d[jj];
          J->b[r] += fabs(J->scale) * (J->rtol * s + fl);
        } else {
          for (int jj = 0; jj < ks; ++jj) s += Ae[ii * ks + jj] * d[jj];
          J->b[r] -= J->scale * s;
        }
      }
    }
  }
  return NULL;
}

static void run_all(job_t* proto)
{
  plan_t* P = proto->plan;
  int T = P->nthreads;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * T);
  job_t* jobs = (job_t*)malloc(sizeof(job_t) * T);
  for (int t = 0; t < T; ++t) {
    jobs[t] = *proto;
    jobs[t].t = t;
    pthread_create(&th[t], NULL, run_job, &jobs[t]);
  }
  for (int t = 0; t < T; ++t) pthread_join(th[t], NULL);
  free(jobs);
  free(th);
}

void cfem_assemble_matrix(void* plan, int kind, const double* coords, const int32_t* cells,
                          const int32_t* dofs, int bs, const double* coeff0, const double* coeff1,
                          const int32_t* row_ptr, const int32_t* col, const uint8_t* markers,
                          double* values, double diagonal, const int32_t* bc_dofs, int64_t n_bc)
{
  job_t J;
  memset(&J, 0, sizeof(J));
  J.plan = (plan_t*)plan;
  J.kind = kind;
  J.bs = bs;
  J.op = 0;
  J.coords = coords;
  J.cells = cells;
  J.dofs = dofs;
  J.coeff0 = coeff0;
  J.coeff1 = coeff1;
  J.row_ptr = row_ptr;
  J.col = col;
  J.markers = markers;
  J.values = values;
  J.diagonal = diagonal;
  J.bc_dofs = bc_dofs;
  J.n_bc = n_bc;
  run_all(&J);
}

void cfem_assemble_vector(void* plan, int kind, const double* coords, const int32_t* cells,
                          const int32_t* dofs, int bs, const double* f, double* b)
{
  job_t J;
  memset(&J, 0, sizeof(J));
  J.plan = (plan_t*)plan;
  J.kind = kind;
  J.bs = bs;
  J.op = 1;
  J.coords = coords;
  J.cells = cells;
  J.dofs = dofs;
  J.f = f;
  J.b = b;
  run_all(&J);
}

void cfem_apply_lifting(void* plan, int kind, const double* coords, const int32_t* cells,
                        const int32_t* dofs, int bs, const double* coeff0, const double* coeff1,
                        const uint8_t* markers, const double* g, const double* x0, double scale,
                        double* b)
{
  job_t J;
  memset(&J, 0, sizeof(J));
  J.plan = (plan_t*)plan;
  J.kind = kind;
  J.bs = bs;
  J.op = 2;
  J.coords = coords;
  J.cells = cells;
  J.dofs = dofs;
  J.coeff0 = coeff0;
  J.coeff1 = coeff1;
  J.markers = markers;
  J.g = g;
  J.x0 = x0;
  J.scale = scale;
  J.b = b;
  run_all(&J);
}

/* Parity bounds of cfem_assemble_matrix and of cfem_assemble_vector +
 * cfem_apply_lifting (per entry: rtol * sum |contributions| + frel * the
 * largest |entry| of each contributing element; fem_oracle.py matrix_bound,
 * vector_bound, lifting_bound); bound[] is overwritten, the set_bc rows are
 * left to the caller (their bound is 0). */
void cfem_matrix_bound(void* plan, int kind, const double* coords, const int32_t* cells, const int32_t* dofs,
                       int bs, const double* coeff0, const double* coeff1, const int32_t* row_ptr,
                       const int32_t* col, const uint8_t* markers, double* bound, double rtol, double frel)
{
  job_t J;
  memset(&J, 0, sizeof(J));
  J.plan = (plan_t*)plan;
  J.kind = kind;
  J.bs = bs;
  J.op = 0;
  J.coords = coords;
  J.cells = cells;
  J.dofs = dofs;
  J.coeff0 = coeff0;
  J.coeff1 = coeff1;
  J.row_ptr = row_ptr;
  J.col = col;
  J.markers = markers;
  J.values = bound;
  J.bound = 1;
  J.rtol = rtol;
  J.frel = frel;
  run_all(&J);
}

void cfem_rhs_bound(void* plan, int kind, const double* coords, const int32_t* cells, const int32_t* dofs, int bs,
                    const double* f, const double* coeff0, const double* coeff1, const uint8_t* markers,
                    const double* g, const double* x0, double scale, double* bound, double rtol, double frel)
{
  job_t J;
  memset(&J, 0, sizeof(J));
  J.plan = (plan_t*)plan;
  J.kind = kind;
  J.bs = bs;
  J.coords = coords;
  J.cells = cells;
  J.dofs = dofs;
  J.f = f;
  J.b = bound;
  J.bound = 1;
  J.rtol = rtol;
  J.frel = frel;
  J.op = 1; /* zeroes the thread's rows, then the load vector's bound */
  run_all(&J);
  J.op = 2;
  J.coeff0 = coeff0;
  J.coeff1 = coeff1;
  J.markers = markers;
  J.g = g;
  J.x0 = x0;
  J.scale = scale;
  run_all(&J);
}

/* ---------------- sparsity ----------------
 * DOLFINx's SparsityPattern of a cell integral (sorted unique block columns
 * of every block row) unrolled to scalar AIJ as cpp/cudolfinx/la/petsc.cpp:45-65
 * does: row bs*R+a holds bs*C+b for each block column C, b = 0..bs-1.  Each
 * thread builds the block rows it owns from the cells touching them. */
typedef struct {
  plan_t* plan;
  int t, k, bs;
  const int32_t* dofs;
  int64_t* blen;      /* [nblocks] block columns per block row */
  int32_t** bcols;    /* per thread: its rows' sorted block columns, concatenated */
  const int32_t* row_ptr;
  int32_t* col;
} pat_job_t;

static void* pattern_job(void* arg)
{
  pat_job_t* J = (pat_job_t*)arg;
  plan_t* P = J->plan;
  const int k = J->k;
  const int64_t lo = P->row_lo[J->t], hi = P->row_lo[J->t + 1], nr = hi - lo;
  const int64_t* my = P->cells[J->t];
  const int64_t nmy = P->ncells[J->t];
  if (J->col == NULL) {
    /* couplings per owned row, then the sorted unique block columns */
    int64_t* start = (int64_t*)calloc((size_t)nr + 1, sizeof(int64_t));
    for (int64_t q = 0; q < nmy; ++q)
      for (int i = 0; i < k; ++i) {
        int64_t R = J->dofs[my[q] * k + i];
        if (R >= lo && R < hi) start[R - lo + 1] += k;
      }
    for (int64_t r = 0; r < nr; ++r) start[r + 1] += start[r];
    int32_t* buf = (int32_t*)malloc(sizeof(int32_t) * (size_t)(start[nr] ? start[nr] : 1));
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nr ? nr : 1));
    for (int64_t r = 0; r < nr; ++r) fill[r] = start[r];
    for (int64_t q = 0; q < nmy; ++q) {
      const int32_t* cd = J->dofs + my[q] * k;
      for (int i = 0; i < k; ++i) {
        int64_t R = cd[i];
        if (R < lo || R >= hi) continue;
        for (int j = 0; j < k; ++j) buf[fill[R - lo]++] = cd[j];
      }
    }
    /* in place: sort each row's list (insertion sort, rows are short), drop repeats */
    int64_t out = 0;
    for (int64_t r = 0; r < nr; ++r) {
      int32_t* a = buf + start[r];
      int64_t n = start[r + 1] - start[r];
      for (int64_t i = 1; i < n; ++i) {
        int32_t v = a[i];
        int64_t j = i - 1;
        while (j >= 0 && a[j] > v) {
          a[j + 1] = a[j];
          --j;
        }
        a[j + 1] = v;
      }
      int64_t m = 0;
      for (int64_t i = 0; i < n; ++i)
        if (m == 0 || buf[out + m - 1] != a[i]) {
          buf[out + m] = a[i];
          ++m;
        }
      J->blen[lo + r] = m;
      out += m;
    }
    J->bcols[J->t] = buf;
    free(fill);
    free(start);
  } else {
    const int bs = J->bs;
    const int32_t* bc = J->bcols[J->t];
    for (int64_t R = lo; R < hi; ++R) {
      const int64_t m = J->blen[R];
      for (int a = 0; a < bs; ++a) {
        int32_t* dst = J->col + J->row_ptr[R * bs + a];
        for (int64_t u = 0; u < m; ++u)
          for (int b = 0; b < bs; ++b) dst[u * bs + b] = bc[u] * bs + b;
      }
      bc += m;
    }
  }
  return NULL;
}

static void run_pattern(pat_job_t* proto)
{
  int T = proto->plan->nthreads;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * T);
  pat_job_t* jobs = (pat_job_t*)malloc(sizeof(pat_job_t) * T);
  for (int t = 0; t < T; ++t) {
    jobs[t] = *proto;
    jobs[t].t = t;
    pthread_create(&th[t], NULL, pattern_job, &jobs[t]);
  }
  for (int t = 0; t < T; ++t) pthread_join(th[t], NULL);
  free(jobs);
  free(th);
}

/* Returns nnz and malloc'd row_ptr [nblocks*bs+1] / col [nnz] (release with
 * cfem_free), or -1 if nnz does not fit int32 indices. */
int64_t cfem_pattern_build(void* plan, const int32_t* dofs, int k, int bs, int64_t nblocks, int32_t** row_ptr,
                           int32_t** col)
{
  plan_t* P = (plan_t*)plan;
  pat_job_t J;
  memset(&J, 0, sizeof(J));
  J.plan = P;
  J.k = k;
  J.bs = bs;
  J.dofs = dofs;
  J.blen = (int64_t*)calloc((size_t)(nblocks ? nblocks : 1), sizeof(int64_t));
  J.bcols = (int32_t**)calloc(P->nthreads, sizeof(int32_t*));
  run_pattern(&J);
  const int64_t nrows = nblocks * bs;
  int32_t* rp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nrows + 1));
  int64_t acc = 0;
  rp[0] = 0;
  for (int64_t R = 0; R < nblocks; ++R)
    for (int a = 0; a < bs; ++a) {
      acc += J.blen[R] * bs;
      if (acc > 2147483647) {
        for (int t = 0; t < P->nthreads; ++t) free(J.bcols[t]);
        free(J.bcols);
        free(J.blen);
        free(rp);
        return -1;
      }
      rp[R * bs + a + 1] = (int32_t)acc;
    }
  int32_t* cl = (int32_t*)malloc(sizeof(int32_t) * (size_t)(acc ? acc : 1));
  J.row_ptr = rp;
  J.col = cl;
  run_pattern(&J);
  for (int t = 0; t < P->nthreads; ++t) free(J.bcols[t]);
  free(J.bcols);
  free(J.blen);
  *row_ptr = rp;
  *col = cl;
  return acc;
}

void cfem_free(void* p) { free(p); }

void cfem_set_bc(double* b, const int32_t* bc_dofs, int64_t n_bc, const double* g,
                 const double* x0, double scale)
{
  for (int64_t q = 0; q < n_bc; ++q) {
    int64_t d = bc_dofs[q];
    b[d] = scale * (g[d] - (x0 ? x0[d] : 0.0));
  }
}
