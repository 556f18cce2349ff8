// ksp_cpu.cc — TEST INFRASTRUCTURE ONLY (CPU oracle / CPU baseline, never the product).
//
// A CPU restatement of the linear solver the reference's SSAFD uses by default:
// PETSc KSPGMRES (restart 30, classical Gram-Schmidt without refinement, left
// preconditioning, preconditioned residual norm) with PCBJACOBI and ILU(0) on
// every block (src/base/stressbalance/ssa/SSAFD.cc:136-161, 1018; the defaults
// are PETSc's, as SSAFD.cc:826-828 notes).  PETSc itself is a third-party
// dependency that is not part of the reference tree ("PETSc 3.5 or later",
// INSTALL.md:21-23, version unpinned); this file restates its published
// algorithms:
//   * ILU(0): incomplete LU on the matrix's own sparsity pattern (explicit zeros
//     included, as a DMDA-preallocated AIJ matrix keeps them), natural ordering;
//   * block Jacobi: one block per MPI rank = a contiguous range of rows in
//     PETSc's rank-major ordering; off-block couplings are dropped;
//   * GMRES(m): Arnoldi with classical Gram-Schmidt, Givens rotations, the
//     residual estimate |g_{k+1}| tested against max(rtol*||B b||, abstol)
//     (KSPConvergedDefault with a nonzero initial guess, SSAFD.cc:124-127).
//
// The blocks run on OpenMP threads, one block per thread, the way
// `mpiexec -n P` runs one block per rank.
//
// C ABI (ctypes):  ksp_gmres_bjacobi_ilu0(...) and ilu0_blocks_apply(...).

#include <cmath>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

struct CSR {
  int n;
  const int *rowptr, *col;
  const double *val;
};

// ILU(0) factors of the diagonal blocks, stored on the block's own pattern.
struct ILU0 {
  int n;
  std::vector<int> rowptr, col, diag;  // diag[i] = position of (i,i)
  std::vector<double> val;
  std::vector<int> block_start;        // nblocks + 1
};

bool build_ilu0(const CSR &A, const int *block_start, int nblocks, ILU0 &F) {
  F.n = A.n;
  F.block_start.assign(block_start, block_start + nblocks + 1);
  F.rowptr.assign(A.n + 1, 0);
  // keep only entries inside the row's block, columns ascending (CSR input is sorted)
  std::vector<int> blk_of_row(A.n);
  for (int b = 0; b < nblocks; ++b)
    for (int i = block_start[b]; i < block_start[b + 1]; ++i) blk_of_row[i] = b;
  for (int i = 0; i < A.n; ++i) {
    int b = blk_of_row[i], lo = block_start[b], hi = block_start[b + 1], cnt = 0;
    for (int p = A.rowptr[i]; p < A.rowptr[i + 1]; ++p)
      if (A.col[p] >= lo && A.col[p] < hi) ++cnt;
    F.rowptr[i + 1] = F.rowptr[i] + cnt;
  }
  F.col.resize(F.rowptr[A.n]);
  F.val.resize(F.rowptr[A.n]);
  F.diag.assign(A.n, -1);
  for (int i = 0; i < A.n; ++i) {
    int b = blk_of_row[i], lo = block_start[b], hi = block_start[b + 1], q = F.rowptr[i];
    for (int p = A.rowptr[i]; p < A.rowptr[i + 1]; ++p)
      if (A.col[p] >= lo && A.col[p] < hi) {
        F.col[q] = A.col[p];
        F.val[q] = A.val[p];
        if (A.col[p] == i) F.diag[i] = q;
        ++q;
      }
    if (F.diag[i] < 0) return false;
  }
  bool ok = true;
#pragma omp parallel for schedule(static, 1) reduction(&& : ok)
  for (int b = 0; b < nblocks; ++b) {
    std::vector<int> pos(A.n, -1);  // scratch: column -> position in current row
    for (int i = block_start[b]; i < block_start[b + 1]; ++i) {
      for (int p = F.rowptr[i]; p < F.rowptr[i + 1]; ++p) pos[F.col[p]] = p;
      // IKJ: for each k < i in row i's pattern, in ascending order
      for (int p = F.rowptr[i]; p < F.rowptr[i + 1] && F.col[p] < i; ++p) {
        int k = F.col[p];
        double piv = F.val[F.diag[k]];
        if (piv == 0.0) { ok = false; break; }
        double lik = F.val[p] / piv;
        F.val[p] = lik;
        for (int r = F.diag[k] + 1; r < F.rowptr[k + 1]; ++r) {
          int c = F.col[r];
          int t = pos[c];
          if (t >= 0) F.val[t] -= lik * F.val[r];
        }
      }
      for (int p = F.rowptr[i]; p < F.rowptr[i + 1]; ++p) pos[F.col[p]] = -1;
    }
  }
  return ok;
}

// z = (LU)^{-1} r block by block
void ilu0_solve(const ILU0 &F, const double *r, double *z) {
  int nb = (int)F.block_start.size() - 1;
#pragma omp parallel for schedule(static, 1)
  for (int b = 0; b < nb; ++b) {
    int lo = F.block_start[b], hi = F.block_start[b + 1];
    for (int i = lo; i < hi; ++i) {
      double s = r[i];
      for (int p = F.rowptr[i]; p < F.diag[i]; ++p) s -= F.val[p] * z[F.col[p]];
      z[i] = s;
    }
    for (int i = hi - 1; i >= lo; --i) {
      double s = z[i];
      for (int p = F.diag[i] + 1; p < F.rowptr[i + 1]; ++p) s -= F.val[p] * z[F.col[p]];
      z[i] = s / F.val[F.diag[i]];
    }
  }
}

void matvec(const CSR &A, const double *x, double *y) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A.n; ++i) {
    double s = 0.0;
    for (int p = A.rowptr[i]; p < A.rowptr[i + 1]; ++p) s += A.val[p] * x[A.col[p]];
    y[i] = s;
  }
}

double dot(int n, const double *a, const double *b) {
  double s = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : s)
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

}  // namespace

extern "C" {

// Returns 0 converged, -3 max iterations (KSP_DIVERGED_ITS), -4 DTOL, -5 breakdown/NaN,
// -9 ILU zero pivot.  *its = iterations, *rnorm = final residual estimate,
// *rnorm0 = ||B b||.
int ksp_gmres_bjacobi_ilu0(int n, const int *rowptr, const int *col, const double *val,
                           int nblocks, const int *block_start, const double *b, double *x,
                           double rtol, double abstol, double dtol, int maxit, int restart,
                           int nthreads, int *its, double *rnorm_out, double *rnorm0_out) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  CSR A{n, rowptr, col, val};
  ILU0 F;
  if (!build_ilu0(A, block_start, nblocks, F)) return -9;
  const int m = restart;
  std::vector<double> V((size_t)(m + 1) * n), H((size_t)(m + 1) * m, 0.0), g(m + 1), cs(m), sn(m),
      w(n), t(n), y(m);
  // rnorm0 = ||B b|| (KSPConvergedDefault, nonzero initial guess, left PC)
  ilu0_solve(F, b, t.data());
  double bnorm = std::sqrt(dot(n, t.data(), t.data()));
  int it_total = 0;
  double ttol = 0.0, rnorm = 0.0, rnorm0 = 0.0;
  bool first = true;
  int reason = 0;
  while (true) {
    // r = B (b - A x)
    matvec(A, x, w.data());
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) w[i] = b[i] - w[i];
    ilu0_solve(F, w.data(), V.data());
    double beta = std::sqrt(dot(n, V.data(), V.data()));
    if (first) {
      rnorm0 = (bnorm != 0.0) ? bnorm : beta;
      ttol = std::fmax(rtol * rnorm0, abstol);
      first = false;
      if (beta < ttol) { rnorm = beta; reason = 0; break; }   // converged at iteration 0
    }
    if (!std::isfinite(beta)) { reason = -5; break; }
    if (beta == 0.0) { rnorm = 0.0; reason = 0; break; }
    double inv = 1.0 / beta;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) V[i] *= inv;
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = beta;
    int k = 0;
    bool done = false;
    for (; k < m && it_total < maxit; ++k) {
      double *vk = &V[(size_t)k * n], *vk1 = &V[(size_t)(k + 1) * n];
      matvec(A, vk, t.data());
      ilu0_solve(F, t.data(), vk1);
      // classical Gram-Schmidt: all dots against the same vector, then one update
      for (int j = 0; j <= k; ++j) H[(size_t)j * m + k] = dot(n, vk1, &V[(size_t)j * n]);
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; ++i) {
        double s = vk1[i];
        for (int j = 0; j <= k; ++j) s -= H[(size_t)j * m + k] * V[(size_t)j * n + i];
        vk1[i] = s;
      }
      double hn = std::sqrt(dot(n, vk1, vk1));
      H[(size_t)(k + 1) * m + k] = hn;
      // apply previous rotations
      for (int j = 0; j < k; ++j) {
        double a = H[(size_t)j * m + k], c = H[(size_t)(j + 1) * m + k];
        H[(size_t)j * m + k] = cs[j] * a + sn[j] * c;
        H[(size_t)(j + 1) * m + k] = -sn[j] * a + cs[j] * c;
      }
      double a = H[(size_t)k * m + k], c = H[(size_t)(k + 1) * m + k];
      double den = std::sqrt(a * a + c * c);
      if (den == 0.0) { reason = -5; done = true; break; }
      cs[k] = a / den;
      sn[k] = c / den;
      H[(size_t)k * m + k] = den;
      H[(size_t)(k + 1) * m + k] = 0.0;
      g[k + 1] = -sn[k] * g[k];
      g[k] = cs[k] * g[k];
      rnorm = std::fabs(g[k + 1]);
      ++it_total;
      if (!std::isfinite(rnorm)) { reason = -5; done = true; break; }
      if (rnorm < ttol) { reason = 0; done = true; ++k; break; }
      if (rnorm > dtol * rnorm0) { reason = -4; done = true; ++k; break; }
      if (hn == 0.0) { reason = 0; done = true; ++k; break; }   // happy breakdown
      double hinv = 1.0 / hn;
#pragma omp parallel for schedule(static)
      for (int i = 0; i < n; ++i) vk1[i] *= hinv;
    }
    // x += V y, H y = g (upper triangular, size k)
    for (int i = k - 1; i >= 0; --i) {
      double s = g[i];
      for (int j = i + 1; j < k; ++j) s -= H[(size_t)i * m + j] * y[j];
      y[i] = s / H[(size_t)i * m + i];
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int j = 0; j < k; ++j) s += y[j] * V[(size_t)j * n + i];
      x[i] += s;
    }
    if (done) break;
    if (it_total >= maxit) { reason = -3; break; }
  }
  *its = it_total;
  *rnorm_out = rnorm;
  *rnorm0_out = rnorm0;
  return reason;
}

// z = B r with B the block-Jacobi ILU(0) preconditioner (for checking).
int ilu0_blocks_apply(int n, const int *rowptr, const int *col, const double *val, int nblocks,
                      const int *block_start, const double *r, double *z) {
  CSR A{n, rowptr, col, val};
  ILU0 F;
  if (!build_ilu0(A, block_start, nblocks, F)) return -9;
  ilu0_solve(F, r, z);
  return 0;
}
}
