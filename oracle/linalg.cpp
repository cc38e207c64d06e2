// Oracle (test infrastructure): dense linear algebra for the CPU restatement.
//
// The reference diagonalises with faer 0.24.4 `self_adjoint_eigen` (src/linalg.rs:231-278),
// a third-party crate whose source is not part of pm7-rs. Converged SCF observables depend
// only on the occupied subspace, so any correct symmetric eigensolver reproduces them. This
// file uses LAPACK dsyevd from the OpenBLAS that ships inside numpy when it has been
// registered with pm7_oracle_set_lapack(), and a cyclic Jacobi solver otherwise.
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "oracle_internal.hpp"

namespace oracle {
namespace {

// ILP64 Fortran LAPACK/BLAS entry points of numpy's bundled OpenBLAS.
typedef void (*dsyevd_fn)(const char *, const char *, const int64_t *, double *, const int64_t *, double *,
                          double *, const int64_t *, int64_t *, const int64_t *, int64_t *, size_t, size_t);
typedef void (*dgemm_fn)(const char *, const char *, const int64_t *, const int64_t *, const int64_t *,
                         const double *, const double *, const int64_t *, const double *, const int64_t *,
                         const double *, double *, const int64_t *, size_t, size_t);
typedef void (*setthreads_fn)(int64_t);

dsyevd_fn g_dsyevd = nullptr;
dgemm_fn g_dgemm = nullptr;

// Cyclic Jacobi eigensolver (fallback), vectors as rows of vt.
void jacobi_eigen(const Mat &a, std::vector<double> &eval, std::vector<double> &vt) {
  int n = a.n;
  std::vector<double> m(a.a);
  vt.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) vt[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) off += m[(size_t)i * n + j] * m[(size_t)i * n + j];
    if (off < 1e-30) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = m[(size_t)p * n + q];
        if (std::fabs(apq) < 1e-300) continue;
        double app = m[(size_t)p * n + p], aqq = m[(size_t)q * n + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double mkp = m[(size_t)k * n + p], mkq = m[(size_t)k * n + q];
          m[(size_t)k * n + p] = c * mkp - s * mkq;
          m[(size_t)k * n + q] = s * mkp + c * mkq;
        }
        for (int k = 0; k < n; ++k) {
          double mpk = m[(size_t)p * n + k], mqk = m[(size_t)q * n + k];
          m[(size_t)p * n + k] = c * mpk - s * mqk;
          m[(size_t)q * n + k] = s * mpk + c * mqk;
        }
        for (int k = 0; k < n; ++k) {
          double vp = vt[(size_t)p * n + k], vq = vt[(size_t)q * n + k];
          vt[(size_t)p * n + k] = c * vp - s * vq;
          vt[(size_t)q * n + k] = s * vp + c * vq;
        }
      }
  }
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return m[(size_t)x * n + x] < m[(size_t)y * n + y]; });
  eval.resize(n);
  std::vector<double> sorted((size_t)n * n);
  for (int k = 0; k < n; ++k) {
    eval[k] = m[(size_t)order[k] * n + order[k]];
    std::memcpy(&sorted[(size_t)k * n], &vt[(size_t)order[k] * n], sizeof(double) * n);
  }
  vt.swap(sorted);
}

}  // namespace

bool set_lapack(const char *path, int threads) {
  void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return false;
  g_dsyevd = (dsyevd_fn)dlsym(h, "scipy_dsyevd_64_");
  g_dgemm = (dgemm_fn)dlsym(h, "scipy_dgemm_64_");
  auto st = (setthreads_fn)dlsym(h, "scipy_openblas_set_num_threads64_");
  if (st && threads > 0) st(threads);
  return g_dsyevd != nullptr;
}

void symmetric_eigen(const Mat &a, std::vector<double> &eval, std::vector<double> &vt) {
  int n = a.n;
  if (n == 0) {
    eval.clear();
    vt.clear();
    return;
  }
  if (!g_dsyevd) {
    jacobi_eigen(a, eval, vt);
    return;
  }
  // Row-major symmetric == column-major symmetric; eigenvectors come back as columns of
  // a column-major matrix, i.e. as contiguous rows of vt.
  vt = a.a;
  eval.assign(n, 0.0);
  int64_t nn = n, lwork = -1, liwork = -1, info = 0, iwq = 0;
  double wq = 0;
  g_dsyevd("V", "L", &nn, vt.data(), &nn, eval.data(), &wq, &lwork, &iwq, &liwork, &info, 1, 1);
  lwork = (int64_t)wq;
  liwork = iwq;
  std::vector<double> work(std::max<int64_t>(lwork, 1));
  std::vector<int64_t> iwork(std::max<int64_t>(liwork, 1));
  g_dsyevd("V", "L", &nn, vt.data(), &nn, eval.data(), work.data(), &lwork, iwork.data(), &liwork, &info, 1, 1);
  if (info != 0) throw Error(PM7_ERR_LINEAR_ALGEBRA, "dsyevd failed, info=" + std::to_string(info));
}

void matmul(const Mat &a, const Mat &b, Mat &c) {
  int n = a.n;
  c = Mat(n);
  if (g_dgemm) {
    // Row-major C = A B  <=>  column-major C^T = B^T A^T.
    int64_t nn = n;
    double one = 1.0, zero = 0.0;
    g_dgemm("N", "N", &nn, &nn, &nn, &one, b.a.data(), &nn, a.a.data(), &nn, &zero, c.a.data(), &nn, 1, 1);
    return;
  }
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    double *ci = &c.a[(size_t)i * n];
    for (int k = 0; k < n; ++k) {
      double aik = a.a[(size_t)i * n + k];
      const double *bk = &b.a[(size_t)k * n];
      for (int j = 0; j < n; ++j) ci[j] += aik * bk[j];
    }
  }
}

void density_from_vectors(const std::vector<double> &vt, int n, int n_occ, double w, Mat &p) {
  p = Mat(n);
  if (n == 0) return;
  if (g_dgemm && n_occ > 0) {
    // vt rows 0..n_occ are the occupied vectors: column-major n x n_occ matrix V.
    // Row-major P = w V V^T is symmetric, so compute column-major P = w V V^T.
    int64_t nn = n, k = n_occ;
    double zero = 0.0;
    g_dgemm("N", "T", &nn, &nn, &k, &w, vt.data(), &nn, vt.data(), &nn, &zero, p.a.data(), &nn, 1, 1);
    return;
  }
#pragma omp parallel for schedule(static)
  for (int mu = 0; mu < n; ++mu)
    for (int nu = 0; nu < n; ++nu) {
      double dot = 0.0;
      for (int k = 0; k < n_occ; ++k) dot += vt[(size_t)k * n + mu] * vt[(size_t)k * n + nu];
      p.a[(size_t)mu * n + nu] = w * dot;
    }
}

}  // namespace oracle
