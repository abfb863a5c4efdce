// Drop-in coding entry points of decomp/decomp.h, running on the B200 engine
// through the C ABI of spams_b200.h.
//
//   omp<T>     decomp/decomp.h:53-57 (declaration), :322-404 (driver)
//   lasso2<T>  decomp/decomp.h:126-135, :1563-1646
//   lasso<T>   decomp/decomp.h:111-116, :735-841 (Cholesky / ols variant)
//
// Same argument meaning: L / eps / lambda pointers with the vec* flags, the
// constraint modes of constraint_type, pos, the optional regularisation path
// of the first signal.  numThreads is accepted and ignored.  Engine failures
// (no CUDA device, out of memory) are thrown as const char* messages, like the
// reference facade's errors.
#ifndef SPAMS_B200_DECOMP_H
#define SPAMS_B200_DECOMP_H

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../spams_b200.h"
#include "linalg.h"

// decomp/decomp.h:95
enum constraint_type { L1COEFFS, L2ERROR, PENALTY, SPARSITY, L2ERROR2, PENALTY2, FISTAMODE };

namespace spams_b200_detail {

inline sc_status call_omp(const float* X, int m, int64_t n, const float* D, int K, const int* L,
                          int64_t nL, const float* e, int64_t nE, const float* la, int64_t nLa,
                          float* path, sc_csc_f32* out) {
  return sc_omp_f32(X, m, n, D, K, L, nL, e, nE, la, nLa, -1, path, nullptr, out);
}
inline sc_status call_omp(const double* X, int m, int64_t n, const double* D, int K, const int* L,
                          int64_t nL, const double* e, int64_t nE, const double* la, int64_t nLa,
                          double* path, sc_csc_f64* out) {
  return sc_omp_f64(X, m, n, D, K, L, nL, e, nE, la, nLa, -1, path, nullptr, out);
}
inline sc_status call_lasso(const float* X, int m, int64_t n, const float* D, int K, int L,
                            float l1, float l2, int mode, int pos, int mlp, float* path,
                            sc_csc_f32* out, int ols = 0, int cholesky = 0) {
  return sc_lasso_f32(X, m, n, D, K, L, l1, l2, mode, pos, ols, -1, mlp, cholesky, path, nullptr,
                      out);
}
inline sc_status call_lasso(const double* X, int m, int64_t n, const double* D, int K, int L,
                            double l1, double l2, int mode, int pos, int mlp, double* path,
                            sc_csc_f64* out, int ols = 0, int cholesky = 0) {
  return sc_lasso_f64(X, m, n, D, K, L, l1, l2, mode, pos, ols, -1, mlp, cholesky, path, nullptr,
                      out);
}
inline sc_status call_lassoQq(const float* X, int m, int64_t n, const float* Q, int K,
                              const float* q, int L, float l1, float l2, int mode, int pos,
                              int mlp, float* path, sc_csc_f32* out, int ols = 0,
                              int cholesky = 0) {
  if (ols || cholesky)
    return sc_lasso_gram_chol_f32(X, m, n, Q, K, q, L, l1, l2, mode, pos, ols, cholesky, -1, mlp,
                                  path, nullptr, out);
  return sc_lasso_gram_f32(X, m, n, Q, K, q, L, l1, l2, mode, pos, -1, mlp, path, nullptr, out);
}
inline sc_status call_lassoQq(const double* X, int m, int64_t n, const double* Q, int K,
                              const double* q, int L, double l1, double l2, int mode, int pos,
                              int mlp, double* path, sc_csc_f64* out, int ols = 0,
                              int cholesky = 0) {
  if (ols || cholesky)
    return sc_lasso_gram_chol_f64(X, m, n, Q, K, q, L, l1, l2, mode, pos, ols, cholesky, -1, mlp,
                                  path, nullptr, out);
  return sc_lasso_gram_f64(X, m, n, Q, K, q, L, l1, l2, mode, pos, -1, mlp, path, nullptr, out);
}
inline sc_status call_omp_mask(const float* X, int m, int64_t n, const float* D, int K,
                               const bool* B, const int* L, int64_t nL, const float* e,
                               int64_t nE, const float* la, int64_t nLa, float* path,
                               sc_csc_f32* out) {
  return sc_omp_mask_f32(X, m, n, D, K, reinterpret_cast<const uint8_t*>(B), L, nL, e, nE, la,
                         nLa, -1, path, nullptr, out);
}
inline sc_status call_omp_mask(const double* X, int m, int64_t n, const double* D, int K,
                               const bool* B, const int* L, int64_t nL, const double* e,
                               int64_t nE, const double* la, int64_t nLa, double* path,
                               sc_csc_f64* out) {
  return sc_omp_mask_f64(X, m, n, D, K, reinterpret_cast<const uint8_t*>(B), L, nL, e, nE, la,
                         nLa, -1, path, nullptr, out);
}
inline sc_status call_lasso_mask(const float* X, int m, int64_t n, const float* D, int K,
                                 const bool* B, int L, float l1, float l2, int mode, int pos,
                                 sc_csc_f32* out) {
  return sc_lasso_mask_f32(X, m, n, D, K, reinterpret_cast<const uint8_t*>(B), L, l1, l2, mode,
                           pos, -1, nullptr, out);
}
inline sc_status call_lasso_mask(const double* X, int m, int64_t n, const double* D, int K,
                                 const bool* B, int L, double l1, double l2, int mode, int pos,
                                 sc_csc_f64* out) {
  return sc_lasso_mask_f64(X, m, n, D, K, reinterpret_cast<const uint8_t*>(B), L, l1, l2, mode,
                           pos, -1, nullptr, out);
}
inline void release(sc_csc_f32* a) { sc_csc_free_f32(a); }
inline void release(sc_csc_f64* a) { sc_csc_free_f64(a); }

template <typename T> struct Csc;
template <> struct Csc<float> { typedef sc_csc_f32 type; };
template <> struct Csc<double> { typedef sc_csc_f64 type; };

// Moves an engine CSC result into a SpMatrix<T> (SpMatrix::convert's output
// layout, linalg/linalg.h:4840-4861).
template <typename T>
void adopt(typename Csc<T>::type& c, SpMatrix<T>& sp) {
  sp.clear();
  if (c.colptr) {
    sp.resize((INTM)c.m, (INTM)c.n, (INTM)c.nnz);
    for (int64_t i = 0; i <= c.n; ++i) sp.pB()[i] = (INTM)c.colptr[i];
    for (int64_t i = 0; i < c.nnz; ++i) {
      sp.r()[i] = (INTM)c.rows[i];
      sp.v()[i] = c.vals[i];
    }
  }
  release(&c);
}

inline void check(sc_status st) {
  if (st != SC_OK) throw sc_last_error();
}

}  // namespace spams_b200_detail

// decomp/decomp.h:322-404
template <typename T>
void omp(const Matrix<T>& X, const Matrix<T>& D, SpMatrix<T>& spalpha, const int* L,
         const T* eps, const T* lambda, const bool vecL = false, const bool vecEps = false,
         const bool vecLambda = false, const int numThreads = -1, Matrix<T>* path = NULL) {
  (void)numThreads;
  namespace d = spams_b200_detail;
  const INTM m = X.m(), n = X.n(), K = D.n();
  const INTM pathL = std::min(m, K);
  std::vector<T> pbuf(path ? (size_t)K * pathL : 0);
  typename d::Csc<T>::type out;
  d::check(d::call_omp(X.X(), (int)m, n, D.X(), (int)K, L, vecL ? n : 1, eps, vecEps ? n : 1,
                       lambda, vecLambda ? n : 1, path ? pbuf.data() : nullptr, &out));
  d::adopt<T>(out, spalpha);
  if (path) {
    const size_t cols = std::min<size_t>((size_t)path->n(), (size_t)pathL);
    for (size_t c = 0; c < cols; ++c)
      memcpy(path->rawX() + c * path->m(), pbuf.data() + c * K, sizeof(T) * std::min<INTM>(K, path->m()));
  }
}

// decomp/decomp.h:1563-1571: G = D^T D + max(lambda2, 1e-10) I, then lasso2.
template <typename T>
void lasso2(const Matrix<T>& X, const Matrix<T>& D, SpMatrix<T>& spalpha, int L,
            const T constraint, const T lambda2 = 0, constraint_type mode = PENALTY,
            const bool pos = false, const int numThreads = -1, Matrix<T>* path = NULL,
            const int length_path = -1) {
  (void)numThreads;
  namespace d = spams_b200_detail;
  const INTM n = X.n(), K = D.n();
  // lasso2 passes length_path straight to coreLARS2, which replaces <= 1 by
  // 4 min(L, K) (decomp/decomp.h:1722)
  const int Lc = std::min<int>(L, (int)K);
  const int mlp = length_path <= 1 ? 4 * Lc : length_path;
  std::vector<T> pbuf(path ? (size_t)K * mlp : 0);
  typename d::Csc<T>::type out;
  d::check(d::call_lasso(X.X(), (int)X.m(), n, D.X(), (int)K, L, constraint, lambda2, (int)mode,
                         pos ? 1 : 0, mlp, path ? pbuf.data() : nullptr, &out));
  d::adopt<T>(out, spalpha);
  if (path) {
    const size_t cols = std::min<size_t>((size_t)path->n(), (size_t)mlp);
    for (size_t c = 0; c < cols; ++c)
      memcpy(path->rawX() + c * path->m(), pbuf.data() + c * K, sizeof(T) * std::min<INTM>(K, path->m()));
  }
}

// decomp/decomp.h:1574-1646 with precomputed G = Q (used as given) and
// DtX = q; X supplies ||x_i||^2.
template <typename T>
void lasso2(const Matrix<T>& X, const Matrix<T>& G, const Matrix<T>& DtX, SpMatrix<T>& spalpha,
            int L, const T constraint, constraint_type mode = PENALTY, const bool pos = false,
            const int numThreads = -1, Matrix<T>* path = NULL, const int length_path = -1) {
  (void)numThreads;
  namespace d = spams_b200_detail;
  const INTM n = X.n(), K = G.n();
  const int Lc = std::min<int>(L, (int)K);
  const int mlp = length_path <= 1 ? 4 * Lc : length_path;
  std::vector<T> pbuf(path ? (size_t)K * mlp : 0);
  typename d::Csc<T>::type out;
  d::check(d::call_lassoQq(X.X(), (int)X.m(), n, G.X(), (int)K, DtX.X(), L, constraint, T(0),
                           (int)mode, pos ? 1 : 0, mlp, path ? pbuf.data() : nullptr, &out));
  d::adopt<T>(out, spalpha);
  if (path) {
    const size_t cols = std::min<size_t>((size_t)path->n(), (size_t)mlp);
    for (size_t c = 0; c < cols; ++c)
      memcpy(path->rawX() + c * path->m(), pbuf.data() + c * K, sizeof(T) * std::min<INTM>(K, path->m()));
  }
}

// decomp/decomp.h:735-745: the Cholesky implementation (coreLARS +
// downDateLasso) with its own stopping rules; ols ends with the
// least-squares fit on the support.  Up to 1024 atoms.
template <typename T>
void lasso(const Matrix<T>& X, const Matrix<T>& D, SpMatrix<T>& spalpha, int L,
           const T constraint, const T lambda2 = 0, constraint_type mode = PENALTY,
           const bool pos = false, const bool ols = false, const int numThreads = -1,
           Matrix<T>* path = NULL, const int length_path = -1) {
  (void)numThreads;
  namespace d = spams_b200_detail;
  const INTM n = X.n(), K = D.n();
  const int Lc = std::min<int>(L, (int)K);
  const int mlp = length_path <= 1 ? 4 * Lc : length_path;
  std::vector<T> pbuf(path ? (size_t)K * mlp : 0);
  typename d::Csc<T>::type out;
  d::check(d::call_lasso(X.X(), (int)X.m(), n, D.X(), (int)K, L, constraint, lambda2, (int)mode,
                         pos ? 1 : 0, mlp, path ? pbuf.data() : nullptr, &out, ols ? 1 : 0, 1));
  d::adopt<T>(out, spalpha);
  if (path) {
    const size_t cols = std::min<size_t>((size_t)path->n(), (size_t)mlp);
    for (size_t c = 0; c < cols; ++c)
      memcpy(path->rawX() + c * path->m(), pbuf.data() + c * K, sizeof(T) * std::min<INTM>(K, path->m()));
  }
}

// decomp/decomp.h:746-842: the Cholesky implementation on precomputed
// G and DtX (used as given); X supplies ||x_i||^2.
template <typename T>
void lasso(const Matrix<T>& X, const Matrix<T>& G, const Matrix<T>& DtX, SpMatrix<T>& spalpha,
           int L, const T lambda, constraint_type mode, const bool pos, const bool ols,
           const int numThreads = -1, Matrix<T>* path = NULL, const int length_path = -1) {
  (void)numThreads;
  namespace d = spams_b200_detail;
  const INTM n = X.n(), K = G.n();
  const int Lc = std::min<int>(L, (int)K);
  const int mlp = length_path <= 1 ? 4 * Lc : length_path;
  std::vector<T> pbuf(path ? (size_t)K * mlp : 0);
  typename d::Csc<T>::type out;
  d::check(d::call_lassoQq(X.X(), (int)X.m(), n, G.X(), (int)K, DtX.X(), L, lambda, T(0),
                           (int)mode, pos ? 1 : 0, mlp, path ? pbuf.data() : nullptr, &out,
                           ols ? 1 : 0, 1));
  d::adopt<T>(out, spalpha);
  if (path) {
    const size_t cols = std::min<size_t>((size_t)path->n(), (size_t)mlp);
    for (size_t c = 0; c < cols; ++c)
      memcpy(path->rawX() + c * path->m(), pbuf.data() + c * K, sizeof(T) * std::min<INTM>(K, path->m()));
  }
}

// decomp/decomp.h:406-519: each column coded from the rows its mask column
// keeps (bool, one byte per entry as in the reference's Matrix<bool>).
template <typename T>
void omp_mask(const Matrix<T>& X, const Matrix<T>& D, SpMatrix<T>& spalpha,
              const Matrix<bool>& mask, const int* L, const T* eps, const T* lambda,
              const bool vecL = false, const bool vecEps = false, const bool vecLambda = false,
              const int numThreads = -1, Matrix<T>* path = NULL) {
  (void)numThreads;
  namespace d = spams_b200_detail;
  const INTM m = X.m(), n = X.n(), K = D.n();
  const INTM pathL = std::min(m, K);
  std::vector<T> pbuf(path ? (size_t)K * pathL : 0);
  typename d::Csc<T>::type out;
  d::check(d::call_omp_mask(X.X(), (int)m, n, D.X(), (int)K, mask.X(), L, vecL ? n : 1, eps,
                            vecEps ? n : 1, lambda, vecLambda ? n : 1,
                            path ? pbuf.data() : nullptr, &out));
  d::adopt<T>(out, spalpha);
  if (path) {
    const size_t cols = std::min<size_t>((size_t)path->n(), (size_t)pathL);
    for (size_t c = 0; c < cols; ++c)
      memcpy(path->rawX() + c * path->m(), pbuf.data() + c * K, sizeof(T) * std::min<INTM>(K, path->m()));
  }
}

// decomp/decomp.h:1466-1561 with L as the _lassoMask facade clamps it.  A
// column with no observed row is empty here (the reference's CSC holds L
// explicit zeros at row 0 for it, the same dense matrix).
template <typename T>
void lasso_mask(const Matrix<T>& X, const Matrix<T>& D, SpMatrix<T>& spalpha,
                const Matrix<bool>& mask, int L, const T constraint, const T lambda2 = 0,
                constraint_type mode = PENALTY, const bool pos = false,
                const int numThreads = -1) {
  (void)numThreads;
  namespace d = spams_b200_detail;
  typename d::Csc<T>::type out;
  d::check(d::call_lasso_mask(X.X(), (int)X.m(), X.n(), D.X(), (int)D.n(), mask.X(), L,
                              constraint, lambda2, (int)mode, pos ? 1 : 0, &out));
  d::adopt<T>(out, spalpha);
}

#endif  // SPAMS_B200_DECOMP_H
