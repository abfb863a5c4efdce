// Drop-in C++ facade of cpp_library/spams.h for the coding path: _omp,
// _lassoD and _lassoQq with the reference's argument checks, default values,
// clamps of L (applied by the engine) and const char* exceptions.
//
//   _lassoD   cpp_library/spams.h:107-143
//   _lassoQq  cpp_library/spams.h:145-188
//   _omp      cpp_library/spams.h:250-293
//   _lassoMask cpp_library/spams.h:191-214, _ompMask :296-343
#ifndef SPAMS_B200_SPAMS_H
#define SPAMS_B200_SPAMS_H

#include "decomp.h"

template <typename T>
SpMatrix<T>* _lassoD(Matrix<T>* X, Matrix<T>* D, Matrix<T>** path, bool return_reg_path, int L,
                     const T constraint, const T lambda2, constraint_type mode, const bool pos,
                     const bool ols, const int numThreads, int max_length_path,
                     const bool verbose, bool cholevsky) {
  (void)numThreads;
  (void)verbose;
  namespace d = spams_b200_detail;
  if (X->m() != D->m()) throw "lasso : incompatible matrix dimensions";
  const int K = (int)D->n();
  const int L0 = L < 0 ? K : L;
  const int mlp = max_length_path < 0 ? 4 * L0 : max_length_path;
  *path = return_reg_path ? new Matrix<T>(K, mlp) : NULL;
  if (*path) (*path)->setZeros();
  SpMatrix<T>* alpha = new SpMatrix<T>();
  typename d::Csc<T>::type out;
  sc_status st = d::call_lasso(X->X(), (int)X->m(), X->n(), D->X(), K, L, constraint, lambda2,
                               (int)mode, pos ? 1 : 0, max_length_path,
                               *path ? (*path)->rawX() : nullptr, &out, ols ? 1 : 0,
                               (cholevsky || ols) ? 1 : 0);
  if (st != SC_OK) {
    delete alpha;
    delete *path;
    *path = NULL;
    throw sc_last_error();
  }
  d::adopt<T>(out, *alpha);
  return alpha;
}

template <typename T>
SpMatrix<T>* _lassoQq(Matrix<T>* X, Matrix<T>* Q, Matrix<T>* q, Matrix<T>** path,
                      bool return_reg_path, int L, const T constraint, const T lambda2,
                      constraint_type mode, const bool pos, const bool ols, const int numThreads,
                      int max_length_path, const bool verbose, bool cholevsky) {
  (void)numThreads;
  (void)verbose;
  namespace d = spams_b200_detail;
  if (Q->m() != Q->n()) throw "lasso : Q must be square";
  if (Q->m() != q->m() || X->n() != q->n()) throw "lasso : incompatible matrix dimensions";
  if (ols) cholevsky = ols;  // cpp_library/spams.h:182
  const int K = (int)Q->m();
  const int L0 = L < 0 ? K : L;
  const int mlp = max_length_path < 0 ? 4 * L0 : max_length_path;
  *path = return_reg_path ? new Matrix<T>(K, mlp) : NULL;
  if (*path) (*path)->setZeros();
  SpMatrix<T>* alpha = new SpMatrix<T>();
  typename d::Csc<T>::type out;
  sc_status st = d::call_lassoQq(X->X(), (int)X->m(), X->n(), Q->X(), K, q->X(), L, constraint,
                                 lambda2, (int)mode, pos ? 1 : 0, max_length_path,
                                 *path ? (*path)->rawX() : nullptr, &out, ols ? 1 : 0,
                                 cholevsky ? 1 : 0);
  if (st != SC_OK) {
    delete alpha;
    delete *path;
    *path = NULL;
    throw sc_last_error();
  }
  d::adopt<T>(out, *alpha);
  return alpha;
}

template <typename T>
SpMatrix<T>* _omp(Matrix<T>* X, Matrix<T>* D, Matrix<T>** path, bool return_reg_path,
                  bool given_L, Vector<int>* L, bool given_eps, Vector<T>* eps,
                  bool given_Lambda, Vector<T>* Lambda, const int numThreads) {
  (void)numThreads;
  namespace d = spams_b200_detail;
  if (X->m() != D->m()) throw "omp : incompatible matrix dimensions";
  if (!given_L && !given_eps && !given_Lambda)
    throw "omp : You should either provide L, eps or lambda";
  const int K = (int)D->n();
  const int scalar_L = (int)std::min<INTM>(X->m(), K);
  *path = return_reg_path ? new Matrix<T>(K, scalar_L) : NULL;
  if (*path) (*path)->setZeros();
  SpMatrix<T>* alpha = new SpMatrix<T>();
  typename d::Csc<T>::type out;
  sc_status st = d::call_omp(X->X(), (int)X->m(), X->n(), D->X(), K,
                             given_L ? L->rawX() : nullptr, given_L ? L->n() : 0,
                             given_eps ? eps->rawX() : nullptr, given_eps ? eps->n() : 0,
                             given_Lambda ? Lambda->rawX() : nullptr,
                             given_Lambda ? Lambda->n() : 0,
                             *path ? (*path)->rawX() : nullptr, &out);
  if (st != SC_OK) {
    delete alpha;
    delete *path;
    *path = NULL;
    throw sc_last_error();
  }
  d::adopt<T>(out, *alpha);
  return alpha;
}

// cpp_library/spams.h:191-214
template <typename T>
SpMatrix<T>* _lassoMask(Matrix<T>* X, Matrix<T>* D, Matrix<bool>* B, int L, const T constraint,
                        const T lambda2, constraint_type mode, const bool pos,
                        const int numThreads, bool verbose) {
  (void)numThreads;
  (void)verbose;
  namespace d = spams_b200_detail;
  if (X->m() != D->m()) throw "lassoMask : incompatible matrix dimensions";
  SpMatrix<T>* alpha = new SpMatrix<T>();
  typename d::Csc<T>::type out;
  sc_status st = d::call_lasso_mask(X->X(), (int)X->m(), X->n(), D->X(), (int)D->n(), B->X(), L,
                                    constraint, lambda2, (int)mode, pos ? 1 : 0, &out);
  if (st != SC_OK) {
    delete alpha;
    throw sc_last_error();
  }
  d::adopt<T>(out, *alpha);
  return alpha;
}

// cpp_library/spams.h:296-343
template <typename T>
SpMatrix<T>* _ompMask(Matrix<T>* X, Matrix<T>* D, Matrix<bool>* B, Matrix<T>** path,
                      bool return_reg_path, bool given_L, Vector<int>* L, bool given_eps,
                      Vector<T>* eps, bool given_Lambda, Vector<T>* Lambda,
                      const int numThreads) {
  (void)numThreads;
  namespace d = spams_b200_detail;
  if (X->m() != D->m()) throw "ompMask : incompatible matrix dimensions";
  if (B->m() != X->m() || B->n() != X->n()) throw "ompMask : Mash has non acceptable dimensions";
  if (!given_L && !given_eps && !given_Lambda)
    throw "omp : You should either provide L, eps or lambda";
  const int K = (int)D->n();
  const int scalar_L = (int)std::min<INTM>(X->m(), K);
  *path = return_reg_path ? new Matrix<T>(K, scalar_L) : NULL;
  if (*path) (*path)->setZeros();
  SpMatrix<T>* alpha = new SpMatrix<T>();
  typename d::Csc<T>::type out;
  sc_status st = d::call_omp_mask(X->X(), (int)X->m(), X->n(), D->X(), K, B->X(),
                                  given_L ? L->rawX() : nullptr, given_L ? L->n() : 0,
                                  given_eps ? eps->rawX() : nullptr, given_eps ? eps->n() : 0,
                                  given_Lambda ? Lambda->rawX() : nullptr,
                                  given_Lambda ? Lambda->n() : 0,
                                  *path ? (*path)->rawX() : nullptr, &out);
  if (st != SC_OK) {
    delete alpha;
    delete *path;
    *path = NULL;
    throw sc_last_error();
  }
  d::adopt<T>(out, *alpha);
  return alpha;
}

#endif  // SPAMS_B200_SPAMS_H
