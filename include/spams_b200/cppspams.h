// Drop-in for cpp_library/cppspams.h (coding path): cppOMP and cppLasso.
//
//   cppOMP    cpp_library/cppspams.h:44-51
//   cppLasso  cpp_library/cppspams.h:105-123
//
// The reference's (X, Q, q) overload of cppLasso calls a _lassoD overload that
// does not exist (cppspams.h:121); here it is routed to _lassoQq, whose
// semantics it documents.
#ifndef SPAMS_B200_CPPSPAMS_H
#define SPAMS_B200_CPPSPAMS_H

#include "spams.h"

template <typename T>
void cppOMP(const Matrix<T>& X, const Matrix<T>& D, SpMatrix<T>& spalpha, const int* L,
            const T* eps, const T* lambda, const bool vecL = false, const bool vecEps = false,
            const bool vecLambda = false, const int numThreads = -1, Matrix<T>* path = NULL) {
  omp(X, D, spalpha, L, eps, lambda, vecL, vecEps, vecLambda, numThreads, path);
}

template <typename T>
SpMatrix<T>* cppLasso(Matrix<T>& X, Matrix<T>& D, Matrix<T>** path, bool return_reg_path, int L,
                      const T constraint, const T lambda2 = 0., constraint_type mode = PENALTY,
                      const bool pos = false, const bool ols = false, const int numThreads = -1,
                      int max_length_path = -1, const bool verbose = false,
                      bool cholevsky = false) {
  return _lassoD(&X, &D, path, return_reg_path, L, constraint, lambda2, mode, pos, ols,
                 numThreads, max_length_path, verbose, cholevsky);
}

template <typename T>
SpMatrix<T>* cppLasso(Matrix<T>& X, Matrix<T>& Q, Matrix<T>& q, Matrix<T>** path,
                      bool return_reg_path, int L, const T constraint, const T lambda2 = 0.,
                      constraint_type mode = PENALTY, const bool pos = false,
                      const bool ols = false, const int numThreads = -1,
                      int max_length_path = -1, const bool verbose = false,
                      bool cholevsky = false) {
  return _lassoQq(&X, &Q, &q, path, return_reg_path, L, constraint, lambda2, mode, pos, ols,
                  numThreads, max_length_path, verbose, cholevsky);
}

#endif  // SPAMS_B200_CPPSPAMS_H
