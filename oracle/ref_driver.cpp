// Test infrastructure only: a C-ABI shim around the SPAMS reference's own
// C++ facade, compiled straight from the reference's header sources by
// oracle/build_ref.sh into oracle/_ref/libspams_ref.so.  It is the ground
// truth the CPU restatement (oracle/sc_oracle.c) and the CUDA engine are
// checked against, and the "reference" CPU baseline that bench.py times.
// Nothing in the shipped engine links or calls it.
//
// Entry points forward to the reference facade unchanged:
//   ref_omp_*    -> _omp<T>     cpp_library/spams.h:250-293
//                   (-> omp<T> decomp/decomp.h:322-404, coreORMP :538-640)
//   ref_lasso_*  -> _lassoD<T>  cpp_library/spams.h:107-143
//                   (-> lasso2<T> decomp/decomp.h:1563-1646, coreLARS2 :1706-1915,
//                    or lasso<T>/coreLARS when cholesky/ols is set)
//   ref_lassoQq_* -> _lassoQq<T> cpp_library/spams.h:145-188
//   ref_omp_mask_*   -> _ompMask<T>   cpp_library/spams.h:296-343 (omp_mask,
//                       decomp/decomp.h:406-519)
//   ref_lasso_mask_* -> _lassoMask<T> cpp_library/spams.h:191-214 (lasso_mask,
//                       decomp/decomp.h:1466-1561)
//   ref_dl_minibatch_f32 -> one minibatch of Trainer<T>::train
//                       (dictLearn/dicts.h:526-603): XtX Gram + ridge, per
//                       signal multTrans + coreLARS2 + sort, per-thread
//                       rank-1 accumulations AT += a a^T, BT += x a^T, summed
//                       into A and B (PENALTY mode, the reference's own code
//                       called in its order; the D update is not part of it)
// Outputs are copied out of the reference's SpMatrix<T> (linalg/linalg.h:775-935)
// into malloc'd CSC arrays released by ref_free().
#include "cppspams.h"
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <vector>

extern "C" {

typedef struct {
  int64_t m, n, nnz;
  int64_t* colptr;  // n+1
  int32_t* rows;    // nnz
  void* vals;       // nnz of T
  char err[128];    // facade exception text, "" on success
} ref_csc;

void ref_free(void* p) { free(p); }

}  // extern "C"

template <typename T>
static void copy_out(SpMatrix<T>* a, ref_csc* out) {
  const int64_t n = a->n();
  out->m = a->m();
  out->n = n;
  const int64_t nnz = n > 0 ? a->pB()[n] : 0;
  out->nnz = nnz;
  out->colptr = (int64_t*)malloc(sizeof(int64_t) * (n + 1));
  out->rows = (int32_t*)malloc(sizeof(int32_t) * (nnz > 0 ? nnz : 1));
  out->vals = malloc(sizeof(T) * (nnz > 0 ? nnz : 1));
  for (int64_t i = 0; i <= n; ++i) out->colptr[i] = n > 0 ? a->pB()[i] : 0;
  for (int64_t i = 0; i < nnz; ++i) {
    out->rows[i] = a->r()[i];
    ((T*)out->vals)[i] = a->v()[i];
  }
}

template <typename T>
static int run_omp(const T* X, int m, int n, const T* D, int K, const int* L,
                   int nL, const T* eps, int nEps, const T* lambda, int nLambda,
                   int numThreads, T* path, ref_csc* out) {
  memset(out, 0, sizeof(*out));
  Matrix<T> mX(const_cast<T*>(X), m, n);
  Matrix<T> mD(const_cast<T*>(D), m, K);
  int Ldummy = 0;
  T edummy = 0, ldummy = 0;
  Vector<int> vL(nL > 0 ? const_cast<int*>(L) : &Ldummy, nL > 0 ? nL : 1);
  Vector<T> vE(nEps > 0 ? const_cast<T*>(eps) : &edummy, nEps > 0 ? nEps : 1);
  Vector<T> vLa(nLambda > 0 ? const_cast<T*>(lambda) : &ldummy,
                nLambda > 0 ? nLambda : 1);
  Matrix<T>* p = NULL;
  SpMatrix<T>* a = NULL;
  try {
    a = _omp<T>(&mX, &mD, &p, path != NULL, nL > 0, &vL, nEps > 0, &vE,
                nLambda > 0, &vLa, numThreads);
  } catch (const char* e) {
    strncpy(out->err, e, sizeof(out->err) - 1);
    return 1;
  }
  copy_out(a, out);
  if (path && p) memcpy(path, p->rawX(), sizeof(T) * p->m() * p->n());
  delete a;
  delete p;
  return 0;
}

template <typename T>
static int run_lasso(const T* X, int m, int n, const T* D, int K, int L,
                     T lambda1, T lambda2, int mode, int pos, int ols,
                     int cholesky, int numThreads, int max_length_path, T* path,
                     ref_csc* out) {
  memset(out, 0, sizeof(*out));
  Matrix<T> mX(const_cast<T*>(X), m, n);
  Matrix<T> mD(const_cast<T*>(D), m, K);
  Matrix<T>* p = NULL;
  SpMatrix<T>* a = NULL;
  try {
    a = _lassoD<T>(&mX, &mD, &p, path != NULL, L, lambda1, lambda2,
                   (constraint_type)mode, pos != 0, ols != 0, numThreads,
                   max_length_path, false, cholesky != 0);
  } catch (const char* e) {
    strncpy(out->err, e, sizeof(out->err) - 1);
    return 1;
  }
  copy_out(a, out);
  if (path && p) memcpy(path, p->rawX(), sizeof(T) * p->m() * p->n());
  delete a;
  delete p;
  return 0;
}

template <typename T>
static int run_lassoQq(const T* X, int m, int n, const T* Q, int K, const T* q,
                       int L, T lambda1, int mode, int pos, int ols, int cholesky,
                       int numThreads, int max_length_path, T* path, ref_csc* out) {
  memset(out, 0, sizeof(*out));
  Matrix<T> mX(const_cast<T*>(X), m, n);
  Matrix<T> mQ(const_cast<T*>(Q), K, K);
  Matrix<T> mq(const_cast<T*>(q), K, n);
  Matrix<T>* p = NULL;
  SpMatrix<T>* a = NULL;
  try {
    a = _lassoQq<T>(&mX, &mQ, &mq, &p, path != NULL, L, lambda1, T(0),
                    (constraint_type)mode, pos != 0, ols != 0, numThreads,
                    max_length_path, false, cholesky != 0);
  } catch (const char* e) {
    strncpy(out->err, e, sizeof(out->err) - 1);
    return 1;
  }
  copy_out(a, out);
  if (path && p) memcpy(path, p->rawX(), sizeof(T) * p->m() * p->n());
  delete a;
  delete p;
  return 0;
}

template <typename T>
static int run_omp_mask(const T* X, int m, int n, const T* D, int K, const uint8_t* B,
                        const int* L, int nL, const T* eps, int nEps, const T* lambda,
                        int nLambda, int numThreads, T* path, ref_csc* out) {
  memset(out, 0, sizeof(*out));
  Matrix<T> mX(const_cast<T*>(X), m, n);
  Matrix<T> mD(const_cast<T*>(D), m, K);
  Matrix<bool> mB(reinterpret_cast<bool*>(const_cast<uint8_t*>(B)), m, n);
  int Ldummy = 0;
  T edummy = 0, ldummy = 0;
  Vector<int> vL(nL > 0 ? const_cast<int*>(L) : &Ldummy, nL > 0 ? nL : 1);
  Vector<T> vE(nEps > 0 ? const_cast<T*>(eps) : &edummy, nEps > 0 ? nEps : 1);
  Vector<T> vLa(nLambda > 0 ? const_cast<T*>(lambda) : &ldummy,
                nLambda > 0 ? nLambda : 1);
  Matrix<T>* p = NULL;
  SpMatrix<T>* a = NULL;
  try {
    a = _ompMask<T>(&mX, &mD, &mB, &p, path != NULL, nL > 0, &vL, nEps > 0, &vE,
                    nLambda > 0, &vLa, numThreads);
  } catch (const char* e) {
    strncpy(out->err, e, sizeof(out->err) - 1);
    return 1;
  }
  copy_out(a, out);
  if (path && p) memcpy(path, p->rawX(), sizeof(T) * p->m() * p->n());
  delete a;
  delete p;
  return 0;
}

template <typename T>
static int run_lasso_mask(const T* X, int m, int n, const T* D, int K, const uint8_t* B,
                          int L, T lambda1, T lambda2, int mode, int pos, int numThreads,
                          ref_csc* out) {
  memset(out, 0, sizeof(*out));
  Matrix<T> mX(const_cast<T*>(X), m, n);
  Matrix<T> mD(const_cast<T*>(D), m, K);
  Matrix<bool> mB(reinterpret_cast<bool*>(const_cast<uint8_t*>(B)), m, n);
  SpMatrix<T>* a = NULL;
  try {
    a = _lassoMask<T>(&mX, &mD, &mB, L, lambda1, lambda2, (constraint_type)mode, pos != 0,
                      numThreads, false);
  } catch (const char* e) {
    strncpy(out->err, e, sizeof(out->err) - 1);
    return 1;
  }
  copy_out(a, out);
  delete a;
  return 0;
}

// One minibatch of the reference's online dictionary learning, coding and
// accumulation part (dictLearn/dicts.h:526-603, PENALTY mode): the same
// calls in the same order on the reference's own classes.  A = beta A +
// gamma sum_j a_j a_j^T, B = beta B + gamma sum_j x_j a_j^T.
template <typename T>
static int run_dl_minibatch(const T* D, int m, int K, const T* X, int M, const int* perm,
                            int iter, int batch, T lambda1, T lambda2, int numThreads, T* A,
                            T* B, T beta, T gamma) {
  Matrix<T> mD(const_cast<T*>(D), m, K);
  Matrix<T> mX(const_cast<T*>(X), m, M);
  Matrix<T> mA(A, K, K), mB(B, m, K);
  const int L = MIN(m, K);
  const int NT = init_omp(numThreads);
  Matrix<T> G;
  mD.XtX(G);
  G.addDiag(MAX(lambda2, T(1e-10)));
  std::vector<Matrix<T>> AT(NT), BT(NT), GsT(NT), GaT(NT), invGsT(NT), workT(NT);
  std::vector<Vector<T>> DtRT(NT), uT(NT), XT(NT);
  std::vector<SpVector<T>> spT(NT);
  for (int t = 0; t < NT; ++t) {
    AT[t].resize(K, K); AT[t].setZeros();
    BT[t].resize(m, K); BT[t].setZeros();
    GsT[t].resize(L, L); invGsT[t].resize(L, L); GaT[t].resize(K, L);
    workT[t].resize(K, 3); workT[t].setZeros();
    DtRT[t].resize(K); uT[t].resize(K); uT[t].setZeros(); XT[t].resize(m);
    spT[t].resize(L);
  }
  int j;
#pragma omp parallel for private(j)
  for (j = 0; j < batch; ++j) {
#ifdef _OPENMP
    const int t = omp_get_thread_num();
#else
    const int t = 0;
#endif
    const int index = perm[((int64_t)j + (int64_t)iter * batch) % M];
    Vector<T>& Xj = XT[t];
    mX.copyCol(index, Xj);
    mD.multTrans(Xj, DtRT[t]);
    SpVector<T>& sp = spT[t];
    sp.setL(L);
    Vector<INTM> ind;
    Vector<T> coeffs;
    sp.refIndices(ind);
    sp.refVal(coeffs);
    T normX = Xj.nrm2sq();
    coeffs.setZeros();
    coreLARS2(DtRT[t], G, GsT[t], GaT[t], invGsT[t], uT[t], coeffs, ind, workT[t], normX,
              PENALTY, lambda1, false);
    int cnt = 0;
    for (int k = 0; k < L; ++k) {
      if (ind[k] == -1) break;
      ++cnt;
    }
    sort(ind.rawX(), coeffs.rawX(), (INTM)0, (INTM)(cnt - 1));
    sp.setL(cnt);
    AT[t].rank1Update(sp);
    BT[t].rank1Update(Xj, sp);
  }
  mA.scal(beta);
  mB.scal(beta);
  for (int t = 0; t < NT; ++t) {
    mA.add(AT[t], gamma);
    mB.add(BT[t], gamma);
  }
  return 0;
}

extern "C" {

int ref_dl_minibatch_f32(const float* D, int m, int K, const float* X, int M, const int* perm,
                         int iter, int batch, float lambda1, int numThreads, float* A, float* B,
                         float beta, float gamma) {
  return run_dl_minibatch<float>(D, m, K, X, M, perm, iter, batch, lambda1, 0.f, numThreads, A,
                                 B, beta, gamma);
}

int ref_omp_mask_f64(const double* X, int m, int n, const double* D, int K, const uint8_t* B,
                     const int* L, int nL, const double* eps, int nEps, const double* lambda,
                     int nLambda, int numThreads, double* path, ref_csc* out) {
  return run_omp_mask<double>(X, m, n, D, K, B, L, nL, eps, nEps, lambda, nLambda, numThreads,
                              path, out);
}
int ref_omp_mask_f32(const float* X, int m, int n, const float* D, int K, const uint8_t* B,
                     const int* L, int nL, const float* eps, int nEps, const float* lambda,
                     int nLambda, int numThreads, float* path, ref_csc* out) {
  return run_omp_mask<float>(X, m, n, D, K, B, L, nL, eps, nEps, lambda, nLambda, numThreads,
                             path, out);
}
int ref_lasso_mask_f64(const double* X, int m, int n, const double* D, int K, const uint8_t* B,
                       int L, double lambda1, double lambda2, int mode, int pos, int numThreads,
                       ref_csc* out) {
  return run_lasso_mask<double>(X, m, n, D, K, B, L, lambda1, lambda2, mode, pos, numThreads,
                                out);
}
int ref_lasso_mask_f32(const float* X, int m, int n, const float* D, int K, const uint8_t* B,
                       int L, float lambda1, float lambda2, int mode, int pos, int numThreads,
                       ref_csc* out) {
  return run_lasso_mask<float>(X, m, n, D, K, B, L, lambda1, lambda2, mode, pos, numThreads,
                               out);
}

int ref_omp_f64(const double* X, int m, int n, const double* D, int K,
                const int* L, int nL, const double* eps, int nEps,
                const double* lambda, int nLambda, int numThreads, double* path,
                ref_csc* out) {
  return run_omp<double>(X, m, n, D, K, L, nL, eps, nEps, lambda, nLambda,
                         numThreads, path, out);
}
int ref_omp_f32(const float* X, int m, int n, const float* D, int K,
                const int* L, int nL, const float* eps, int nEps,
                const float* lambda, int nLambda, int numThreads, float* path,
                ref_csc* out) {
  return run_omp<float>(X, m, n, D, K, L, nL, eps, nEps, lambda, nLambda,
                        numThreads, path, out);
}
int ref_lasso_f64(const double* X, int m, int n, const double* D, int K, int L,
                  double lambda1, double lambda2, int mode, int pos, int ols,
                  int cholesky, int numThreads, int max_length_path,
                  double* path, ref_csc* out) {
  return run_lasso<double>(X, m, n, D, K, L, lambda1, lambda2, mode, pos, ols,
                           cholesky, numThreads, max_length_path, path, out);
}
int ref_lasso_f32(const float* X, int m, int n, const float* D, int K, int L,
                  float lambda1, float lambda2, int mode, int pos, int ols,
                  int cholesky, int numThreads, int max_length_path,
                  float* path, ref_csc* out) {
  return run_lasso<float>(X, m, n, D, K, L, lambda1, lambda2, mode, pos, ols,
                          cholesky, numThreads, max_length_path, path, out);
}
int ref_lassoQq_f64(const double* X, int m, int n, const double* Q, int K,
                    const double* q, int L, double lambda1, int mode, int pos,
                    int ols, int cholesky, int numThreads, int max_length_path,
                    double* path, ref_csc* out) {
  return run_lassoQq<double>(X, m, n, Q, K, q, L, lambda1, mode, pos, ols,
                             cholesky, numThreads, max_length_path, path, out);
}
int ref_lassoQq_f32(const float* X, int m, int n, const float* Q, int K,
                    const float* q, int L, float lambda1, int mode, int pos,
                    int ols, int cholesky, int numThreads, int max_length_path,
                    float* path, ref_csc* out) {
  return run_lassoQq<float>(X, m, n, Q, K, q, L, lambda1, mode, pos, ols,
                            cholesky, numThreads, max_length_path, path, out);
}

}  // extern "C"
