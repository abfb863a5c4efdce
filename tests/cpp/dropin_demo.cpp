// Drives the drop-in C++ API (include/spams_b200/cppspams.h) the way the
// reference's own demo drives cppspams.h (cpp_library/test_decomp.cpp:14-64):
// OMP and LARS-Lasso on a dictionary and a batch of signals, through
// cppOMP / cppLasso / _omp / _lassoD / lasso2(G, DtX) / lasso(G, DtX) / _lassoQq /
// _ompMask / _lassoMask.  Inputs and outputs are
// raw binary files in a directory given on the command line; the GPU test
// suite compares the outputs with the oracle.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "spams_b200/cppspams.h"

template <typename T>
static std::vector<T> read_all(const std::string& fn, size_t n) {
  std::vector<T> v(n);
  FILE* f = fopen(fn.c_str(), "rb");
  if (!f || fread(v.data(), sizeof(T), n, f) != n) { fprintf(stderr, "read %s\n", fn.c_str()); exit(2); }
  fclose(f);
  return v;
}

template <typename T>
static void write_csc(const std::string& fn, const SpMatrix<T>& a) {
  FILE* f = fopen(fn.c_str(), "wb");
  long long hdr[3] = {(long long)a.m(), (long long)a.n(), (long long)a.nnz()};
  fwrite(hdr, sizeof(hdr), 1, f);
  for (INTM j = 0; j <= a.n(); ++j) { long long p = a.pB()[j]; fwrite(&p, 8, 1, f); }
  for (INTM k = 0; k < a.nnz(); ++k) { int r = (int)a.r()[k]; fwrite(&r, 4, 1, f); }
  for (INTM k = 0; k < a.nnz(); ++k) { double v = a.v()[k]; fwrite(&v, 8, 1, f); }
  fclose(f);
}

template <typename T>
static int run(const std::string& dir, int m, int n, int K) {
  std::vector<T> x = read_all<T>(dir + "/X.bin", (size_t)m * n);
  std::vector<T> dd = read_all<T>(dir + "/D.bin", (size_t)m * K);
  Matrix<T> X(x.data(), m, n);
  Matrix<T> D(dd.data(), m, K);
  // cppOMP, L = 6, eps = 0, lambda = 0 (cpp_library/test_decomp.cpp:14-34)
  {
    const int L = 6;
    T eps = 0, lambda = 0;
    SpMatrix<T> spa;
    cppOMP(X, D, spa, &L, &eps, &lambda);
    write_csc(dir + "/omp.csc", spa);
  }
  // _omp with eps only and a path
  {
    Vector<T> eps(1);
    eps[0] = T(0.05);
    Vector<int> Lv(1);
    Lv[0] = 0;
    Vector<T> la(1);
    la[0] = 0;
    Matrix<T>* path = nullptr;
    SpMatrix<T>* spa = _omp(&X, &D, &path, true, false, &Lv, true, &eps, false, &la, -1);
    write_csc(dir + "/omp_eps.csc", *spa);
    delete spa;
    delete path;
  }
  // cppLasso(X, D, &path, false, 10, 0.15) (cpp_library/test_decomp.cpp:36-65)
  {
    Matrix<T>* path = nullptr;
    SpMatrix<T>* spa = cppLasso(X, D, &path, false, 10, T(0.15));
    write_csc(dir + "/lasso_L10.csc", *spa);
    delete spa;
  }
  // _lassoD with defaults (L = -1) and pos
  {
    Matrix<T>* path = nullptr;
    SpMatrix<T>* spa = _lassoD(&X, &D, &path, false, -1, T(0.1), T(0), PENALTY, true, false, -1,
                               -1, false, false);
    write_csc(dir + "/lasso_pos.csc", *spa);
    delete spa;
  }
  // lasso2 with precomputed G = D^T D (+1e-10) and D^T X
  {
    Matrix<T> G(K, K), DtX(K, n);
    for (int a = 0; a < K; ++a)
      for (int b = 0; b < K; ++b) {
        double s = 0;
        for (int r = 0; r < m; ++r) s += (double)dd[(size_t)a * m + r] * dd[(size_t)b * m + r];
        G(a, b) = (T)s + (a == b ? T(1e-10) : T(0));
      }
    for (int a = 0; a < K; ++a)
      for (int i = 0; i < n; ++i) {
        double s = 0;
        for (int r = 0; r < m; ++r) s += (double)dd[(size_t)a * m + r] * x[(size_t)i * m + r];
        DtX(a, i) = (T)s;
      }
    SpMatrix<T> spa;
    lasso2(X, G, DtX, spa, std::min(m, K), T(0.15));
    write_csc(dir + "/lasso_gram.csc", spa);
    // cppLasso(X, Q, q, ...) overload
    Matrix<T>* path = nullptr;
    SpMatrix<T>* sp2 = cppLasso(X, G, DtX, &path, false, -1, T(0.15));
    write_csc(dir + "/lasso_qq.csc", *sp2);
    delete sp2;
    // the Cholesky implementation on the same products: lasso(X, G, DtX, ...,
    // ols) (decomp/decomp.h:746) and _lassoQq with ols (cpp_library/spams.h:145)
    SpMatrix<T> spc;
    lasso(X, G, DtX, spc, std::min(m, K), T(1.0), L1COEFFS, false, false);
    write_csc(dir + "/lasso_gram_chol_l1.csc", spc);
    SpMatrix<T>* sp3 = _lassoQq(&X, &G, &DtX, &path, false, -1, T(0.05), T(0), L2ERROR, false,
                                true, -1, -1, false, false);
    write_csc(dir + "/lasso_qq_ols_l2err.csc", *sp3);
    delete sp3;
  }
  // _lassoD with the Cholesky implementation in L2ERROR mode
  {
    Matrix<T>* path = nullptr;
    SpMatrix<T>* spa = _lassoD(&X, &D, &path, false, -1, T(0.05), T(0), L2ERROR, false, false, -1,
                               -1, false, true);
    write_csc(dir + "/lasso_chol_l2err.csc", *spa);
    delete spa;
  }
  // masked variants: row r of signal i observed unless (7 r + 3 i) % 10 >= 7;
  // signal 0 fully observed, signal 1 not at all
  {
    std::vector<char> bm((size_t)m * n);
    for (int i = 0; i < n; ++i)
      for (int r = 0; r < m; ++r)
        bm[(size_t)i * m + r] = i == 0 ? 1 : (i == 1 ? 0 : ((7 * r + 3 * i) % 10 < 7));
    Matrix<bool> B(reinterpret_cast<bool*>(bm.data()), m, n);
    Vector<int> Lv(1);
    Lv[0] = 6;
    Vector<T> eps(1), la(1);
    eps[0] = 0;
    la[0] = 0;
    Matrix<T>* path = nullptr;
    SpMatrix<T>* spa = _ompMask(&X, &D, &B, &path, false, true, &Lv, true, &eps, true, &la, -1);
    write_csc(dir + "/omp_mask.csc", *spa);
    delete spa;
    SpMatrix<T>* spl = _lassoMask(&X, &D, &B, -1, T(0.1), T(0), PENALTY, false, -1, false);
    write_csc(dir + "/lasso_mask.csc", *spl);
    delete spl;
  }
  // facade error path
  {
    Matrix<T> Dbad(dd.data(), m - 1, K);
    try {
      SpMatrix<T> spa;
      Matrix<T>* path = nullptr;
      SpMatrix<T>* s = _lassoD(&X, &Dbad, &path, false, 5, T(0.1), T(0), PENALTY, false, false,
                               -1, -1, false, false);
      delete s;
      printf("no exception\n");
      return 1;
    } catch (const char* e) {
      printf("caught: %s\n", e);
    }
  }
  return 0;
}

int main(int argc, char** argv) {
  if (argc != 6) { fprintf(stderr, "usage: dropin_demo DIR m n K f32|f64\n"); return 2; }
  const std::string dir = argv[1];
  const int m = atoi(argv[2]), n = atoi(argv[3]), K = atoi(argv[4]);
  return std::string(argv[5]) == "f64" ? run<double>(dir, m, n, K) : run<float>(dir, m, n, K);
}
