// Drop-in containers for the SPAMS coding API, backed by the B200 engine.
//
// Matrix<T>, Vector<T> and SpMatrix<T> keep the storage layout, ownership
// rules and accessors of the reference containers that the coding entry points
// and their callers use (linalg/linalg.h: Matrix :205-548, Vector :551-772,
// SpMatrix :775-935): column-major dense storage, CSC sparse storage with
// pE = pB + 1, a constructor over an external pointer that does not own it,
// and an (m, n) constructor that allocates.  Only the members the coding path
// and its callers touch are provided; the arithmetic lives on the GPU.
#ifndef SPAMS_B200_LINALG_H
#define SPAMS_B200_LINALG_H

#include <cstddef>
#include <cstdint>
#include <cstring>

#ifdef INT_64BITS
typedef long long int INTM;
#else
typedef int INTM;
#endif

template <typename T> class Matrix {
 public:
  // over existing data: the matrix does not own X (linalg.h:1077-1078)
  Matrix(T* X, INTM m, INTM n) : _externAlloc(true), _X(X), _m(m), _n(n) {}
  // new m x n matrix, uninitialised (linalg.h:1082-1088)
  Matrix(INTM m, INTM n) : _externAlloc(false), _X(new T[(size_t)m * n]), _m(m), _n(n) {}
  Matrix() : _externAlloc(false), _X(nullptr), _m(0), _n(0) {}
  ~Matrix() { clear(); }
  Matrix(const Matrix&) = delete;
  Matrix& operator=(const Matrix&) = delete;

  inline INTM m() const { return _m; }
  inline INTM n() const { return _n; }
  inline T& operator()(INTM i, INTM j) { return _X[(size_t)j * _m + i]; }
  inline T operator()(INTM i, INTM j) const { return _X[(size_t)j * _m + i]; }
  inline T& operator[](INTM i) { return _X[i]; }
  inline T operator[](INTM i) const { return _X[i]; }
  inline T* rawX() const { return _X; }
  inline const T* X() const { return _X; }
  inline void setZeros() { if (_X) memset(_X, 0, sizeof(T) * (size_t)_m * _n); }
  inline void resize(INTM m, INTM n, bool set_zeros = true) {
    if (m == _m && n == _n) return;
    clear();
    _m = m;
    _n = n;
    _externAlloc = false;
    _X = new T[(size_t)m * n];
    if (set_zeros) setZeros();
  }
  inline void clear() {
    if (!_externAlloc) delete[] _X;
    _X = nullptr;
    _m = _n = 0;
    _externAlloc = true;
  }

 private:
  bool _externAlloc;
  T* _X;
  INTM _m, _n;
};

template <typename T> class Vector {
 public:
  Vector(T* X, INTM n) : _externAlloc(true), _X(X), _n(n) {}
  explicit Vector(INTM n) : _externAlloc(false), _X(new T[n]), _n(n) {}
  Vector() : _externAlloc(false), _X(nullptr), _n(0) {}
  ~Vector() { if (!_externAlloc) delete[] _X; }
  Vector(const Vector&) = delete;
  Vector& operator=(const Vector&) = delete;
  inline INTM n() const { return _n; }
  inline T* rawX() const { return _X; }
  inline T& operator[](INTM i) { return _X[i]; }
  inline T operator[](INTM i) const { return _X[i]; }
  inline T maxval() const {
    T v = _X[0];
    for (INTM i = 1; i < _n; ++i) v = _X[i] > v ? _X[i] : v;
    return v;
  }

 private:
  bool _externAlloc;
  T* _X;
  INTM _n;
};

// Compressed sparse column matrix (linalg.h:775-935).
template <typename T> class SpMatrix {
 public:
  SpMatrix(T* v, INTM* r, INTM* pB, INTM* pE, INTM m, INTM n, INTM nzmax)
      : _externAlloc(true), _v(v), _r(r), _pB(pB), _pE(pE), _m(m), _n(n), _nzmax(nzmax) {}
  SpMatrix(INTM m, INTM n, INTM nzmax) : _externAlloc(true), _v(nullptr), _r(nullptr),
      _pB(nullptr), _pE(nullptr), _m(0), _n(0), _nzmax(0) { resize(m, n, nzmax); }
  SpMatrix() : _externAlloc(true), _v(nullptr), _r(nullptr), _pB(nullptr), _pE(nullptr),
      _m(0), _n(0), _nzmax(0) {}
  ~SpMatrix() { clear(); }
  SpMatrix(const SpMatrix&) = delete;
  SpMatrix& operator=(const SpMatrix&) = delete;

  inline INTM pB(INTM i) const { return _pB[i]; }
  inline INTM r(INTM i) const { return _r[i]; }
  inline T v(INTM i) const { return _v[i]; }
  inline INTM nzmax() const { return _nzmax; }
  inline INTM n() const { return _n; }
  inline INTM m() const { return _m; }
  inline INTM* pB() const { return _pB; }
  inline INTM* pE() const { return _pE; }
  inline INTM* r() const { return _r; }
  inline T* v() const { return _v; }
  inline INTM nnz() const { return _pB ? _pB[_n] : 0; }

  // (linalg.h:4258-4272)
  inline void clear() {
    if (!_externAlloc) {
      delete[] _r;
      delete[] _v;
      delete[] _pB;
    }
    _n = _m = _nzmax = 0;
    _v = nullptr;
    _r = nullptr;
    _pB = _pE = nullptr;
    _externAlloc = true;
  }
  // (linalg.h:4275-4291): zeroed column pointers
  inline void resize(INTM m, INTM n, INTM nzmax) {
    if (n == _n && m == _m && nzmax == _nzmax) return;
    clear();
    _n = n;
    _m = m;
    _nzmax = nzmax;
    _externAlloc = false;
    _v = new T[nzmax > 0 ? nzmax : 1];
    _r = new INTM[nzmax > 0 ? nzmax : 1];
    _pB = new INTM[_n + 1];
    _pE = _pB + 1;
    for (INTM i = 0; i <= _n; ++i) _pB[i] = 0;
  }
  // dense copy (linalg.h SpMatrix::toFull)
  inline void toFull(Matrix<T>& full) const {
    full.resize(_m, _n);
    full.setZeros();
    for (INTM j = 0; j < _n; ++j)
      for (INTM k = _pB[j]; k < _pE[j]; ++k) full(_r[k], j) = _v[k];
  }

 private:
  bool _externAlloc;
  T* _v;
  INTM* _r;
  INTM* _pB;
  INTM* _pE;
  INTM _m, _n, _nzmax;
};

#endif  // SPAMS_B200_LINALG_H
