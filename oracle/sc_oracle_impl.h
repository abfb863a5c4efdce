/* Test infrastructure only (the oracle): a plain-C restatement of the SPAMS
 * reference's OMP and LARS-Lasso coding path, used by tests/ and by bench.py's
 * CPU-baseline leg as the checker.  The shipped engine never links it.
 *
 * This file is included twice by sc_oracle.c, once with T=double/SUF=f64 and
 * once with T=float/SUF=f32, so every routine exists in both precisions like
 * the reference's templates.  Loops replace the reference's BLAS calls, so
 * low-order bits can differ from a BLAS build (summation order); the control
 * flow, stopping rules and tie-breaks are the reference's.
 */
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define F(name) CAT(name, SUF)
/* MIN macro of linalg/utils.h:46 (a NaN first argument is kept). */
#define ORC_MIN(a, b) (((a) > (b)) ? (b) : (a))

/* cblas_iamax semantics (linalg/cblas_alt_template.h:787-797 -> BLAS i?amax):
 * first index of the largest magnitude. */
static int F(orc_iamax)(int n, const T* x) {
  int best = 0;
  T bv = n > 0 ? (T)fabs((double)x[0]) : 0;
  for (int j = 1; j < n; ++j) {
    T v = (T)fabs((double)x[j]);
    if (v > bv) { bv = v; best = j; }
  }
  return best;
}

/* Vector<T>::max (linalg/linalg.h:2769-2780): first index of the largest value. */
static int F(orc_argmax)(int n, const T* x) {
  int best = 0;
  T bv = x[0];
  for (int j = 1; j < n; ++j)
    if (x[j] > bv) { bv = x[j]; best = j; }
  return best;
}

/* The reference's own cblas_iamin (linalg/cblas_alt_template.h:1094-1105):
 * first index of the smallest magnitude, comparisons in double. */
static int F(orc_iamin)(int n, const T* x) {
  int imin = 0;
  double mn = fabs((double)x[0]);
  for (int j = 1; j < n; ++j) {
    double cur = fabs((double)x[j]);
    if (cur < mn) { imin = j; mn = cur; }
  }
  return imin;
}

/* x[0:n] <- U[0:n,0:n] x, U upper triangular, column-major with leading
 * dimension ld (BLAS trmv Upper/NoTrans/NonUnit). */
static void F(orc_trmv_upper)(int n, const T* U, int ld, T* x) {
  for (int r = 0; r < n; ++r) {
    T s = 0;
    for (int k = r; k < n; ++k) s += U[r + (size_t)k * ld] * x[k];
    x[r] = s;
  }
}

/* y = A x for symmetric A of order n stored in its upper triangle
 * (BLAS symv Upper). */
static void F(orc_symv_upper)(int n, const T* A, int ld, const T* x, T* y) {
  for (int r = 0; r < n; ++r) {
    T s = 0;
    for (int c = 0; c < n; ++c) {
      const T a = r <= c ? A[r + (size_t)c * ld] : A[c + (size_t)r * ld];
      s += a * x[c];
    }
    y[r] = s;
  }
}

/* A += alpha x x^T on the upper triangle (BLAS syr Upper). */
static void F(orc_syr_upper)(int n, T alpha, const T* x, T* A, int ld) {
  for (int c = 0; c < n; ++c) {
    const T t = alpha * x[c];
    for (int r = 0; r <= c; ++r) A[r + (size_t)c * ld] += t * x[r];
  }
}

/* G = D^T D (+ ridge on the diagonal): Matrix::XtX (linalg/linalg.h:1967-1972)
 * followed by ProdMatrix::addDiag when ridge != 0. */
void F(orc_gram)(const T* D, int m, int K, T ridge, T* G) {
  for (int a = 0; a < K; ++a)
    for (int b = a; b < K; ++b) {
      T s = 0;
      for (int r = 0; r < m; ++r) s += D[r + (size_t)a * m] * D[r + (size_t)b * m];
      G[a + (size_t)b * K] = s;
      G[b + (size_t)a * K] = s;
    }
  if (ridge != 0)
    for (int a = 0; a < K; ++a) G[a + (size_t)a * K] += ridge;
}

/* y = D^T x (Matrix::multTrans, linalg/linalg.h:1751-1756). */
static void F(orc_dtx)(const T* D, int m, int K, const T* x, T* y) {
  for (int k = 0; k < K; ++k) {
    T s = 0;
    for (int r = 0; r < m; ++r) s += D[r + (size_t)k * m] * x[r];
    y[k] = s;
  }
}

/* coreORMP (decomp/decomp.h:538-640) for one signal.
 *   Rdn:  D^T x on entry (overwritten with the residual correlations)
 *   Lcap: the driver's clamped L (Gs.n() in the reference); L: this signal's L
 *   ind:  Lcap entries, -1 terminated on return; RUn: Lcap coefficients
 *   path: K x Lcap or NULL
 * Returns the number of selected atoms. */
int F(orc_omp_signal)(const T* G, int K, T* Rdn, T normX, int Lcap, int Lsig,
                      T eps_in, T lambda, int* ind, T* RUn, T* path) {
  const T eps = (T)fabs((double)eps_in);
  const int L = Lsig < Lcap ? Lsig : Lcap;
  for (int j = 0; j < Lcap; ++j) { ind[j] = -1; RUn[j] = 0; }
  /* L < 0 reaches undefined behaviour in the reference (negative memset
   * when a path is requested); it selects nothing otherwise. */
  if (normX <= eps || L <= 0) return 0;
  T* scores = (T*)malloc(sizeof(T) * K);
  T* norm = (T*)malloc(sizeof(T) * K);
  T* Un = (T*)calloc((size_t)L * L, sizeof(T));
  T* Undn = (T*)calloc((size_t)K * L, sizeof(T));
  for (int k = 0; k < K; ++k) { scores[k] = Rdn[k]; norm[k] = 1; }
  if (path) memset(path, 0, sizeof(T) * (size_t)K * L);
  int j;
  for (j = 0; j < L; ++j) {
    const int c = F(orc_iamax)(K, scores);
    if (norm[c] < 1e-8) { ind[j] = -1; break; }
    const T invNorm = (T)1.0 / (T)sqrt((double)norm[c]);
    const T RU = Rdn[c] * invNorm;
    const T delta = RU * RU;
    if (delta < 2 * lambda) break;
    RUn[j] = RU;
    normX -= delta;
    ind[j] = c;
    /* new inverse-Cholesky column: Un[:,j] = invNorm [ -Un_j Undn[c,0:j] ; 1 ] */
    T* col = Un + (size_t)j * L;
    col[j] = -1;
    for (int k = 0; k < j; ++k) col[k] = Undn[c + (size_t)k * K];
    F(orc_trmv_upper)(j, Un, L, col);
    for (int k = 0; k <= j; ++k) col[k] *= -invNorm;
    if (j == L - 1 || normX <= eps) { ++j; break; }
    if (path) {
      T* last = path + (size_t)(L - 1) * K;
      for (int k = 0; k <= j; ++k) last[k] = RUn[k];
      F(orc_trmv_upper)(j + 1, Un, L, last);
      for (int k = 0; k <= j; ++k) path[(size_t)j * K + ind[k]] = last[k];
    }
    /* Undn[:,j] = G[:, ind[0:j+1]] Un[0:j+1, j] */
    T* und = Undn + (size_t)j * K;
    for (int r = 0; r < K; ++r) {
      T s = 0;
      for (int k = 0; k <= j; ++k) s += G[r + (size_t)ind[k] * K] * col[k];
      und[r] = s;
    }
    for (int r = 0; r < K; ++r) {
      Rdn[r] += und[r] * (-RUn[j]);
      norm[r] -= und[r] * und[r];
      scores[r] = (Rdn[r] * Rdn[r]) / norm[r];
    }
    for (int k = 0; k <= j; ++k) scores[ind[k]] = 0;
  }
  F(orc_trmv_upper)(j, Un, L, RUn);
  if (path) {
    memset(path + (size_t)(L - 1) * K, 0, sizeof(T) * L);
    for (int k = 0; k < j; ++k) path[(size_t)(j - 1) * K + ind[k]] = RUn[k];
  }
  free(scores); free(norm); free(Un); free(Undn);
  return j;
}

/* coreLARS2 (decomp/decomp.h:1706-1915) for one signal.
 *   DtR: D^T x on entry (overwritten);  G includes the ridge.
 *   LL:  the driver's L;  coeffs/ind: LL entries.
 *   path: K x length_path or NULL.  Returns the number of active atoms. */
int F(orc_lars_signal)(const T* G, int K, T* DtR, T normX, int LL, int mode,
                       T constraint, int pos, int length_path, int* ind,
                       T* coeffs, T* path) {
  const int L = LL < K ? LL : K;
  if (length_path <= 1) length_path = 4 * L;
  for (int j = 0; j < LL; ++j) { coeffs[j] = 0; ind[j] = -1; }
  if (L <= 0) return 0;
  int cur = pos ? F(orc_argmax)(K, DtR) : F(orc_iamax)(K, DtR);
  if (mode == 2 && fabs((double)DtR[cur]) < constraint) return 0;
  if (mode == 1 && normX < constraint) return 0;
  T* Gs = (T*)calloc((size_t)LL * LL, sizeof(T));
  T* invGs = (T*)calloc((size_t)LL * LL, sizeof(T));
  T* Ga = (T*)calloc((size_t)K * LL, sizeof(T));
  T* work = (T*)calloc((size_t)K * 3, sizeof(T));
  T* u = (T*)calloc((size_t)K, sizeof(T));
  const T INF = (T)INFINITY;
  int newAtom = 1, i, iter = 0;
  T thrs = 0;
  for (i = 0; i < L; ++i) {
    ++iter;
    if (newAtom) {
      ind[i] = cur;
      memcpy(Ga + (size_t)i * K, G + (size_t)cur * K, sizeof(T) * K);
      for (int j = 0; j <= i; ++j) Gs[(size_t)i * LL + j] = Ga[(size_t)i * K + ind[j]];
      if (i == 0) {
        invGs[0] = (T)1.0 / Gs[0];
      } else {
        F(orc_symv_upper)(i, invGs, LL, Gs + (size_t)i * LL, u);
        T d = 0;
        for (int j = 0; j < i; ++j) d += u[j] * Gs[(size_t)i * LL + j];
        const T schur = (T)1.0 / (Gs[(size_t)i * LL + i] - d);
        invGs[(size_t)i * LL + i] = schur;
        for (int j = 0; j < i; ++j) invGs[(size_t)i * LL + j] = -schur * u[j];
        F(orc_syr_upper)(i, schur, u, invGs, LL);
      }
    }
    for (int j = 0; j <= i; ++j) work[j] = DtR[ind[j]] > 0 ? (T)1.0 : (T)-1.0;
    F(orc_symv_upper)(i + 1, invGs, LL, work, u);
    T step_max = INF;
    int first_zero = -1;
    for (int j = 0; j <= i; ++j) {
      const T ratio = -coeffs[j] / u[j];
      if (ratio > 0 && ratio <= step_max) { step_max = ratio; first_zero = j; }
    }
    const T C = (T)fabs((double)DtR[ind[0]]);
    T* A = work + 2 * (size_t)K;
    for (int r = 0; r < K; ++r) {
      T s = 0;
      for (int j = 0; j <= i; ++j) s += Ga[r + (size_t)j * K] * u[j];
      A[r] = s;
    }
    for (int r = 0; r < K; ++r) { work[r] = A[r]; work[r + K] = A[r]; }
    for (int j = 0; j <= i; ++j) { work[ind[j]] = INF; work[ind[j] + K] = INF; }
    for (int r = 0; r < K; ++r)
      work[r] = (work[r] < INF && work[r] > (T)-1.0) ? (DtR[r] + C) / ((T)1.0 + work[r]) : INF;
    for (int r = 0; r < K; ++r)
      work[r + K] = (work[r + K] < INF && work[r + K] < (T)1.0) ? (C - DtR[r]) / ((T)1.0 - work[r + K]) : INF;
    if (pos)
      for (int r = 0; r < K; ++r) work[r] = INF;
    const int index = F(orc_iamin)(2 * K, work);
    T step = work[index];
    cur = index % K;
    T coeff1 = 0, coeff2 = 0;
    for (int j = 0; j <= i; ++j) coeff1 += DtR[ind[j]] > 0 ? u[j] : -u[j];
    for (int j = 0; j <= i; ++j) coeff2 += DtR[ind[j]] * u[j];
    const T coeff3 = normX - constraint;
    T step_max2;
    if (mode == 2) {
      step_max2 = C - constraint;
    } else if (mode == 1) {
      const T delta = coeff2 * coeff2 - coeff1 * coeff3;
      step_max2 = delta < 0 ? INF : (coeff2 - (T)sqrt((double)delta)) / coeff1;
      step_max2 = ORC_MIN(C, step_max2);
    } else {
      step_max2 = coeff1 < 0 ? INF : (constraint - thrs) / coeff1;
      step_max2 = ORC_MIN(C, step_max2);
    }
    step = ORC_MIN(ORC_MIN(step, step_max2), step_max);
    if (step == INF) break;
    for (int j = 0; j <= i; ++j) coeffs[j] += step * u[j];
    if (pos)
      for (int j = 0; j <= i; ++j) if (coeffs[j] < 0) coeffs[j] = 0;
    for (int r = 0; r < K; ++r) DtR[r] += (-step) * A[r];
    normX += coeff1 * step * step - 2 * coeff2 * step;
    thrs += step * coeff1;
    if (path)
      for (int k = 0; k <= i; ++k) path[(size_t)iter * K + ind[k]] = coeffs[k];
    if (step == step_max) {
      const int fz = first_zero;
      for (int j = fz; j < i; ++j) {
        memcpy(Ga + (size_t)j * K, Ga + (size_t)(j + 1) * K, sizeof(T) * K);
        ind[j] = ind[j + 1];
        coeffs[j] = coeffs[j + 1];
      }
      ind[i] = -1;
      coeffs[i] = 0;
      for (int j = fz; j < i; ++j) {
        memmove(Gs + (size_t)j * LL, Gs + (size_t)(j + 1) * LL, sizeof(T) * fz);
        memmove(Gs + (size_t)j * LL + fz, Gs + (size_t)(j + 1) * LL + fz + 1, sizeof(T) * (i - fz));
      }
      const T schur = invGs[(size_t)fz * LL + fz];
      for (int j = 0; j < fz; ++j) u[j] = invGs[(size_t)fz * LL + j];
      for (int j = fz; j < i; ++j) u[j] = invGs[(size_t)(j + 1) * LL + fz];
      for (int j = fz; j < i; ++j) {
        memmove(invGs + (size_t)j * LL, invGs + (size_t)(j + 1) * LL, sizeof(T) * fz);
        memmove(invGs + (size_t)j * LL + fz, invGs + (size_t)(j + 1) * LL + fz + 1, sizeof(T) * (i - fz));
      }
      F(orc_syr_upper)(i, (T)-1.0 / schur, u, invGs, LL);
      newAtom = 0;
      i = i - 2;
    } else {
      newAtom = 1;
    }
    if ((iter >= length_path - 1) || fabs((double)step) < 1e-15 || step == step_max2 ||
        (normX < 1e-15) || (i == (L - 1)) ||
        (mode == 1 && normX - constraint < 1e-15) ||
        (mode == 0 && (constraint - thrs < 1e-15)))
      break;
  }
  free(Gs); free(invGs); free(Ga); free(work); free(u);
  int cnt = 0;
  while (cnt < LL && ind[cnt] >= 0) ++cnt;
  return cnt;
}

/* downDateLasso (decomp/decomp.h:1096-1203): drop position mb of the
 * active set 0..*j of coreLARS's state (all L x L matrices column-major with
 * leading dimension LL, Gs K x LL).  Decrements *j. */
static void F(orc_chol_downdate)(int* pj, int mb, T* normX, int ols, int pos, T* Rdn, int* ind,
                                 T* coeffs, T* sig, T* av, T* Xdn, T* RUn, T* Un, T* Gs,
                                 T* Gsa, T* Unds, T* R, int LL, int K) {
  const int j = *pj;
  const int L = LL;
  const int indB = ind[mb];
  if (!pos && sig[mb] < 0) {
    Rdn[indB] = -Rdn[indB];
    if (ols) Xdn[indB] = -Xdn[indB];
  }
  const int num = j - mb;
  for (int k = 0; k < num * num; ++k) R[k] = 0;
  for (int k = 0; k < num; ++k) R[k * num + k] = 1;
  for (int k = mb + 1; k <= j; ++k) {
    const T a = -Un[k * L + mb] / Un[mb * L + mb];
    av[k - mb - 1] = a;
    for (int r = 0; r < mb; ++r) Un[k * L + r] += a * Un[mb * L + r];
  }
  for (int k = mb + 1; k <= j; ++k) {
    for (int r = 0; r < mb; ++r) Un[(k - 1) * L + r] = Un[k * L + r];
    for (int r = 0; r < num; ++r) Un[(k - 1) * L + mb + r] = Un[k * L + mb + 1 + r];
  }
  T alpha = 1, alphab, gamma;
  for (int k = 0; k < num; ++k) {
    alphab = alpha + av[k] * av[k];
    R[k * num + k] = (T)sqrt((double)(alphab / alpha));
    gamma = av[k] * R[k * num + k] / alphab;
    alpha = alphab;
    for (int r = k + 1; r < num; ++r) R[k * num + r] = gamma * av[r];
  }
  if (num > 0) {
    /* trtri(lower, non-unit): R <- R^-1, column by column */
    for (int k = 0; k < num; ++k) {
      R[k * num + k] = (T)1.0 / R[k * num + k];
      for (int r = k + 1; r < num; ++r) {
        T s2 = 0;
        for (int q = k; q < r; ++q) s2 += R[q * num + r] * R[k * num + q];
        R[k * num + r] = -s2 / R[r * num + r];
      }
    }
    /* trmm(Right, Lower, Trans): Un(0:j, mb:mb+num) <- Un(0:j, mb:mb+num) R^T */
    for (int r = 0; r < j; ++r)
      for (int c = num - 1; c >= 0; --c) {
        T s2 = 0;
        for (int q = 0; q <= c; ++q) s2 += Un[(mb + q) * L + r] * R[q * num + c];
        Un[(mb + c) * L + r] = s2;
      }
  }
  /* Unds */
  for (int k = mb + 1; k <= j; ++k)
    for (int r = 0; r < j - mb; ++r) Unds[k * L + mb + 1 + r] += av[k - mb - 1] * Unds[mb * L + mb + 1 + r];
  for (int k = 0; k < mb; ++k)
    for (int l = mb + 1; l <= j; ++l) Unds[k * L + l - 1] = Unds[k * L + l];
  for (int k = mb + 1; k <= j; ++k)
    for (int r = 0; r < j - mb; ++r) Unds[(k - 1) * L + mb + r] = Unds[k * L + mb + 1 + r];
  if (num > 0) {
    /* trmm(Right, Lower, Trans) on Unds(mb:j, mb:mb+num), j - mb rows */
    for (int r = 0; r < j - mb; ++r)
      for (int c = num - 1; c >= 0; --c) {
        T s2 = 0;
        for (int q = 0; q <= c; ++q) s2 += Unds[(mb + q) * L + mb + r] * R[q * num + c];
        Unds[(mb + c) * L + mb + r] = s2;
      }
  }
  for (int k = mb + 1; k <= j; ++k)
    for (int l = 0; l < k; ++l) Unds[k * L + l] = 0;
  /* Gs */
  for (int k = mb + 1; k <= j; ++k) memcpy(Gs + (size_t)(k - 1) * K, Gs + (size_t)k * K, sizeof(T) * K);
  if (!pos && sig[mb] < 0)
    for (int k = 0; k < j; ++k) Gs[(size_t)k * K + indB] = -Gs[(size_t)k * K + indB];
  /* Gsa */
  for (int k = mb + 1; k <= j; ++k) {
    for (int r = 0; r < mb; ++r) Gsa[(k - 1) * L + r] = Gsa[k * L + r];
    for (int r = 0; r < j - mb; ++r) Gsa[(k - 1) * L + mb + r] = Gsa[k * L + mb + 1 + r];
  }
  for (int k = 0; k < mb; ++k)
    for (int l = mb + 1; l <= j; ++l) Gsa[k * L + l - 1] = Gsa[k * L + l];
  for (int k = mb + 1; k <= j && !pos; ++k) sig[k - 1] = sig[k];
  for (int k = mb + 1; k <= j; ++k) ind[k - 1] = ind[k];
  ind[j] = -1;
  for (int k = mb + 1; k <= j; ++k) coeffs[k - 1] = coeffs[k];
  coeffs[j] = 0;
  if (ols) {
    for (int k = mb; k <= j; ++k) *normX += RUn[k] * RUn[k];
    for (int k = mb; k < j; ++k) {
      RUn[k] = 0;
      for (int l = 0; l <= k; ++l) RUn[k] += Xdn[ind[l]] * Un[k * L + l];
      *normX -= RUn[k] * RUn[k];
    }
  }
  *pj = j - 1;
}

/* coreLARS (decomp/decomp.h:844-1093), the Cholesky implementation of the
 * Lasso homotopy, for one signal: Rdn (K) = D^T x on entry (overwritten),
 * ind / coeffs (LL) out, -1 terminated; returns the number of entries. */
int F(orc_larschol_signal)(const T* G, int K, T* Rdn, T normX, int LL, int mode, T constraint,
                           int pos, int ols, int length_path, int* ind, T* coeffs, T* path) {
  for (int k = 0; k < LL; ++k) { coeffs[k] = 0; ind[k] = -1; }
  if (mode == 1 && normX < constraint) return 0;
  const int L = ORC_MIN(LL, K);
  if (length_path <= 1) length_path = 4 * L;
  const int Lm = LL;  /* leading dimension of the L x L state */
  T* Xdn = (T*)calloc((size_t)K, sizeof(T));
  T* A = (T*)calloc((size_t)K, sizeof(T));
  T* u = (T*)calloc((size_t)Lm, sizeof(T));
  T* sig = (T*)calloc((size_t)Lm, sizeof(T));
  T* av = (T*)calloc((size_t)Lm, sizeof(T));
  T* RUn = (T*)calloc((size_t)Lm, sizeof(T));
  T* Un = (T*)calloc((size_t)Lm * Lm, sizeof(T));
  T* Unds = (T*)calloc((size_t)Lm * Lm, sizeof(T));
  T* Gs = (T*)calloc((size_t)K * Lm, sizeof(T));
  T* Gsa = (T*)calloc((size_t)Lm * Lm, sizeof(T));
  T* work = (T*)calloc((size_t)2 * K + Lm, sizeof(T));
  T* R = (T*)calloc((size_t)Lm * Lm, sizeof(T));
  const T INF = (T)INFINITY;
  if (ols) memcpy(Xdn, Rdn, sizeof(T) * K);
  int cur = pos ? F(orc_argmax)(K, Rdn) : F(orc_iamax)(K, Rdn);
  int newAtom = 1, iter = 1, j;
  T Cmax = 0, thrs = 0;
  for (j = 0; j < L; ++j) {
    if (newAtom) {
      ind[j] = cur;
      if (pos) { Cmax = Rdn[cur]; sig[j] = 1; }
      else { Cmax = (T)fabs((double)Rdn[cur]); sig[j] = Rdn[cur] < 0 ? (T)-1.0 : (T)1.0; }
      for (int k = 0; k <= j; ++k) Un[j * Lm + k] = 0;
      Un[j * Lm + j] = 1;
      memcpy(Gs + (size_t)K * j, G + (size_t)cur * K, sizeof(T) * K);
      for (int k = 0; k < j; ++k) Gs[(size_t)K * j + ind[k]] *= sig[k];
      if (sig[j] < 0) {
        Rdn[cur] = -Rdn[cur];
        if (ols) Xdn[cur] = -Xdn[cur];
        for (int r = 0; r < K; ++r) Gs[(size_t)K * j + r] *= sig[j];
        for (int k = 0; k <= j; ++k) Gs[cur + (size_t)K * k] *= sig[j];
      }
      for (int k = 0; k <= j; ++k) Gsa[j * Lm + k] = Gs[cur + (size_t)K * k];
      for (int k = 0; k < j; ++k) Gsa[k * Lm + j] = Gsa[j * Lm + k];
      for (int k = 0; k < j; ++k) Unds[k * Lm + j] = Gsa[j * Lm + k];
      /* trmv(Upper, Trans, j + 1) on Unds row j (stride Lm) */
      for (int k = j; k >= 0; --k) {
        T s2 = 0;
        for (int l = 0; l <= k; ++l) s2 += Un[k * Lm + l] * Unds[l * Lm + j];
        work[k] = s2;
      }
      for (int k = 0; k <= j; ++k) Unds[k * Lm + j] = work[k];
      T norm2 = Gsa[j * Lm + j];
      for (int k = 0; k < j; ++k) norm2 -= Unds[k * Lm + j] * Unds[k * Lm + j];
      if (norm2 < 1e-15) { ind[j] = -1; break; }
      Un[j * Lm + j] = -1;
      for (int k = 0; k < j; ++k) Un[j * Lm + k] = Unds[k * Lm + j];
      /* trmv(Upper, NoTrans, j) on Un(0:j, j) */
      for (int r = 0; r < j; ++r) {
        T s2 = 0;
        for (int k = r; k < j; ++k) s2 += Un[k * Lm + r] * Un[j * Lm + k];
        work[r] = s2;
      }
      for (int r = 0; r < j; ++r) Un[j * Lm + r] = work[r];
      const T invNorm = (T)1.0 / (T)sqrt((double)norm2);
      for (int k = 0; k <= j; ++k) Un[j * Lm + k] *= -invNorm;
      T d = 0;
      for (int k = 0; k <= j; ++k) d += Un[j * Lm + k] * Gsa[j * Lm + k];
      Unds[j * Lm + j] = d;
    }
    /* direction: w = Un^T 1, a = 1 / ||w||, u = a Un w */
    for (int k = j; k >= 0; --k) {
      T s2 = 0;
      for (int l = 0; l <= k; ++l) s2 += Un[k * Lm + l];
      u[k] = s2;
    }
    T nr = 0;
    for (int k = 0; k <= j; ++k) nr += u[k] * u[k];
    const T a = (T)1.0 / (T)sqrt((double)nr);
    for (int r = 0; r <= j; ++r) {
      T s2 = 0;
      for (int k = r; k <= j; ++k) s2 += Un[k * Lm + r] * u[k];
      work[r] = s2;
    }
    for (int r = 0; r <= j; ++r) u[r] = a * work[r];
    for (int r = 0; r < K; ++r) {
      T s2 = 0;
      for (int k = 0; k <= j; ++k) s2 += Gs[r + (size_t)K * k] * u[k];
      A[r] = s2;
    }
    T potentNorm = 0;
    if (!ols)
      for (int k = 0; k <= j; ++k) potentNorm += Rdn[ind[k]] * u[k];
    if (pos) {
      for (int k = 0; k < K; ++k) {
        const T diff = a - A[k];
        work[k] = diff <= 0 ? INF : (Cmax - Rdn[k]) / diff;
      }
      for (int k = 0; k <= j; ++k) work[ind[k]] = INF;
      for (int k = 0; k < K; ++k) if (work[k] <= 0) work[k] = INF;
      cur = F(orc_iamin)(K, work);
    } else {
      memset(work, 0, sizeof(T) * 2 * K);
      for (int k = 0; k <= j; ++k) { work[2 * ind[k]] = INF; work[2 * ind[k] + 1] = INF; }
      for (int k = 0; k < K; ++k) {
        if (!work[2 * k]) {
          const T d1 = a - A[k];
          work[2 * k] = d1 <= 0 ? INF : (Cmax - Rdn[k]) / d1;
          const T d2 = a + A[k];
          work[2 * k + 1] = d2 <= 0 ? INF : (Cmax + Rdn[k]) / d2;
        }
      }
      cur = F(orc_iamin)(2 * K, work);
    }
    T gamma = work[cur];
    T gammaMin = 0;
    int minBasis = 0;
    if (mode == 2) gamma = ORC_MIN(gamma, (Cmax - constraint) / a);
    for (int k = 0; k <= j; ++k) work[k] = -(coeffs[k] / u[k]);
    for (int k = 0; k <= j; ++k) if (coeffs[k] == 0 || work[k] <= 0) work[k] = INF;
    minBasis = F(orc_iamin)(j + 1, work);
    gammaMin = work[minBasis];
    if (gammaMin < gamma) gamma = gammaMin;
    if (mode == 0) {
      T Tu = 0;
      for (int k = 0; k <= j; ++k) Tu += u[k];
      if (Tu > 10e-10) gamma = ORC_MIN(gamma, (constraint - thrs) / Tu);
      thrs += gamma * Tu;
    }
    if (!ols) {
      const T t = gamma * gamma - 2 * gamma * potentNorm;
      if (t > 0 || isnan((double)t) || isinf((double)t)) { ind[j] = -1; break; }
      normX += t;
    } else if (newAtom) {
      RUn[j] = 0;
      for (int k = 0; k <= j; ++k) RUn[j] += Xdn[ind[k]] * Un[j * Lm + k];
      normX -= RUn[j] * RUn[j];
    }
    for (int k = 0; k <= j; ++k) coeffs[k] += gamma * u[k];
    if (pos)
      for (int k = 0; k <= j; ++k) if (coeffs[k] < 0) coeffs[k] = 0;
    for (int r = 0; r < K; ++r) Rdn[r] += (-gamma) * A[r];
    if (!pos) cur /= 2;
    if (path)
      for (int k = 0; k <= j; ++k) path[(size_t)iter * K + ind[k]] = coeffs[k] * sig[k];
    if (gamma == gammaMin) {
      F(orc_chol_downdate)(&j, minBasis, &normX, ols, pos, Rdn, ind, coeffs, sig, av, Xdn, RUn,
                           Un, Gs, Gsa, Unds, R, Lm, K);
      newAtom = 0;
      Cmax = (T)fabs((double)Rdn[ind[0]]);
      --j;
    } else {
      newAtom = 1;
    }
    ++iter;
    if (mode == 2) thrs = (T)fabs((double)Rdn[ind[0]]);
    if ((j == L - 1) || (mode == 2 && (thrs - constraint < 1e-15)) ||
        (mode == 0 && (thrs - constraint > -1e-15)) ||
        (newAtom && mode == 1 && (normX - constraint < 1e-15)) || (normX < 1e-15) ||
        (iter >= length_path))
      break;
  }
  if (ols) {
    for (int r = 0; r <= j; ++r) {
      T s2 = 0;
      for (int k = r; k <= j; ++k) s2 += Un[k * Lm + r] * RUn[k];
      work[r] = s2;
    }
    for (int r = 0; r <= j; ++r) coeffs[r] = work[r];
  }
  for (int k = 0; k <= j && k < LL; ++k) coeffs[k] *= sig[k];
  free(Xdn); free(A); free(u); free(sig); free(av); free(RUn); free(Un); free(Unds); free(Gs);
  free(Gsa); free(work); free(R);
  int cnt = 0;
  while (cnt < LL && ind[cnt] >= 0) ++cnt;
  return cnt;
}

/* lasso<T> with cholesky / ols (decomp/decomp.h:735-842): Gram with the
 * ridge max(lambda2, 1e-10), or the caller's Q and q (Q used as given). */
void F(orc_lasso_chol)(const T* X, int m, int64_t n, const T* D, const T* Q, const T* q, int K,
                       int L, T lambda1, T lambda2, int mode, int pos, int ols, int length_path,
                       T* vM, int* rM, T* path) {
  if (L <= 0) return;
  T* G = (T*)malloc(sizeof(T) * (size_t)K * K);
  T* Rdn = (T*)malloc(sizeof(T) * (size_t)K);
  if (Q) {
    memcpy(G, Q, sizeof(T) * (size_t)K * K);
  } else {
    const T ridge = lambda2 > (T)1e-10 ? lambda2 : (T)1e-10;
    F(orc_gram)(D, m, K, ridge, G);
  }
  for (int64_t i = 0; i < n; ++i) {
    const T* x = X + (size_t)i * m;
    T normX = 0;
    for (int r = 0; r < m; ++r) normX += x[r] * x[r];
    if (Q) memcpy(Rdn, q + (size_t)i * K, sizeof(T) * K);
    else F(orc_dtx)(D, m, K, x, Rdn);
    F(orc_larschol_signal)(G, K, Rdn, normX, L, mode, lambda1, pos, ols, length_path,
                           rM + (size_t)i * L, vM + (size_t)i * L, (path && i == 0) ? path : NULL);
  }
  free(G); free(Rdn);
}

/* SpMatrix::convert (linalg/linalg.h:4840-4861): dense L x n (value, row)
 * pairs, -1 terminated per column, to CSC with rows sorted ascending
 * (misc.h:137-166 quicksort; any correct sort gives the same result since
 * rows are distinct).  colptr has n+1 entries. */
int64_t F(orc_convert)(const T* vM, const int* rM, int L, int64_t n,
                       int64_t* colptr, int* rows, T* vals) {
  int64_t cnt = 0;
  for (int64_t i = 0; i < n; ++i) {
    colptr[i] = cnt;
    const int64_t beg = cnt;
    for (int j = 0; j < L; ++j) {
      const int r = rM[(size_t)i * L + j];
      if (r == -1) break;
      if (rows) {
        /* insertion into the sorted run [beg, cnt) */
        int64_t p = cnt;
        while (p > beg && rows[p - 1] > r) { rows[p] = rows[p - 1]; vals[p] = vals[p - 1]; --p; }
        rows[p] = r;
        vals[p] = vM[(size_t)i * L + j];
      }
      ++cnt;
    }
  }
  colptr[n] = cnt;
  return cnt;
}

/* omp<T> driver (decomp/decomp.h:322-404) with the _omp facade's defaults
 * (cpp_library/spams.h:250-293) already resolved by the caller:
 *   Lv/nL: scalar (nL == 1) or per-column L; likewise eps and lambda.
 * Writes vM (Lc x n) and rM (Lc x n) where Lc = the clamped L (returned). */
int F(orc_omp)(const T* X, int m, int64_t n, const T* D, int K, const int* Lv,
               int nL, const T* eps, int nEps, const T* lambda, int nLambda,
               T* vM, int* rM, T* path, int Lc_cap) {
  int L = Lv[0];
  if (nL > 1)
    for (int64_t i = 1; i < n; ++i) if (Lv[i] > L) L = Lv[i];
  if (L <= 0) return 0;
  if (L > K) L = K;
  if (L > m) L = m;
  if (Lc_cap > 0 && L > Lc_cap) return -1;
  T* G = (T*)malloc(sizeof(T) * (size_t)K * K);
  T* Rdn = (T*)malloc(sizeof(T) * (size_t)K);
  F(orc_gram)(D, m, K, 0, G);
  for (int64_t i = 0; i < n; ++i) {
    const T* x = X + (size_t)i * m;
    T normX = 0;
    for (int r = 0; r < m; ++r) normX += x[r] * x[r];
    F(orc_dtx)(D, m, K, x, Rdn);
    F(orc_omp_signal)(G, K, Rdn, normX, L, nL > 1 ? Lv[i] : Lv[0],
                      nEps > 1 ? eps[i] : eps[0], nLambda > 1 ? lambda[i] : lambda[0],
                      rM + (size_t)i * L, vM + (size_t)i * L, (path && i == 0) ? path : NULL);
  }
  free(G); free(Rdn);
  return L;
}

/* Facade clamps of _lassoD (cpp_library/spams.h:107-130): returns the L that
 * lasso2 receives and writes the path length through *max_length_path. */
int F(orc_lasso_clamp)(int m, int K, int L, T lambda1, T lambda2, int mode,
                       int pos, int* max_length_path) {
  if (L < 0) L = K;
  if (*max_length_path < 0) *max_length_path = 4 * L;
  if (L > m && !(mode == 2 && fabs((double)lambda1) < 1e-99 && !pos && lambda2 > 0)) L = m;
  if (L > K) L = K;
  return L;
}

/* lasso2<T>(X, D, ...) driver (decomp/decomp.h:1563-1646), L already clamped:
 * G = D^T D + max(lambda2, 1e-10) I, per-column D^T x, coreLARS2. */
void F(orc_lasso)(const T* X, int m, int64_t n, const T* D, int K, int L,
                  T lambda1, T lambda2, int mode, int pos, int length_path,
                  T* vM, int* rM, T* path) {
  if (L <= 0) return;
  T* G = (T*)malloc(sizeof(T) * (size_t)K * K);
  T* DtR = (T*)malloc(sizeof(T) * (size_t)K);
  const T ridge = lambda2 > (T)1e-10 ? lambda2 : (T)1e-10;
  F(orc_gram)(D, m, K, ridge, G);
  for (int64_t i = 0; i < n; ++i) {
    const T* x = X + (size_t)i * m;
    T normX = 0;
    for (int r = 0; r < m; ++r) normX += x[r] * x[r];
    F(orc_dtx)(D, m, K, x, DtR);
    F(orc_lars_signal)(G, K, DtR, normX, L, mode, lambda1, pos, length_path,
                       rM + (size_t)i * L, vM + (size_t)i * L, (path && i == 0) ? path : NULL);
  }
  free(G); free(DtR);
}

/* Vector::copyMask / Matrix::copyMask (linalg/linalg.h:4082-4107): the
 * observed rows of x and of D, compacted; returns their number. */
static int F(orc_copy_mask)(const T* D, int m, int K, const T* x, const unsigned char* b,
                            T* Dm, T* xm) {
  int count = 0;
  for (int r = 0; r < m; ++r) if (b[r]) xm[count++] = x[r];
  for (int k = 0; k < K; ++k) {
    int p = 0;
    for (int r = 0; r < m; ++r)
      if (b[r]) Dm[(size_t)k * count + p++] = D[(size_t)k * m + r];
  }
  return count;
}

/* omp_mask<T> driver (decomp/decomp.h:406-519), facade defaults resolved as
 * in orc_omp.  B: m x n bytes, nonzero = observed row.  A column with no
 * observed row keeps ind = -1 (empty); a full mask codes with D^T D; otherwise
 * the observed rows' Gram + 1e-10 I, eps scaled by count / m. */
int F(orc_omp_mask)(const T* X, int m, int64_t n, const T* D, int K, const unsigned char* B,
                    const int* Lv, int nL, const T* eps, int nEps, const T* lambda,
                    int nLambda, T* vM, int* rM, T* path) {
  int L = Lv[0];
  if (nL > 1)
    for (int64_t i = 1; i < n; ++i) if (Lv[i] > L) L = Lv[i];
  if (L <= 0) return 0;
  if (L > K) L = K;
  if (L > m) L = m;
  T* G = (T*)malloc(sizeof(T) * (size_t)K * K);
  T* Gm = (T*)malloc(sizeof(T) * (size_t)K * K);
  T* Rdn = (T*)malloc(sizeof(T) * (size_t)K);
  T* Dm = (T*)malloc(sizeof(T) * (size_t)m * K);
  T* xm = (T*)malloc(sizeof(T) * (size_t)m);
  F(orc_gram)(D, m, K, 0, G);
  for (int64_t i = 0; i < n; ++i) {
    const T* x = X + (size_t)i * m;
    const unsigned char* b = B + (size_t)i * m;
    int* ind = rM + (size_t)i * L;
    for (int j = 0; j < L; ++j) ind[j] = -1;
    int count = 0;
    for (int r = 0; r < m; ++r) count += b[r] != 0;
    if (count == 0) continue;
    const int Li = nL > 1 ? Lv[i] : Lv[0];
    const T ei = nEps > 1 ? eps[i] : eps[0];
    const T li = nLambda > 1 ? lambda[i] : lambda[0];
    T* pth = (path && i == 0) ? path : NULL;
    if (count == m) {
      T normX = 0;
      for (int r = 0; r < m; ++r) normX += x[r] * x[r];
      F(orc_dtx)(D, m, K, x, Rdn);
      F(orc_omp_signal)(G, K, Rdn, normX, L, Li, ei, li, ind, vM + (size_t)i * L, pth);
    } else {
      F(orc_copy_mask)(D, m, K, x, b, Dm, xm);
      T normX = 0;
      for (int r = 0; r < count; ++r) normX += xm[r] * xm[r];
      F(orc_dtx)(Dm, count, K, xm, Rdn);
      F(orc_gram)(Dm, count, K, (T)1e-10, Gm);
      const T eps_mask = ei * (T)count / (T)m;
      F(orc_omp_signal)(Gm, K, Rdn, normX, L, Li, eps_mask, li, ind, vM + (size_t)i * L, pth);
    }
  }
  free(G); free(Gm); free(Rdn); free(Dm); free(xm);
  return L;
}

/* lasso_mask<T> driver (decomp/decomp.h:1466-1561), L already clamped as in
 * _lassoMask.  rM must come zero-filled (Matrix::resize): a column with no
 * observed row is left untouched there, so convert turns it into L zero
 * entries at row 0, as the reference does.  Full masks code with
 * D^T D + ridge; others with the observed rows' Gram + ridge and, in PENALTY
 * and L2ERROR modes, the constraint scaled by count / m; coreLARS2 runs with
 * its default path length. */
void F(orc_lasso_mask)(const T* X, int m, int64_t n, const T* D, int K, const unsigned char* B,
                       int L, T lambda1, T lambda2, int mode, int pos, T* vM, int* rM) {
  if (L <= 0) return;
  const T ridge = lambda2 > (T)1e-10 ? lambda2 : (T)1e-10;
  T* G = (T*)malloc(sizeof(T) * (size_t)K * K);
  T* Gm = (T*)malloc(sizeof(T) * (size_t)K * K);
  T* DtR = (T*)malloc(sizeof(T) * (size_t)K);
  T* Dm = (T*)malloc(sizeof(T) * (size_t)m * K);
  T* xm = (T*)malloc(sizeof(T) * (size_t)m);
  F(orc_gram)(D, m, K, ridge, G);
  for (int64_t i = 0; i < n; ++i) {
    const T* x = X + (size_t)i * m;
    const unsigned char* b = B + (size_t)i * m;
    int count = 0;
    for (int r = 0; r < m; ++r) count += b[r] != 0;
    if (count == 0) continue;
    if (count == m) {
      T normX = 0;
      for (int r = 0; r < m; ++r) normX += x[r] * x[r];
      F(orc_dtx)(D, m, K, x, DtR);
      F(orc_lars_signal)(G, K, DtR, normX, L, mode, lambda1, pos, -1, rM + (size_t)i * L,
                         vM + (size_t)i * L, NULL);
    } else {
      F(orc_copy_mask)(D, m, K, x, b, Dm, xm);
      const T cm = (mode == 2 || mode == 1) ? lambda1 * (T)count / (T)m : lambda1;
      T normX = 0;
      for (int r = 0; r < count; ++r) normX += xm[r] * xm[r];
      F(orc_dtx)(Dm, count, K, xm, DtR);
      F(orc_gram)(Dm, count, K, ridge, Gm);
      F(orc_lars_signal)(Gm, K, DtR, normX, L, mode, cm, pos, -1, rM + (size_t)i * L,
                         vM + (size_t)i * L, NULL);
    }
  }
  free(G); free(Gm); free(DtR); free(Dm); free(xm);
}

#undef F
#undef ORC_MIN
#undef CAT
#undef CAT2
