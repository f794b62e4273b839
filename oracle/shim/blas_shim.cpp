// Test infrastructure (oracle only): the three Fortran BLAS routines the
// reference defmm reaches on its matvec path (dgemm_, zgemm_, zgemv_; call
// sites include/gaia/gaia_blas3.hpp:41-96 and gaia_blas2.hpp:41-74), written
// from the BLAS reference definitions (column-major, C = alpha*op(A)*op(B) +
// beta*C; y = alpha*op(A)*x + beta*y).  No system BLAS exists in this image.
// Only the non-transposed forms are implemented; any other form aborts, so a
// silent mismatch with the reference's calls cannot happen.
#include <complex>
#include <cstdlib>

namespace {

template <typename T, typename I>
void gemm_nn(const char* ta, const char* tb, const I* m_, const I* n_,
             const I* k_, const T* alpha, const T* A, const I* lda_,
             const T* B, const I* ldb_, const T* beta, T* C, const I* ldc_) {
  if ((*ta != 'N' && *ta != 'n') || (*tb != 'N' && *tb != 'n')) std::abort();
  const long m = (long)*m_, n = (long)*n_, k = (long)*k_;
  const long lda = (long)*lda_, ldb = (long)*ldb_, ldc = (long)*ldc_;
  const T a = *alpha, b = *beta;
  for (long j = 0; j < n; ++j) {
    T* c = C + j * ldc;
    if (b == T(0)) {
      for (long i = 0; i < m; ++i) c[i] = T(0);
    } else if (b != T(1)) {
      for (long i = 0; i < m; ++i) c[i] *= b;
    }
    for (long p = 0; p < k; ++p) {
      const T s = a * B[p + j * ldb];
      const T* ac = A + p * lda;
      for (long i = 0; i < m; ++i) c[i] += ac[i] * s;
    }
  }
}

}  // namespace

extern "C" {

void dgemm_(const char* ta, const char* tb, const unsigned* m,
            const unsigned* n, const unsigned* k, const double* alpha,
            const double* A, const unsigned* lda, const double* B,
            const unsigned* ldb, const double* beta, double* C,
            const unsigned* ldc) {
  gemm_nn<double, unsigned>(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C,
                            ldc);
}

void zgemm_(const char* ta, const char* tb, const unsigned* m,
            const unsigned* n, const unsigned* k,
            const std::complex<double>* alpha, const std::complex<double>* A,
            const unsigned* lda, const std::complex<double>* B,
            const unsigned* ldb, const std::complex<double>* beta,
            std::complex<double>* C, const unsigned* ldc) {
  gemm_nn<std::complex<double>, unsigned>(ta, tb, m, n, k, alpha, A, lda, B,
                                          ldb, beta, C, ldc);
}

void zgemv_(const char* trans, const int* m_, const int* n_,
            const std::complex<double>* alpha, const std::complex<double>* A,
            const int* lda_, const std::complex<double>* x, const int* incx_,
            const std::complex<double>* beta, std::complex<double>* y,
            const int* incy_) {
  if (*trans != 'N' && *trans != 'n') std::abort();
  const long m = *m_, n = *n_, lda = *lda_, incx = *incx_, incy = *incy_;
  const std::complex<double> a = *alpha, b = *beta;
  for (long i = 0; i < m; ++i) {
    if (b == 0.0)
      y[i * incy] = 0.0;
    else if (b != 1.0)
      y[i * incy] *= b;
  }
  for (long j = 0; j < n; ++j) {
    const std::complex<double> s = a * x[j * incx];
    const std::complex<double>* ac = A + j * lda;
    for (long i = 0; i < m; ++i) y[i * incy] += ac[i] * s;
  }
}

}  // extern "C"
