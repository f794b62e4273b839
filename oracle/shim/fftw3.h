/*
 * Test infrastructure (oracle only): the subset of the FFTW3 C API that the
 * reference defmm calls, so that its unmodified headers compile here without
 * libfftw3.  FFTW3 itself (unpinned `-lfftw3` in the reference's makefile:7)
 * is absent from this image.
 *
 * Call sites in the reference: include/thetis/titan_dft.hpp:39-232,
 * include/calculus/circulant.hpp:60-71 and :103-113,
 * include/traversals/m2fpass.hpp:72-104.
 *
 * Semantics restated from FFTW's published definition: the forward transform
 * (sign -1) is Y[k] = sum_j X[j] exp(-2 pi i j k / n), the backward transform
 * (sign +1) uses exp(+2 pi i j k / n); neither is normalised; multi-dimensional
 * arrays are row-major (last index fastest).
 */
#ifndef DEFMM_ORACLE_FFTW3_SHIM_H
#define DEFMM_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct oracle_fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft(int rank, const int* n, fftw_complex* in,
                        fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany,
                             fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed,
                             int ostride, int odist, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
