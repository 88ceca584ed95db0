/* FFTW-API shim for building the reference CPU code without FFTW.
 *
 * Test infrastructure only: this header lets the reference's own FFT wrapper
 * (src/base/fft.hh:18-57, src/base/fft.cc:15-38) compile against a
 * project-written FP64 power-of-two complex FFT (fftw_shim.c). It declares
 * exactly the FFTW3 calls the reference makes and nothing else.
 *
 * Semantics follow the FFTW3 manual: fftw_plan_dft is a row-major
 * (last axis fastest), unnormalised complex DFT with sign -1 (forward) or +1
 * (backward); in and out may alias.
 */
#ifndef CONAN_FFTW_SHIM_H
#define CONAN_FFTW_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct conan_shim_plan *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void *fftw_malloc(size_t n);
void fftw_free(void *p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
fftw_plan fftw_plan_dft(int rank, const int *n, fftw_complex *in,
                        fftw_complex *out, int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
/* The reference's allocator passes a const hint pointer (src/base/fft.hh:33). */
inline void fftw_free(const void *p) { fftw_free(const_cast<void *>(p)); }
#endif

#endif
