/*
 * Compile-only stand-in for <fftw3.h> (FFTW 3 is not installed here), used ONLY to build
 * the reference's whole driver (tremor_main + the adaptive planner) as a test oracle.
 * The reference's FFT branch is kept off at run time with TREMOR_NO_FFT=1
 * (fft_fallback.cpp:115), so no transform below is ever executed; each one stops the
 * process if it is. Oracle infrastructure: nothing in the product library includes it.
 */
#ifndef TM_REF_SHIM_FFTW3_H
#define TM_REF_SHIM_FFTW3_H

#include <cstdio>
#include <cstdlib>

typedef double fftw_complex[2];
typedef struct tm_shim_fftw_plan_s *fftw_plan;

#define FFTW_ESTIMATE (1U << 6)

static inline double *fftw_alloc_real(size_t n) { return (double *)std::malloc(n * sizeof(double)); }
static inline fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)std::malloc(n * sizeof(fftw_complex)); }
static inline void fftw_free(void *p) { std::free(p); }

static inline void tm_shim_fftw_unavailable()
{
    std::fprintf(stderr, "fftw3 stand-in: FFTW is not available in this build (set TREMOR_NO_FFT=1)\n");
    std::abort();
}
static inline fftw_plan fftw_plan_dft_r2c_1d(int, double *, fftw_complex *, unsigned)
{
    tm_shim_fftw_unavailable();
    return nullptr;
}
static inline fftw_plan fftw_plan_dft_c2r_1d(int, fftw_complex *, double *, unsigned)
{
    tm_shim_fftw_unavailable();
    return nullptr;
}
static inline void fftw_execute_dft_r2c(const fftw_plan, double *, fftw_complex *) { tm_shim_fftw_unavailable(); }
static inline void fftw_execute_dft_c2r(const fftw_plan, fftw_complex *, double *) { tm_shim_fftw_unavailable(); }
static inline void fftw_destroy_plan(fftw_plan) {}

#endif
