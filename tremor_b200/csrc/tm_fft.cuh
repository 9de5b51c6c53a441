// The FFT contraction's launchers and constants (tm_fft.cu).
#pragma once

#include "tm_internal.cuh"
#include "tm_prefix.cuh"

namespace tmb {

constexpr int kFftL = 32768;             // piece length (samples); templates up to kFftS
constexpr int kFftS = kFftL / 2;         // piece step
constexpr int kFftH = kFftL / 2 + 1;     // complex bins of a real FFT
constexpr uint32_t kFftBatch = 1024;     // pieces per inverse-FFT batch

struct FftEpiArgs
{
    const double *out;     // count x kFftL correlation outputs of pieces p0 ..
    uint32_t p0, count;
    uint32_t t;            // template row
    TemplParam p;          // its constants, in the launch's parameter space (one broadcast copy)
    double e_fac;          // sqrt(m) (2 sqrt(m) + sqrt(kFftL)): the template's factor of the output error
    uint64_t w0;           // window range start (windows are relative to it)
    PrefixView pv;
    const uint16_t *run;
    const float *raw;
    const double *shifts, *norms;
    uint32_t *bmin_u, *bmin_l;
    uint32_t nb;
    Candidate *cand;
    uint32_t *cand_count, cand_cap;
    float *dbg_d, *dbg_e; // diagnostics: d and e of every window, [t][W]; null in searches
    uint32_t W;
};

uint32_t fft_pieces(uint64_t n);
cudaError_t launch_fft_gather(const float *clean, uint64_t n, const double *centres, uint32_t p0, uint32_t count,
                              double *pieces, double *shifts, double *norms, cudaStream_t s);
cudaError_t launch_fft_template(const float *q, int m, double *y, cudaStream_t s);
cudaError_t launch_fft_mul(const double2 *X, const double2 *Y, double2 *Z, uint32_t count, cudaStream_t s);
cudaError_t launch_fft_epilogue(const FftEpiArgs &f, cudaStream_t s);

} // namespace tmb
