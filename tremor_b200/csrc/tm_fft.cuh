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

// The in-tree fused FFT branch (tm_fftk.cu) for templates of up to kF2S samples: pieces
// of kF2L samples every kF2S samples, real transforms through complex ones of kF2N points.
constexpr int kF2L = 16384;
constexpr int kF2S = 8192;
constexpr int kF2N = kF2L / 2;
constexpr int kF2H = kF2L / 2 + 1;

struct Fft2Args
{
    const double2 *X;             // piece spectra, kF2H bins per piece
    const double *shifts, *norms; // per piece: its shift s_p and ||x - s_p||_2
    uint32_t p_first, p_count;    // pieces of this launch
    const double2 *Y;             // template spectra, kF2H bins per entry of rows
    const int *rows;              // the launch's template rows (indices into tp)
    int nrows;
    const TemplParam *tp;
    const double2 *roots;         // twiddle tables (fft2_roots)
    uint64_t w0;                  // window range start (windows are relative to it)
    uint32_t W;
    PrefixView pv;
    const uint16_t *run;
    const float *raw;
    uint32_t *bmin_u, *bmin_l;
    uint32_t nb;
    Candidate *cand;
    uint32_t *cand_count, cand_cap;
    float *dbg_d, *dbg_e; // diagnostics: d and e of every window, [t][W]; null in searches
};

uint32_t fft2_pieces(uint64_t n);
void fft2_roots(double2 *host256);
cudaError_t launch_fft2_pieces(const float *clean, uint64_t n, const double *centres, uint32_t p0, uint32_t count,
                               const double2 *roots, double2 *X, double *shifts, double *norms, cudaStream_t s);
cudaError_t launch_fft2_templates(const float *q, const TemplParam *tp, const int *rows, int nrows,
                                  const double2 *roots, double2 *Y, cudaStream_t s);
cudaError_t launch_fft2_corr(const Fft2Args &a, int sms, cudaStream_t s);

uint32_t fft_pieces(uint64_t n);
cudaError_t launch_fft_gather(const float *clean, uint64_t n, const double *centres, uint32_t p0, uint32_t count,
                              double *pieces, double *shifts, double *norms, cudaStream_t s);
cudaError_t launch_fft_template(const float *q, int m, double *y, cudaStream_t s);
cudaError_t launch_fft_mul(const double2 *X, const double2 *Y, double2 *Z, uint32_t count, cudaStream_t s);
cudaError_t launch_fft_epilogue(const FftEpiArgs &f, cudaStream_t s);

} // namespace tmb
