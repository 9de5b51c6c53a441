// The FFT branch's constants, launch arguments and launchers (tm_fftk.cu).
#pragma once

#include "tm_internal.cuh"
#include "tm_prefix.cuh"

namespace tmb {

// Pieces of kF2L samples every kF2S samples serve templates of up to kF2S samples; pieces of
// kF3L samples every kF3S serve the longer ones, up to kFftMaxM. Real transforms of length L
// go through complex ones of L / 2 points.
constexpr int kF2L = 16384;
constexpr int kF2S = 8192;
constexpr int kF2N = kF2L / 2;
constexpr int kF2H = kF2L / 2 + 1;
constexpr int kF3L = 32768;
constexpr int kF3S = 16384;
constexpr int kF3N = kF3L / 2;
constexpr int kF3H = kF3L / 2 + 1;
constexpr int kFftMaxM = kF3S; // longest template of the FFT branch

struct Fft2Args
{
    const double2 *X;             // piece spectra, kF2H (or kF3H) bins per piece
    const double *shifts, *norms; // per piece: its shift s_p and ||x - s_p||_2
    uint32_t p_first, p_count;    // pieces of this launch
    const double2 *Y;             // template spectra, one per entry of rows
    const int *rows;              // the launch's template rows (indices into tp)
    int nrows;
    const TemplParam *tp;
    const double2 *roots;         // twiddle tables (fft_roots)
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
    float4 *stats;        // per block, kFftCache windows' folded statistics of the current piece (a lane's scratch)
    // per template row t, the largest bound coefficients of the launch's templates of its
    // length: gmax[2 t] = (a1_main, a2, a5, a6), gmax[2 t + 1] = (qs, |s1|, 0, 0)
    const float4 *gmax;
};

// Work items of one half of a kF3 piece's epilogue (one complex output each, two windows),
// rounded up; a block's statistics cache holds two windows per item of both halves.
constexpr int kF3Items = 4104;
constexpr int kFftCache = 4 * kF3Items;

constexpr int kFftRoots = 384; // entries of the twiddle tables
constexpr int kFftScratchPts = 8192; // complex points of a block's slice of the forward scratch

uint32_t fft2_pieces(uint64_t n);
uint32_t fft3_pieces(uint64_t n);
void fft_roots(double2 *host384);
cudaError_t launch_fft2_pieces(const float *clean, uint64_t n, const double *centres, uint32_t p0, uint32_t count,
                               const double2 *roots, double2 *X, double *shifts, double *norms, cudaStream_t s);
cudaError_t launch_fft2_templates(const float *q, const TemplParam *tp, const int *rows, int nrows,
                                  const double2 *roots, double2 *Y, cudaStream_t s);
cudaError_t launch_fft2_corr(const Fft2Args &a, int sms, cudaStream_t s);
cudaError_t launch_fft3_pieces(const float *clean, uint64_t n, const double *centres, uint32_t p0, uint32_t count,
                               const double2 *roots, double2 *X, double *shifts, double *norms, double2 *scratch,
                               int blocks, cudaStream_t s);
cudaError_t launch_fft3_templates(const float *q, const TemplParam *tp, const int *rows, int nrows,
                                  const double2 *roots, double2 *Y, double2 *scratch, int blocks, cudaStream_t s);
cudaError_t launch_fft3_corr(const Fft2Args &a, int sms, cudaStream_t s);

} // namespace tmb
