// Test infrastructure only (oracle build).  Declarations of the single-precision FFTW calls that
// the reference's src/fft.cpp makes (one-dimensional complex, real-to-complex and
// complex-to-real transforms of one line at a time), so that its distributed 3-D transform
// compiles where it lies; oracle/ic_probe.cpp defines them as plain discrete Fourier sums.
#pragma once
typedef float fftwf_complex[2];
typedef struct fftwf_plan_s* fftwf_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex* in, fftwf_complex* out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float* in, fftwf_complex* out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex* in, float* out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
