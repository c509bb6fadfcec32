/*
 * fftw3.h -- minimal FFTW3-compatible interface, written for this project.
 *
 * TEST INFRASTRUCTURE ONLY.  This header and fftw_shim.c exist so that the
 * unmodified K-Litho CPU programs (K-Litho-TCC/klitho_tcc.cpp,
 * K-Litho-SOCS/klitho_socs.cpp) can be compiled as an oracle on a machine
 * without libfftw3.  Nothing in the shipped product links against it.
 *
 * Only the entry points those programs call are provided
 * (klitho_tcc.cpp:461-462, klitho_socs.cpp:208,212,286-287):
 *   fftw_plan_dft_r2c_2d, fftw_plan_dft_c2r_2d, fftw_plan_dft_2d,
 *   fftw_execute, fftw_destroy_plan.
 * Semantics follow FFTW's documented conventions: row-major n0 x n1 arrays,
 * FORWARD = exp(-2*pi*i*k*x/n), BACKWARD = exp(+2*pi*i*k*x/n), no
 * normalisation, r2c output n0 x (n1/2+1), c2r input n0 x (n1/2+1) with the
 * Hermitian-symmetric remainder implied.  The FFT algorithm is the project's
 * own (radix-2 Cooley-Tukey for powers of two, Bluestein chirp-z otherwise),
 * in IEEE double precision.
 */
#ifndef KLITHO_ORACLE_FFTW3_SHIM_H
#define KLITHO_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct kl_shim_plan* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

/* Project extension (not FFTW API): in-place 1-D complex transform of length n
 * with the given sign, used by the restated oracle. */
void kl_shim_fft1d(double* data_interleaved, int n, int sign);

#ifdef __cplusplus
}
#endif
#endif
