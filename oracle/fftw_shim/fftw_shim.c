/*
 * fftw_shim.c -- project-written double-precision FFT behind the FFTW3 subset
 * declared in fftw3.h.
 *
 * TEST INFRASTRUCTURE ONLY (oracle).  Used to compile the unmodified K-Litho
 * reference sources and the restated FP64 oracle on a machine without FFTW.
 * It is never linked into the GPU library, the CLIs or the benchmark's timed
 * GPU path.
 *
 * Algorithms: iterative radix-2 Cooley-Tukey for power-of-two lengths and
 * Bluestein's chirp-z transform (over a power-of-two convolution) for every
 * other length, so odd SOCS grids such as 53, 105 or 213 points are exact to
 * double rounding.  2-D transforms are row transforms followed by column
 * transforms on gathered column blocks.
 */
#include "fftw3.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define KL_PI 3.14159265358979323846264338327950288

typedef struct {
  int n;
  int sign;
  int pow2;
  double* tw;      /* pow2: exp(sign*2*pi*i*j/n), j < n/2 (interleaved)      */
  /* Bluestein */
  int m;           /* convolution length, power of two >= 2n-1               */
  double* chirp;   /* c[k] = exp(sign*pi*i*k^2/n), k < n                     */
  double* bhat;    /* FFT_m of conj chirp sequence                           */
  double* twm_f;   /* forward twiddles for length m                          */
  double* twm_b;   /* backward twiddles for length m                         */
  double* work;    /* m complex scratch                                      */
} fft1d;

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static double* make_twiddles(int n, int sign) {
  int h = n / 2 > 0 ? n / 2 : 1;
  double* tw = (double*)malloc(sizeof(double) * 2 * (size_t)h);
  for (int j = 0; j < h; ++j) {
    double ang = 2.0 * KL_PI * (double)j / (double)n;
    tw[2 * j] = cos(ang);
    tw[2 * j + 1] = (double)sign * sin(ang);
  }
  return tw;
}

static void fft_pow2_inplace(double* a, int n, const double* tw) {
  if (n <= 1) return;
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double tr = a[2 * i], ti = a[2 * i + 1];
      a[2 * i] = a[2 * j];
      a[2 * i + 1] = a[2 * j + 1];
      a[2 * j] = tr;
      a[2 * j + 1] = ti;
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1, step = n / len;
    for (int i = 0; i < n; i += len) {
      for (int k = 0; k < half; ++k) {
        double wr = tw[2 * (k * step)], wi = tw[2 * (k * step) + 1];
        double* u = a + 2 * (i + k);
        double* v = a + 2 * (i + k + half);
        double vr = v[0] * wr - v[1] * wi;
        double vi = v[0] * wi + v[1] * wr;
        v[0] = u[0] - vr;
        v[1] = u[1] - vi;
        u[0] += vr;
        u[1] += vi;
      }
    }
  }
}

static fft1d* fft1d_create(int n, int sign) {
  fft1d* p = (fft1d*)calloc(1, sizeof(fft1d));
  p->n = n;
  p->sign = sign;
  p->pow2 = is_pow2(n);
  if (p->pow2) {
    p->tw = make_twiddles(n, sign);
    return p;
  }
  int m = 1;
  while (m < 2 * n - 1) m <<= 1;
  p->m = m;
  p->chirp = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    /* k^2 mod 2n keeps the angle in [0, 2*pi) without precision loss */
    int64_t q = ((int64_t)k * (int64_t)k) % (2 * (int64_t)n);
    double ang = KL_PI * (double)q / (double)n;
    p->chirp[2 * k] = cos(ang);
    p->chirp[2 * k + 1] = (double)sign * sin(ang);
  }
  p->twm_f = make_twiddles(m, -1);
  p->twm_b = make_twiddles(m, +1);
  p->bhat = (double*)calloc(2 * (size_t)m, sizeof(double));
  for (int k = 0; k < n; ++k) {
    double br = p->chirp[2 * k], bi = -p->chirp[2 * k + 1]; /* conj chirp */
    p->bhat[2 * k] = br;
    p->bhat[2 * k + 1] = bi;
    if (k > 0) {
      p->bhat[2 * (m - k)] = br;
      p->bhat[2 * (m - k) + 1] = bi;
    }
  }
  fft_pow2_inplace(p->bhat, m, p->twm_f);
  p->work = (double*)malloc(sizeof(double) * 2 * (size_t)m);
  return p;
}

static void fft1d_destroy(fft1d* p) {
  if (!p) return;
  free(p->tw);
  free(p->chirp);
  free(p->bhat);
  free(p->twm_f);
  free(p->twm_b);
  free(p->work);
  free(p);
}

/* in-place transform of one contiguous interleaved complex vector */
static void fft1d_run(fft1d* p, double* a) {
  int n = p->n;
  if (p->pow2) {
    fft_pow2_inplace(a, n, p->tw);
    return;
  }
  int m = p->m;
  double* w = p->work;
  memset(w, 0, sizeof(double) * 2 * (size_t)m);
  for (int k = 0; k < n; ++k) {
    double xr = a[2 * k], xi = a[2 * k + 1];
    double cr = p->chirp[2 * k], ci = p->chirp[2 * k + 1];
    w[2 * k] = xr * cr - xi * ci;
    w[2 * k + 1] = xr * ci + xi * cr;
  }
  fft_pow2_inplace(w, m, p->twm_f);
  for (int k = 0; k < m; ++k) {
    double xr = w[2 * k], xi = w[2 * k + 1];
    double br = p->bhat[2 * k], bi = p->bhat[2 * k + 1];
    w[2 * k] = xr * br - xi * bi;
    w[2 * k + 1] = xr * bi + xi * br;
  }
  fft_pow2_inplace(w, m, p->twm_b);
  double inv = 1.0 / (double)m;
  for (int k = 0; k < n; ++k) {
    double xr = w[2 * k] * inv, xi = w[2 * k + 1] * inv;
    double cr = p->chirp[2 * k], ci = p->chirp[2 * k + 1];
    a[2 * k] = xr * cr - xi * ci;
    a[2 * k + 1] = xr * ci + xi * cr;
  }
}

/* 2-D in-place complex transform of a row-major n0 x n1 array */
static void fft2d_inplace(double* a, int n0, int n1, fft1d* prow, fft1d* pcol) {
  for (int r = 0; r < n0; ++r) fft1d_run(prow, a + 2 * (size_t)r * n1);
  enum { BLK = 16 };
  double* col = (double*)malloc(sizeof(double) * 2 * (size_t)n0 * BLK);
  for (int c0 = 0; c0 < n1; c0 += BLK) {
    int nb = (n1 - c0) < BLK ? (n1 - c0) : BLK;
    for (int r = 0; r < n0; ++r) {
      const double* src = a + 2 * ((size_t)r * n1 + c0);
      for (int b = 0; b < nb; ++b) {
        col[2 * ((size_t)b * n0 + r)] = src[2 * b];
        col[2 * ((size_t)b * n0 + r) + 1] = src[2 * b + 1];
      }
    }
    for (int b = 0; b < nb; ++b) fft1d_run(pcol, col + 2 * (size_t)b * n0);
    for (int r = 0; r < n0; ++r) {
      double* dst = a + 2 * ((size_t)r * n1 + c0);
      for (int b = 0; b < nb; ++b) {
        dst[2 * b] = col[2 * ((size_t)b * n0 + r)];
        dst[2 * b + 1] = col[2 * ((size_t)b * n0 + r) + 1];
      }
    }
  }
  free(col);
}

enum { KIND_R2C = 1, KIND_C2R = 2, KIND_C2C = 3 };

struct kl_shim_plan {
  int kind, n0, n1, sign;
  void* in;
  void* out;
  fft1d* prow;
  fft1d* pcol;
};

static fftw_plan make_plan(int kind, int n0, int n1, int sign, void* in, void* out) {
  fftw_plan p = (fftw_plan)calloc(1, sizeof(struct kl_shim_plan));
  p->kind = kind;
  p->n0 = n0;
  p->n1 = n1;
  p->sign = sign;
  p->in = in;
  p->out = out;
  p->prow = fft1d_create(n1, sign);
  p->pcol = fft1d_create(n0, sign);
  return p;
}

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags) {
  (void)flags;
  return make_plan(KIND_R2C, n0, n1, FFTW_FORWARD, in, out);
}

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags) {
  (void)flags;
  return make_plan(KIND_C2R, n0, n1, FFTW_BACKWARD, in, out);
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned flags) {
  (void)flags;
  return make_plan(KIND_C2C, n0, n1, sign, in, out);
}

void fftw_execute(const fftw_plan p) {
  int n0 = p->n0, n1 = p->n1, wt = n1 / 2 + 1;
  size_t nn = (size_t)n0 * n1;
  if (p->kind == KIND_C2C) {
    double* buf = (double*)malloc(sizeof(double) * 2 * nn);
    memcpy(buf, p->in, sizeof(double) * 2 * nn);
    fft2d_inplace(buf, n0, n1, p->prow, p->pcol);
    memcpy(p->out, buf, sizeof(double) * 2 * nn);
    free(buf);
  } else if (p->kind == KIND_R2C) {
    const double* in = (const double*)p->in;
    double* out = (double*)p->out;
    double* buf = (double*)malloc(sizeof(double) * 2 * nn);
    for (size_t i = 0; i < nn; ++i) {
      buf[2 * i] = in[i];
      buf[2 * i + 1] = 0.0;
    }
    fft2d_inplace(buf, n0, n1, p->prow, p->pcol);
    for (int r = 0; r < n0; ++r)
      memcpy(out + 2 * (size_t)r * wt, buf + 2 * (size_t)r * n1, sizeof(double) * 2 * (size_t)wt);
    free(buf);
  } else {
    const double* in = (const double*)p->in;
    double* out = (double*)p->out;
    double* buf = (double*)malloc(sizeof(double) * 2 * nn);
    for (int r = 0; r < n0; ++r) {
      for (int c = 0; c < n1; ++c) {
        double re, im;
        if (c < wt) {
          re = in[2 * ((size_t)r * wt + c)];
          im = in[2 * ((size_t)r * wt + c) + 1];
        } else { /* Hermitian completion X[r][c] = conj X[-r][-c] */
          int rr = (n0 - r) % n0, cc = n1 - c;
          re = in[2 * ((size_t)rr * wt + cc)];
          im = -in[2 * ((size_t)rr * wt + cc) + 1];
        }
        buf[2 * ((size_t)r * n1 + c)] = re;
        buf[2 * ((size_t)r * n1 + c) + 1] = im;
      }
    }
    fft2d_inplace(buf, n0, n1, p->prow, p->pcol);
    for (size_t i = 0; i < nn; ++i) out[i] = buf[2 * i];
    free(buf);
  }
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  fft1d_destroy(p->prow);
  fft1d_destroy(p->pcol);
  free(p);
}

void kl_shim_fft1d(double* data, int n, int sign) {
  fft1d* p = fft1d_create(n, sign);
  fft1d_run(p, data);
  fft1d_destroy(p);
}
