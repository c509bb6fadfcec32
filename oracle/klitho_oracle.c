/*
 * klitho_oracle.c -- restated FP64 CPU oracle of K-Litho's Hopkins/SOCS path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library, and
 * only as the checker (or the timed CPU baseline).  The GPU product never
 * links or calls it.
 *
 * Each function restates one reference function, step for step, including
 * the single-precision roundings the reference performs inside its "double"
 * code (float coordinates, float loop bounds, cosf/sinf pupil phases), so
 * that on NA <= 1 inputs the results are bit-identical to the reference
 * compiled with the project's FFT shim (checked by tests/test_oracle_pin.py).
 * The one generalisation is `n_medium`: the defocus phase uses
 * sqrt(n_medium^2 - rho^2 NA^2) so that immersion configurations (NA > 1)
 * are defined; n_medium = 1 reproduces klitho_tcc.cpp:220 exactly.
 *
 * Complex numbers are interleaved (re, im) doubles.  Products are written out
 * as the same real operations the reference's std::complex<double> code
 * performs (x86-64, no FMA contraction), in the same order.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_shim/fftw3.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* zheevr_ comes from lapack_shim/zheevr_fwd.c (same prototype as
 * K-Litho-TCC/klitho_tcc.cpp:294-297). */
void zheevr_(const char* jobz, const char* range, const char* uplo, int* n, void* a, int* lda,
             double* vl, double* vu, int* il, int* iu, double* abstol, int* m, double* w, void* z,
             int* ldz, int* isuppz, void* work, int* lwork, double* rwork, int* lrwork, int* iwork,
             int* liwork, int* info);

/* number of out-of-band pupil writes skipped (reference would index outside
 * its table there); tests assert it stays 0 */
static long g_out_of_band = 0;
long kor_out_of_band_count(void) { return g_out_of_band; }

/* ---------------------------------------------------------------------- */
/* Source analysis and band sizing                                          */
/* ---------------------------------------------------------------------- */

/* getOuterSigma: K-Litho-TCC/klitho_tcc.cpp:52-67 */
float kor_outer_sigma(const float* src, int srcSize) {
  int center = (srcSize - 1) / 2;
  float far = 0.0f;
  for (int y = 0; y < srcSize; ++y) {
    for (int x = 0; x < srcSize; ++x) {
      if (src[y * srcSize + x] != 0.0f) {
        int r2 = (y - center) * (y - center) + (x - center) * (x - center);
        float d = (float)sqrt((double)r2);
        if (d > far) far = d;
      }
    }
  }
  return far / (float)center;
}

/* Band half-widths: K-Litho-TCC/klitho_tcc.cpp:479-486 (sigma clamp at :480-483) */
void kor_band(double NA, int Lx, int Ly, float outerSigma, float lambda, int* Nx, int* Ny) {
  float s = outerSigma > 1.0f ? 1.0f : outerSigma;
  float na = (float)NA;
  *Nx = (int)floorf(na * (float)Lx * (1.0f + s) / lambda);
  *Ny = (int)floorf(na * (float)Ly * (1.0f + s) / lambda);
}

/* ---------------------------------------------------------------------- */
/* Pupil sampling and TCC: K-Litho-TCC/klitho_tcc.cpp:186-267              */
/* ---------------------------------------------------------------------- */

typedef struct {
  int src_id;
  float J;
  float sx, sy;
  int nxmin, nxmax, nymin, nymax;
} kor_pt;

typedef struct {
  int Nx, Ny, N, S;
  kor_pt* pts;
  double* P; /* N x S interleaved complex, 0 outside the shifted pupil */
} kor_pupil;

/* Active source points in the reference's raster order (:202-205) and their
 * pupil values (:206-224). */
static void pupil_build(kor_pupil* pu, const float* src, int srcSize, float outerSigma,
                        float lambda, float NA, float defocus, double n_medium, int Lx, int Ly,
                        int Nx, int Ny) {
  int sh = (int)((srcSize - 1) / 2.0);
  int oSgm = (int)ceilf((float)sh * outerSigma);
  float dz = defocus / (NA * NA / lambda);
  float k = (float)(2 * M_PI / lambda);
  float Lx_norm = (float)Lx * NA / lambda, Ly_norm = (float)Ly * NA / lambda;
  double nm2 = n_medium * n_medium;
  int bw = 2 * Nx + 1;
  pu->Nx = Nx;
  pu->Ny = Ny;
  pu->N = bw * (2 * Ny + 1);
  int cap = (2 * oSgm + 1) * (2 * oSgm + 1);
  pu->pts = (kor_pt*)malloc(sizeof(kor_pt) * (size_t)(cap > 0 ? cap : 1));
  int S = 0;
  for (int q = -oSgm; q <= oSgm; ++q) {
    for (int p = -oSgm; p <= oSgm; ++p) {
      int id = (q + sh) * srcSize + p + sh;
      if (src[id] != 0.0f && (p * p + q * q) <= sh * sh) {
        kor_pt* t = &pu->pts[S++];
        t->src_id = id;
        t->J = src[id];
        t->sx = (float)p / (float)sh;
        t->sy = (float)q / (float)sh;
        t->nxmin = (int)((-1.0f - t->sx) * Lx_norm);
        t->nxmax = (int)((1.0f - t->sx) * Lx_norm);
        t->nymin = (int)((-1.0f - t->sy) * Ly_norm);
        t->nymax = (int)((1.0f - t->sy) * Ly_norm);
      }
    }
  }
  pu->S = S;
  pu->P = (double*)calloc(2 * (size_t)pu->N * (size_t)(S > 0 ? S : 1), sizeof(double));
  for (int s = 0; s < S; ++s) {
    kor_pt* t = &pu->pts[s];
    for (int ny = t->nymin; ny <= t->nymax; ++ny) {
      float fy = (float)ny / Ly_norm + t->sy;
      if (fy * fy <= 1.0f) {
        for (int nx = t->nxmin; nx <= t->nxmax; ++nx) {
          float fx = (float)nx / Lx_norm + t->sx;
          float rho2 = fx * fx + fy * fy;
          if (rho2 <= 1.0f) {
            float ph = (float)((double)(dz * k) * sqrt(nm2 - (double)(rho2 * NA * NA)));
            if (ny < -Ny || ny > Ny || nx < -Nx || nx > Nx) {
              ++g_out_of_band;
              continue;
            }
            size_t f = (size_t)((ny + Ny) * bw + nx + Nx);
            pu->P[2 * (f * S + s)] = (double)cosf(ph);
            pu->P[2 * (f * S + s) + 1] = (double)sinf(ph);
          }
        }
      }
    }
  }
}

static void pupil_free(kor_pupil* pu) {
  free(pu->pts);
  free(pu->P);
}

/* Active source point count (size of the TCC factor A = sqrt(J) P). */
int kor_source_point_count(const float* src, int srcSize, float outerSigma) {
  int sh = (int)((srcSize - 1) / 2.0);
  int oSgm = (int)ceilf((float)sh * outerSigma);
  int S = 0;
  for (int q = -oSgm; q <= oSgm; ++q)
    for (int p = -oSgm; p <= oSgm; ++p) {
      int id = (q + sh) * srcSize + p + sh;
      if (src[id] != 0.0f && (p * p + q * q) <= sh * sh) ++S;
    }
  return S;
}

/* Pupil table restricted to active points: P_out is N x S complex, src_ids
 * and J give each column's source pixel and weight. */
int kor_pupil_matrix(const float* src, int srcSize, float outerSigma, float lambda, float NA,
                     float defocus, double n_medium, int Lx, int Ly, int Nx, int Ny,
                     double* P_out, int* src_ids, float* J_out, int maxS) {
  kor_pupil pu;
  pupil_build(&pu, src, srcSize, outerSigma, lambda, NA, defocus, n_medium, Lx, Ly, Nx, Ny);
  int S = pu.S;
  if (S <= maxS) {
    memcpy(P_out, pu.P, sizeof(double) * 2 * (size_t)pu.N * (size_t)S);
    for (int s = 0; s < S; ++s) {
      src_ids[s] = pu.pts[s].src_id;
      J_out[s] = pu.pts[s].J;
    }
  }
  pupil_free(&pu);
  return S;
}

/* calcTCC: upper-triangle accumulation in the reference loop order
 * (:230-260), then the Hermitian mirror (:261-266). */
int kor_calc_tcc(const float* src, int srcSize, float outerSigma, float lambda, float NA,
                 float defocus, double n_medium, int Lx, int Ly, int Nx, int Ny, double* tcc) {
  kor_pupil pu;
  pupil_build(&pu, src, srcSize, outerSigma, lambda, NA, defocus, n_medium, Lx, Ly, Nx, Ny);
  int N = pu.N, S = pu.S, bw = 2 * Nx + 1;
  memset(tcc, 0, sizeof(double) * 2 * (size_t)N * (size_t)N);
  for (int s = 0; s < S; ++s) {
    const kor_pt* t = &pu.pts[s];
    double J = (double)t->J;
    for (int ny = t->nymin; ny <= t->nymax; ++ny) {
      for (int nx = t->nxmin; nx <= t->nxmax; ++nx) {
        if (ny < -Ny || ny > Ny || nx < -Nx || nx > Nx) continue;
        size_t id1 = (size_t)((ny + Ny) * bw + nx + Nx);
        double pr = pu.P[2 * (id1 * S + s)], pi = pu.P[2 * (id1 * S + s) + 1];
        if (pr == 0.0 && pi == 0.0) continue;
        double tr = pr * J, ti = pi * J;
        for (int my = ny; my <= t->nymax; ++my) {
          int mx0 = (my == ny) ? nx : t->nxmin;
          for (int mx = mx0; mx <= t->nxmax; ++mx) {
            if (my < -Ny || my > Ny || mx < -Nx || mx > Nx) continue;
            size_t id2 = (size_t)((my + Ny) * bw + mx + Nx);
            double cr = pu.P[2 * (id2 * S + s)], ci = pu.P[2 * (id2 * S + s) + 1];
            double* d = tcc + 2 * (id1 * N + id2);
            d[0] += tr * cr + ti * ci;
            d[1] += ti * cr - tr * ci;
          }
        }
      }
    }
  }
  for (size_t i = 0; i < (size_t)N; ++i)
    for (size_t j = i + 1; j < (size_t)N; ++j) {
      tcc[2 * (j * N + i)] = tcc[2 * (i * N + j)];
      tcc[2 * (j * N + i) + 1] = -tcc[2 * (i * N + j) + 1];
    }
  pupil_free(&pu);
  return N;
}

/* ---------------------------------------------------------------------- */
/* FFT helpers: myShift / FT_r2c / FT_c2r, K-Litho-TCC/klitho_tcc.cpp:37-183 */
/* ---------------------------------------------------------------------- */

/* myShift (:37-50): out[(y+yh)%sy][(x+xh)%sx] = in[y][x] */
static void shift_d(const double* in, double* out, int sx, int sy, int halfX, int halfY) {
  int xh = halfX ? sx / 2 : (sx + 1) / 2;
  int yh = halfY ? sy / 2 : (sy + 1) / 2;
  for (int y = 0; y < sy; ++y)
    for (int x = 0; x < sx; ++x)
      out[(size_t)((y + yh) % sy) * sx + (x + xh) % sx] = in[(size_t)y * sx + x];
}

/* FT_r2c (:97-148): centred spectrum, DC at [Ly/2][Lx/2], scaled 1/(Lx*Ly) */
void kor_ft_r2c(const float* mask, int sizeX, int sizeY, double* out) {
  size_t nn = (size_t)sizeX * sizeY;
  int wt = sizeX / 2 + 1, sizeXh = sizeX / 2;
  double* tmp = (double*)malloc(sizeof(double) * nn);
  double* datar = (double*)malloc(sizeof(double) * nn);
  double* datac = (double*)calloc(2 * (size_t)wt * sizeY, sizeof(double));
  for (size_t i = 0; i < nn; ++i) tmp[i] = (double)mask[i];
  shift_d(tmp, datar, sizeX, sizeY, 0, 0);
  fftw_plan pl = fftw_plan_dft_r2c_2d(sizeY, sizeX, datar, (fftw_complex*)datac, FFTW_ESTIMATE);
  fftw_execute(pl);
  fftw_destroy_plan(pl);
  int AY = (sizeY + 1) / 2, BY = sizeY - AY;
  double* R = (double*)calloc(2 * (size_t)wt * sizeY, sizeof(double));
  double* Lh = (double*)calloc(2 * (size_t)wt * sizeY, sizeof(double));
  for (int y = 0; y < sizeY; ++y) {
    int y2 = (y < BY) ? y + AY : y - BY;
    memcpy(R + 2 * (size_t)y * wt, datac + 2 * (size_t)y2 * wt, sizeof(double) * 2 * wt);
  }
  for (int y = 0; y < sizeY; ++y) {
    int y2 = (sizeY % 2 == 0) ? (y == 0 ? 0 : sizeY - y) : sizeY - 1 - y;
    for (int x = 0; x < wt; ++x) {
      int x2 = wt - 1 - x;
      Lh[2 * ((size_t)y * wt + x)] = R[2 * ((size_t)y2 * wt + x2)];
      Lh[2 * ((size_t)y * wt + x) + 1] = -R[2 * ((size_t)y2 * wt + x2) + 1];
    }
  }
  for (int y = 0; y < sizeY; ++y)
    for (int x = 0; x < wt; ++x) {
      out[2 * ((size_t)y * sizeX + x)] = Lh[2 * ((size_t)y * wt + x)];
      out[2 * ((size_t)y * sizeX + x) + 1] = Lh[2 * ((size_t)y * wt + x) + 1];
    }
  for (int y = 0; y < sizeY; ++y)
    for (int x = sizeXh, x2 = 0; x < sizeX; ++x, ++x2) {
      out[2 * ((size_t)y * sizeX + x)] = R[2 * ((size_t)y * wt + x2)];
      out[2 * ((size_t)y * sizeX + x) + 1] = R[2 * ((size_t)y * wt + x2) + 1];
    }
  double d = (double)(sizeX * sizeY);
  for (size_t i = 0; i < nn; ++i) {
    out[2 * i] /= d;
    out[2 * i + 1] /= d;
  }
  free(tmp);
  free(datar);
  free(datac);
  free(R);
  free(Lh);
}

/* FT_c2r (:150-183), double result before the reference's float store.
 * The reference's first column write (x = xh-1) lands one row on in the
 * half-spectrum buffer and, for the wrapped row, past its end; both writes
 * carry the (always zero) nx = -1 entry of the half-plane image spectrum.
 * The in-bounds aliases are reproduced; the past-the-end one is dropped. */
void kor_ft_c2r_d(const double* in, int sizeX, int sizeY, double* out) {
  int wt = sizeX / 2 + 1;
  int xh = (sizeX + 1) / 2, yh = (sizeY + 1) / 2;
  size_t nc = (size_t)wt * sizeY, nn = (size_t)sizeX * sizeY;
  double* datac = (double*)calloc(2 * nc, sizeof(double));
  double* datar = (double*)malloc(sizeof(double) * nn);
  for (int y = 0; y < sizeY; ++y)
    for (int x = xh - 1; x < sizeX; ++x) {
      int sx = (x + xh) % sizeX, sy = (y + yh) % sizeY;
      size_t o = (size_t)sy * wt + sx;
      if (o < nc) {
        datac[2 * o] = in[2 * ((size_t)y * sizeX + x)];
        datac[2 * o + 1] = in[2 * ((size_t)y * sizeX + x) + 1];
      }
    }
  if (sizeX % 2 == 0) {
    for (int y = 0; y < sizeY; ++y) {
      int y2 = (y == 0) ? 0 : sizeY - y;
      datac[2 * ((size_t)y * wt + wt - 1)] = in[2 * ((size_t)y2 * sizeX)];
      datac[2 * ((size_t)y * wt + wt - 1) + 1] = -in[2 * ((size_t)y2 * sizeX) + 1];
    }
  }
  fftw_plan pl = fftw_plan_dft_c2r_2d(sizeY, sizeX, (fftw_complex*)datac, datar, FFTW_ESTIMATE);
  fftw_execute(pl);
  fftw_destroy_plan(pl);
  shift_d(datar, out, sizeX, sizeY, 0, 0);
  free(datac);
  free(datar);
}

/* calcImage (:269-290): half-plane Hopkins spectrum from the TCC */
void kor_calc_image(const double* msk, int Lx, int Ly, const double* tcc, int N, int Nx, int Ny,
                    double* imgf) {
  int tch = (N - 1) / 2, Lxh = Lx / 2, Lyh = Ly / 2, bw = 2 * Nx + 1;
  memset(imgf, 0, sizeof(double) * 2 * (size_t)Lx * Ly);
  for (int ny2 = -2 * Ny; ny2 <= 2 * Ny; ++ny2) {
    for (int nx2 = 0; nx2 <= 2 * Nx; ++nx2) {
      double vr = 0.0, vi = 0.0;
      for (int ny1 = -Ny; ny1 <= Ny; ++ny1) {
        for (int nx1 = -Nx; nx1 <= Nx; ++nx1) {
          if (abs(nx2 + nx1) <= Nx && abs(ny2 + ny1) <= Ny) {
            const double* a = msk + 2 * ((size_t)(ny2 + ny1 + Lyh) * Lx + (nx2 + nx1 + Lxh));
            const double* b = msk + 2 * ((size_t)(ny1 + Lyh) * Lx + (nx1 + Lxh));
            const double* t =
                tcc + 2 * ((size_t)(ny1 * bw + nx1 + tch) * N + (size_t)((ny2 + ny1) * bw + (nx2 + nx1) + tch));
            double pr = a[0] * b[0] + a[1] * b[1]; /* a * conj(b) */
            double pi = a[1] * b[0] - a[0] * b[1];
            vr += pr * t[0] - pi * t[1];
            vi += pr * t[1] + pi * t[0];
          }
        }
      }
      imgf[2 * ((size_t)(ny2 + Lyh) * Lx + (nx2 + Lxh))] = vr;
      imgf[2 * ((size_t)(ny2 + Lyh) * Lx + (nx2 + Lxh)) + 1] = vi;
    }
  }
}

/* ---------------------------------------------------------------------- */
/* calcKernels (:300-377): LAPACK zheevr top-nk, reversed order and index    */
/* ---------------------------------------------------------------------- */
int kor_calc_kernels(const double* tcc, int n, int nk, double* krns, float* scales,
                     double* evals_d) {
  int lda = n, ldz = n, il = n - (nk - 1), iu = n, m = iu - il + 1, info = 0;
  double abstol = -1.0, vl = 0.0, vu = 0.0;
  int* isuppz = (int*)malloc(sizeof(int) * 2 * (size_t)m);
  double* a = (double*)malloc(sizeof(double) * 2 * (size_t)n * n);
  double* z = (double*)malloc(sizeof(double) * 2 * (size_t)n * m);
  double* w = (double*)malloc(sizeof(double) * (size_t)n);
  /* the reference hands LAPACK the transposed row-major copy (:313-317) */
  for (size_t i = 0; i < (size_t)n; ++i)
    for (size_t j = 0; j < (size_t)n; ++j) {
      a[2 * (i * n + j)] = tcc[2 * (j * n + i)];
      a[2 * (i * n + j) + 1] = tcc[2 * (j * n + i) + 1];
    }
  int lwork = -1, lrwork = -1, liwork = -1, iwkopt = 0;
  double wkopt[2] = {0, 0}, rwkopt = 0;
  zheevr_("V", "I", "U", &n, a, &lda, &vl, &vu, &il, &iu, &abstol, &m, w, z, &ldz, isuppz, wkopt,
          &lwork, &rwkopt, &lrwork, &iwkopt, &liwork, &info);
  lwork = (int)wkopt[0];
  lrwork = (int)rwkopt;
  liwork = iwkopt;
  double* work = (double*)malloc(sizeof(double) * 2 * (size_t)lwork);
  double* rwork = (double*)malloc(sizeof(double) * (size_t)lrwork);
  int* iwork = (int*)malloc(sizeof(int) * (size_t)liwork);
  zheevr_("V", "I", "U", &n, a, &lda, &vl, &vu, &il, &iu, &abstol, &m, w, z, &ldz, isuppz, work,
          &lwork, rwork, &lrwork, iwork, &liwork, &info);
  for (int j = m - 1; j >= 0; --j) {
    scales[m - 1 - j] = (float)w[j];
    if (evals_d) evals_d[m - 1 - j] = w[j];
  }
  /* kernel i = eigenvector (m-1-i) with its index reversed, f -> -f (:358-362);
   * the loop at :350-356 writes the same array and is fully overwritten */
  for (size_t i = 0; i < (size_t)m; ++i)
    for (size_t j = 0; j < (size_t)n; ++j) {
      krns[2 * (i * n + j)] = z[2 * ((m - 1 - i) * n + (n - 1 - j))];
      krns[2 * (i * n + j) + 1] = z[2 * ((m - 1 - i) * n + (n - 1 - j)) + 1];
    }
  free(work);
  free(rwork);
  free(iwork);
  free(isuppz);
  free(a);
  free(z);
  free(w);
  return info;
}

/* ---------------------------------------------------------------------- */
/* calcSOCS + FI: K-Litho-SOCS/klitho_socs.cpp:158-241                      */
/* ---------------------------------------------------------------------- */

/* FI (:158-194) with double output (the reference stores float) */
static void fourier_interp(const double* in, int isx, int isy, double* out, int osx, int osy) {
  int difY = osy - isy;
  size_t ni = (size_t)isx * isy, no = (size_t)osx * osy;
  int iw = isx / 2 + 1, ow = osx / 2 + 1;
  double* r2cr = (double*)calloc(ni, sizeof(double));
  double* r2cc = (double*)calloc(2 * (size_t)iw * isy, sizeof(double));
  double* c2rc = (double*)calloc(2 * (size_t)ow * osy, sizeof(double));
  double* c2rr = (double*)calloc(no, sizeof(double));
  shift_d(in, r2cr, isx, isy, 0, 0);
  fftw_plan p1 = fftw_plan_dft_r2c_2d(isy, isx, r2cr, (fftw_complex*)r2cc, FFTW_ESTIMATE);
  fftw_execute(p1);
  fftw_destroy_plan(p1);
  double d = (double)(isx * isy);
  for (size_t i = 0; i < (size_t)isy * iw; ++i) {
    r2cc[2 * i] /= d;
    r2cc[2 * i + 1] /= d;
  }
  for (int y = 0; y < isy / 2 + 1; ++y)
    for (int x = 0; x < iw; ++x) {
      c2rc[2 * ((size_t)y * ow + x)] = r2cc[2 * ((size_t)y * iw + x)];
      c2rc[2 * ((size_t)y * ow + x) + 1] = r2cc[2 * ((size_t)y * iw + x) + 1];
    }
  for (int y = isy / 2 + 1; y < isy; ++y)
    for (int x = 0; x < iw; ++x) {
      c2rc[2 * ((size_t)(y + difY) * ow + x)] = r2cc[2 * ((size_t)y * iw + x)];
      c2rc[2 * ((size_t)(y + difY) * ow + x) + 1] = r2cc[2 * ((size_t)y * iw + x) + 1];
    }
  fftw_plan p2 = fftw_plan_dft_c2r_2d(osy, osx, (fftw_complex*)c2rc, c2rr, FFTW_ESTIMATE);
  fftw_execute(p2);
  fftw_destroy_plan(p2);
  shift_d(c2rr, out, osx, osy, 0, 0);
  free(r2cr);
  free(r2cc);
  free(c2rc);
  free(c2rr);
}

/* calcSOCS (:196-241): krns is nk x (2Nx+1)(2Ny+1) complex (from float files),
 * scales the float eigenvalues, msk the centred spectrum from kor_ft_r2c. */
void kor_calc_socs(const double* msk, int Lx, int Ly, const double* krns, const float* scales,
                   int nk, int Nx, int Ny, double* image) {
  int sizeX = 4 * Nx + 1, sizeY = 4 * Ny + 1;
  int difX = sizeX - (2 * Nx + 1), difY = sizeY - (2 * Ny + 1);
  int Lxh = Lx / 2, Lyh = Ly / 2, bw = 2 * Nx + 1;
  size_t ng = (size_t)sizeX * sizeY;
  double* bin = (double*)calloc(2 * ng, sizeof(double));
  double* bout = (double*)calloc(2 * ng, sizeof(double));
  double* acc = (double*)calloc(ng, sizeof(double));
  double* accp = (double*)calloc(ng, sizeof(double));
  fftw_plan pb =
      fftw_plan_dft_2d(sizeY, sizeX, (fftw_complex*)bin, (fftw_complex*)bout, FFTW_BACKWARD, FFTW_ESTIMATE);
  for (int k = 0; k < nk; ++k) {
    const double* h = krns + 2 * (size_t)k * bw * (2 * Ny + 1);
    for (int y = -Ny; y <= Ny; ++y)
      for (int x = -Nx; x <= Nx; ++x) {
        const double* hk = h + 2 * ((size_t)(y + Ny) * bw + x + Nx);
        const double* m = msk + 2 * ((size_t)(y + Lyh) * Lx + x + Lxh);
        double* o = bin + 2 * ((size_t)(difY + y + Ny) * sizeX + difX + x + Nx);
        o[0] = hk[0] * m[0] - hk[1] * m[1];
        o[1] = hk[0] * m[1] + hk[1] * m[0];
      }
    fftw_execute(pb);
    double sc = (double)scales[k];
    for (size_t i = 0; i < ng; ++i)
      acc[i] += sc * (bout[2 * i] * bout[2 * i] + bout[2 * i + 1] * bout[2 * i + 1]);
  }
  fftw_destroy_plan(pb);
  shift_d(acc, accp, sizeX, sizeY, 1, 1);
  fourier_interp(accp, sizeX, sizeY, image, Lx, Ly);
  free(bin);
  free(bout);
  free(acc);
  free(accp);
}

/* Small-grid SOCS intensity (before FI), for tests of the spectral stage:
 * the (4Nx+1)x(4Ny+1) accumulator after the reference's myShift(:233). */
void kor_socs_small_grid(const double* msk, int Lx, int Ly, const double* krns,
                         const float* scales, int nk, int Nx, int Ny, double* out) {
  int sizeX = 4 * Nx + 1, sizeY = 4 * Ny + 1;
  int difX = sizeX - (2 * Nx + 1), difY = sizeY - (2 * Ny + 1);
  int Lxh = Lx / 2, Lyh = Ly / 2, bw = 2 * Nx + 1;
  size_t ng = (size_t)sizeX * sizeY;
  double* bin = (double*)calloc(2 * ng, sizeof(double));
  double* bout = (double*)calloc(2 * ng, sizeof(double));
  double* acc = (double*)calloc(ng, sizeof(double));
  fftw_plan pb =
      fftw_plan_dft_2d(sizeY, sizeX, (fftw_complex*)bin, (fftw_complex*)bout, FFTW_BACKWARD, FFTW_ESTIMATE);
  for (int k = 0; k < nk; ++k) {
    const double* h = krns + 2 * (size_t)k * bw * (2 * Ny + 1);
    for (int y = -Ny; y <= Ny; ++y)
      for (int x = -Nx; x <= Nx; ++x) {
        const double* hk = h + 2 * ((size_t)(y + Ny) * bw + x + Nx);
        const double* m = msk + 2 * ((size_t)(y + Lyh) * Lx + x + Lxh);
        double* o = bin + 2 * ((size_t)(difY + y + Ny) * sizeX + difX + x + Nx);
        o[0] = hk[0] * m[0] - hk[1] * m[1];
        o[1] = hk[0] * m[1] + hk[1] * m[0];
      }
    fftw_execute(pb);
    double sc = (double)scales[k];
    for (size_t i = 0; i < ng; ++i)
      acc[i] += sc * (bout[2 * i] * bout[2 * i] + bout[2 * i + 1] * bout[2 * i + 1]);
  }
  fftw_destroy_plan(pb);
  shift_d(acc, out, sizeX, sizeY, 1, 1);
  free(bin);
  free(bout);
  free(acc);
}
