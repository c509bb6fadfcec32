// ref_harness_tcc.cpp -- C entry points onto the reference's own klitho_tcc
// functions, for pinning the restated oracle and the product's host code.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile together with the
// UNMODIFIED reference sources K-Litho-TCC/klitho_tcc.cpp (its main renamed
// with -Dmain=), K-Litho-TCC/source.cpp, common/mask.cpp and
// common/file_io.cpp, read in place from the reference checkout, plus the
// project's fftw3.h shim and zheevr_ forwarder.  Output: oracle/_ref/.
// Nothing here is linked into the product.
#include <complex>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "fftw3.h"
#include "file_io.hpp"
#include "mask.hpp"
#include "source.hpp"

using namespace std;
typedef complex<double> Complex;

// calcKernels (klitho_tcc.cpp:312) allocates zheevr's W with m entries while
// LAPACK documents W as length N; inside a long-lived test process the
// difference corrupts the heap.  Array allocations made by the reference code
// in this library get slack at the end so such writes stay inside them.
// Results are unaffected.
void* operator new[](size_t n) {
  void* p = std::malloc(n + (1u << 20));
  if (!p) throw std::bad_alloc();
  return p;
}
void operator delete[](void* p) noexcept { std::free(p); }
void operator delete[](void* p, size_t) noexcept { std::free(p); }

// Prototypes of functions defined in K-Litho-TCC/klitho_tcc.cpp (line of
// definition in parentheses); the signatures must match to link.
void FT_r2c(vector<float>& in, vector<Complex>& out, int sizeX, int sizeY, fftw_plan& fwd,
            vector<double>& datar, vector<Complex>& datac);  // (:98)
void FT_c2r(vector<Complex>& in, vector<float>& out, int sizeX, int sizeY, fftw_plan& bwd,
            vector<Complex>& datac, vector<double>& datar);  // (:151)
void calcTCC(vector<Complex>& tcc, int tccSize, vector<float>& src, int srcSize, float outerSigma,
             float lambda, float NA, float defocus, int Lx, int Ly, int Nx, int Ny);  // (:187)
void calcImage(vector<Complex>& imgf, vector<Complex>& msk, int Lx, int Ly, vector<Complex>& tcc,
               int tccSize, int Nx, int Ny);  // (:270)
int calcKernels(vector<vector<Complex>>& krns, vector<float>& scales, int nk,
                vector<Complex>& tcc, int tccSize, int Nx, int Ny);  // (:301)
float getOuterSigma(vector<float>& src, int srcSize);               // (:52)

extern "C" {

// createSource (K-Litho-TCC/source.cpp:105-142) with the argv-style parameters
int kref_create_source(int srcSize, const char* type, float innerR, float outerR, float radius,
                       float offset, int onXAxis, float ptX, float ptY, const char* file,
                       float* out) {
  vector<float> src(srcSize * srcSize);
  Annular an;
  an.innerRadius = innerR;
  an.outerRadius = outerR;
  Dipole di;
  CrossQuadrupole cq;
  di.radius = cq.radius = radius;
  di.offset = cq.offset = offset;
  di.onXAxis = onXAxis != 0;
  Point pt;
  pt.x = ptX;
  pt.y = ptY;
  stringstream ss;
  createSource(src, srcSize, string(type), an, di, cq, pt, string(file ? file : ""), ss);
  // an imported file can leave the vector longer than srcSize^2
  // (readFloatArrayFromBinary sizes it by the byte count, file_io.cpp:245)
  memcpy(out, src.data(), sizeof(float) * (size_t)srcSize * srcSize);
  return 0;
}

// createMask (common/mask.cpp:31-60)
int kref_create_mask(int Lx, int Ly, int msx, int msy, const char* type, int lw, int sw, int horiz,
                     const char* file, float dose, float* out) {
  vector<float> msk(Lx * Ly, 0);
  LineSpace ls;
  ls.lineWidth = lw;
  ls.spaceWidth = sw;
  ls.isHorizontal = horiz != 0;
  stringstream ss;
  createMask(msk, Lx, Ly, msx, msy, string(type), ls, string(file ? file : ""), ss, dose);
  memcpy(out, msk.data(), sizeof(float) * msk.size());
  return 0;
}

float kref_outer_sigma(const float* src, int srcSize) {
  vector<float> s(src, src + srcSize * srcSize);
  return getOuterSigma(s, srcSize);
}

// calcTCC (K-Litho-TCC/klitho_tcc.cpp:187-267); tcc_out is N*N interleaved
int kref_calc_tcc(const float* src, int srcSize, float outerSigma, float lambda, float NA,
                  float defocus, int Lx, int Ly, int Nx, int Ny, double* tcc_out) {
  int N = (2 * Nx + 1) * (2 * Ny + 1);
  vector<float> s(src, src + srcSize * srcSize);
  vector<Complex> tcc((size_t)N * N, 0);
  calcTCC(tcc, N, s, srcSize, outerSigma, lambda, NA, defocus, Lx, Ly, Nx, Ny);
  memcpy(tcc_out, tcc.data(), sizeof(Complex) * tcc.size());
  return N;
}

// FT_r2c as main() drives it (:458-462, :510)
int kref_ft_r2c(const float* mask, int Lx, int Ly, double* out) {
  int Lxy = Lx * Ly;
  vector<float> msk(mask, mask + Lxy);
  vector<Complex> mskf(Lxy);
  vector<double> realDataLxy(Lxy, 0);
  vector<Complex> complexDataLxy(Ly * (Lx / 2 + 1), 0);
  fftw_plan r2c = fftw_plan_dft_r2c_2d(Ly, Lx, realDataLxy.data(),
                                       reinterpret_cast<fftw_complex*>(complexDataLxy.data()),
                                       FFTW_ESTIMATE);
  FT_r2c(msk, mskf, Lx, Ly, r2c, realDataLxy, complexDataLxy);
  fftw_destroy_plan(r2c);
  memcpy(out, mskf.data(), sizeof(Complex) * Lxy);
  return 0;
}

// Hopkins image as main() computes it: FT_r2c, calcImage, FT_c2r (:510,:534,:537)
int kref_hopkins_image(const float* mask, const double* tcc_in, int Lx, int Ly, int Nx, int Ny,
                       float* img_out) {
  int Lxy = Lx * Ly, N = (2 * Nx + 1) * (2 * Ny + 1);
  vector<float> msk(mask, mask + Lxy);
  vector<Complex> mskf(Lxy), imgf(Lxy);
  vector<float> img(Lxy);
  vector<Complex> tcc((size_t)N * N);
  memcpy(tcc.data(), tcc_in, sizeof(Complex) * tcc.size());
  vector<double> realDataLxy(Lxy, 0);
  // FT_c2r (klitho_tcc.cpp:162-167) stores the nx = -1 column one row ahead,
  // which for the last row is Lx/2-2 elements past the buffer: the slack
  // keeps that (zero-valued) store inside this allocation
  vector<Complex> complexDataLxy(Ly * (Lx / 2 + 1) + Lx, 0);
  fftw_plan r2c = fftw_plan_dft_r2c_2d(Ly, Lx, realDataLxy.data(),
                                       reinterpret_cast<fftw_complex*>(complexDataLxy.data()),
                                       FFTW_ESTIMATE);
  fftw_plan c2r = fftw_plan_dft_c2r_2d(Ly, Lx,
                                       reinterpret_cast<fftw_complex*>(complexDataLxy.data()),
                                       realDataLxy.data(), FFTW_ESTIMATE);
  FT_r2c(msk, mskf, Lx, Ly, r2c, realDataLxy, complexDataLxy);
  calcImage(imgf, mskf, Lx, Ly, tcc, N, Nx, Ny);
  FT_c2r(imgf, img, Lx, Ly, c2r, complexDataLxy, realDataLxy);
  fftw_destroy_plan(r2c);
  fftw_destroy_plan(c2r);
  memcpy(img_out, img.data(), sizeof(float) * Lxy);
  return 0;
}

// calcKernels (:301-377); krn_out nk*N interleaved, scales_out nk floats
int kref_calc_kernels(const double* tcc_in, int N, int Nx, int Ny, int nk, double* krn_out,
                      float* scales_out) {
  vector<Complex> tcc((size_t)N * N);
  memcpy(tcc.data(), tcc_in, sizeof(Complex) * tcc.size());
  vector<vector<Complex>> krns(nk, vector<Complex>(N));
  vector<float> scales(nk);
  int info = calcKernels(krns, scales, nk, tcc, N, Nx, Ny);
  for (int i = 0; i < nk; ++i) memcpy(krn_out + 2 * (size_t)i * N, krns[i].data(), sizeof(Complex) * N);
  memcpy(scales_out, scales.data(), sizeof(float) * nk);
  return info;
}

// writeKernelInfo / readKernelInfo (common/file_io.cpp:262-307)
int kref_write_kernel_info(const char* path, int kx, int ky, int nk, const float* scales) {
  vector<float> s(scales, scales + nk);
  writeKernelInfo(string(path), kx, ky, nk, s);
  return 0;
}

int kref_read_kernel_info(const char* path, int* kx, int* ky, int* nk, float* scales, int cap) {
  vector<float> s;
  int a = 0, b = 0, n = 0;
  readKernelInfo(string(path), a, b, n, s);
  *kx = a;
  *ky = b;
  *nk = n;
  for (int i = 0; i < (int)s.size() && i < cap; ++i) scales[i] = s[i];
  return (int)s.size();
}

// readFloatArrayFromBinary / readFloatArrayFromTxt (common/file_io.cpp:204-260)
int kref_read_float_file(const char* path, int size, float* out) {
  vector<float> d;
  string p(path);
  if (p.substr(p.find_last_of(".") + 1) == "bin")
    readFloatArrayFromBinary(p, d, size);
  else
    readFloatArrayFromTxt(p, d, size);
  int n = (int)d.size() < size ? (int)d.size() : size;
  memcpy(out, d.data(), sizeof(float) * n);
  return (int)d.size();
}

// the reference's PNG writers (common/file_io.cpp:7-135, stb_image_write):
// mode 0 grayscale, 1 seven colours, 2 continuous colour
int kref_write_png(const char* path, const float* data, int sx, int sy, float mn, float mx, int mode) {
  vector<float> d(data, data + (size_t)sx * sy);
  if (mode == 0)
    writeFloatArrayToPNGWithGrayscale(sx, sy, d, mn, mx, string(path));
  else if (mode == 1)
    writeFloatArrayToPNGWith7Colors(sx, sy, d, string(path), mn, mx);
  else
    writeFloatArrayToPNGWithContinuousColor(sx, sy, d, string(path), mn, mx);
  return 0;
}

}  // extern "C"
