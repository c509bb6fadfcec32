// ref_harness_socs.cpp -- C entry points onto the reference's own klitho_socs
// functions, for pinning the restated oracle.
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile with the UNMODIFIED
// reference sources K-Litho-SOCS/klitho_socs.cpp (main renamed by -Dmain=),
// common/mask.cpp and common/file_io.cpp, plus the project's fftw3.h shim.
// klitho_socs.cpp repeats FT_r2c and other helpers of klitho_tcc.cpp, so it
// goes into a library of its own.
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "fftw3.h"
#include "file_io.hpp"
#include "mask.hpp"

using namespace std;
typedef complex<double> Complex;

// Prototypes of functions defined in K-Litho-SOCS/klitho_socs.cpp
void FT_r2c(vector<float>& in, vector<Complex>& out, int sizeX, int sizeY, fftw_plan& fwd,
            vector<double>& datar, vector<Complex>& datac);  // (:71)
void calcSOCS(vector<float>& image, vector<Complex>& msk, int Lx, int Ly,
              vector<vector<Complex>>& krns, vector<float>& scales, int nk, int Nx, int Ny,
              fftw_plan& LxyC2R_plan, vector<Complex>& complexDataLxy,
              vector<double>& realDataLxy);  // (:196)

extern "C" {

// main()'s imaging sequence (klitho_socs.cpp:283-343) on an already embedded
// Lx x Ly mask and float kernel planes.
int kref_socs_image(const float* mask, int Lx, int Ly, const float* krn_r, const float* krn_i,
                    const float* scales_in, int nk, int Nx, int Ny, float* img_out) {
  int Lxy = Lx * Ly, n = (2 * Nx + 1) * (2 * Ny + 1);
  vector<Complex> complexDataLxy(Ly * (Lx / 2 + 1));
  vector<double> realDataLxy(Lxy);
  fftw_plan c2r = fftw_plan_dft_c2r_2d(Ly, Lx,
                                       reinterpret_cast<fftw_complex*>(complexDataLxy.data()),
                                       realDataLxy.data(), FFTW_ESTIMATE);
  fftw_plan r2c = fftw_plan_dft_r2c_2d(Ly, Lx, realDataLxy.data(),
                                       reinterpret_cast<fftw_complex*>(complexDataLxy.data()),
                                       FFTW_ESTIMATE);
  vector<Complex> mskf(Lxy);
  vector<float> msk(mask, mask + Lxy);
  vector<float> img(Lxy);
  vector<float> scales(scales_in, scales_in + nk);
  vector<vector<Complex>> krns(nk, vector<Complex>(n));
  for (int i = 0; i < nk; ++i)
    for (int j = 0; j < n; ++j) krns[i][j] = Complex(krn_r[(size_t)i * n + j], krn_i[(size_t)i * n + j]);
  FT_r2c(msk, mskf, Lx, Ly, r2c, realDataLxy, complexDataLxy);
  calcSOCS(img, mskf, Lx, Ly, krns, scales, nk, Nx, Ny, c2r, complexDataLxy, realDataLxy);
  fftw_destroy_plan(c2r);
  fftw_destroy_plan(r2c);
  memcpy(img_out, img.data(), sizeof(float) * Lxy);
  return 0;
}

}  // extern "C"
