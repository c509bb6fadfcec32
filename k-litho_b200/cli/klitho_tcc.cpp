// klitho_tcc -- drop-in replacement for K-Litho-TCC/klitho_tcc.
//
// Same 22 positional arguments (klitho_tcc.cpp:386-429), validation and
// console output; writes ./out/image.bin (Hopkins image), and, for nk > 0,
// ./out/kernels/krn_<i>_{r,i}.bin and ./out/kernels/kernel_info.txt in the
// reference's formats, plus the reference's PNG previews (KLITHO_PNG=0 skips
// them).  The TCC is assembled on the tensor cores, the SOCS kernels come from
// the GPU eigensolver, and the image from the fused imaging pipeline
// (libklitho_gpu), for any period Lx x Ly the reference accepts.
//
// The kernels are computed and written before the image, so that a failure of
// one stage leaves the other's files in place; the console reports the two
// stages in the reference's order (calcImage, then calcKernels).
//
// Extensions that leave the argv form unchanged (environment variables):
//   KLITHO_N_MEDIUM   immersion index n (default 1 = the reference's pupil);
//                     NA up to n is then accepted instead of NA <= 1
//   KLITHO_PRECISION  "fast" (default) or "fp64": plain FP64 TCC + eigen, and
//                     the FP64 Hopkins image where Lx and Ly are powers of two
#include <cstdlib>
#include <string>
#include <vector>

#include "cli_common.h"

// TARGET_INTENSITY of klitho_tcc.cpp:442, the top of image_s.png's colour scale
constexpr float kTargetIntensity = 0.225f;

int main(int argc, char* argv[]) {
  klcli::banner_start();
  auto start = std::chrono::system_clock::now();
  if (argc != 23) {
    std::cerr << "Error: Invalid number of arguments: " << argc << ". Expected 23 arguments."
              << std::endl;
    return 1;
  }
  const int Lx = std::stoi(argv[1]);
  const int Ly = std::stoi(argv[2]);
  const int msx = std::stoi(argv[3]);
  const int msy = std::stoi(argv[4]);
  const std::string maskType = argv[5];
  const int lineWidth = std::stoi(argv[6]);
  const int spaceWidth = std::stoi(argv[7]);
  const int isHorizontal = std::stoi(argv[8]);
  const std::string maskFile = argv[9];
  const int srcSize = std::stoi(argv[10]);
  const std::string srcType = argv[11];
  const float innerR = std::stof(argv[12]);
  const float outerR = std::stof(argv[13]);
  const float radius = std::stof(argv[14]);
  const float offset = std::stof(argv[15]);
  const bool onXAxis = static_cast<bool>(std::stoi(argv[16]));
  const float ptX = std::stof(argv[17]);
  const float ptY = std::stof(argv[18]);
  const std::string sourceFile = argv[19];
  const double NA = std::stof(argv[20]);
  const float defocus = std::stof(argv[21]);
  int nk = std::stoi(argv[22]);

  if (Lx <= 0 || Ly <= 0 || msx <= 0 || msy <= 0 || Lx < msx || Ly < msy || srcSize <= 0) {
    std::cerr << "Error: Invalid input parameters. Please check the values." << std::endl;
    return 1;
  }
  double n_medium = 1.0;
  if (const char* e = std::getenv("KLITHO_N_MEDIUM")) n_medium = std::atof(e);
  int precision = KL_PREC_FAST;
  if (const char* e = std::getenv("KLITHO_PRECISION"))
    if (std::string(e) == "fp64") precision = KL_PREC_FP64;
  const double na_max = n_medium > 1.0 ? n_medium : 1.0;
  if (NA < 0 || NA > na_max) {
    if (na_max == 1.0)
      std::cerr << "Error: NA must be in the range [0, 1]." << std::endl;
    else
      std::cerr << "Error: NA must be in the range [0, " << na_max << "]." << std::endl;
    return 1;
  }
  const float wavelength = 193;
  const float dose = 1.0;

  std::vector<float> src((size_t)srcSize * srcSize, 0.0f);
  if (kl_create_source(srcSize, srcType.c_str(), innerR, outerR, radius, offset, onXAxis ? 1 : 0,
                       ptX, ptY, sourceFile.c_str(), src.data()) != KL_OK)
    std::exit(1);
  klcli::png("./out/source.png", src, srcSize, srcSize, klcli::min_of(src), klcli::max_of(src), KL_PNG_GRAY);
  std::stringstream ssrc;
  ssrc << "Source Size: " << srcSize << " x " << srcSize << "\nSource Type: " << srcType << "\n";
  if (srcType == "Annular")
    ssrc << "Inner Radius: " << innerR << "\nOuter Radius: " << outerR << "\n";
  else if (srcType == "Dipole")
    ssrc << "Radius: " << radius << "\nOffset: " << offset << "\nOnXAxis: " << onXAxis << "\n";
  else if (srcType == "CrossQuadrupole")
    ssrc << "Radius: " << radius << "\nOffset: " << offset << "\n";
  else if (srcType == "Point")
    ssrc << "Point Position: (" << ptX << ", " << ptY << ")\n";

  std::vector<float> msk((size_t)Lx * Ly, 0.0f);
  if (kl_create_mask(Lx, Ly, msx, msy, maskType.c_str(), lineWidth, spaceWidth, isHorizontal,
                     maskFile.c_str(), dose, msk.data()) != KL_OK)
    std::exit(1);
  klcli::png("./out/mask.png", msk, Lx, Ly, klcli::min_of(msk), klcli::max_of(msk), KL_PNG_GRAY);

  float outerSigma = kl_outer_sigma(src.data(), srcSize);
  if (outerSigma > 1) {
    std::cout << "Warning: Outer Sigma is greater than 1. Setting outerSigma = 1." << std::endl;
    outerSigma = 1;
  }
  int Nx = 0, Ny = 0;
  kl_band_size(NA, Lx, Ly, outerSigma, &Nx, &Ny);
  const int tccSize = (2 * Nx + 1) * (2 * Ny + 1);
  if (tccSize < nk) {
    std::cout << "Warning: Number of kernels (nk) is greater than TCC size (tccSize). Setting nk = tccSize."
              << std::endl;
    nk = tccSize;
  }

  std::cout << std::endl << "Simulation Parameters:" << std::endl;
  std::cout << "-------------------" << std::endl;
  std::cout << klcli::mask_params(Lx, Ly, msx, msy, maskType, lineWidth, spaceWidth);
  std::cout << ssrc.str();
  std::cout << "Wavelength: " << wavelength << " nm" << std::endl;
  std::cout << "NA: " << NA << std::endl;
  std::cout << "Defocus: " << defocus << std::endl;
  std::cout << "Dose: " << dose << std::endl;
  std::cout << "Nx: " << Nx << ", Ny: " << Ny << std::endl;
  std::cout << "TCC Size: " << tccSize << " x " << tccSize << std::endl;
  std::cout << "Number of Kernels: " << nk << std::endl << std::endl;

  klcli::banner_section("Calculating FFT Mask...");
  kl_tcc_plan plan = nullptr;
  if (kl_tcc_plan_create(&plan, src.data(), srcSize, NA, defocus, n_medium, Lx, Ly, KL_PREC_FAST) != KL_OK)
    return klcli::fail("kl_tcc_plan_create");

  klcli::banner_section("Starting calcTCC...");
  if (klcli::png_enabled()) {
    std::vector<float> tr((size_t)tccSize * tccSize), ti((size_t)tccSize * tccSize);
    if (kl_tcc_build_host(plan, tr.data(), ti.data()) != KL_OK) return klcli::fail("kl_tcc_build_host");
    float mx = klcli::max_of(tr), mn = klcli::min_of(tr);
    std::cout << "Max. TCC Real Value: " << mx << std::endl;
    klcli::png("./out/tcc_r.png", tr, tccSize, tccSize, mn, mx, KL_PNG_CONTINUOUS);
    mx = klcli::max_of(ti);
    mn = klcli::min_of(ti);
    std::cout << "Max. TCC Imag Value: " << mx << std::endl;
    klcli::png("./out/tcc_i.png", ti, tccSize, tccSize, mn, mx, KL_PNG_CONTINUOUS);
  } else {
    double mm[4];
    if (kl_tcc_build_minmax(plan, mm) != KL_OK) return klcli::fail("kl_tcc_build_minmax");
    std::cout << "Max. TCC Real Value: " << (float)mm[0] << std::endl;
    std::cout << "Max. TCC Imag Value: " << (float)mm[2] << std::endl;
  }

  // calcKernels first (its files are written even if the image fails)
  std::vector<float> kre((size_t)nk * tccSize), kim((size_t)nk * tccSize), scales(nk);
  std::vector<double> ev(nk);
  int eig_rc = KL_OK;
  std::string eig_err;
  if (nk > 0) {
    kl_tcc_plan eplan = plan;
    kl_tcc_plan plan64 = nullptr;
    if (precision == KL_PREC_FP64) {
      if (kl_tcc_plan_create(&plan64, src.data(), srcSize, NA, defocus, n_medium, Lx, Ly, KL_PREC_FP64) != KL_OK)
        return klcli::fail("kl_tcc_plan_create");
      eplan = plan64;
    }
    int iters = 0;
    eig_rc = kl_topk_eig(eplan, nk, 0, kre.data(), kim.data(), scales.data(), ev.data(), &iters);
    if (eig_rc != KL_OK) eig_err = kl_last_error();
    if (plan64) kl_tcc_plan_destroy(plan64);
    if (eig_rc == KL_OK) {
      for (int i = 0; i < nk; ++i) {
        const std::string b = "./out/kernels/krn_" + std::to_string(i);
        if (kl_write_float_file((b + "_r.bin").c_str(), kre.data() + (size_t)i * tccSize, tccSize) != KL_OK ||
            kl_write_float_file((b + "_i.bin").c_str(), kim.data() + (size_t)i * tccSize, tccSize) != KL_OK)
          std::exit(1);
        const std::vector<float> kr(kre.begin() + (size_t)i * tccSize, kre.begin() + (size_t)(i + 1) * tccSize);
        const std::vector<float> ki(kim.begin() + (size_t)i * tccSize, kim.begin() + (size_t)(i + 1) * tccSize);
        const std::string pb = "./out/kernels/png/krn_" + std::to_string(i);
        klcli::png(pb + "_r.png", kr, 2 * Nx + 1, 2 * Ny + 1, klcli::min_of(kr), klcli::max_of(kr), KL_PNG_CONTINUOUS);
        klcli::png(pb + "_i.png", ki, 2 * Nx + 1, 2 * Ny + 1, klcli::min_of(ki), klcli::max_of(ki), KL_PNG_CONTINUOUS);
      }
      if (kl_write_kernel_info("./out/kernels/kernel_info.txt", 2 * Nx + 1, 2 * Ny + 1, nk, scales.data()) != KL_OK)
        std::exit(1);
    }
  }

  klcli::banner_section("Starting calcImage...");
  int img_rc = KL_OK;
  {
    std::vector<float> img((size_t)Lx * Ly);
    const bool pow2 = (Lx & (Lx - 1)) == 0 && (Ly & (Ly - 1)) == 0;
    if (precision == KL_PREC_FP64 && pow2) {
      kl_tcc_plan plan64 = nullptr;
      img_rc = kl_tcc_plan_create(&plan64, src.data(), srcSize, NA, defocus, n_medium, Lx, Ly, KL_PREC_FP64);
      if (img_rc == KL_OK) img_rc = kl_fp64_hopkins_image_host(plan64, msk.data(), img.data());
      if (plan64) kl_tcc_plan_destroy(plan64);
    } else {
      if (precision == KL_PREC_FP64)
        std::cerr << "Note: the FP64 Hopkins image needs power-of-two periods; using the fast path." << std::endl;
      img_rc = kl_hopkins_image_host(plan, msk.data(), img.data());
    }
    if (img_rc != KL_OK) {
      std::cerr << "Error: calcImage failed: " << kl_last_error() << std::endl;
    } else {
      const float mx = klcli::max_of(img), mn = klcli::min_of(img);
      std::cout << "Max. Intensity: " << mx << std::endl;
      if (kl_write_float_file("./out/image.bin", img.data(), Lx * Ly) != KL_OK) std::exit(1);
      klcli::png("./out/image.png", img, Lx, Ly, mn, mx, KL_PNG_CONTINUOUS);
      klcli::png("./out/image_s.png", img, Lx, Ly, 0.0f, kTargetIntensity, KL_PNG_7COLORS);
    }
  }

  if (nk > 0) {
    klcli::banner_section("Starting calcKernels...");
    std::cout << "Solving eigenproblem..." << std::endl;
    if (eig_rc != KL_OK) {
      std::cerr << "Kernels derivation failed with info = " << eig_rc << " (" << eig_err << ")" << std::endl;
      kl_tcc_plan_destroy(plan);
      return 1;
    }
    std::cout << "Eigenvalues: " << std::endl;
    for (int j = 0; j < nk; ++j) std::cout << ev[j] << " ";
    std::cout << std::endl;
  }
  if (img_rc != KL_OK) {
    kl_tcc_plan_destroy(plan);
    return 1;
  }
  kl_tcc_plan_destroy(plan);
  klcli::banner_end(start);
  return 0;
}
