// klitho_socs -- drop-in replacement for K-Litho-SOCS/klitho_socs.
//
// Same 10 positional arguments (klitho_socs.cpp:251-270), same validation and
// console output, same inputs (kernel_info.txt + krn_<i>_{r,i}.bin from the
// kernel directory, float32 mask) and the same ./out/image.bin.  The image is
// computed on the GPU by the fused SOCS pipeline of libklitho_gpu
// (kl_socs_forward_host) instead of FFTW, for any period Lx x Ly.  The
// reference's PNG previews (mask.png, image.png, image_s.png) are written by
// the library's own PNG writer; KLITHO_PNG=0 skips them.
#include <cstdlib>
#include <string>
#include <vector>

#include "cli_common.h"

// TARGET_INTENSITY of klitho_socs.cpp:275, the top of image_s.png's colour scale
constexpr float kTargetIntensity = 0.225f;

int main(int argc, char* argv[]) {
  klcli::banner_start();
  auto start = std::chrono::system_clock::now();
  if (argc != 11) {
    std::cerr << "Error: Invalid number of arguments: " << argc << ". Expected 11 arguments."
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
  const std::string krnDir = argv[10];
  if (Lx <= 0 || Ly <= 0 || msx <= 0 || msy <= 0 || Lx < msx || Ly < msy) {
    std::cerr << "Error: Invalid input parameters. Please check the values." << std::endl;
    return 1;
  }

  int kx = 0, ky = 0, nk = 0;
  std::vector<float> scales(1 << 16, 0.0f);
  if (kl_read_kernel_info((krnDir + "kernel_info.txt").c_str(), &kx, &ky, &nk, scales.data(),
                          (int)scales.size()) != KL_OK)
    return 1;
  if (kx % 2 == 0 || ky % 2 == 0) {
    std::cerr << "Error: Kernel size must be odd." << std::endl;
    return 1;
  }
  if (nk <= 0) {
    std::cerr << "Error: kernel_info.txt declares no kernels." << std::endl;
    return 1;
  }
  scales.resize(nk);
  const int Nx = (kx - 1) / 2, Ny = (ky - 1) / 2;
  const size_t nb = (size_t)kx * ky;
  std::vector<float> kre(nb * nk), kim(nb * nk);
  for (int i = 0; i < nk; ++i) {
    const std::string fr = krnDir + "krn_" + std::to_string(i) + "_r.bin";
    const std::string fi = krnDir + "krn_" + std::to_string(i) + "_i.bin";
    std::cout << "Read Kernel " << i << " : " << fr << std::endl;
    if (kl_read_float_file(fr.c_str(), (int)nb, kre.data() + nb * i, nullptr) != KL_OK) return 1;
    std::cout << "Read Kernel " << i << " : " << fi << std::endl;
    if (kl_read_float_file(fi.c_str(), (int)nb, kim.data() + nb * i, nullptr) != KL_OK) return 1;
  }

  std::vector<float> msk((size_t)Lx * Ly);
  if (kl_create_mask(Lx, Ly, msx, msy, maskType.c_str(), lineWidth, spaceWidth, isHorizontal,
                     maskFile.c_str(), 1.0f, msk.data()) != KL_OK)
    return 1;
  klcli::png("./out/mask.png", msk, Lx, Ly, klcli::min_of(msk), klcli::max_of(msk), KL_PNG_GRAY);

  std::cout << std::endl << "Simulation Parameters:" << std::endl;
  std::cout << "-------------------" << std::endl;
  std::cout << klcli::mask_params(Lx, Ly, msx, msy, maskType, lineWidth, spaceWidth);
  std::cout << "Nx: " << Nx << ",  Ny: " << Ny << std::endl;
  std::cout << "Number of Kernels: " << nk << std::endl << std::endl;

  klcli::banner_section("Calculating FFT Mask...");
  kl_socs_plan plan = nullptr;
  if (kl_socs_plan_create(&plan, Lx, Ly, Nx, Ny, nk, 1, 1) != KL_OK)
    return klcli::fail("kl_socs_plan_create");
  if (kl_socs_set_kernels(plan, 0, kre.data(), kim.data(), scales.data()) != KL_OK)
    return klcli::fail("kl_socs_set_kernels");
  klcli::banner_section("Calc Image...");
  std::vector<float> img((size_t)Lx * Ly);
  if (kl_socs_forward_host(plan, msk.data(), 1, img.data(), nullptr) != KL_OK)
    return klcli::fail("kl_socs_forward_host");
  kl_socs_plan_destroy(plan);

  const float mx = klcli::max_of(img), mn = klcli::min_of(img);
  std::cout << "Max. Intensity: " << mx << std::endl;
  if (kl_write_float_file("./out/image.bin", img.data(), Lx * Ly) != KL_OK) std::exit(1);
  klcli::png("./out/image.png", img, Lx, Ly, mn, mx, KL_PNG_CONTINUOUS);
  klcli::png("./out/image_s.png", img, Lx, Ly, 0.0f, kTargetIntensity, KL_PNG_7COLORS);
  klcli::banner_end(start);
  return 0;
}
