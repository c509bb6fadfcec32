// cli_common.h -- pieces shared by the drop-in klitho_tcc / klitho_socs CLIs:
// the reference's console banners and parameter echo, and timing.
#pragma once

#include <chrono>
#include <iostream>
#include <sstream>
#include <cstdlib>
#include <string>
#include <vector>

#include "klitho_gpu.h"

namespace klcli {

inline void banner_start() {
  std::cout << "************************************" << std::endl;
  std::cout << "* Lithography Simulation initiated..." << std::endl;
  std::cout << "************************************" << std::endl;
}

inline void banner_section(const char* title) {
  std::cout << std::endl << "------------------------------------" << std::endl;
  std::cout << title << std::endl;
}

inline void banner_end(std::chrono::system_clock::time_point start) {
  auto us = std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::system_clock::now() -
                                                                  start)
                .count();
  std::cout << std::endl << "------------------------------------" << std::endl;
  std::cout << "Simulation completed." << std::endl;
  std::cout << "Total Execution Time: " << us * 1.0e-06 << " sec." << std::endl;
  std::cout << "************************************" << std::endl;
}

// Parameter echo of common/mask.cpp:214,217
inline std::string mask_params(int Lx, int Ly, int msx, int msy, const std::string& type, int lw,
                               int sw) {
  std::stringstream ss;
  ss << "Mask Period: " << Lx << " x " << Ly << "\nMask Size: " << msx << " x " << msy
     << "\nMask Type: " << type << "\n";
  if (type == "LineSpace") ss << "Line Width: " << lw << "\nSpace Width: " << sw << "\n";
  return ss.str();
}

// the reference's optional PNG outputs (common/file_io.cpp:7-135); KLITHO_PNG=0
// skips them
inline bool png_enabled() {
  const char* e = std::getenv("KLITHO_PNG");
  return !(e && std::string(e) == "0");
}

inline float min_of(const std::vector<float>& v) {
  float m = v.empty() ? 0.f : v[0];
  for (float x : v) m = x < m ? x : m;
  return m;
}
inline float max_of(const std::vector<float>& v) {
  float m = v.empty() ? 0.f : v[0];
  for (float x : v) m = x > m ? x : m;
  return m;
}

// writes a PNG like the reference: on failure, the message and exit(1)
inline void png(const std::string& path, const std::vector<float>& data, int sx, int sy, float mn, float mx,
                int colormap) {
  if (!png_enabled()) return;
  if (kl_write_png(path.c_str(), data.data(), sx, sy, mn, mx, colormap) != KL_OK) {
    std::cerr << kl_last_error() << std::endl;
    std::exit(1);
  }
}

inline int fail(const char* what) {
  std::cerr << "Error: " << what << ": " << kl_last_error() << std::endl;
  return 1;
}

}  // namespace klcli
