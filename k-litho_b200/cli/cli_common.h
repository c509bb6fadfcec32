// cli_common.h -- pieces shared by the drop-in klitho_tcc / klitho_socs CLIs:
// the reference's console banners and parameter echo, and timing.
#pragma once

#include <chrono>
#include <iostream>
#include <sstream>
#include <string>

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

inline int fail(const char* what) {
  std::cerr << "Error: " << what << ": " << kl_last_error() << std::endl;
  return 1;
}

}  // namespace klcli
