// kl_host.cpp -- host-side inputs of the imaging path: source and mask
// builders, band sizing, and the reference's on-disk formats.  These run on
// the CPU by design (they are O(srcSize^2) / O(L^2) setup work that feeds
// the GPU); their results must match the reference bit for bit, so each
// one follows the reference's arithmetic types (float vs double) exactly.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "kl_internal.h"

namespace kl {

static thread_local std::string t_err;
void set_error(const std::string& msg) { t_err = msg; }

// The library's own stream-ordered pool per device (cudaMemPoolCreate), which
// keeps freed blocks (release threshold at its maximum) so repeated calls
// neither synchronise nor allocate afresh.  The device's default pool -- the
// host program's cudaMallocAsync -- is left as the program configured it.
int scratch_alloc(void** p, size_t bytes, cudaStream_t st, const char* what) {
  static std::mutex mu;
  static std::vector<std::pair<int, cudaMemPool_t>> pools;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(mu);
    for (auto& e : pools)
      if (e.first == dev) pool = e.second;
    if (!pool) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        pools.emplace_back(dev, pool);
      } else {
        pool = nullptr;
        set_error("scratch pool creation failed");
        return KL_ERR_NOMEM;
      }
    }
  }
  *p = nullptr;
  const cudaError_t e = cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, st);
  if (e != cudaSuccess) {
    *p = nullptr;
    set_error(std::string("device allocation failed (") + what + ", " + std::to_string(bytes) +
              " bytes): " + cudaGetErrorString(e));
    return KL_ERR_NOMEM;
  }
  return KL_OK;
}

void scratch_free(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}
const char* last_error() { return t_err.c_str(); }

namespace {

std::string extension_of(const std::string& path) {
  return path.substr(path.find_last_of('.') + 1);
}

// Raw float32 file -> `size` floats.  common/file_io.cpp:232-260 keeps the
// first fileSize/4 floats, zero-pads, and warns when the byte count differs.
int read_bin(const std::string& path, int size, std::vector<float>& out, int* count) {
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) {
    set_error("Error: Failed to open file " + path);
    std::cerr << "Error: Failed to open file " << path << std::endl;
    return KL_ERR_IO;
  }
  f.seekg(0, std::ios::end);
  long long bytes = (long long)f.tellg();
  f.seekg(0, std::ios::beg);
  std::vector<char> raw((size_t)(bytes > 0 ? bytes : 0));
  if (bytes > 0) f.read(raw.data(), bytes);
  if (!f) {
    set_error("Error: Failed to read data from file " + path);
    std::cerr << "Error: Failed to read data from file " << path << std::endl;
    return KL_ERR_IO;
  }
  out.assign((size_t)size, 0.0f);
  size_t nfl = (size_t)bytes / sizeof(float);
  size_t ncopy = nfl < (size_t)size ? nfl : (size_t)size;
  if (ncopy) std::memcpy(out.data(), raw.data(), ncopy * sizeof(float));
  if (bytes != (long long)size * (long long)sizeof(float)) {
    std::cerr << "Warning: File size (" << bytes
              << " bytes) does not match the expected data size (" << size * sizeof(float)
              << " bytes)" << std::endl;
  }
  if (count) *count = (int)nfl;
  return KL_OK;
}

// Whitespace-separated text.  common/file_io.cpp:204-230.
int read_txt(const std::string& path, int size, std::vector<float>& out, int* count) {
  std::ifstream f(path);
  if (!f.is_open()) {
    set_error("Error: Failed to open file " + path);
    std::cerr << "Error: Failed to open file " << path << std::endl;
    return KL_ERR_IO;
  }
  std::vector<float> vals;
  float v;
  while (f >> v) vals.push_back(v);
  if (!f.eof()) {
    set_error("Error: Failed to read data from file " + path);
    std::cerr << "Error: Failed to read data from file " << path << std::endl;
    return KL_ERR_IO;
  }
  if ((int)vals.size() != size) {
    std::cerr << "Warning: Data size (" << vals.size() << ") does not match the expected size ("
              << size << ")" << std::endl;
  }
  if (count) *count = (int)vals.size();
  vals.resize((size_t)size, 0.0f);
  out.swap(vals);
  return KL_OK;
}

int read_any(const std::string& path, int size, std::vector<float>& out, int* count) {
  if (extension_of(path) == "bin") return read_bin(path, size, out, count);
  return read_txt(path, size, out, count);
}

}  // namespace
}  // namespace kl

using kl::set_error;

extern "C" {

int kl_version(void) { return 10000; }
const char* kl_last_error(void) { return kl::last_error(); }

int kl_read_float_file(const char* path, int size, float* out, int* count) {
  KL_CHECK_ARG(path && out && size >= 0, "kl_read_float_file: bad arguments");
  std::vector<float> v;
  int rc = kl::read_any(path, size, v, count);
  if (rc) return rc;
  if (size) std::memcpy(out, v.data(), sizeof(float) * (size_t)size);
  return KL_OK;
}

int kl_write_float_file(const char* path, const float* data, int size) {
  KL_CHECK_ARG(path && (data || size == 0) && size >= 0, "kl_write_float_file: bad arguments");
  std::ofstream f(path, std::ios::binary);
  if (!f.is_open()) {
    set_error(std::string("Error: Failed to open file ") + path);
    std::cerr << "Error: Failed to open file " << path << std::endl;
    return KL_ERR_IO;
  }
  f.write(reinterpret_cast<const char*>(data), (std::streamsize)size * sizeof(float));
  if (!f) {
    set_error(std::string("Error: Failed to write data to file ") + path);
    std::cerr << "Error: Failed to write data to file " << path << std::endl;
    return KL_ERR_IO;
  }
  return KL_OK;
}

// Text layout of common/file_io.cpp:269-277; eigenvalues are printed with
// the stream's default 6 significant digits.
int kl_write_kernel_info(const char* path, int krnSizeX, int krnSizeY, int nk,
                         const float* scales) {
  KL_CHECK_ARG(path && (scales || nk == 0), "kl_write_kernel_info: bad arguments");
  std::ofstream f(path);
  if (!f) {
    set_error(std::string("Error opening file for writing: ") + path);
    std::cerr << "Error opening file for writing: " << path << std::endl;
    return KL_ERR_IO;
  }
  f << "# Kernel Information\n";
  f << "## Kernel Size and Count\n";
  f << "- Kernel Size: " << krnSizeX << "x" << krnSizeY << "\n";
  f << "- Number of Kernels: " << nk << "\n";
  f << "## Eigenvalues of Each Kernel\n";
  for (int i = 0; i < nk; ++i) f << "Eigenvalue " << i << ": " << scales[i] << "\n";
  return f ? KL_OK : KL_ERR_IO;
}

// Parser with the reference's matching rules (file_io.cpp:289-304): lines are
// recognised by substring, numbers read with the same sscanf patterns, and an
// eigenvalue index is accepted when 0 <= index < the kernel count seen so far.
int kl_read_kernel_info(const char* path, int* krnSizeX, int* krnSizeY, int* nk, float* scales,
                        int cap) {
  KL_CHECK_ARG(path && krnSizeX && krnSizeY && nk, "kl_read_kernel_info: bad arguments");
  std::ifstream f(path);
  if (!f) {
    set_error(std::string("Error opening file for reading: ") + path);
    std::cerr << "Error opening file for reading: " << path << std::endl;
    return KL_ERR_IO;
  }
  int kx = *krnSizeX, ky = *krnSizeY, n = *nk;
  std::string line;
  while (std::getline(f, line)) {
    if (line.find("Kernel Size:") != std::string::npos) {
      std::sscanf(line.c_str(), "- Kernel Size: %dx%d", &kx, &ky);
    } else if (line.find("Number of Kernels:") != std::string::npos) {
      std::sscanf(line.c_str(), "- Number of Kernels: %d", &n);
    } else if (line.find("Eigenvalue") != std::string::npos) {
      int idx = -1;
      double val = 0.0;
      std::sscanf(line.c_str(), "Eigenvalue %d: %lf", &idx, &val);
      if (idx >= 0 && idx < n && scales && idx < cap) scales[idx] = (float)val;
    }
  }
  *krnSizeX = kx;
  *krnSizeY = ky;
  *nk = n;
  return KL_OK;
}

// --------------------------------------------------------------------------
// Source shapes: K-Litho-TCC/source.cpp
// --------------------------------------------------------------------------
int kl_create_source(int n, const char* type, float innerRadius, float outerRadius, float radius,
                     float offset, int onXAxis, float ptX, float ptY, const char* sourceFile,
                     float* out) {
  KL_CHECK_ARG(n > 0 && type && out, "kl_create_source: bad arguments");
  const std::string t(type);
  const size_t nn = (size_t)n * n;
  const int half = (n - 1) / 2;
  if (t == "Annular") {  // source.cpp:5-24
    const int rin = (int)(innerRadius * (float)half);
    const int rout = (int)(outerRadius * (float)half);
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        const double dx = (double)(x - half), dy = (double)(y - half);
        const double d = std::sqrt(dx * dx + dy * dy);
        out[(size_t)y * n + x] = (d >= (double)rin && d <= (double)rout) ? 1.0f : 0.0f;
      }
  } else if (t == "Dipole" || t == "CrossQuadrupole") {  // source.cpp:25-88
    const int off = (int)(offset * (float)half);
    const int rad = (int)(radius * (float)half);
    int cxy[4][2];
    int npoles;
    if (t == "Dipole") {  // centre n/2, poles along x or y
      const int c = n / 2;
      const int ox = onXAxis ? off : 0, oy = onXAxis ? 0 : off;
      cxy[0][0] = c + ox; cxy[0][1] = c + oy;
      cxy[1][0] = c - ox; cxy[1][1] = c - oy;
      npoles = 2;
    } else {  // centre (n-1)/2, poles on both axes
      const int c = half;
      cxy[0][0] = c; cxy[0][1] = c + off;
      cxy[1][0] = c; cxy[1][1] = c - off;
      cxy[2][0] = c + off; cxy[2][1] = c;
      cxy[3][0] = c - off; cxy[3][1] = c;
      npoles = 4;
    }
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        bool in = false;
        for (int i = 0; i < npoles && !in; ++i) {
          const double dx = (double)(x - cxy[i][0]), dy = (double)(y - cxy[i][1]);
          in = std::sqrt(dx * dx + dy * dy) <= (double)rad;
        }
        out[(size_t)y * n + x] = in ? 1.0f : 0.0f;
      }
  } else if (t == "Point") {  // source.cpp:122-129, on a zero map
    std::memset(out, 0, sizeof(float) * nn);
    int ix = (int)std::round((double)(ptX * (float)n) / 2.0 + n / 2.0);
    int iy = (int)std::round((double)(-1.0f * ptY * (float)n) / 2.0 + n / 2.0);
    if (ptX >= 0) ix -= 1;
    if (-1.0f * ptY >= 0) iy -= 1;
    if (ix < 0 || ix >= n || iy < 0 || iy >= n) {
      set_error("kl_create_source: point outside the source grid");
      return KL_ERR_INVALID;
    }
    out[(size_t)iy * n + ix] = 1.0f;
  } else if (t == "Import") {  // source.cpp:130-139
    std::cout << "Read Source: " << (sourceFile ? sourceFile : "") << std::endl;
    std::vector<float> v;
    int rc = kl::read_any(sourceFile ? sourceFile : "", (int)nn, v, nullptr);
    if (rc) return rc;
    std::memcpy(out, v.data(), sizeof(float) * nn);
  } else {
    // unknown type: the reference leaves the (zero) map untouched
    std::memset(out, 0, sizeof(float) * nn);
  }
  // normalizeMatrix (source.cpp:89-103): float running sum, then divide
  float sum = 0.0f;
  for (size_t i = 0; i < nn; ++i) sum += out[i];
  if (sum != 0.0f)
    for (size_t i = 0; i < nn; ++i) out[i] /= sum;
  return KL_OK;
}

// --------------------------------------------------------------------------
// Mask: common/mask.cpp
// --------------------------------------------------------------------------
int kl_create_mask(int Lx, int Ly, int msx, int msy, const char* type, int lineWidth,
                   int spaceWidth, int isHorizontal, const char* maskFile, float dose,
                   float* out) {
  KL_CHECK_ARG(Lx > 0 && Ly > 0 && msx > 0 && msy > 0 && msx <= Lx && msy <= Ly && type && out,
               "kl_create_mask: bad arguments");
  const std::string t(type);
  std::vector<float> in((size_t)msx * msy, 0.0f);
  if (t == "LineSpace") {  // mask.cpp:5-29
    const int period = lineWidth + spaceWidth;
    KL_CHECK_ARG(period > 0, "kl_create_mask: lineWidth + spaceWidth must be positive");
    for (int y = 0; y < msy; ++y)
      for (int x = 0; x < msx; ++x) {
        const int u = isHorizontal ? y : x;
        in[(size_t)y * msx + x] = (u % period) < lineWidth ? 1.0f : 0.0f;
      }
  } else if (t == "Import") {  // mask.cpp:42-52
    std::cout << "Read Mask: " << (maskFile ? maskFile : "") << std::endl;
    int rc = kl::read_any(maskFile ? maskFile : "", msx * msy, in, nullptr);
    if (rc) return rc;
  }
  std::memset(out, 0, sizeof(float) * (size_t)Lx * Ly);
  const int oy = (Ly - msy) / 2, ox = (Lx - msx) / 2;  // mask.cpp:53-59
  for (int y = 0; y < msy; ++y)
    for (int x = 0; x < msx; ++x)
      out[(size_t)(y + oy) * Lx + x + ox] = in[(size_t)y * msx + x] * dose;
  return KL_OK;
}

// getOuterSigma: klitho_tcc.cpp:52-67
float kl_outer_sigma(const float* src, int n) {
  if (!src || n <= 0) return 0.0f;
  const int c = (n - 1) / 2;
  float far = 0.0f;
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < n; ++x)
      if (src[(size_t)y * n + x] != 0.0f) {
        const float d = (float)std::sqrt((double)((y - c) * (y - c) + (x - c) * (x - c)));
        if (d > far) far = d;
      }
  return far / (float)c;
}

// klitho_tcc.cpp:479-486, float arithmetic throughout
int kl_band_size(double NA, int Lx, int Ly, float outerSigma, int* Nx, int* Ny) {
  KL_CHECK_ARG(Nx && Ny && Lx > 0 && Ly > 0, "kl_band_size: bad arguments");
  const float s = outerSigma > 1.0f ? 1.0f : outerSigma;
  const float na = (float)NA, lambda = 193.0f;
  *Nx = (int)std::floor(na * (float)Lx * (1.0f + s) / lambda);
  *Ny = (int)std::floor(na * (float)Ly * (1.0f + s) / lambda);
  return KL_OK;
}

// klitho_tcc.cpp:202-205
int kl_source_point_count(const float* src, int n, float outerSigma) {
  if (!src || n <= 0) return 0;
  const float s = outerSigma > 1.0f ? 1.0f : outerSigma;
  const int sh = (int)((n - 1) / 2.0);
  const int os = (int)std::ceil((float)sh * s);
  int S = 0;
  for (int q = -os; q <= os; ++q)
    for (int p = -os; p <= os; ++p) {
      const int id = (q + sh) * n + p + sh;
      if (src[id] != 0.0f && p * p + q * q <= sh * sh) ++S;
    }
  return S;
}

}  // extern "C"
