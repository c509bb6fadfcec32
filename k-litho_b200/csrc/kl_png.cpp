// kl_png.cpp -- the optional PNG outputs of the reference programs
// (common/file_io.cpp:7-135: grayscale, 7-colour and continuous colour maps
// of a float array between given min and max), written by the library's own
// PNG encoder: 8-bit grey or RGB, one IDAT chunk deflated by the system zlib,
// no row filters.  The pixel values follow the reference's conversion
// arithmetic (a float ratio clamped to [0, 1], then the colour map, then a
// truncating cast to unsigned char); the compressed bytes differ from the
// reference's (another deflate encoder), the decoded pixels do not.
#include <zlib.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "kl_internal.h"

namespace {

void put_be32(std::vector<unsigned char>& v, uint32_t x) {
  v.push_back((unsigned char)(x >> 24));
  v.push_back((unsigned char)(x >> 16));
  v.push_back((unsigned char)(x >> 8));
  v.push_back((unsigned char)x);
}

void put_chunk(std::vector<unsigned char>& out, const char type[4], const unsigned char* data, size_t n) {
  put_be32(out, (uint32_t)n);
  const size_t at = out.size();
  out.insert(out.end(), type, type + 4);
  out.insert(out.end(), data, data + n);
  const uLong crc = crc32(0L, out.data() + at, (uInt)(n + 4));
  put_be32(out, (uint32_t)crc);
}

// ratio in [0, 1] as the reference forms it: float arithmetic, clamp
inline float unit(float v, float mn, float mx) { return std::max(0.0f, std::min(1.0f, (v - mn) / (mx - mn))); }

void seven_colors(double value, unsigned char* rgb) {
  unsigned char R = 0, G = 0, B = 0;
  if (value < 1.0 / 6.0) {
    B = 255;
  } else if (value < 2.0 / 6.0) {
    G = 127;
    B = 255;
  } else if (value < 3.0 / 6.0) {
    G = 255;
    B = 127;
  } else if (value < 4.0 / 6.0) {
    G = 255;
  } else if (value < 5.0 / 6.0) {
    R = 127;
    G = 255;
  } else if (value < 1.0) {
    R = 255;
    G = 127;
  } else {
    R = 255;
  }
  rgb[0] = R;
  rgb[1] = G;
  rgb[2] = B;
}

// piecewise-linear blue -> aqua -> green -> yellow -> orange -> red
void continuous(double value, unsigned char* rgb) {
  unsigned char R = 0, G = 0, B = 0;
  if (value < 1.0 / 6.0) {
    B = 255;
    G = (unsigned char)(value * 6 * 127);
  } else if (value < 2.0 / 6.0) {
    G = 127 + (unsigned char)((value - 1.0 / 6.0) * 6 * 128);
    B = (unsigned char)(255 - (value - 1.0 / 6.0) * 6 * 127);
  } else if (value < 3.0 / 6.0) {
    G = 255;
    B = (unsigned char)(128 - (value - 2.0 / 6.0) * 6 * 128);
  } else if (value < 4.0 / 6.0) {
    R = (unsigned char)((value - 3.0 / 6.0) * 6 * 127);
    G = 255;
  } else if (value < 5.0 / 6.0) {
    R = 127 + (unsigned char)((value - 4.0 / 6.0) * 6 * 128);
    G = (unsigned char)(255 - (value - 4.0 / 6.0) * 6 * 127);
  } else {
    R = 255;
    G = (unsigned char)(128 - (value - 5.0 / 6.0) * 6 * 128);
  }
  rgb[0] = R;
  rgb[1] = G;
  rgb[2] = B;
}

}  // namespace

extern "C" int kl_write_png(const char* path, const float* data, int sizeX, int sizeY, float mn, float mx,
                            int colormap) {
  KL_CHECK_ARG(path && data && sizeX > 0 && sizeY > 0, "kl_write_png: bad argument");
  KL_CHECK_ARG(colormap >= 0 && colormap <= 2, "kl_write_png: colormap must be 0 (grey), 1 (7 colours) or 2 (continuous)");
  const int ch = colormap == 0 ? 1 : 3;
  const size_t row = (size_t)sizeX * ch + 1;  // filter byte + pixels
  std::vector<unsigned char> raw(row * sizeY);
  for (int y = 0; y < sizeY; ++y) {
    unsigned char* r = raw.data() + (size_t)y * row;
    r[0] = 0;  // no filter
    for (int x = 0; x < sizeX; ++x) {
      const float v = data[(size_t)y * sizeX + x];
      unsigned char* px = r + 1 + (size_t)x * ch;
      if (colormap == 0) {
        px[0] = (unsigned char)(unit(v, mn, mx) * 255.0f);
      } else if (mn == mx) {  // the reference's uniform-image case: all green
        px[0] = 0;
        px[1] = 255;
        px[2] = 0;
      } else if (colormap == 1) {
        seven_colors((double)unit(v, mn, mx), px);
      } else {
        continuous((double)unit(v, mn, mx), px);
      }
    }
  }
  uLongf zlen = compressBound((uLong)raw.size());
  std::vector<unsigned char> z(zlen);
  if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) {
    kl::set_error(std::string("kl_write_png: compression failed for ") + path);
    return KL_ERR_IO;
  }
  std::vector<unsigned char> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
  std::vector<unsigned char> ihdr;
  put_be32(ihdr, (uint32_t)sizeX);
  put_be32(ihdr, (uint32_t)sizeY);
  ihdr.push_back(8);                              // bit depth
  ihdr.push_back(colormap == 0 ? 0 : 2);          // grey or RGB
  ihdr.push_back(0);                              // deflate
  ihdr.push_back(0);                              // adaptive filtering (type 0 rows)
  ihdr.push_back(0);                              // no interlace
  put_chunk(out, "IHDR", ihdr.data(), ihdr.size());
  put_chunk(out, "IDAT", z.data(), zlen);
  put_chunk(out, "IEND", nullptr, 0);
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    kl::set_error(std::string("Error: Failed to write PNG: ") + path);
    return KL_ERR_IO;
  }
  const size_t w = std::fwrite(out.data(), 1, out.size(), f);
  std::fclose(f);
  if (w != out.size()) {
    kl::set_error(std::string("Error: Failed to write PNG: ") + path);
    return KL_ERR_IO;
  }
  return KL_OK;
}
