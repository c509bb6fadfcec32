// resist.cu -- resist image and printed contour of aerial images.
//
// The reference thresholds its aerial image only for display: klitho_tcc
// draws image_s.png with a colour scale topped at TARGET_INTENSITY = 0.225
// (K-Litho-TCC/klitho_tcc.cpp:442, :547).  Here the threshold feeds the two
// outputs a lithography flow reads next: the sigmoid resist image
// s = 1 / (1 + exp(-alpha (I - threshold))) -- the resist model of the
// adjoint (socs_vjp.cu) -- and the printed pattern I >= threshold with its
// contour (printed pixels that have a 4-neighbour, periodic across the clip,
// that does not print).  One pass over the image: a tile of rows is staged in
// shared memory with a one-row halo above and below, so every image pixel is
// read from HBM about once.
#include <cstdint>

#include "kl_internal.h"

namespace kl {
namespace {
constexpr int kRows = 8;  // image rows per CTA tile
constexpr int kT = 256;

__global__ void __launch_bounds__(kT) k_resist(const float* __restrict__ img, int Lx, int Ly, float alpha,
                                               float thr, float* __restrict__ resist, uint8_t* __restrict__ printed,
                                               uint8_t* __restrict__ edges, unsigned long long* __restrict__ count) {
  extern __shared__ float tile[];  // [kRows + 2][Lx]
  const int n = blockIdx.y;
  const int y0 = blockIdx.x * kRows;
  const int rows = min(kRows, Ly - y0);
  const float* im = img + (size_t)n * Lx * Ly;
  // rows y0-1 .. y0+rows (periodic)
  for (int r = 0; r < rows + 2; ++r) {
    int y = y0 - 1 + r;
    y = y < 0 ? y + Ly : (y >= Ly ? y - Ly : y);
    const float* src = im + (size_t)y * Lx;
    for (int x = threadIdx.x; x < Lx; x += kT) tile[(size_t)r * Lx + x] = __ldg(src + x);
  }
  __syncthreads();
  unsigned long long local = 0;
  for (int r = 1; r <= rows; ++r) {
    const size_t o = (size_t)n * Lx * Ly + (size_t)(y0 + r - 1) * Lx;
    const float* t = tile + (size_t)r * Lx;
    for (int x = threadIdx.x; x < Lx; x += kT) {
      const float v = t[x];
      const bool p = v >= thr;
      if (resist) resist[o + x] = __frcp_rn(1.0f + __expf(-alpha * (v - thr)));
      if (printed) printed[o + x] = p ? 1 : 0;
      if (edges || count) {
        const int xl = x == 0 ? Lx - 1 : x - 1, xr = x == Lx - 1 ? 0 : x + 1;
        const bool e = p && (t[xl] < thr || t[xr] < thr || t[x - Lx] < thr || t[x + Lx] < thr);
        if (edges) edges[o + x] = e ? 1 : 0;
        local += e ? 1 : 0;
      }
    }
  }
  if (count) {
    for (int s = 16; s > 0; s >>= 1) local += __shfl_xor_sync(0xffffffffu, local, s);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count + n, local);
  }
}
}  // namespace
}  // namespace kl

extern "C" int kl_resist_contour(const float* images_dev, int nimg, int Lx, int Ly, float alpha, float threshold,
                                 float* resist_dev, unsigned char* printed_dev, unsigned char* edges_dev,
                                 unsigned long long* edge_count_dev, void* stream) {
  KL_CHECK_ARG(images_dev, "kl_resist_contour: images_dev is NULL");
  KL_CHECK_ARG(nimg >= 0 && Lx > 0 && Ly > 0, "kl_resist_contour: bad sizes");
  KL_CHECK_ARG(nimg <= 65535, "kl_resist_contour: at most 65535 images per call");
  const size_t smem = sizeof(float) * (size_t)(kl::kRows + 2) * Lx;
  KL_CHECK_ARG(smem <= 200 * 1024, "kl_resist_contour: rows wider than 5120 pixels");
  if (nimg == 0) return KL_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (edge_count_dev) KL_CUDA_TRY(cudaMemsetAsync(edge_count_dev, 0, sizeof(unsigned long long) * nimg, st));
  if (smem > 48 * 1024)
    KL_CUDA_TRY(cudaFuncSetAttribute(kl::k_resist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  dim3 grid((Ly + kl::kRows - 1) / kl::kRows, nimg);
  kl::k_resist<<<grid, kl::kT, smem, st>>>(images_dev, Lx, Ly, alpha, threshold, resist_dev,
                                            reinterpret_cast<uint8_t*>(printed_dev),
                                            reinterpret_cast<uint8_t*>(edges_dev), edge_count_dev);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}
