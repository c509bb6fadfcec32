// socs_noalloc.cu -- SOCS imaging that allocates no memory at all.
//
// Some callers cannot allocate device memory while they run: a host program
// that hands this library a fixed memory budget and forbids allocation after
// start-up, an allocator-owning framework that must see every device byte,
// or code running where a cudaMalloc would synchronise the device or fail.
// kl_socs_forward_noalloc serves them: the caller owns every input and output
// buffer, and the pipeline's scratch (strip partial spectra, intensity
// spectra, twiddle tables) lives in one fixed-size file-scope device array
// below instead of in cudaMalloc'd plan buffers.
//
// The array is part of the module: every GPU that loads the library holds it
// (kNoallocScratchBytes) until the process exits.  All calls share it and it
// keeps whatever the last call left there; calls that overlap on the GPU
// (other streams, other host threads) race on it and must be serialised by
// the caller.  Every scratch element is written before it is read within a
// call, so no part of it has to start at zero.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "kl_internal.h"

namespace {

// 8 MiB: room for about 38 clips of 1024^2 at NA 1.35 (about 210 KB each)
constexpr size_t kNoallocScratchBytes = size_t(8) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// Device address of g_noalloc_scratch per device.  In host code the symbol
// name is only a host-side handle, never a device address, so the address is
// looked up once per device with that device current.  The address belongs
// to the device's primary context: it is remembered together with that
// context and looked up again when the context is a new one (after a
// cudaDeviceReset, for instance).
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};
CUcontext g_ctx[kMaxDevices] = {};

// cuCtxGetCurrent through the runtime's driver entry point (the library does
// not link the driver library directly)
CUcontext current_context() {
  using Fn = CUresult (*)(CUcontext*);
  static Fn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<Fn>(p);
  }();
  CUcontext c = nullptr;
  if (fn) fn(&c);
  return c;
}

int scratch_address(void** out) {
  int dev = 0;
  KL_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    kl::set_error("kl_socs_forward_noalloc: device index out of range");
    return KL_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  CUcontext ctx = current_context();
  if (!g_addr[dev] || !ctx || ctx != g_ctx[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      kl::set_error(std::string("kl_socs_forward_noalloc: cudaGetSymbolAddress failed: ") +
                    cudaGetErrorString(e));
      return KL_ERR_CUDA;
    }
    g_addr[dev] = p;
    g_ctx[dev] = current_context();  // the look-up made the primary context current
  }
  *out = g_addr[dev];
  return KL_OK;
}

size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

extern "C" int kl_socs_forward_noalloc(const float* masks_dev, int nclips, int Lx, int Ly, int Nx,
                                       int Ny, const float* kernels_dev, const float* scales_dev,
                                       int nk, float* images_dev, void* stream) {
  KL_CHECK_ARG(masks_dev && kernels_dev && scales_dev && images_dev,
               "kl_socs_forward_noalloc: NULL argument");
  KL_CHECK_ARG(nclips >= 0 && nk > 0, "kl_socs_forward_noalloc: bad nclips or nk");
  if (nclips == 0) return KL_OK;
  kl::SocsGeom g;
  int rc = kl::socs_geometry(Lx, Ly, Nx, Ny, &g);
  if (rc) return rc;
  const int nsplit = kl::socs_choose_split(g, nclips, 1, nk);
  const size_t b_tx = up256(sizeof(float2) * kl::socs_table_x_elems(g));
  const size_t b_ty = up256(sizeof(float2) * kl::socs_table_y_elems(g));
  const size_t b_part = up256(kl::socs_partial_bytes(g, nclips));
  const size_t b_T = up256(kl::socs_spectrum_bytes(g, nclips, 1, nsplit));
  const size_t need = b_tx + b_ty + b_part + b_T;
  if (need > kNoallocScratchBytes) {
    kl::set_error("kl_socs_forward_noalloc: " + std::to_string(nclips) + " clips of " +
                  std::to_string(Lx) + "x" + std::to_string(Ly) + " need " + std::to_string(need) +
                  " bytes of scratch; the static workspace holds " +
                  std::to_string(kNoallocScratchBytes) + " bytes (use fewer clips per call)");
    return KL_ERR_INVALID;
  }
  void* base = nullptr;
  if ((rc = scratch_address(&base))) return rc;
  unsigned char* p = static_cast<unsigned char*>(base);
  float2* tx = reinterpret_cast<float2*>(p);
  float2* ty = reinterpret_cast<float2*>(p + b_tx);
  float2* partial = reinterpret_cast<float2*>(p + b_tx + b_ty);
  float2* T = reinterpret_cast<float2*>(p + b_tx + b_ty + b_part);
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = kl::socs_build_tables(g, tx, ty, st))) return rc;
  if ((rc = kl::socs_launch_forward(g, tx, ty, masks_dev, nclips, partial, st))) return rc;
  if ((rc = kl::socs_launch_spectral(g, partial, nclips, reinterpret_cast<const float2*>(kernels_dev),
                                     scales_dev, nk, 1, nsplit, T, st)))
    return rc;
  return kl::socs_launch_inverse(g, tx, ty, T, nclips, 1, nsplit, images_dev, st);
}
