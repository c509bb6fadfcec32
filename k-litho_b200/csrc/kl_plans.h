// kl_plans.h -- plan objects behind the opaque handles of include/klitho_gpu.h.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "kl_internal.h"
#include "kl_tcc.h"

struct kl_socs_plan_s {
  kl::SocsGeom g{};
  int K = 0, nsets = 0, max_clips = 0;
  int device = 0;
  bool adjoint = false;
  float2* H = nullptr;       // nsets x K x nby x nbx
  float* lam = nullptr;      // nsets x K
  float2* partial = nullptr; // max_clips strip partials
  float2* T = nullptr;       // intensity spectra (clip x set x kernel slice)
  float2* tx = nullptr;      // plan-time twiddle tables
  float2* ty = nullptr;
  float* stage_in = nullptr; // host-entry staging (lazily allocated)
  float* stage_out = nullptr;
  size_t stage_clips = 0;
  // host-entry pipeline: copy-in, compute, copy-out streams and their hand-offs
  cudaStream_t hs[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t hev[3] = {nullptr, nullptr, nullptr};
  // adjoint state (kl_socs_plan_create_adjoint)
  float2* gpart = nullptr;   // strip partials of the spectrum of dL/dI
  float2* gam = nullptr;     // per-slice Gam partials
  float2* Tg = nullptr;      // half-plane spectrum of dL/dm
  int last_vjp_clips = 0;
  // optional stage timing: 4 events per kl_socs_forward
  bool timing = false;
  std::vector<cudaEvent_t> events;
  // launch shape chosen by kl_socs_autotune for batches of tune_clips clips
  int tcap = 0;  // clip x kernel-slice products the spectra buffer holds
  int tune_clips = 0, tune_nsplit = 0, tune_spc = 0;  // tune_spc < 0: tensor-core synthesis
  // synthesis engine of the specialised pipeline (KL_SYNTH_*), the tensor-core
  // basis (FP16 hi / lo halves, [Lx][Kp]) and its pipeline status word
  int synth = 0;
  void* bhi = nullptr;
  void* blo = nullptr;
  int* status = nullptr;
  // the transposed basis ([64][Lx]) of the tensor-core mask transform and, on
  // adjoint plans with vjp_tc, of the tensor-core adjoint
  void* thi = nullptr;
  void* tlo = nullptr;
  bool vjp_tc = false;
  // general-geometry pipeline (socs_gen.cu): any period, bands up to 4N+1 <= 256.
  // Used when the specialised kernels above do not cover the geometry (or on
  // request); `g` then only carries the sizes.
  bool gen = false;
  kl::GenGeom gg{};
  float2* gtab = nullptr;   // x twiddles, chunk twiddles, roots of unity of Ly
  float2* R = nullptr;      // row bins of the masks (Nx+1 per row)
  float2* band = nullptr;   // band partials of the masks
  float2* Q = nullptr;      // per-row synthesis coefficients of every image; the
                            // adjoint overwrites them with the row bins of dL/dI
  int nparts_max = 0;       // band partials per clip the band buffer holds
  float2* gband = nullptr;  // adjoint: band partials of dL/dI per image
  int gparts_max = 0;
  int last_nparts = 0, last_gparts = 0;  // partial counts of the last kl_socs_vjp
};

namespace kl {
// one forward pass of a plan on `st`; ev4 (optional) receives the stage
// boundaries, otherwise the plan's own timing marks are used
int socs_run_forward(kl_socs_plan_s* p, const float* masks, int nclips, float* images, cudaStream_t st,
                     const cudaEvent_t* ev4);
}  // namespace kl

struct kl_tcc_plan_s {
  int precision = KL_PREC_FAST;
  int Lx = 0, Ly = 0, srcSize = 0;
  float outerSigma = 0.f;
  kl::PupilParams pp{};
  std::vector<kl::SrcPoint> pts;
  kl::SrcPoint* pts_dev = nullptr;
  float2* A = nullptr;        // fast path: N x S FP32 factor
  double2* P = nullptr;       // FP64 path: N x S pupil table (host libm)
  float* J = nullptr;         // S weights (both paths)
  int* src_id = nullptr;      // S source-map indices (both paths)
  double2* tcc64 = nullptr;   // FP64 path: TCC (built on demand)
  int* err = nullptr;
  struct kl_socs_plan_s* hopkins = nullptr;  // SOCS plan of the Abbe form (lazy)
  int hopkins_clips = 0;
};

namespace kl {
// adjoint launchers (socs_vjp.cu)
int vjp_supported(const SocsGeom& g);
size_t vjp_gpart_bytes(const SocsGeom& g, int nimg);
int vjp_launch_inverse(const SocsGeom& g, const float2* tx, const float2* ty, const float2* T,
                       int nclips, int nsets, int nsplit, const float* targets, float alpha,
                       float thr, float* images, double* loss, float2* gpart, cudaStream_t st);
int vjp_launch_spectral(const SocsGeom& g, const float2* partial, const float2* gpart, int nclips,
                        const float2* H, const float* lam, int K, int nsets, int nsplit,
                        float2* gam_out, cudaStream_t st);
int vjp_launch_gradT(const SocsGeom& g, const float2* gam, int nclips, int nparts, float2* T,
                     cudaStream_t st);
int vjp_launch_source(const SocsGeom& g, const float2* partial, const float2* gpart, int nimg,
                      int nsets, const float2* Hs, const float* Jw, const int* src_id, int S,
                      int nsplit, float* grad_src, cudaStream_t st);
}  // namespace kl

namespace kl {
namespace f64 {
// the plain FP64 imaging path (fp64_path.cu); device pointers, one clip at a time
int socs_forward(const float* masks, int nclips, int Lx, int Ly, int Nx, int Ny, const float2* H,
                 const float* lam, int nk, double* images, cudaStream_t st);
int hopkins_image(const float* masks, int nclips, int Lx, int Ly, int Nx, int Ny, const double2* tcc,
                  double* images, cudaStream_t st);
int mask_spectrum(const float* mask, int Lx, int Ly, double2* out, cudaStream_t st);
int socs_vjp(const float* masks, const float* targets, int nclips, int Lx, int Ly, int Nx, int Ny,
             const float2* H, const float* lam, int nk, double alpha, double thr, double* images, double* grad,
             double* loss, cudaStream_t st);
}  // namespace f64
}  // namespace kl
