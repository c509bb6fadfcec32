// kl_internal.h -- host-side internal types shared by the library sources.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "../../include/klitho_gpu.h"

namespace kl {

// thread-local last error text, returned by kl_last_error()
void set_error(const std::string& msg);

// Per-call scratch: stream-ordered allocations from the current device's
// default memory pool, which keeps freed blocks cached, so temporaries cost
// neither a device synchronisation nor a fresh cudaMalloc on repeat calls.
// scratch_alloc returns KL_OK or KL_ERR_NOMEM (with the message set).
int scratch_alloc(void** p, size_t bytes, cudaStream_t st, const char* what);
void scratch_free(void* p, cudaStream_t st);
const char* last_error();

#define KL_CUDA_TRY(expr)                                                      \
  do {                                                                         \
    cudaError_t _e = (expr);                                                   \
    if (_e != cudaSuccess) {                                                   \
      ::kl::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));     \
      return KL_ERR_CUDA;                                                      \
    }                                                                          \
  } while (0)

#define KL_CHECK_ARG(cond, msg)        \
  do {                                 \
    if (!(cond)) {                     \
      ::kl::set_error(msg);            \
      return KL_ERR_INVALID;           \
    }                                  \
  } while (0)

// Geometry of the fused FP32 SOCS pipeline for one clip size.
struct SocsGeom {
  int Lx, Ly;      // clip period in pixels (1 nm each)
  int Nx, Ny;      // kernel band half-widths
  int nbx, nby;    // 2N+1
  int nf;          // Nx+1 row-DFT bins kept by the forward pass (fx >= 0)
  int ntx, nty;    // 2Nx+1 and 4Ny+1: intensity spectrum half plane
  int P;           // points per lane in the row transforms
  int V;           // virtual lanes per row, Lx = V * P
  int J;           // rows per strip (power of two >= max(32, 2Ny+1))
  int nS;          // strips per clip, Ly = nS * J
  int G;           // spectral grid (power of two >= max(32, 4Nx+1, 4Ny+1))
  int dx, dy;      // one-pixel output shift of odd periods (0 or 1)
  int NFM, NBM;    // padded forward / inverse bin counts (16, 32 or 64)
  int KX;          // rows of the x twiddle table, max(NFM, NBM)
};

// Largest number of kernel slices the spectral stage splits a (clip, set) into.
constexpr int kSocsMaxSplit = 8;

// Fill geometry; returns KL_OK or KL_ERR_UNSUPPORTED with a message.  With
// `adjoint`, strips are tall enough (J >= 4Ny+1) to carry the band of the
// loss gradient dL/dI as well.
int socs_geometry(int Lx, int Ly, int Nx, int Ny, SocsGeom* g, bool adjoint = false);

// Device workspace sizes.
size_t socs_partial_bytes(const SocsGeom& g, int nclips);
size_t socs_spectrum_bytes(const SocsGeom& g, int nclips, int nsets, int nsplit);
size_t socs_table_x_elems(const SocsGeom& g);  // float2 elements of tx
size_t socs_table_y_elems(const SocsGeom& g);  // float2 elements of ty
// kernel slices per (clip, set) for a launch of `nclips` clips
int socs_choose_split(const SocsGeom& g, int nclips, int nsets, int K);

// Plan-time twiddle tables (stream-ordered).
int socs_build_tables(const SocsGeom& g, float2* tx, float2* ty, cudaStream_t st);

// Launchers (stream-ordered).  Buffers are device pointers.
int socs_launch_forward(const SocsGeom& g, const float2* tx, const float2* ty, const float* masks,
                        int nclips, float2* partial, cudaStream_t st);
int socs_launch_spectral(const SocsGeom& g, const float2* partial, int nclips, const float2* H,
                         const float* lam, int K, int nsets, int nsplit, float2* T,
                         cudaStream_t st);
// spc: strips per CTA of the inverse kernel (0 = chosen from the batch size)
int socs_launch_inverse(const SocsGeom& g, const float2* tx, const float2* ty, const float2* T,
                        int nclips, int nsets, int nsplit, float* images, cudaStream_t st, int spc = 0);
// Image synthesis on the tensor cores (socs_synth_tc.cu): the inverse stage as
// an FP16x3 split GEMM of the row coefficients against a cos/sin basis.
bool synth_tc_supported(const SocsGeom& g);
int synth_tc_kp(const SocsGeom& g);  // padded K (64 or 128) of the basis rows
bool synth_tc_aligned(const float* images);  // TMA stores need 16-byte aligned images
// basis [Lx][Kp] as FP16 hi and lo halves (each Lx * Kp * 2 bytes)
int synth_tc_build_basis(const SocsGeom& g, void* bhi, void* blo, cudaStream_t st);
// err: device status word, set to a nonzero code if a pipeline wait times out
int synth_tc_launch(const SocsGeom& g, const float2* T, const float2* ty, int nsplit, const void* bhi,
                    const void* blo, int nimg, float* images, int* err, cudaStream_t st);
// The mask transform (strip partial band spectra) on the tensor cores
// (socs_fwd_tc.cu), in place of socs_launch_forward; thi / tlo: the transposed
// basis of vjp_tc_build_basis_t.  Mask values must lie within +-2^15 (the
// status word reports others).
bool fwd_tc_supported(const SocsGeom& g);
int fwd_tc_launch(const SocsGeom& g, const float* masks, int nclips, const float2* ty, const void* thi,
                  const void* tlo, float2* partial, int* err, cudaStream_t st);
// The adjoint's image + resist + loss + row DFT of dL/dI on the tensor cores
// (socs_vjp_tc.cu), in place of vjp_launch_inverse: same outputs (images,
// loss, strip partials of the spectrum of dL/dI).
bool vjp_tc_supported(const SocsGeom& g);
// transposed row-DFT basis [64][Lx] as FP16 hi and lo halves (each 64 * Lx * 2 bytes)
int vjp_tc_build_basis_t(const SocsGeom& g, void* thi, void* tlo, cudaStream_t st);
// bhi / blo: the synthesis basis of synth_tc_build_basis (Kp = 64)
int vjp_tc_launch(const SocsGeom& g, const float2* T, const float2* ty, int nclips, int nsets, int nsplit,
                  const void* bhi, const void* blo, const void* thi, const void* tlo, const float* targets,
                  float alpha, float thr, float* images, double* loss, float2* gpart, int* err, cudaStream_t st);
// centred band of FT_r2c (DC at the band centre), complex64 nby x nbx per clip
int socs_launch_band(const SocsGeom& g, const float2* partial, int nclips, float2* band,
                     cudaStream_t st);

// ---------------------------------------------------------------------------
// General-geometry fused SOCS pipeline (socs_gen.cu, socs_gen_vjp.cu): any
// period Lx x Ly, bands up to 4N+1 <= 256.  Five stream-ordered stages:
//   row_fwd  mask rows -> row bins R[y][fx], fx in [0, Nx]       (HBM-bound)
//   col_fwd  R -> band spectrum, |fy| <= Ny                      (small)
//   spectral band -> intensity spectrum T (cluster of G/32 CTAs per image)
//   col_inv  T -> per-row coefficients Q[y][b], b in [0, 2Nx]    (small)
//   row_inv  Q rows -> image rows                                (HBM-bound)
// ---------------------------------------------------------------------------
struct GenGeom {
  int Lx, Ly, Nx, Ny;
  int nbx, nby, nf;  // 2Nx+1, 2Ny+1, Nx+1
  int ntx, nty;      // 2Nx+1, 4Ny+1 (intensity half plane)
  int G, RG;         // spectral grid G = 32 RG (power of two >= 4N+1); RG CTAs per image
  int P, V;          // row synthesis: Lx = P V, P a power of two <= 64
  int Pf, Vf;        // row transforms of masks and of dL/dI: Pf = min(P, 32)
  int nC;            // lane chunks of 32 covering max(V, Vf)
  int NBX;           // bin count of the x tables (multiple of 32 and of P, >= 2Nx+1)
  int ystrip;        // 1: Ly % 32 == 0, strips of 32 rows spaced nS apart; 0: 32-row blocks
  int nS;            // strips (ystrip) or row blocks per clip
  int dx, dy;        // one-pixel output shift of odd periods (0 or 1)
};

constexpr int kGenMaxSplit = 8;
// the chunk twiddles of the row kernels are staged in shared memory up to 32 KB
__host__ __device__ inline bool gen_t2_in_smem(const GenGeom& g) { return (size_t)g.nC * g.NBX * 8 <= 32 * 1024; }

int gen_geometry(int Lx, int Ly, int Nx, int Ny, GenGeom* g);
size_t gen_rowbins_bytes(const GenGeom& g, int nrows_img, int nbins);  // R / Q buffers
size_t gen_band_bytes(const GenGeom& g, int n, int nparts, int nrows, int ncols);
size_t gen_T_bytes(const GenGeom& g, int nimg, int nsplit);
size_t gen_table_elems(const GenGeom& g);  // twb + twl + tw2 + rootLy (float2)
int gen_build_tables(const GenGeom& g, float2* tables, cudaStream_t st);
// kernel slices per image of a spectral launch with `per_sm` resident CTAs per SM
// (2 for the forward core, 1 for the adjoint's)
int gen_choose_split(const GenGeom& g, int nimg, int K, int per_sm = 2);
int gen_choose_parts(const GenGeom& g, int n, int ncols);

// stage launchers (device pointers, stream-ordered)
int gen_launch_rowfwd(const GenGeom& g, const float2* tables, const float* src, int nrows, float2* R,
                      cudaStream_t st);
int gen_launch_colfwd(const GenGeom& g, const float2* tables, const float2* R, int n, int ncols, int Yb,
                      float scale, int nparts, float2* band, cudaStream_t st);
int gen_launch_spectral(const GenGeom& g, const float2* band, int nparts, int nclips, const float2* H,
                        const float* lam, int K, int nsets, int nsplit, float2* T, cudaStream_t st);
int gen_launch_colinv(const GenGeom& g, const float2* tables, const float2* T, int nimg, int nsplit, int A,
                      int nbins, float2* Q, cudaStream_t st);
int gen_launch_rowinv(const GenGeom& g, const float2* tables, const float2* Q, int nimg, int nbins,
                      float* images, cudaStream_t st);
int gen_launch_bandout(const GenGeom& g, const float2* band, int nparts, int nclips, float2* out,
                       cudaStream_t st);
// adjoint stages (socs_gen_vjp.cu).  row_vjp overwrites Q (2Nx+1 bins per row)
// with the row bins of dL/dI; col_fwd then gives its band (|gy| <= 2Ny).
int gen_launch_rowvjp(const GenGeom& g, const float2* tables, float2* Q, int nimg, int nsets, const float* targets,
                      float alpha, float thr, float* images, double* loss, cudaStream_t st);
int gen_launch_vjp_spectral(const GenGeom& g, const float2* band, int nparts, const float2* gband, int gparts,
                            int nclips, const float2* H, const float* lam, int K, int nsets, int nsplit, float2* gam,
                            cudaStream_t st);
int gen_launch_gradT(const GenGeom& g, const float2* gam, int nclips, int nparts, float2* Tg, cudaStream_t st);
int gen_launch_vjp_source(const GenGeom& g, const float2* band, int nparts, const float2* gband, int gparts,
                          int nimg, int nsets, const float2* Hs, int S, const float* Jw, const int* src_id,
                          int nsplit, float* grad_src, cudaStream_t st);

}  // namespace kl

// Internal: upload kernel set `set` of a SOCS plan from device memory
// (H_dev: nk x band complex64, lam_dev: nk floats; device-to-device copies).
extern "C" int kl_socs_set_kernels_device(struct kl_socs_plan_s* plan, int set,
                                          const float2* H_dev, const float* lam_dev,
                                          cudaStream_t st);
