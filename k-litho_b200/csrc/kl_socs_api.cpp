// kl_socs_api.cpp -- C ABI for SOCS imaging plans (see include/klitho_gpu.h).
#include <cuda_runtime.h>

#include <cstdint>
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "kl_internal.h"
#include "kl_plans.h"

namespace {
void drop_events(kl_socs_plan p) {
  for (cudaEvent_t e : p->events) cudaEventDestroy(e);
  p->events.clear();
}

void free_plan(kl_socs_plan p) {
  if (!p) return;
  drop_events(p);
  for (int i = 0; i < 3; ++i) {
    if (p->hs[i]) {
      cudaStreamSynchronize(p->hs[i]);
      cudaStreamDestroy(p->hs[i]);
    }
    if (p->hev[i]) cudaEventDestroy(p->hev[i]);
  }
  cudaFree(p->H);
  cudaFree(p->lam);
  cudaFree(p->partial);
  cudaFree(p->T);
  cudaFree(p->tx);
  cudaFree(p->ty);
  cudaFree(p->stage_in);
  cudaFree(p->stage_out);
  cudaFree(p->gpart);
  cudaFree(p->gam);
  cudaFree(p->Tg);
  cudaFree(p->gtab);
  cudaFree(p->R);
  cudaFree(p->band);
  cudaFree(p->Q);
  cudaFree(p->gband);
  cudaFree(p->bhi);
  cudaFree(p->blo);
  cudaFree(p->status);
  cudaFree(p->thi);
  cudaFree(p->tlo);
  delete p;
}

int alloc(void** ptr, size_t bytes, const char* what) {
  cudaError_t e = cudaMalloc(ptr, bytes ? bytes : 16);
  if (e != cudaSuccess) {
    kl::set_error(std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
    cudaGetLastError();
    return KL_ERR_NOMEM;
  }
  return KL_OK;
}

int mark(kl_socs_plan p, cudaStream_t st) {
  if (!p->timing) return KL_OK;
  cudaEvent_t e;
  KL_CUDA_TRY(cudaEventCreate(&e));
  p->events.push_back(e);
  KL_CUDA_TRY(cudaEventRecord(e, st));
  return KL_OK;
}

int stage_mark(kl_socs_plan p, cudaStream_t st, const cudaEvent_t* ev4, int i) {
  if (!ev4) return mark(p, st);
  // inside a stream capture the record must become an event node of the graph
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  KL_CUDA_TRY(cudaStreamIsCapturing(st, &cs));
  KL_CUDA_TRY(cudaEventRecordWithFlags(ev4[i], st,
                                       cs == cudaStreamCaptureStatusActive ? cudaEventRecordExternal
                                                                           : cudaEventRecordDefault));
  return KL_OK;
}

// the launch shape for a batch of nclips: the autotuned one when it was tuned
// for this batch size, else the heuristic
void launch_shape(kl_socs_plan p, int nclips, int* nsplit, int* spc) {
  if (p->tune_clips == nclips && p->tune_nsplit > 0) {
    *nsplit = p->tune_nsplit;
    *spc = p->tune_spc;
  } else {
    *nsplit = kl::socs_choose_split(p->g, nclips, p->nsets, p->K);
    *spc = 0;
  }
}

// general-geometry pipeline: row transform, column transform, spectral core,
// column synthesis, row synthesis
int run_forward_gen(kl_socs_plan p, const float* masks, int nclips, float* images, cudaStream_t st,
                    const cudaEvent_t* ev4) {
  const kl::GenGeom& g = p->gg;
  const int nimg = nclips * p->nsets;
  int nsplit = kl::gen_choose_split(g, nimg, p->K);
  if (p->tune_clips == nclips && p->tune_nsplit > 0) nsplit = p->tune_nsplit;
  const int nparts = kl::gen_choose_parts(g, nclips, g.nf);
  int rc;
  if ((rc = stage_mark(p, st, ev4, 0))) return rc;
  if ((rc = kl::gen_launch_rowfwd(g, p->gtab, masks, nclips * g.Ly, p->R, st))) return rc;
  if ((rc = kl::gen_launch_colfwd(g, p->gtab, p->R, nclips, g.nf, g.Ny, 1.0f / ((float)g.Lx * (float)g.Ly), nparts,
                                  p->band, st)))
    return rc;
  if ((rc = stage_mark(p, st, ev4, 1))) return rc;
  if ((rc = kl::gen_launch_spectral(g, p->band, nparts, nclips, p->H, p->lam, p->K, p->nsets, nsplit, p->T, st)))
    return rc;
  if ((rc = stage_mark(p, st, ev4, 2))) return rc;
  if ((rc = kl::gen_launch_colinv(g, p->gtab, p->T, nimg, nsplit, 2 * g.Ny, g.ntx, p->Q, st))) return rc;
  if ((rc = kl::gen_launch_rowinv(g, p->gtab, p->Q, nimg, g.ntx, images, st))) return rc;
  return stage_mark(p, st, ev4, 3);
}

// synthesis on the tensor cores for a batch of nclips clips: when requested,
// or when the autotuner picked it for this batch size
bool use_tc_synthesis(kl_socs_plan p, int nclips) {
  if (p->gen || !p->bhi) return false;
  if (p->synth == KL_SYNTH_TENSOR_CORES) return true;
  if (p->synth == KL_SYNTH_CUDA_CORES) return false;
  return p->tune_clips == nclips && p->tune_nsplit > 0 && p->tune_spc < 0;
}

// mask transform on the tensor cores: with the tensor-core engine forced, or
// when the autotuner picked it (tune_spc == -2) for this batch size
bool use_tc_forward(kl_socs_plan p, int nclips, const float* masks) {
  if (p->gen || !p->thi || !kl::fwd_tc_supported(p->g) || ((uintptr_t)masks & 15)) return false;
  if (p->synth == KL_SYNTH_TENSOR_CORES) return true;
  if (p->synth == KL_SYNTH_CUDA_CORES) return false;
  return p->tune_clips == nclips && p->tune_nsplit > 0 && p->tune_spc == -2;
}

int run_forward(kl_socs_plan p, const float* masks, int nclips, float* images, cudaStream_t st,
                const cudaEvent_t* ev4 = nullptr) {
  if (p->gen) return run_forward_gen(p, masks, nclips, images, st, ev4);
  int rc;
  if ((rc = stage_mark(p, st, ev4, 0))) return rc;
  int nsplit, spc;
  launch_shape(p, nclips, &nsplit, &spc);
  const bool tc = use_tc_synthesis(p, nclips) && kl::synth_tc_aligned(images);
  spc = spc > 0 ? spc : 0;
  if (use_tc_forward(p, nclips, masks))
    rc = kl::fwd_tc_launch(p->g, masks, nclips, p->ty, p->thi, p->tlo, p->partial, p->status, st);
  else
    rc = kl::socs_launch_forward(p->g, p->tx, p->ty, masks, nclips, p->partial, st);
  if (rc) return rc;
  if ((rc = stage_mark(p, st, ev4, 1))) return rc;
  rc = kl::socs_launch_spectral(p->g, p->partial, nclips, p->H, p->lam, p->K, p->nsets, nsplit,
                                p->T, st);
  if (rc) return rc;
  if ((rc = stage_mark(p, st, ev4, 2))) return rc;
  rc = tc ? kl::synth_tc_launch(p->g, p->T, p->ty, nsplit, p->bhi, p->blo, nclips * p->nsets, images, p->status, st)
          : kl::socs_launch_inverse(p->g, p->tx, p->ty, p->T, nclips, p->nsets, nsplit, images, st, spc);
  if (rc) return rc;
  return stage_mark(p, st, ev4, 3);
}
// plan on the general-geometry pipeline
int create_gen_plan(kl_socs_plan* plan, int Lx, int Ly, int Nx, int Ny, int nk, int nsets, int max_clips,
                    bool adjoint) {
  kl::GenGeom gg;
  int rc = kl::gen_geometry(Lx, Ly, Nx, Ny, &gg);
  if (rc) return rc;
  kl_socs_plan p = new (std::nothrow) kl_socs_plan_s;
  if (!p) {
    kl::set_error("kl_socs_plan_create: out of host memory");
    return KL_ERR_NOMEM;
  }
  p->gen = true;
  p->adjoint = adjoint;
  p->gg = gg;
  // sizes only, for callers that read them
  p->g.Lx = Lx;
  p->g.Ly = Ly;
  p->g.Nx = Nx;
  p->g.Ny = Ny;
  p->g.nbx = gg.nbx;
  p->g.nby = gg.nby;
  p->g.nf = gg.nf;
  p->g.ntx = gg.ntx;
  p->g.nty = gg.nty;
  p->g.G = gg.G;
  p->g.nS = gg.nS;
  p->g.dx = gg.dx;
  p->g.dy = gg.dy;
  p->K = nk;
  p->nsets = nsets;
  p->max_clips = max_clips;
  cudaGetDevice(&p->device);
  const size_t nb2 = (size_t)gg.nby * gg.nbx;
  // spectra buffer: the largest (image, kernel slice) count any batch size or
  // autotuned split needs
  int tcap = 0, pmax = 0;
  for (int n = 1; n <= max_clips; ++n) {
    tcap = std::max(tcap, n * nsets * kl::gen_choose_split(gg, n * nsets, nk));
    if (adjoint) tcap = std::max(tcap, n * nsets * kl::gen_choose_split(gg, n * nsets, nk, 1));
    pmax = std::max(pmax, kl::gen_choose_parts(gg, n, gg.nf));
  }
  for (int ns = 1; ns <= kl::kGenMaxSplit; ns *= 2) tcap = std::max(tcap, std::min(ns, nk) * nsets);
  p->tcap = tcap;
  p->nparts_max = pmax;
  if ((rc = alloc((void**)&p->H, sizeof(float2) * nb2 * nk * nsets, "kernels")) ||
      (rc = alloc((void**)&p->lam, sizeof(float) * (size_t)nk * nsets, "eigenvalues")) ||
      (rc = alloc((void**)&p->gtab, sizeof(float2) * kl::gen_table_elems(gg), "tables")) ||
      (rc = alloc((void**)&p->R, kl::gen_rowbins_bytes(gg, max_clips, gg.nf), "row bins")) ||
      (rc = alloc((void**)&p->band, kl::gen_band_bytes(gg, max_clips, pmax, gg.nby, gg.nf), "band partials")) ||
      (rc = alloc((void**)&p->T, kl::gen_T_bytes(gg, tcap, 1), "spectra")) ||
      (rc = alloc((void**)&p->Q, kl::gen_rowbins_bytes(gg, max_clips * nsets, gg.ntx), "row coefficients")) ||
      (rc = kl::gen_build_tables(gg, p->gtab, nullptr))) {
    free_plan(p);
    return rc;
  }
  if (adjoint) {
    int gmax = 0;
    for (int n = 1; n <= max_clips; ++n) gmax = std::max(gmax, kl::gen_choose_parts(gg, n * nsets, gg.ntx));
    p->gparts_max = gmax;
    if ((rc = alloc((void**)&p->gband, kl::gen_band_bytes(gg, max_clips * nsets, gmax, gg.nty, gg.ntx),
                    "dL/dI bands")) ||
        (rc = alloc((void**)&p->gam, sizeof(float2) * nb2 * tcap, "adjoint partials")) ||
        (rc = alloc((void**)&p->Tg, sizeof(float2) * (size_t)max_clips * gg.nf * gg.nby, "gradient spectra"))) {
      free_plan(p);
      return rc;
    }
  }
  if (cudaStreamSynchronize(nullptr) != cudaSuccess) {
    kl::set_error(std::string("kl_socs_plan_create: ") + cudaGetErrorString(cudaGetLastError()));
    free_plan(p);
    return KL_ERR_CUDA;
  }
  cudaMemset(p->H, 0, sizeof(float2) * nb2 * nk * nsets);
  cudaMemset(p->lam, 0, sizeof(float) * (size_t)nk * nsets);
  *plan = p;
  return KL_OK;
}

int create_plan(kl_socs_plan* plan, int Lx, int Ly, int Nx, int Ny, int nk, int nsets,
                int max_clips, bool adjoint, bool general = false) {
  KL_CHECK_ARG(plan != nullptr, "kl_socs_plan_create: plan is NULL");
  *plan = nullptr;
  KL_CHECK_ARG(nk > 0 && nsets > 0 && max_clips > 0, "kl_socs_plan_create: nk, nsets, max_clips must be positive");
  kl::SocsGeom g;
  int rc = general ? KL_ERR_UNSUPPORTED : kl::socs_geometry(Lx, Ly, Nx, Ny, &g, adjoint);
  if (!rc && adjoint) rc = kl::vjp_supported(g);
  // geometries outside the specialised kernels run on the general pipeline
  if (rc == KL_ERR_UNSUPPORTED) return create_gen_plan(plan, Lx, Ly, Nx, Ny, nk, nsets, max_clips, adjoint);
  if (rc) return rc;
  kl_socs_plan p = new (std::nothrow) kl_socs_plan_s;
  if (p) p->adjoint = adjoint;
  if (!p) {
    kl::set_error("kl_socs_plan_create: out of host memory");
    return KL_ERR_NOMEM;
  }
  p->g = g;
  p->K = nk;
  p->nsets = nsets;
  p->max_clips = max_clips;
  cudaGetDevice(&p->device);
  const size_t nb2 = (size_t)g.nby * g.nbx;
  if ((rc = alloc((void**)&p->H, sizeof(float2) * nb2 * nk * nsets, "kernels")) ||
      (rc = alloc((void**)&p->lam, sizeof(float) * (size_t)nk * nsets, "eigenvalues")) ||
      (rc = alloc((void**)&p->partial, kl::socs_partial_bytes(g, max_clips), "partials")) ||
      (rc = alloc((void**)&p->tx, sizeof(float2) * kl::socs_table_x_elems(g), "x twiddles")) ||
      (rc = alloc((void**)&p->ty, sizeof(float2) * kl::socs_table_y_elems(g), "y twiddles"))) {
    free_plan(p);
    return rc;
  }
  // spectra buffer: the largest clips x slices product any batch size needs
  int tcap = 0;
  for (int n = 1; n <= max_clips; ++n) {
    const int c = n * kl::socs_choose_split(g, n, nsets, nk);
    tcap = c > tcap ? c : tcap;
  }
  p->tcap = tcap;
  if ((rc = alloc((void**)&p->T, kl::socs_spectrum_bytes(g, tcap, nsets, 1), "spectra")) ||
      (rc = kl::socs_build_tables(g, p->tx, p->ty, nullptr))) {
    free_plan(p);
    return rc;
  }
  if (kl::synth_tc_supported(g)) {
    const size_t bb = (size_t)g.Lx * kl::synth_tc_kp(g) * 2;
    if ((rc = alloc(&p->bhi, bb, "synthesis basis")) || (rc = alloc(&p->blo, bb, "synthesis basis")) ||
        (rc = alloc((void**)&p->status, sizeof(int), "status word")) ||
        (rc = kl::synth_tc_build_basis(g, p->bhi, p->blo, nullptr))) {
      free_plan(p);
      return rc;
    }
    cudaMemset(p->status, 0, sizeof(int));
    // the transposed basis of the row DFTs: the tensor-core mask transform and,
    // on adjoint plans, the row DFT of dL/dI
    p->vjp_tc = adjoint && kl::synth_tc_kp(g) == 64 && kl::vjp_tc_supported(g);
    if (kl::fwd_tc_supported(g) || p->vjp_tc) {
      const size_t tb = (size_t)64 * g.Lx * 2;
      if ((rc = alloc(&p->thi, tb, "row DFT basis")) || (rc = alloc(&p->tlo, tb, "row DFT basis")) ||
          (rc = kl::vjp_tc_build_basis_t(g, p->thi, p->tlo, nullptr))) {
        free_plan(p);
        return rc;
      }
    }
  }
  if (adjoint) {
    const size_t nb2s = (size_t)g.nby * g.nbx;
    if ((rc = alloc((void**)&p->gpart, kl::vjp_gpart_bytes(g, max_clips * nsets), "dL/dI partials")) ||
        (rc = alloc((void**)&p->gam, sizeof(float2) * nb2s * tcap * nsets, "adjoint partials")) ||
        (rc = alloc((void**)&p->Tg, sizeof(float2) * (size_t)max_clips * g.nty * g.ntx, "gradient spectra"))) {
      free_plan(p);
      return rc;
    }
  }
  if (cudaStreamSynchronize(nullptr) != cudaSuccess) {
    kl::set_error(std::string("kl_socs_plan_create: ") + cudaGetErrorString(cudaGetLastError()));
    free_plan(p);
    return KL_ERR_CUDA;
  }
  cudaMemset(p->H, 0, sizeof(float2) * nb2 * nk * nsets);
  cudaMemset(p->lam, 0, sizeof(float) * (size_t)nk * nsets);
  *plan = p;
  return KL_OK;
}
}  // namespace

namespace {
// adjoint on the general pipeline: forward to T, image + resist + dL/dI row
// bins, dL/dI band, Gam, gradient spectrum, gradient image
int vjp_gen(kl_socs_plan p, const float* masks, const float* targets, int nclips, float alpha, float threshold,
            float* images, float* grad, double* loss, cudaStream_t st) {
  const kl::GenGeom& g = p->gg;
  const int nimg = nclips * p->nsets;
  const int ns = kl::gen_choose_split(g, nimg, p->K);
  const int ns_adj = kl::gen_choose_split(g, nimg, p->K, 1);
  const int nparts = kl::gen_choose_parts(g, nclips, g.nf);
  const int gparts = kl::gen_choose_parts(g, nimg, g.ntx);
  int rc;
  if ((rc = kl::gen_launch_rowfwd(g, p->gtab, masks, nclips * g.Ly, p->R, st))) return rc;
  if ((rc = kl::gen_launch_colfwd(g, p->gtab, p->R, nclips, g.nf, g.Ny, 1.0f / ((float)g.Lx * (float)g.Ly), nparts,
                                  p->band, st)))
    return rc;
  if ((rc = kl::gen_launch_spectral(g, p->band, nparts, nclips, p->H, p->lam, p->K, p->nsets, ns, p->T, st)))
    return rc;
  if ((rc = kl::gen_launch_colinv(g, p->gtab, p->T, nimg, ns, 2 * g.Ny, g.ntx, p->Q, st))) return rc;
  KL_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(double) * (size_t)nimg, st));
  if ((rc = kl::gen_launch_rowvjp(g, p->gtab, p->Q, nimg, p->nsets, targets, alpha, threshold, images, loss, st)))
    return rc;
  if ((rc = kl::gen_launch_colfwd(g, p->gtab, p->Q, nimg, g.ntx, 2 * g.Ny, 1.0f, gparts, p->gband, st))) return rc;
  if ((rc = kl::gen_launch_vjp_spectral(g, p->band, nparts, p->gband, gparts, nclips, p->H, p->lam, p->K, p->nsets,
                                        ns_adj, p->gam, st)))
    return rc;
  if ((rc = kl::gen_launch_gradT(g, p->gam, nclips, p->nsets * ns_adj, p->Tg, st))) return rc;
  if ((rc = kl::gen_launch_colinv(g, p->gtab, p->Tg, nclips, 1, g.Ny, g.nf, p->Q, st))) return rc;
  if ((rc = kl::gen_launch_rowinv(g, p->gtab, p->Q, nclips, g.nf, grad, st))) return rc;
  p->last_vjp_clips = nclips;
  p->last_nparts = nparts;
  p->last_gparts = gparts;
  return KL_OK;
}
}  // namespace

int kl::socs_run_forward(kl_socs_plan_s* p, const float* masks, int nclips, float* images, cudaStream_t st,
                         const cudaEvent_t* ev4) {
  return run_forward(p, masks, nclips, images, st, ev4);
}

extern "C" {

int kl_socs_plan_create(kl_socs_plan* plan, int Lx, int Ly, int Nx, int Ny, int nk, int nsets,
                        int max_clips) {
  return create_plan(plan, Lx, Ly, Nx, Ny, nk, nsets, max_clips, false);
}

int kl_socs_plan_create_adjoint(kl_socs_plan* plan, int Lx, int Ly, int Nx, int Ny, int nk,
                                int nsets, int max_clips) {
  return create_plan(plan, Lx, Ly, Nx, Ny, nk, nsets, max_clips, true);
}

int kl_socs_plan_create_ex(kl_socs_plan* plan, int Lx, int Ly, int Nx, int Ny, int nk, int nsets,
                           int max_clips, int flags) {
  KL_CHECK_ARG((flags & ~(KL_SOCS_ADJOINT | KL_SOCS_GENERAL)) == 0, "kl_socs_plan_create_ex: unknown flags");
  return create_plan(plan, Lx, Ly, Nx, Ny, nk, nsets, max_clips, (flags & KL_SOCS_ADJOINT) != 0,
                     (flags & KL_SOCS_GENERAL) != 0);
}

int kl_socs_plan_engine(kl_socs_plan plan) { return plan ? (plan->gen ? 1 : 0) : -1; }

int kl_socs_vjp(kl_socs_plan p, const float* masks, const float* targets, int nclips, float alpha,
                float threshold, float* images, float* grad, double* loss, void* stream) {
  KL_CHECK_ARG(p && masks && targets && grad && loss, "kl_socs_vjp: NULL argument");
  KL_CHECK_ARG((reinterpret_cast<uintptr_t>(targets) & 15) == 0, "kl_socs_vjp: targets_dev must be 16-byte aligned");
  KL_CHECK_ARG(p->adjoint, "kl_socs_vjp: the plan was not created by kl_socs_plan_create_adjoint");
  KL_CHECK_ARG(nclips >= 0 && nclips <= p->max_clips, "kl_socs_vjp: nclips exceeds the plan");
  cudaStream_t st = (cudaStream_t)stream;
  if (nclips == 0) return KL_OK;
  if (p->gen) return vjp_gen(p, masks, targets, nclips, alpha, threshold, images, grad, loss, st);
  const kl::SocsGeom& g = p->g;
  int rc;
  const int ns1 = kl::socs_choose_split(g, nclips, p->nsets, p->K);
  if (p->synth == KL_SYNTH_TENSOR_CORES && use_tc_forward(p, nclips, masks))
    rc = kl::fwd_tc_launch(g, masks, nclips, p->ty, p->thi, p->tlo, p->partial, p->status, st);
  else
    rc = kl::socs_launch_forward(g, p->tx, p->ty, masks, nclips, p->partial, st);
  if (rc) return rc;
  if ((rc = kl::socs_launch_spectral(g, p->partial, nclips, p->H, p->lam, p->K, p->nsets, ns1, p->T, st)))
    return rc;
  KL_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(double) * (size_t)nclips * p->nsets, st));
  // image, resist, loss and the row DFT of dL/dI: on the tensor cores where
  // the plan has them, unless it asks for the CUDA-core engine
  const bool tca = p->vjp_tc && p->synth != KL_SYNTH_CUDA_CORES &&
                   (((uintptr_t)targets | (uintptr_t)images) & 15) == 0;
  rc = tca ? kl::vjp_tc_launch(g, p->T, p->ty, nclips, p->nsets, ns1, p->bhi, p->blo, p->thi, p->tlo, targets, alpha,
                               threshold, images, loss, p->gpart, p->status, st)
           : kl::vjp_launch_inverse(g, p->tx, p->ty, p->T, nclips, p->nsets, ns1, targets, alpha, threshold, images,
                                    loss, p->gpart, st);
  if (rc) return rc;
  const int ns2 = kl::socs_choose_split(g, nclips, p->nsets, p->K);
  if ((rc = kl::vjp_launch_spectral(g, p->partial, p->gpart, nclips, p->H, p->lam, p->K, p->nsets,
                                    ns2, p->gam, st)))
    return rc;
  if ((rc = kl::vjp_launch_gradT(g, p->gam, nclips, p->nsets * ns2, p->Tg, st))) return rc;
  // the gradient is a band-limited synthesis like the image: on the tensor
  // cores unless the plan asks for the CUDA-core engine
  const bool tcg = p->bhi && p->synth != KL_SYNTH_CUDA_CORES && kl::synth_tc_aligned(grad);
  rc = tcg ? kl::synth_tc_launch(g, p->Tg, p->ty, 1, p->bhi, p->blo, nclips, grad, p->status, st)
           : kl::socs_launch_inverse(g, p->tx, p->ty, p->Tg, nclips, 1, 1, grad, st);
  if (rc) return rc;
  p->last_vjp_clips = nclips;
  return KL_OK;
}

int kl_socs_set_synthesis(kl_socs_plan p, int mode) {
  KL_CHECK_ARG(p != nullptr, "kl_socs_set_synthesis: plan is NULL");
  KL_CHECK_ARG(mode == KL_SYNTH_AUTO || mode == KL_SYNTH_CUDA_CORES || mode == KL_SYNTH_TENSOR_CORES,
               "kl_socs_set_synthesis: mode must be KL_SYNTH_AUTO, KL_SYNTH_CUDA_CORES or KL_SYNTH_TENSOR_CORES");
  if (mode == KL_SYNTH_TENSOR_CORES && !p->bhi) {
    kl::set_error(p->gen ? "kl_socs_set_synthesis: the general pipeline has no tensor-core synthesis"
                         : "kl_socs_set_synthesis: the tensor-core synthesis needs Lx, Ly multiples of 128 and "
                           "2(2Nx+1) <= 128");
    return KL_ERR_UNSUPPORTED;
  }
  p->synth = mode;
  return KL_OK;
}

int kl_socs_synthesis(kl_socs_plan p, int nclips) {
  if (!p) return KL_ERR_INVALID;
  return use_tc_synthesis(p, nclips) ? KL_SYNTH_TENSOR_CORES : KL_SYNTH_CUDA_CORES;
}

int kl_socs_plan_status(kl_socs_plan p) {
  KL_CHECK_ARG(p != nullptr, "kl_socs_plan_status: plan is NULL");
  KL_CUDA_TRY(cudaDeviceSynchronize());
  if (!p->status) return KL_OK;
  int code = 0;
  KL_CUDA_TRY(cudaMemcpy(&code, p->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (!code) return KL_OK;
  KL_CUDA_TRY(cudaMemset(p->status, 0, sizeof(int)));
  kl::set_error("tensor-core synthesis: pipeline wait timed out (code " + std::to_string(code) + ")");
  return KL_ERR_CUDA;
}

int kl_socs_plan_destroy(kl_socs_plan plan) {
  free_plan(plan);
  return KL_OK;
}

int kl_socs_set_kernels(kl_socs_plan p, int set, const float* re, const float* im,
                        const float* scales) {
  KL_CHECK_ARG(p && re && im && scales, "kl_socs_set_kernels: NULL argument");
  KL_CHECK_ARG(set >= 0 && set < p->nsets, "kl_socs_set_kernels: set out of range");
  const size_t nb2 = (size_t)p->g.nby * p->g.nbx;
  std::vector<float2> h(nb2 * p->K);
  for (size_t i = 0; i < h.size(); ++i) h[i] = make_float2(re[i], im[i]);
  KL_CUDA_TRY(cudaMemcpy(p->H + (size_t)set * p->K * nb2, h.data(), sizeof(float2) * h.size(),
                         cudaMemcpyHostToDevice));
  KL_CUDA_TRY(cudaMemcpy(p->lam + (size_t)set * p->K, scales, sizeof(float) * p->K,
                         cudaMemcpyHostToDevice));
  return KL_OK;
}

int kl_socs_set_kernels_device(kl_socs_plan p, int set, const float2* H_dev, const float* lam_dev,
                               cudaStream_t st) {
  KL_CHECK_ARG(p && H_dev && lam_dev, "kl_socs_set_kernels_device: NULL argument");
  KL_CHECK_ARG(set >= 0 && set < p->nsets, "kl_socs_set_kernels_device: set out of range");
  const size_t nb2 = (size_t)p->g.nby * p->g.nbx;
  KL_CUDA_TRY(cudaMemcpyAsync(p->H + (size_t)set * p->K * nb2, H_dev, sizeof(float2) * nb2 * p->K,
                              cudaMemcpyDeviceToDevice, st));
  KL_CUDA_TRY(cudaMemcpyAsync(p->lam + (size_t)set * p->K, lam_dev, sizeof(float) * p->K,
                              cudaMemcpyDeviceToDevice, st));
  return KL_OK;
}

int kl_socs_forward(kl_socs_plan p, const float* masks, int nclips, float* images, void* stream) {
  KL_CHECK_ARG(p && masks && images, "kl_socs_forward: NULL argument");
  KL_CHECK_ARG(nclips >= 0 && nclips <= p->max_clips, "kl_socs_forward: nclips exceeds the plan");
  return run_forward(p, masks, nclips, images, (cudaStream_t)stream);
}

int kl_socs_forward_host(kl_socs_plan p, const float* masks_host, int nclips, float* images_host,
                         void* stream) {
  KL_CHECK_ARG(p && masks_host && images_host, "kl_socs_forward_host: NULL argument");
  KL_CHECK_ARG(nclips >= 0 && nclips <= p->max_clips, "kl_socs_forward_host: nclips exceeds the plan");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t px = (size_t)p->g.Lx * p->g.Ly;
  if (p->stage_clips < (size_t)nclips) {
    cudaFree(p->stage_in);
    cudaFree(p->stage_out);
    p->stage_in = p->stage_out = nullptr;
    p->stage_clips = 0;
    int rc;
    if ((rc = alloc((void**)&p->stage_in, sizeof(float) * px * nclips, "mask staging")) ||
        (rc = alloc((void**)&p->stage_out, sizeof(float) * px * nclips * p->nsets, "image staging")))
      return rc;
    p->stage_clips = (size_t)nclips;
  }
  if (nclips == 0) return KL_OK;
  // chunks flow through three streams: copy-in, compute (in order, so the
  // plan's scratch is reused safely), copy-out; the two copy directions and
  // the kernels of neighbouring chunks overlap
  if (!p->hs[0]) {
    for (int i = 0; i < 3; ++i) {
      KL_CUDA_TRY(cudaStreamCreateWithFlags(&p->hs[i], cudaStreamNonBlocking));
      KL_CUDA_TRY(cudaEventCreateWithFlags(&p->hev[i], cudaEventDisableTiming));
    }
  }
  cudaStream_t sin = p->hs[0], scomp = p->hs[1], sout = p->hs[2];
  KL_CUDA_TRY(cudaEventRecord(p->hev[0], st));  // after earlier work on the caller's stream
  for (int i = 0; i < 3; ++i) KL_CUDA_TRY(cudaStreamWaitEvent(p->hs[i], p->hev[0], 0));
  // chunks of about 64 MB of images (up to 16): the copy-out stream idles only
  // while the first chunk is copied in and imaged, and the last copied out
  const size_t outpx = px * p->nsets;
  const size_t outbytes = sizeof(float) * outpx * (size_t)nclips;
  const int nchunks = (int)std::min<size_t>({(size_t)16, std::max<size_t>(1, outbytes >> 26), (size_t)nclips});
  for (int c = 0; c < nchunks; ++c) {
    const int a = (int)((long long)nclips * c / nchunks), b = (int)((long long)nclips * (c + 1) / nchunks);
    if (b == a) continue;
    KL_CUDA_TRY(cudaMemcpyAsync(p->stage_in + px * a, masks_host + px * a, sizeof(float) * px * (b - a),
                                cudaMemcpyHostToDevice, sin));
    KL_CUDA_TRY(cudaEventRecord(p->hev[1], sin));
    KL_CUDA_TRY(cudaStreamWaitEvent(scomp, p->hev[1], 0));
    int rc = run_forward(p, p->stage_in + px * a, b - a, p->stage_out + outpx * a, scomp);
    if (rc) return rc;
    KL_CUDA_TRY(cudaEventRecord(p->hev[2], scomp));
    KL_CUDA_TRY(cudaStreamWaitEvent(sout, p->hev[2], 0));
    KL_CUDA_TRY(cudaMemcpyAsync(images_host + outpx * a, p->stage_out + outpx * a, sizeof(float) * outpx * (b - a),
                                cudaMemcpyDeviceToHost, sout));
  }
  KL_CUDA_TRY(cudaEventRecord(p->hev[0], sout));
  KL_CUDA_TRY(cudaStreamWaitEvent(st, p->hev[0], 0));
  KL_CUDA_TRY(cudaStreamSynchronize(st));
  return p->status ? kl_socs_plan_status(p) : KL_OK;
}

int kl_socs_enable_timing(kl_socs_plan p, int enable) {
  KL_CHECK_ARG(p, "kl_socs_enable_timing: NULL plan");
  p->timing = enable != 0;
  if (!p->timing) drop_events(p);
  return KL_OK;
}

int kl_socs_stage_times(kl_socs_plan p, double* ms, int* launches) {
  KL_CHECK_ARG(p && ms && launches, "kl_socs_stage_times: NULL argument");
  for (int i = 0; i < 3; ++i) {
    ms[i] = 0.0;
    launches[i] = 0;
  }
  for (size_t b = 0; b + 3 < p->events.size(); b += 4) {
    KL_CUDA_TRY(cudaEventSynchronize(p->events[b + 3]));
    for (int i = 0; i < 3; ++i) {
      float t = 0.f;
      KL_CUDA_TRY(cudaEventElapsedTime(&t, p->events[b + i], p->events[b + i + 1]));
      ms[i] += t;
      launches[i] += 1;
    }
  }
  drop_events(p);
  return KL_OK;
}

int kl_mask_spectrum(kl_socs_plan p, const float* masks, int nclips, float* band, void* stream) {
  KL_CHECK_ARG(p && masks && band, "kl_mask_spectrum: NULL argument");
  KL_CHECK_ARG(nclips >= 0 && nclips <= p->max_clips, "kl_mask_spectrum: nclips exceeds the plan");
  cudaStream_t st = (cudaStream_t)stream;
  if (p->gen) {
    const kl::GenGeom& g = p->gg;
    const int nparts = kl::gen_choose_parts(g, nclips, g.nf);
    int rc = kl::gen_launch_rowfwd(g, p->gtab, masks, nclips * g.Ly, p->R, st);
    if (!rc)
      rc = kl::gen_launch_colfwd(g, p->gtab, p->R, nclips, g.nf, g.Ny, 1.0f / ((float)g.Lx * (float)g.Ly), nparts,
                                 p->band, st);
    if (!rc) rc = kl::gen_launch_bandout(g, p->band, nparts, nclips, reinterpret_cast<float2*>(band), st);
    return rc;
  }
  int rc = kl::socs_launch_forward(p->g, p->tx, p->ty, masks, nclips, p->partial, st);
  if (rc) return rc;
  return kl::socs_launch_band(p->g, p->partial, nclips, reinterpret_cast<float2*>(band), st);
}

int kl_fp64_socs_forward(const float* masks, int nclips, int Lx, int Ly, int Nx, int Ny, const float* kernels,
                         const float* scales, int nk, double* images, void* stream) {
  return kl::f64::socs_forward(masks, nclips, Lx, Ly, Nx, Ny, reinterpret_cast<const float2*>(kernels), scales,
                               nk, images, (cudaStream_t)stream);
}

int kl_fp64_socs_vjp(const float* masks, const float* targets, int nclips, int Lx, int Ly, int Nx, int Ny,
                     const float* kernels, const float* scales, int nk, double alpha, double threshold,
                     double* images, double* grad, double* loss, void* stream) {
  return kl::f64::socs_vjp(masks, targets, nclips, Lx, Ly, Nx, Ny, reinterpret_cast<const float2*>(kernels), scales,
                           nk, alpha, threshold, images, grad, loss, (cudaStream_t)stream);
}

int kl_fp64_mask_spectrum(const float* mask, int Lx, int Ly, double* spectrum, void* stream) {
  return kl::f64::mask_spectrum(mask, Lx, Ly, reinterpret_cast<double2*>(spectrum), (cudaStream_t)stream);
}

}  // extern "C"
