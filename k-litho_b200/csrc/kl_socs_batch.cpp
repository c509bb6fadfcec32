// kl_socs_batch.cpp -- launch-shape autotuning of a SOCS plan, and batches of
// plans (one per clip size, each with its kernel sets, e.g. focus values)
// imaged by one CUDA graph whose branches run concurrently, so that the
// on-chip spectral stage of one size class overlaps the HBM-bound stages of
// the others.  No counterpart in the reference, which images one clip per
// process (K-Litho-SOCS/klitho_socs.cpp:245-362).
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <string>
#include <vector>

#include "kl_internal.h"
#include "kl_plans.h"

struct kl_socs_batch_s {
  std::vector<kl_socs_plan> plans;
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> join;
  std::vector<cudaEvent_t> stage;  // 4 per plan when timing is on
  cudaStream_t origin = nullptr;
  cudaEvent_t fork = nullptr, entry = nullptr, done = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool timing = false;
  // what the instantiated graph was captured for
  std::vector<const float*> key_masks;
  std::vector<float*> key_images;
  std::vector<int> key_clips;
  int graph_builds = 0;
};

namespace {

void destroy_batch(kl_socs_batch_s* b) {
  if (!b) return;
  if (b->origin) cudaStreamSynchronize(b->origin);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  for (cudaStream_t s : b->branch) cudaStreamDestroy(s);
  for (cudaEvent_t e : b->join) cudaEventDestroy(e);
  for (cudaEvent_t e : b->stage) cudaEventDestroy(e);
  if (b->origin) cudaStreamDestroy(b->origin);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->entry) cudaEventDestroy(b->entry);
  if (b->done) cudaEventDestroy(b->done);
  delete b;
}

// fork on `origin`, one branch per plan, join back on `origin`
int enqueue_branches(kl_socs_batch_s* b, const float* const* masks, const int* nclips, float* const* images) {
  KL_CUDA_TRY(cudaEventRecord(b->fork, b->origin));
  for (size_t i = 0; i < b->plans.size(); ++i) {
    KL_CUDA_TRY(cudaStreamWaitEvent(b->branch[i], b->fork, 0));
    const cudaEvent_t* ev4 = b->timing ? &b->stage[4 * i] : nullptr;
    if (ev4 || nclips[i] > 0) {
      const int rc = kl::socs_run_forward(b->plans[i], masks[i], nclips[i], images[i], b->branch[i], ev4);
      if (rc) return rc;
    }
    KL_CUDA_TRY(cudaEventRecord(b->join[i], b->branch[i]));
    KL_CUDA_TRY(cudaStreamWaitEvent(b->origin, b->join[i], 0));
  }
  return KL_OK;
}

bool same_key(const kl_socs_batch_s* b, const float* const* masks, const int* nclips, float* const* images) {
  if (!b->exec) return false;
  for (size_t i = 0; i < b->plans.size(); ++i)
    if (b->key_masks[i] != masks[i] || b->key_images[i] != images[i] || b->key_clips[i] != nclips[i]) return false;
  return true;
}

}  // namespace

extern "C" {

int kl_socs_autotune(kl_socs_plan p, const float* masks, int nclips, float* images, void* stream, int* nsplit_out,
                     int* spc_out) {
  KL_CHECK_ARG(p && masks && images, "kl_socs_autotune: NULL argument");
  KL_CHECK_ARG(nclips > 0 && nclips <= p->max_clips, "kl_socs_autotune: nclips must be in [1, max_clips]");
  cudaStream_t st = (cudaStream_t)stream;
  const bool timing = p->timing;
  p->timing = false;
  std::vector<int> splits, spcs;
  // the spectra buffer holds tcap (clip, slice) pairs per kernel set on the
  // specialised kernels, tcap (image, slice) pairs on the general pipeline
  const int per_slice = p->gen ? nclips * p->nsets : nclips;
  for (int ns = 1; ns <= kl::kSocsMaxSplit; ns *= 2)
    if (ns * per_slice <= p->tcap && ns <= p->K) splits.push_back(ns);
  // strips per CTA of the synthesis: specialised kernels only
  if (!p->gen)
    for (int c = 1; c <= 16 && c <= p->g.nS; c *= 2) spcs.push_back(c);
  cudaEvent_t e0, e1;
  KL_CUDA_TRY(cudaEventCreate(&e0));
  KL_CUDA_TRY(cudaEventCreate(&e1));
  int rc = KL_OK;
  auto time_shape = [&](int ns, int spc, float* ms) -> int {
    p->tune_clips = nclips;
    p->tune_nsplit = ns;
    p->tune_spc = spc;
    int r = kl::socs_run_forward(p, masks, nclips, images, st, nullptr);  // warm-up
    if (r) return r;
    KL_CUDA_TRY(cudaEventRecord(e0, st));
    for (int k = 0; k < 3 && !r; ++k) r = kl::socs_run_forward(p, masks, nclips, images, st, nullptr);
    if (r) return r;
    KL_CUDA_TRY(cudaEventRecord(e1, st));
    KL_CUDA_TRY(cudaEventSynchronize(e1));
    KL_CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
    return KL_OK;
  };
  int best_ns = splits.empty() ? 1 : splits[0], best_spc = 0;
  float best = 1e30f, t = 0.f;
  // kernel slices of the spectral stage, with the default inverse shape ...
  for (int ns : splits) {
    if ((rc = time_shape(ns, 0, &t))) break;
    if (t < best) {
      best = t;
      best_ns = ns;
    }
  }
  // ... then strips per CTA of the inverse stage, and the tensor-core synthesis
  if (!p->gen && p->bhi && p->synth == KL_SYNTH_AUTO) {
    spcs.push_back(-1);                                  // tensor-core synthesis
    if (p->thi && kl::fwd_tc_supported(p->g)) spcs.push_back(-2);  // ... and mask transform
  }
  for (size_t i = 0; i < spcs.size() && !rc; ++i) {
    if ((rc = time_shape(best_ns, spcs[i], &t))) break;
    if (t < best) {
      best = t;
      best_spc = spcs[i];
    }
  }
  if (!rc && p->status) rc = kl_socs_plan_status(p);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  p->timing = timing;
  if (rc) {
    p->tune_clips = p->tune_nsplit = p->tune_spc = 0;
    return rc;
  }
  p->tune_clips = nclips;
  p->tune_nsplit = best_ns;
  p->tune_spc = best_spc;
  // leave the images of the chosen shape in the output
  if ((rc = kl::socs_run_forward(p, masks, nclips, images, st, nullptr))) return rc;
  if (nsplit_out) *nsplit_out = best_ns;
  if (spc_out) *spc_out = best_spc;
  return KL_OK;
}

int kl_socs_batch_create(kl_socs_batch* batch, const kl_socs_plan* plans, int nplans) {
  KL_CHECK_ARG(batch && plans && nplans > 0, "kl_socs_batch_create: bad arguments");
  *batch = nullptr;
  for (int i = 0; i < nplans; ++i) KL_CHECK_ARG(plans[i], "kl_socs_batch_create: NULL plan");
  kl_socs_batch_s* b = new (std::nothrow) kl_socs_batch_s;
  if (!b) return KL_ERR_NOMEM;
  b->plans.assign(plans, plans + nplans);
  b->branch.assign(nplans, nullptr);
  b->join.assign(nplans, nullptr);
  bool ok = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->entry, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < nplans && ok; ++i)
    ok = cudaStreamCreateWithFlags(&b->branch[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    kl::set_error(std::string("kl_socs_batch_create: ") + cudaGetErrorString(cudaGetLastError()));
    destroy_batch(b);
    return KL_ERR_CUDA;
  }
  *batch = b;
  return KL_OK;
}

int kl_socs_batch_destroy(kl_socs_batch batch) {
  destroy_batch(batch);
  return KL_OK;
}

int kl_socs_batch_enable_timing(kl_socs_batch b, int enable) {
  KL_CHECK_ARG(b, "kl_socs_batch_enable_timing: NULL batch");
  if ((enable != 0) == b->timing) return KL_OK;
  if (b->origin) KL_CUDA_TRY(cudaStreamSynchronize(b->origin));
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;  // the graph is captured again with (or without) the stage events
  for (cudaEvent_t e : b->stage) cudaEventDestroy(e);
  b->stage.clear();
  b->timing = enable != 0;
  if (b->timing) {
    b->stage.assign(4 * b->plans.size(), nullptr);
    for (cudaEvent_t& e : b->stage) KL_CUDA_TRY(cudaEventCreate(&e));
  }
  return KL_OK;
}

int kl_socs_batch_forward(kl_socs_batch b, const float* const* masks, const int* nclips, float* const* images,
                          void* stream) {
  KL_CHECK_ARG(b && masks && nclips && images, "kl_socs_batch_forward: NULL argument");
  const size_t n = b->plans.size();
  for (size_t i = 0; i < n; ++i) {
    KL_CHECK_ARG(nclips[i] >= 0 && nclips[i] <= b->plans[i]->max_clips,
                 "kl_socs_batch_forward: nclips exceeds a plan's max_clips");
    KL_CHECK_ARG(nclips[i] == 0 || (masks[i] && images[i]), "kl_socs_batch_forward: NULL buffer");
  }
  cudaStream_t caller = (cudaStream_t)stream;
  KL_CUDA_TRY(cudaEventRecord(b->entry, caller));
  KL_CUDA_TRY(cudaStreamWaitEvent(b->origin, b->entry, 0));
  int rc;
  if (!same_key(b, masks, nclips, images)) {
    // first call for these buffers: run directly (this also sets the kernels'
    // shared-memory attributes), then capture the same work as a graph
    if ((rc = enqueue_branches(b, masks, nclips, images))) return rc;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    KL_CUDA_TRY(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_branches(b, masks, nclips, images);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(b->origin, &graph);
    if (rc || ce != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      if (!rc) {
        kl::set_error(std::string("kl_socs_batch_forward: capture failed: ") + cudaGetErrorString(ce));
        rc = KL_ERR_CUDA;
      }
      cudaGetLastError();
      return rc;
    }
    const cudaError_t ie = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      b->exec = nullptr;
      kl::set_error(std::string("kl_socs_batch_forward: graph instantiation failed: ") + cudaGetErrorString(ie));
      cudaGetLastError();
      return KL_ERR_CUDA;
    }
    b->key_masks.assign(masks, masks + n);
    b->key_images.assign(images, images + n);
    b->key_clips.assign(nclips, nclips + n);
    ++b->graph_builds;
  } else {
    KL_CUDA_TRY(cudaGraphLaunch(b->exec, b->origin));
  }
  KL_CUDA_TRY(cudaEventRecord(b->done, b->origin));
  KL_CUDA_TRY(cudaStreamWaitEvent(caller, b->done, 0));
  return KL_OK;
}

int kl_socs_batch_stage_times(kl_socs_batch b, int plan, double* ms) {
  KL_CHECK_ARG(b && ms && plan >= 0 && plan < (int)b->plans.size(), "kl_socs_batch_stage_times: bad argument");
  KL_CHECK_ARG(b->timing, "kl_socs_batch_stage_times: timing is not enabled");
  KL_CUDA_TRY(cudaEventSynchronize(b->stage[4 * plan + 3]));
  for (int i = 0; i < 3; ++i) {
    float t = 0.f;
    KL_CUDA_TRY(cudaEventElapsedTime(&t, b->stage[4 * plan + i], b->stage[4 * plan + i + 1]));
    ms[i] = t;
  }
  return KL_OK;
}

int kl_socs_batch_graph_builds(kl_socs_batch b) { return b ? b->graph_builds : -1; }

}  // extern "C"
