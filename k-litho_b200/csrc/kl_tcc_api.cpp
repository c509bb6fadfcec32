// kl_tcc_api.cpp -- C ABI of TCC assembly, top-K SOCS kernels and the
// Hopkins image (see include/klitho_gpu.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "kl_internal.h"
#include "kl_plans.h"
#include "kl_tcc.h"

namespace {
// Plan buffers and host-synchronous temporaries come from the device's pooled
// scratch allocator on the legacy stream; dalloc waits for the block to be
// usable from any stream, dfree is called only after the work using the
// block has been synchronised.
void dfree(void* p) { kl::scratch_free(p, nullptr); }

void free_plan(kl_tcc_plan p) {
  if (!p) return;
  cudaDeviceSynchronize();
  dfree(p->pts_dev);
  dfree(p->A);
  dfree(p->P);
  dfree(p->J);
  dfree(p->src_id);
  dfree(p->tcc64);
  dfree(p->err);
  if (p->hopkins) kl_socs_plan_destroy(p->hopkins);
  delete p;
}

int dalloc(void** ptr, size_t bytes, const char* what) {
  const int rc = kl::scratch_alloc(ptr, bytes, nullptr, what);
  if (rc) return rc;
  KL_CUDA_TRY(cudaStreamSynchronize(nullptr));
  return KL_OK;
}

int ensure_tcc64(kl_tcc_plan p, cudaStream_t st) {
  if (p->tcc64) return KL_OK;
  const size_t N = (size_t)p->pp.N;
  int rc = dalloc((void**)&p->tcc64, sizeof(double2) * N * N, "FP64 TCC");
  if (rc) return rc;
  return kl::tcc_direct_fp64(p->P, p->J, p->pp.N, p->pp.S, p->tcc64, st);
}
}  // namespace

extern "C" {

int kl_tcc_plan_create(kl_tcc_plan* plan, const float* src, int srcSize, double NA, double defocus,
                       double n_medium, int Lx, int Ly, int precision) {
  KL_CHECK_ARG(plan, "kl_tcc_plan_create: plan is NULL");
  *plan = nullptr;
  KL_CHECK_ARG(src && srcSize > 2 && Lx > 0 && Ly > 0 && NA > 0 && n_medium > 0,
               "kl_tcc_plan_create: bad arguments");
  KL_CHECK_ARG(precision == KL_PREC_FAST || precision == KL_PREC_FP64,
               "kl_tcc_plan_create: unknown precision");
  kl_tcc_plan p = new (std::nothrow) kl_tcc_plan_s;
  if (!p) return KL_ERR_NOMEM;
  p->precision = precision;
  p->Lx = Lx;
  p->Ly = Ly;
  p->srcSize = srcSize;
  float sig = kl_outer_sigma(src, srcSize);
  if (sig > 1.0f) sig = 1.0f;  // klitho_tcc.cpp:480-483
  p->outerSigma = sig;
  int Nx = 0, Ny = 0;
  kl_band_size(NA, Lx, Ly, sig, &Nx, &Ny);
  kl::tcc_source_points(src, srcSize, sig, 193.0f, (float)NA, (float)defocus, n_medium, Lx, Ly,
                        Nx, Ny, p->pts, p->pp);
  const kl::PupilParams& pp = p->pp;
  if (pp.S == 0) {
    free_plan(p);
    kl::set_error("kl_tcc_plan_create: the source has no points inside the pupil");
    return KL_ERR_INVALID;
  }
  if (n_medium * n_medium < NA * NA) {
    free_plan(p);
    kl::set_error("kl_tcc_plan_create: NA exceeds n_medium; the defocus phase is undefined");
    return KL_ERR_INVALID;
  }
  int rc;
  if ((rc = dalloc((void**)&p->err, sizeof(int), "status"))) {
    free_plan(p);
    return rc;
  }
  cudaMemset(p->err, 0, sizeof(int));
  const size_t NS = (size_t)pp.N * pp.S;
  {
    std::vector<float> Jh(pp.S);
    std::vector<int> ids(pp.S);
    for (int s = 0; s < pp.S; ++s) {
      Jh[s] = p->pts[s].J;
      ids[s] = p->pts[s].src_id;
    }
    if ((rc = dalloc((void**)&p->J, sizeof(float) * pp.S, "source weights")) ||
        (rc = dalloc((void**)&p->src_id, sizeof(int) * pp.S, "source indices"))) {
      free_plan(p);
      return rc;
    }
    cudaMemcpy(p->J, Jh.data(), sizeof(float) * pp.S, cudaMemcpyHostToDevice);
    cudaMemcpy(p->src_id, ids.data(), sizeof(int) * pp.S, cudaMemcpyHostToDevice);
  }
  if (precision == KL_PREC_FAST) {
    if ((rc = dalloc((void**)&p->pts_dev, sizeof(kl::SrcPoint) * pp.S, "source points")) ||
        (rc = dalloc((void**)&p->A, sizeof(float2) * NS, "TCC factor"))) {
      free_plan(p);
      return rc;
    }
    cudaMemcpy(p->pts_dev, p->pts.data(), sizeof(kl::SrcPoint) * pp.S, cudaMemcpyHostToDevice);
    if ((rc = kl::tcc_build_A(p->pts_dev, pp, p->A, nullptr))) {
      free_plan(p);
      return rc;
    }
  } else {
    std::vector<double> P(2 * NS);
    kl::tcc_pupil_host(p->pts, pp, P.data());
    if ((rc = dalloc((void**)&p->P, sizeof(double2) * NS, "pupil table"))) {
      free_plan(p);
      return rc;
    }
    cudaMemcpy(p->P, P.data(), sizeof(double2) * NS, cudaMemcpyHostToDevice);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    kl::set_error(std::string("kl_tcc_plan_create: ") + cudaGetErrorString(cudaGetLastError()));
    free_plan(p);
    return KL_ERR_CUDA;
  }
  *plan = p;
  return KL_OK;
}

int kl_tcc_plan_destroy(kl_tcc_plan plan) {
  free_plan(plan);
  return KL_OK;
}

int kl_tcc_plan_info(kl_tcc_plan p, int* Nx, int* Ny, int* N, int* S, float* outerSigma) {
  KL_CHECK_ARG(p, "kl_tcc_plan_info: NULL plan");
  if (Nx) *Nx = p->pp.Nx;
  if (Ny) *Ny = p->pp.Ny;
  if (N) *N = p->pp.N;
  if (S) *S = p->pp.S;
  if (outerSigma) *outerSigma = p->outerSigma;
  return KL_OK;
}

int kl_tcc_factor(kl_tcc_plan p, float* A_dev, void* stream) {
  KL_CHECK_ARG(p && A_dev, "kl_tcc_factor: NULL argument");
  KL_CHECK_ARG(p->precision == KL_PREC_FAST, "kl_tcc_factor: FP32 factor exists on the fast path only");
  KL_CUDA_TRY(cudaMemcpyAsync(A_dev, p->A, sizeof(float2) * (size_t)p->pp.N * p->pp.S,
                              cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return KL_OK;
}

int kl_tcc_build(kl_tcc_plan p, void* tcc_dev, void* stream) {
  KL_CHECK_ARG(p && tcc_dev, "kl_tcc_build: NULL argument");
  cudaStream_t st = (cudaStream_t)stream;
  const int N = p->pp.N, S = p->pp.S;
  if (p->precision == KL_PREC_FP64) {
    int rc = kl::tcc_direct_fp64(p->P, p->J, N, S, (double2*)tcc_dev, st);
    if (rc) return rc;
    return KL_OK;
  }
  const int K2p = kl::tcc_kp(S);
  void* ops = nullptr;
  int rc;
  if ((rc = kl::scratch_alloc(&ops, sizeof(uint16_t) * 4 * (size_t)N * K2p, st, "split operands"))) return rc;
  if (cudaMemsetAsync(p->err, 0, sizeof(int), st) != cudaSuccess) {
    kl::set_error(std::string("kl_tcc_build: ") + cudaGetErrorString(cudaGetLastError()));
    rc = KL_ERR_CUDA;
  }
  if (!rc) rc = kl::tcc_split_operands(p->A, N, S, K2p, ops, st);
  if (!rc) rc = kl::tcc_gemm_tc(ops, N, K2p, (float2*)tcc_dev, p->err, st);
  int herr = 0;
  if (!rc) {
    cudaMemcpyAsync(&herr, p->err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      kl::set_error(std::string("kl_tcc_build: ") + cudaGetErrorString(cudaGetLastError()));
      rc = KL_ERR_CUDA;
    } else if (herr) {
      kl::set_error("kl_tcc_build: tensor-core pipeline wait timed out (code " + std::to_string(herr) + ")");
      rc = KL_ERR_CUDA;
    }
  }
  kl::scratch_free(ops, st);
  return rc;
}

int kl_tcc_minmax(kl_tcc_plan p, const void* tcc_dev, double* out4, void* stream) {
  KL_CHECK_ARG(p && tcc_dev && out4, "kl_tcc_minmax: NULL argument");
  const size_t n = (size_t)p->pp.N * p->pp.N;
  if (p->precision == KL_PREC_FP64)
    return kl::tcc_minmax_c128((const double2*)tcc_dev, n, out4, (cudaStream_t)stream);
  return kl::tcc_minmax_c64((const float2*)tcc_dev, n, out4, (cudaStream_t)stream);
}

int kl_tcc_build_host(kl_tcc_plan p, float* re_host, float* im_host) {
  KL_CHECK_ARG(p && re_host && im_host, "kl_tcc_build_host: NULL argument");
  const size_t n = (size_t)p->pp.N * p->pp.N;
  const bool f64 = p->precision == KL_PREC_FP64;
  void* tcc = nullptr;
  int rc = kl::scratch_alloc(&tcc, (f64 ? sizeof(double2) : sizeof(float2)) * n, nullptr, "TCC");
  if (rc) return rc;
  rc = kl_tcc_build(p, tcc, nullptr);
  if (!rc) {
    if (f64) {
      std::vector<double2> h(n);
      if (cudaMemcpy(h.data(), tcc, sizeof(double2) * n, cudaMemcpyDeviceToHost) != cudaSuccess) rc = KL_ERR_CUDA;
      for (size_t i = 0; i < n && !rc; ++i) {
        re_host[i] = (float)h[i].x;
        im_host[i] = (float)h[i].y;
      }
    } else {
      std::vector<float2> h(n);
      if (cudaMemcpy(h.data(), tcc, sizeof(float2) * n, cudaMemcpyDeviceToHost) != cudaSuccess) rc = KL_ERR_CUDA;
      for (size_t i = 0; i < n && !rc; ++i) {
        re_host[i] = h[i].x;
        im_host[i] = h[i].y;
      }
    }
    if (rc) kl::set_error(std::string("kl_tcc_build_host: ") + cudaGetErrorString(cudaGetLastError()));
  }
  kl::scratch_free(tcc, nullptr);
  return rc;
}

int kl_tcc_build_minmax(kl_tcc_plan p, double* out4) {
  KL_CHECK_ARG(p && out4, "kl_tcc_build_minmax: NULL argument");
  const size_t n = (size_t)p->pp.N * p->pp.N;
  void* tcc = nullptr;
  int rc = kl::scratch_alloc(&tcc, (p->precision == KL_PREC_FP64 ? sizeof(double2) : sizeof(float2)) * n,
                             nullptr, "TCC");
  if (rc) return rc;
  rc = kl_tcc_build(p, tcc, nullptr);
  if (!rc) rc = kl_tcc_minmax(p, tcc, out4, nullptr);
  kl::scratch_free(tcc, nullptr);
  return rc;
}

namespace {

// device buffers of one top-K solve
// device buffers of one top-K solve; c64: the kernels interleaved (re holds
// 2 N K floats, im is unused) instead of as two planes
struct TopkBuffers {
  double2* U = nullptr;
  double* ev = nullptr;
  float *re = nullptr, *im = nullptr;
  kl::EigenResult res{};
  int alloc(int N, int K, bool c64) {
    int rc;
    if ((rc = kl::scratch_alloc((void**)&U, sizeof(double2) * (size_t)N * K, nullptr, "eigenvectors")) ||
        (rc = kl::scratch_alloc((void**)&ev, sizeof(double) * K, nullptr, "eigenvalues")) ||
        (rc = kl::scratch_alloc((void**)&re, sizeof(float) * (size_t)N * K * (c64 ? 2 : 1), nullptr, "kernels")) ||
        (!c64 && (rc = kl::scratch_alloc((void**)&im, sizeof(float) * (size_t)N * K, nullptr, "kernels"))))
      return rc;
    return KL_OK;
  }
  ~TopkBuffers() {
    kl::scratch_free(U, nullptr);
    kl::scratch_free(ev, nullptr);
    kl::scratch_free(re, nullptr);
    kl::scratch_free(im, nullptr);
  }
};

kl::EigenOptions topk_options(int K, int block) {
  kl::EigenOptions opt;
  opt.K = K;
  opt.B = block > 0 ? block : std::min(K + std::max(16, K / 2), std::max(K, 2 * K));
  opt.max_iter = 400;
  opt.tol = 1e-13;
  opt.seed = 0x6b6c697468ull;
  return opt;
}

// kernels (reference layout) and eigenvalues to the host; the nk - K kernels
// beyond the TCC's rank are zero
// kernels, scales and eigenvalues to the host; krn_im_host null: the kernels
// go interleaved (complex64) into krn_re_host
int topk_finish(TopkBuffers& b, int N, int K, int nk, float* krn_re_host, float* krn_im_host,
                float* scales_host, double* evals_host, int* iterations, cudaStream_t st) {
  const bool c64 = krn_im_host == nullptr;
  int rc = kl::eig_to_kernels(b.U, N, K, b.re, c64 ? nullptr : b.im, st);
  if (rc) return rc;
  std::vector<double> evh(K);
  cudaMemcpy(krn_re_host, b.re, sizeof(float) * (size_t)N * K * (c64 ? 2 : 1), cudaMemcpyDeviceToHost);
  if (!c64) cudaMemcpy(krn_im_host, b.im, sizeof(float) * (size_t)N * K, cudaMemcpyDeviceToHost);
  cudaMemcpy(evh.data(), b.ev, sizeof(double) * K, cudaMemcpyDeviceToHost);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    kl::set_error(std::string("kl_topk_eig: ") + cudaGetErrorString(cudaGetLastError()));
    return KL_ERR_CUDA;
  }
  for (int k = 0; k < nk; ++k) {
    const double v = k < K ? evh[k] : 0.0;
    scales_host[k] = (float)v;
    if (evals_host) evals_host[k] = v;
  }
  for (int k = K; k < nk; ++k) {
    if (c64) {
      std::memset(krn_re_host + 2 * (size_t)k * N, 0, 2 * sizeof(float) * N);
      continue;
    }
    std::memset(krn_re_host + (size_t)k * N, 0, sizeof(float) * N);
    std::memset(krn_im_host + (size_t)k * N, 0, sizeof(float) * N);
  }
  if (iterations) *iterations = b.res.iterations;
  return KL_OK;
}

}  // namespace

int kl_factor_gram(const void* A_dev, int N, int S, void* G_dev, void* stream) {
  KL_CHECK_ARG(A_dev && G_dev && N >= 1 && S >= 1, "kl_factor_gram: NULL argument or empty factor");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int* err = nullptr;
  if (int rc = kl::scratch_alloc((void**)&err, sizeof(int), st, "kl_factor_gram status")) return rc;
  int rc = KL_OK, herr = 0;
  if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) {
    kl::set_error("kl_factor_gram: cudaMemsetAsync failed");
    rc = KL_ERR_CUDA;
  }
  if (!rc) rc = kl::gram_factor(static_cast<const float2*>(A_dev), N, S, static_cast<double2*>(G_dev), err, st);
  if (!rc && (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
              cudaStreamSynchronize(st) != cudaSuccess)) {
    kl::set_error(std::string("kl_factor_gram: ") + cudaGetErrorString(cudaGetLastError()));
    rc = KL_ERR_CUDA;
  }
  kl::scratch_free(err, st);
  if (!rc && herr) {
    kl::set_error("kl_factor_gram: a tensor-core pipeline wait gave up (code " + std::to_string(herr) + ")");
    rc = KL_ERR_CUDA;
  }
  return rc;
}

int kl_hermitian_topk(const void* H_dev, int B, int K, double* evals_dev, void* vecs_dev, void* stream) {
  KL_CHECK_ARG(H_dev && evals_dev && vecs_dev, "kl_hermitian_topk: NULL argument");
  KL_CHECK_ARG(B >= kl::kTridiagMinB && B <= kl::kTridiagMaxB, "kl_hermitian_topk: B must be in [64, 256]");
  KL_CHECK_ARG(K >= 1 && K <= B, "kl_hermitian_topk: K must be in [1, B]");
  KL_CHECK_ARG(kl::tridiag_eig_supported(B),
               "kl_hermitian_topk: this device cannot co-schedule the 8-CTA cluster of the reduction");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t n2 = sizeof(double2) * B * B, nv = sizeof(double) * B * K;
  const size_t nwy = sizeof(double2) * 64 * (size_t)kl::tridiag_wy_blocks(B);
  const size_t bytes = n2 + nwy + sizeof(double) * B + sizeof(double2) * B + 2 * nv + 16;
  void* buf = nullptr;
  if (int rc = kl::scratch_alloc(&buf, bytes, st, "kl_hermitian_topk work")) return rc;
  char* c = static_cast<char*>(buf);
  kl::TridiagJob j{};
  j.H = static_cast<const double2*>(H_dev);
  j.refl = reinterpret_cast<double2*>(c);
  j.wy = reinterpret_cast<double2*>(c + n2);
  c += nwy;
  j.e = reinterpret_cast<double2*>(c + n2);
  j.d = reinterpret_cast<double*>(c + n2 + sizeof(double2) * B);
  j.lw = reinterpret_cast<double*>(c + n2 + sizeof(double2) * B + sizeof(double) * B);
  j.Y = j.lw + (size_t)B * K;
  j.w = evals_dev;
  j.Q = static_cast<double2*>(vecs_dev);
  j.B = B;
  j.K = K;
  j.ldq = K;
  j.err = reinterpret_cast<int*>(j.Y + (size_t)B * K);
  int rc = KL_OK, herr = 0;
  if (cudaMemsetAsync(j.err, 0, sizeof(int), st) != cudaSuccess) {
    kl::set_error("kl_hermitian_topk: cudaMemsetAsync failed");
    rc = KL_ERR_CUDA;
  }
  if (!rc) rc = kl::tridiag_eig_batch({j}, st);
  if (!rc && (cudaMemcpyAsync(&herr, j.err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
              cudaStreamSynchronize(st) != cudaSuccess)) {
    kl::set_error(std::string("kl_hermitian_topk: ") + cudaGetErrorString(cudaGetLastError()));
    rc = KL_ERR_CUDA;
  }
  kl::scratch_free(buf, st);
  if (!rc && herr) {
    kl::set_error("kl_hermitian_topk: the reduction's exchange wait gave up (code " + std::to_string(herr) + ")");
    rc = KL_ERR_CUDA;
  }
  return rc;
}

namespace {

// kl_topk_eig; krn_im_host null: interleaved kernels (kl_topk_eig_c64)
int topk_one(kl_tcc_plan p, int nk, int block, float* krn_re_host, float* krn_im_host, float* scales_host,
             double* evals_host, int* iterations) {
  const int N = p->pp.N, S = p->pp.S;
  KL_CHECK_ARG(nk > 0 && nk <= N, "kl_topk_eig: nk must be in [1, N]");
  cudaStream_t st = nullptr;
  // kernels beyond the TCC's rank (<= S) have eigenvalue 0: the solver
  // returns the nonzero part, the rest are zero kernels
  const int K = std::min(nk, std::min(N, S));
  const kl::EigenOptions opt = topk_options(K, block);
  TopkBuffers b;
  int rc = b.alloc(N, K, krn_im_host == nullptr);
  if (rc) return rc;
  if (p->precision == KL_PREC_FAST) {
    rc = kl::eig_topk_factor(p->A, N, S, opt, b.U, b.ev, &b.res, st);
  } else {
    rc = ensure_tcc64(p, st);
    if (!rc) rc = kl::eig_topk_dense(p->tcc64, N, opt, b.U, b.ev, &b.res, st);
  }
  if (rc) return rc;
  return topk_finish(b, N, K, nk, krn_re_host, krn_im_host, scales_host, evals_host, iterations, st);
}

// kl_topk_eig_batch; krn_im_host null: interleaved kernels (kl_topk_eig_batch_c64)
int topk_batch(const kl_tcc_plan* plans, int nplans, int nk, int block, float* krn_re_host, float* krn_im_host,
               float* scales_host, double* evals_host, int* iterations) {
  const bool c64 = krn_im_host == nullptr;
  const int N = plans[0] ? plans[0]->pp.N : 0;
  bool fast = true;
  for (int i = 0; i < nplans; ++i) {
    KL_CHECK_ARG(plans[i], "kl_topk_eig_batch: NULL plan");
    KL_CHECK_ARG(plans[i]->pp.N == N, "kl_topk_eig_batch: plans must share the pupil band (same N)");
    fast = fast && plans[i]->precision == KL_PREC_FAST;
  }
  KL_CHECK_ARG(nk > 0 && nk <= N, "kl_topk_eig_batch: nk must be in [1, N]");
  const size_t kstride = (size_t)nk * N;
  const size_t rstride = kstride * (c64 ? 2 : 1);  // floats of one plan's kernels in krn_re_host
  if (!fast) {  // the FP64 path solves one plan after another
    for (int i = 0; i < nplans; ++i) {
      const int rc = topk_one(plans[i], nk, block, krn_re_host + i * rstride,
                              c64 ? nullptr : krn_im_host + i * kstride, scales_host + (size_t)i * nk,
                              evals_host ? evals_host + (size_t)i * nk : nullptr, iterations ? iterations + i : nullptr);
      if (rc) return rc;
    }
    return KL_OK;
  }
  cudaStream_t st = nullptr;
  std::vector<TopkBuffers> bufs(nplans);
  std::vector<kl::FactorProblem> pr(nplans);
  int kmax = 1;
  for (int i = 0; i < nplans; ++i) {
    const int K = std::min(nk, std::min(N, plans[i]->pp.S));
    kmax = std::max(kmax, K);
    int rc = bufs[i].alloc(N, K, c64);
    if (rc) return rc;
    pr[i] = kl::FactorProblem{plans[i]->A, N, plans[i]->pp.S, K, bufs[i].U, bufs[i].ev, &bufs[i].res};
  }
  int rc = kl::eig_topk_factor_batch(pr, topk_options(kmax, block), st);
  if (rc) return rc;
  for (int i = 0; i < nplans; ++i) {
    rc = topk_finish(bufs[i], N, pr[i].K, nk, krn_re_host + i * rstride, c64 ? nullptr : krn_im_host + i * kstride,
                     scales_host + (size_t)i * nk, evals_host ? evals_host + (size_t)i * nk : nullptr,
                     iterations ? iterations + i : nullptr, st);
    if (rc) return rc;
  }
  return KL_OK;
}

}  // namespace

int kl_topk_eig(kl_tcc_plan p, int nk, int block, float* krn_re_host, float* krn_im_host, float* scales_host,
                double* evals_host, int* iterations) {
  KL_CHECK_ARG(p && krn_re_host && krn_im_host && scales_host, "kl_topk_eig: NULL argument");
  return topk_one(p, nk, block, krn_re_host, krn_im_host, scales_host, evals_host, iterations);
}

int kl_topk_eig_c64(kl_tcc_plan p, int nk, int block, float* krn_host, float* scales_host, double* evals_host,
                    int* iterations) {
  KL_CHECK_ARG(p && krn_host && scales_host, "kl_topk_eig_c64: NULL argument");
  return topk_one(p, nk, block, krn_host, nullptr, scales_host, evals_host, iterations);
}

int kl_topk_eig_batch(const kl_tcc_plan* plans, int nplans, int nk, int block, float* krn_re_host,
                      float* krn_im_host, float* scales_host, double* evals_host, int* iterations) {
  KL_CHECK_ARG(plans && nplans > 0 && krn_re_host && krn_im_host && scales_host,
               "kl_topk_eig_batch: NULL argument or empty batch");
  return topk_batch(plans, nplans, nk, block, krn_re_host, krn_im_host, scales_host, evals_host, iterations);
}

int kl_topk_eig_batch_c64(const kl_tcc_plan* plans, int nplans, int nk, int block, float* krn_host,
                          float* scales_host, double* evals_host, int* iterations) {
  KL_CHECK_ARG(plans && nplans > 0 && krn_host && scales_host, "kl_topk_eig_batch_c64: NULL argument or empty batch");
  return topk_batch(plans, nplans, nk, block, krn_host, nullptr, scales_host, evals_host, iterations);
}

int kl_fp64_hopkins_image(kl_tcc_plan p, const float* masks_dev, int nclips, double* images_dev, void* stream) {
  KL_CHECK_ARG(p && masks_dev && images_dev, "kl_fp64_hopkins_image: NULL argument");
  KL_CHECK_ARG(p->precision == KL_PREC_FP64, "kl_fp64_hopkins_image: needs a plan of KL_PREC_FP64 precision");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = ensure_tcc64(p, st);
  if (rc) return rc;
  return kl::f64::hopkins_image(masks_dev, nclips, p->Lx, p->Ly, p->pp.Nx, p->pp.Ny, p->tcc64, images_dev, st);
}

int kl_hopkins_image(kl_tcc_plan p, const float* masks_dev, int nclips, float* images_dev,
                     void* stream) {
  KL_CHECK_ARG(p && masks_dev && images_dev, "kl_hopkins_image: NULL argument");
  KL_CHECK_ARG(p->precision == KL_PREC_FAST, "kl_hopkins_image: plans of FP64 precision image through kl_fp64_hopkins_image");
  cudaStream_t st = (cudaStream_t)stream;
  const int N = p->pp.N, S = p->pp.S;
  if (!p->hopkins || nclips > p->hopkins_clips) {
    if (p->hopkins) kl_socs_plan_destroy(p->hopkins);
    p->hopkins = nullptr;
    int rc = kl_socs_plan_create(&p->hopkins, p->Lx, p->Ly, p->pp.Nx, p->pp.Ny, S, 1,
                                 std::max(1, nclips));
    if (rc) return rc;
    p->hopkins_clips = std::max(1, nclips);
    float2* H = nullptr;
    float* lam = nullptr;
    if ((rc = dalloc((void**)&H, sizeof(float2) * (size_t)N * S, "Abbe kernels")) ||
        (rc = dalloc((void**)&lam, sizeof(float) * S, "Abbe weights"))) {
      dfree(H);
      return rc;
    }
    rc = kl::tcc_factor_kernels(p->A, N, S, H, lam, st);
    if (!rc) rc = kl_socs_set_kernels_device(p->hopkins, 0, H, lam, st);
    cudaStreamSynchronize(st);
    dfree(H);
    dfree(lam);
    if (rc) return rc;
  }
  return kl_socs_forward(p->hopkins, masks_dev, nclips, images_dev, stream);
}

int kl_socs_vjp_source(kl_socs_plan sp, kl_tcc_plan tp, float* grad_src, void* stream) {
  KL_CHECK_ARG(sp && tp && grad_src, "kl_socs_vjp_source: NULL argument");
  KL_CHECK_ARG(sp->adjoint && sp->last_vjp_clips > 0, "kl_socs_vjp_source: run kl_socs_vjp first");
  KL_CHECK_ARG(sp->nsets == 1, "kl_socs_vjp_source: one kernel set (one optical setting) per plan");
  KL_CHECK_ARG(tp->precision == KL_PREC_FAST, "kl_socs_vjp_source: needs the fast-path TCC plan");
  KL_CHECK_ARG(tp->pp.Nx == sp->g.Nx && tp->pp.Ny == sp->g.Ny && tp->Lx == sp->g.Lx && tp->Ly == sp->g.Ly,
               "kl_socs_vjp_source: TCC plan and SOCS plan describe different bands");
  cudaStream_t st = (cudaStream_t)stream;
  const int N = tp->pp.N, S = tp->pp.S, nimg = sp->last_vjp_clips;
  float2* H = nullptr;
  float* lam = nullptr;
  int rc;
  if ((rc = dalloc((void**)&H, sizeof(float2) * (size_t)N * S, "source kernels")) ||
      (rc = dalloc((void**)&lam, sizeof(float) * S, "source weights"))) {
    dfree(H);
    return rc;
  }
  KL_CUDA_TRY(cudaMemsetAsync(grad_src, 0, sizeof(float) * (size_t)tp->srcSize * tp->srcSize, st));
  rc = kl::tcc_factor_kernels(tp->A, N, S, H, lam, st);
  int nsplit = 1;
  while (nsplit < S && nimg * nsplit < 2 * 148) nsplit *= 2;
  if (nsplit > S) nsplit = S;
  if (!rc && sp->gen)
    rc = kl::gen_launch_vjp_source(sp->gg, sp->band, sp->last_nparts, sp->gband, sp->last_gparts, nimg, sp->nsets, H,
                                   S, tp->J, tp->src_id, nsplit, grad_src, st);
  else if (!rc)
    rc = kl::vjp_launch_source(sp->g, sp->partial, sp->gpart, nimg, sp->nsets, H, tp->J, tp->src_id,
                               S, nsplit, grad_src, st);
  cudaStreamSynchronize(st);
  dfree(H);
  dfree(lam);
  return rc;
}

int kl_hopkins_image_host(kl_tcc_plan p, const float* mask_host, float* image_host) {
  KL_CHECK_ARG(p && mask_host && image_host, "kl_hopkins_image_host: NULL argument");
  const size_t bytes = sizeof(float) * (size_t)p->Lx * p->Ly;
  float *md = nullptr, *id = nullptr;
  int rc;
  if ((rc = dalloc((void**)&md, bytes, "mask")) || (rc = dalloc((void**)&id, bytes, "image"))) {
    dfree(md);
    return rc;
  }
  cudaMemcpy(md, mask_host, bytes, cudaMemcpyHostToDevice);
  rc = kl_hopkins_image(p, md, 1, id, nullptr);
  if (!rc && cudaMemcpy(image_host, id, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
    kl::set_error(std::string("kl_hopkins_image_host: ") + cudaGetErrorString(cudaGetLastError()));
    rc = KL_ERR_CUDA;
  }
  dfree(md);
  dfree(id);
  return rc;
}

int kl_fp64_hopkins_image_host(kl_tcc_plan p, const float* mask_host, float* image_host) {
  KL_CHECK_ARG(p && mask_host && image_host, "kl_fp64_hopkins_image_host: NULL argument");
  KL_CHECK_ARG(p->precision == KL_PREC_FP64, "kl_fp64_hopkins_image_host: needs a plan of KL_PREC_FP64 precision");
  const size_t n = (size_t)p->Lx * p->Ly;
  float* md = nullptr;
  double* id = nullptr;
  int rc;
  if ((rc = dalloc((void**)&md, sizeof(float) * n, "mask")) || (rc = dalloc((void**)&id, sizeof(double) * n, "image"))) {
    dfree(md);
    return rc;
  }
  std::vector<double> img(n);
  if (cudaMemcpy(md, mask_host, sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
    kl::set_error(std::string("kl_fp64_hopkins_image_host: ") + cudaGetErrorString(cudaGetLastError()));
    rc = KL_ERR_CUDA;
  }
  if (!rc) rc = kl_fp64_hopkins_image(p, md, 1, id, nullptr);
  if (!rc && cudaMemcpy(img.data(), id, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
    kl::set_error(std::string("kl_fp64_hopkins_image_host: ") + cudaGetErrorString(cudaGetLastError()));
    rc = KL_ERR_CUDA;
  }
  // the reference stores the float cast of its double image (klitho_tcc.cpp:537-544)
  if (!rc)
    for (size_t i = 0; i < n; ++i) image_host[i] = (float)img[i];
  dfree(md);
  dfree(id);
  return rc;
}

}  // extern "C"
