// kl_tcc.h -- internal interfaces of the TCC assembly and eigen-decomposition
// (K-Litho-TCC/klitho_tcc.cpp:186-267 calcTCC, :300-377 calcKernels).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace kl {

// One active source pixel, in the reference's raster order
// (klitho_tcc.cpp:202-205), with its shifted-pupil loop bounds (:206-211).
struct SrcPoint {
  float sx, sy, J;
  int nxmin, nxmax, nymin, nymax;
  int src_id;
};

// Scalars of the pupil evaluation, computed on the host with the reference's
// float arithmetic (klitho_tcc.cpp:189-197).
struct PupilParams {
  int Nx, Ny, N, S;
  float Lx_norm, Ly_norm;  // L*NA/lambda
  float dzk;               // (defocus / (NA^2/lambda)) * (2 pi / lambda), float product
  float NA;
  double n_medium2;        // n_medium^2 (1 reproduces the reference)
};

// Host: enumerate the TCC's source points; fills pp (except N/S sizes derived).
void tcc_source_points(const float* src, int srcSize, float outerSigma, float lambda, float NA,
                       float defocus, double n_medium, int Lx, int Ly, int Nx, int Ny,
                       std::vector<SrcPoint>& pts, PupilParams& pp);

// Host: pupil table P[f][s] (N x S complex128) with the host libm's cosf/sinf,
// bit-identical to the reference's table (used by the FP64 path).
void tcc_pupil_host(const std::vector<SrcPoint>& pts, const PupilParams& pp, double* P);

// Device: A[f][s] = sqrt(J_s) P(f, s) in FP32 (N x S complex64, row-major).
int tcc_build_A(const SrcPoint* pts_dev, const PupilParams& pp, float2* A, cudaStream_t st);

// Device: bf16 split operands for TCC = A A^H on the tensor cores: four
// planes X1h, X2h, X1l, X2l of N x K2p bf16 in one buffer (4 N K2p elements),
// K2p = round_up(2 S, 32) = tcc_kp(S).
int tcc_split_operands(const float2* A, int N, int S, int K2p, void* ops, cudaStream_t st);
int tcc_kp(int S);

// Device: Hermitian TCC (N x N complex64) = X1 Y^T + i X2 Y^T (Y = X1, three
// split terms) by tcgen05 MMA, upper tiles computed, lower tiles mirrored.
// err_dev receives a nonzero code if a pipeline wait gave up.
int tcc_gemm_tc(const void* ops, int N, int K2p, float2* tcc, int* err_dev, cudaStream_t st);

// Device: FP64 TCC by direct accumulation over source points (the plain FP64
// path): tcc[i][j] = sum_s J_s P[i][s] conj(P[j][s]).  P is N x S complex128.
int tcc_direct_fp64(const double2* P, const float* J, int N, int S, double2* tcc, cudaStream_t st);

// Device: SOCS-layout kernels of the Abbe (source-point) form of the Hopkins
// image: H_s[f] = conj A[f][s] (S x N complex64), lam = 1.
int tcc_factor_kernels(const float2* A, int N, int S, float2* H, float* lam, cudaStream_t st);

// Device: min/max of the real and imaginary parts of a complex64/128 matrix
// (klitho_tcc.cpp:521-528 prints the maxima).  out4 = {max re, min re, max im, min im}.
int tcc_minmax_c64(const float2* m, size_t n, double* out4_host, cudaStream_t st);
int tcc_minmax_c128(const double2* m, size_t n, double* out4_host, cudaStream_t st);

// ---------------------------------------------------------------------------
// Eigen-decomposition by blocked subspace iteration (FP64 Rayleigh-Ritz)
// ---------------------------------------------------------------------------
struct EigenOptions {
  int K;          // kernels wanted
  int B;          // block size (>= K)
  int max_iter;   // iteration cap (KL_ERR_NOT_CONVERGED beyond it)
  double tol;     // relative change of the top-K Ritz values between checks
  uint64_t seed;  // start block
};

struct EigenResult {
  int iterations;   // subspace iterations; Jacobi sweeps of a one-step Gram solve (1 when it
                    // ran the tridiagonal solver)
  double residual;  // max relative Ritz-value change at the last check
};

// One top-K problem on a TCC factor A (N x S), for the batched solver.
struct FactorProblem {
  const float2* A;
  int N, S, K;
  double2* U;      // N x K eigenvectors (row-major)
  double* evals;   // K eigenvalues, descending
  EigenResult* res;
};

// Top-K eigenpairs of several TCC = A A^H at once (e.g. one per focus value):
// factors with S <= 256 columns share one batched Gram eigensolve; the rest
// are solved one after another by subspace iteration.
int eig_topk_factor_batch(const std::vector<FactorProblem>& problems, const EigenOptions& opt,
                          cudaStream_t st);

// Operator TCC = A A^H given by its FP32 factor A (N x S).
int eig_topk_factor(const float2* A, int N, int S, const EigenOptions& opt, double2* U,
                    double* evals, EigenResult* res, cudaStream_t st);
// Operator given by a materialised FP64 TCC (N x N).
int eig_topk_dense(const double2* tcc, int N, const EigenOptions& opt, double2* U, double* evals,
                   EigenResult* res, cudaStream_t st);
// Operator given by a materialised FP32 TCC (N x N).
int eig_topk_dense_c64(const float2* tcc, int N, const EigenOptions& opt, double2* U,
                       double* evals, EigenResult* res, cudaStream_t st);

// G = A^H A (S x S complex128, row-major) of an FP32 factor A (N x S complex64),
// exact to the factor's precision, by an integer-digit split on the tcgen05
// tensor cores (gram_i8.cu).  err_dev (zeroed by the caller) receives a
// nonzero code if a pipeline wait gave up.
constexpr int kGramI8MaxS = 256;
bool gram_i8_supported(int N, int S);
int gram_i8(const float2* A, int N, int S, double2* G, int* err_dev, cudaStream_t st);
// G = A^H A by gram_i8 where it applies, else by the FP64 CUDA-core GEMM
int gram_factor(const float2* A, int N, int S, double2* G, int* err_dev, cudaStream_t st);

// Top-K eigenpairs of a Hermitian B x B matrix, kTridiagMinB <= B <= kTridiagMaxB, by
// Householder tridiagonalisation on a thread-block cluster, bisection and inverse
// iteration (eig_tridiag.cu).  The work buffers belong to the caller.
constexpr int kTridiagMinB = 64;
constexpr int kTridiagMaxB = 256;
struct TridiagJob {
  const double2* H;  // B x B Hermitian, row-major (read only)
  double2* refl;     // B x B work: Householder vector k in row k, columns k+1 .. B-1
  double* d;         // B work: diagonal of the tridiagonal T
  double2* e;        // B work: e[k] = T[k+1][k]
  double* w;         // K eigenvalues, descending
  double* lw;        // B x K work: multipliers of the inverse-iteration solves
  double* Y;         // B x K work: eigenvectors of the real tridiagonal
  double2* Q;        // B x ldq, row-major: column j < K = eigenvector j
  double2* wy;       // tridiag_wy_blocks(B) x 8 x 8 work: compact WY factors of the reflector blocks
  int* err;          // optional: set nonzero if an exchange wait of the reduction gave up
  int B, K, ldq;
};
// reflector blocks of the back-transform of an order-B reduction
inline int tridiag_wy_blocks(int B) { return (B - 2 + 7) / 8; }
// true when the device can run the cluster reduction for order B
bool tridiag_eig_supported(int B);
int tridiag_eig_batch(const std::vector<TridiagJob>& jobs, cudaStream_t st);

// Kernels in the reference layout: krn[k][j] = U[n-1-j][k] (klitho_tcc.cpp:358-362),
// as separate float32 planes, or interleaved complex64 in re (2 N K floats) when im is null.
int eig_to_kernels(const double2* U, int N, int K, float* re, float* im, cudaStream_t st);

}  // namespace kl
