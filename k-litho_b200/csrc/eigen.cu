// eigen.cu -- top-K eigenpairs of the TCC by blocked subspace iteration with
// FP64 CholeskyQR2 re-orthogonalisation and FP64 Rayleigh-Ritz (replaces the
// LAPACK zheevr call of K-Litho-TCC/klitho_tcc.cpp:300-377).
//
// The operator is either the TCC's FP32 factor A (TCC = A A^H, matvecs
// A (A^H X) at cost 2 N S B) or a materialised TCC (N^2 B).  All block
// arithmetic is complex FP64 on the CUDA cores; products of the FP32 factor
// are formed exactly in FP64.  The B x B problems (Cholesky, triangular
// inverse, Hermitian eigensolve by cyclic Jacobi) run in one CTA each.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "kl_internal.h"
#include "kl_tcc.h"

namespace kl {

namespace {

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}

// ---------------------------------------------------------------------------
// Tiled complex FP64 GEMM C[m][n] (+)= sum_k a(m,k) b(k,n), with the operand
// accessors chosen by MODE.  32 x 32 output tile, k-step 16, 256 threads,
// 2 x 2 outputs per thread.  gridDim.z > 1 splits k and accumulates with
// double atomics into a zeroed C.
// ---------------------------------------------------------------------------
enum GemmMode {
  G_AHX = 0,   // a = conj(A32[k][m]) (A32: K x lda float2), b = X[k][n] (ldb)
  G_AY = 1,    // a = A32[m][k],                             b = Y[k][n]
  G_DX = 2,    // a = T64[m][k] (double2),                   b = X[k][n]
  G_FX = 3,    // a = T32[m][k] (float2),                    b = X[k][n]
  G_HH = 4,    // a = conj(W[k][m]),                         b = V[k][n]   (W^H V)
  G_NN = 5     // a = W[m][k],                               b = R[k][n]
};

template <int MODE>
__device__ __forceinline__ double2 load_a(const void* A, int lda, int m, int k) {
  if (MODE == G_AHX) {
    float2 v = reinterpret_cast<const float2*>(A)[(size_t)k * lda + m];
    return make_double2(v.x, -v.y);
  } else if (MODE == G_AY || MODE == G_FX) {
    float2 v = reinterpret_cast<const float2*>(A)[(size_t)m * lda + k];
    return make_double2(v.x, v.y);
  } else if (MODE == G_DX || MODE == G_NN) {
    return reinterpret_cast<const double2*>(A)[(size_t)m * lda + k];
  } else {  // G_HH
    double2 v = reinterpret_cast<const double2*>(A)[(size_t)k * lda + m];
    return make_double2(v.x, -v.y);
  }
}

template <int MODE>
__global__ void __launch_bounds__(256) k_zgemm(const void* __restrict__ A, int lda,
                                               const double2* __restrict__ Bm, int ldb,
                                               double2* __restrict__ C, int ldc, int M, int N,
                                               int K, int accumulate) {
  constexpr int TM = 32, TN = 32, TK = 16;
  __shared__ double2 sa[TK][TM + 1];
  __shared__ double2 sb[TK][TN + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
  const int kchunk = (K + gridDim.z - 1) / gridDim.z;
  const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
  double2 acc[2][2];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) acc[i][j] = make_double2(0.0, 0.0);
  for (int k0 = kbeg; k0 < kend; k0 += TK) {
    for (int i = threadIdx.x; i < TK * TM; i += 256) {
      const int kk = i / TM, mm = i - kk * TM;
      const int m = m0 + mm, k = k0 + kk;
      sa[kk][mm] = (m < M && k < kend) ? load_a<MODE>(A, lda, m, k) : make_double2(0.0, 0.0);
    }
    for (int i = threadIdx.x; i < TK * TN; i += 256) {
      const int kk = i / TN, nn = i - kk * TN;
      const int n = n0 + nn, k = k0 + kk;
      sb[kk][nn] = (n < N && k < kend) ? Bm[(size_t)k * ldb + n] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TK; ++kk) {
      const double2 a0 = sa[kk][ty], a1 = sa[kk][ty + 16];
      const double2 b0 = sb[kk][tx], b1 = sb[kk][tx + 16];
      acc[0][0] = zfma(a0, b0, acc[0][0]);
      acc[0][1] = zfma(a0, b1, acc[0][1]);
      acc[1][0] = zfma(a1, b0, acc[1][0]);
      acc[1][1] = zfma(a1, b1, acc[1][1]);
    }
    __syncthreads();
  }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      const int m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
      if (m < M && n < N) {
        double2* c = C + (size_t)m * ldc + n;
        if (gridDim.z > 1) {
          atomicAdd(&c->x, acc[i][j].x);
          atomicAdd(&c->y, acc[i][j].y);
        } else if (accumulate) {
          *c = zadd(*c, acc[i][j]);
        } else {
          *c = acc[i][j];
        }
      }
    }
}

template <int MODE>
int zgemm(const void* A, int lda, const double2* Bm, int ldb, double2* C, int ldc, int M, int N,
          int K, cudaStream_t st) {
  const int gx = (M + 31) / 32, gy = (N + 31) / 32;
  int gz = 1;
  const int tiles = gx * gy;
  if (tiles < 296 && K >= 512) gz = std::min(std::max(1, 296 / tiles), std::max(1, K / 256));
  if (gz > 1) KL_CUDA_TRY(cudaMemsetAsync(C, 0, sizeof(double2) * (size_t)M * ldc, st));
  k_zgemm<MODE><<<dim3(gx, gy, gz), 256, 0, st>>>(A, lda, Bm, ldb, C, ldc, M, N, K, 0);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

// deterministic start block, entries uniform in [-1, 1] + i[-1, 1]
__global__ void k_rand_block(double2* X, int N, int B, uint64_t seed) {
  const size_t n = (size_t)N * B;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double a = (double)(z >> 11) * (1.0 / 9007199254740992.0);
    uint64_t w = z * 0xD6E8FEB86659FD93ull + 0x9E3779B97F4A7C15ull;
    w ^= w >> 32;
    const double b = (double)(w >> 11) * (1.0 / 9007199254740992.0);
    X[i] = make_double2(2.0 * a - 1.0, 2.0 * b - 1.0);
  }
}

// ---------------------------------------------------------------------------
// One-CTA dense helpers on B x B matrices (B <= 128)
// ---------------------------------------------------------------------------

// Upper Cholesky G + shift*I = R^H R, then Rinv = R^{-1}.  G, Rinv row-major
// B x B.  status[0] set to 1 on a non-positive pivot.
__global__ void __launch_bounds__(256) k_chol_inv(const double2* __restrict__ G, int B,
                                                  double rel_shift, double2* __restrict__ Rinv,
                                                  int* __restrict__ status) {
  extern __shared__ double2 sm[];
  double2* R = sm;  // B x B
  __shared__ double s_shift;
  __shared__ int s_bad;
  for (int i = threadIdx.x; i < B * B; i += blockDim.x) R[i] = G[i];
  if (threadIdx.x == 0) {
    double tr = 0.0;
    for (int i = 0; i < B; ++i) tr = fmax(tr, G[(size_t)i * B + i].x);
    s_shift = rel_shift * tr;
    s_bad = 0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < B; i += blockDim.x) R[i * B + i].x += s_shift;
  __syncthreads();
  for (int j = 0; j < B; ++j) {
    const double d2 = R[j * B + j].x;
    const double d = d2 > 0.0 ? sqrt(d2) : 0.0;
    __syncthreads();
    if (threadIdx.x == 0 && !(d2 > 0.0)) s_bad = 1;
    const double inv = d > 0.0 ? 1.0 / d : 0.0;
    for (int i = j + 1 + threadIdx.x; i < B; i += blockDim.x) R[j * B + i] = make_double2(R[j * B + i].x * inv, R[j * B + i].y * inv);
    if (threadIdx.x == 0) R[j * B + j] = make_double2(d, 0.0);
    __syncthreads();
    // trailing update R[i][l] -= conj(R[j][i]) R[j][l], j < i <= l
    const int rem = B - j - 1;
    for (int t = threadIdx.x; t < rem * rem; t += blockDim.x) {
      const int i = j + 1 + t / rem, l = j + 1 + t % rem;
      if (l >= i) R[i * B + l] = zsub(R[i * B + l], zmul(zconj(R[j * B + i]), R[j * B + l]));
    }
    __syncthreads();
  }
  // zero the strict lower part
  for (int t = threadIdx.x; t < B * B; t += blockDim.x) {
    const int i = t / B, l = t % B;
    if (l < i) R[t] = make_double2(0.0, 0.0);
  }
  __syncthreads();
  // Rinv column c by back substitution: R x = e_c
  for (int c = threadIdx.x; c < B; c += blockDim.x) {
    for (int i = B - 1; i >= 0; --i) {
      double2 s = make_double2(i == c ? 1.0 : 0.0, 0.0);
      for (int l = i + 1; l <= c; ++l) s = zsub(s, zmul(R[i * B + l], Rinv[(size_t)l * B + c]));
      const double2 r = R[i * B + i];
      const double den = r.x;  // real positive diagonal
      Rinv[(size_t)i * B + c] = (i <= c && den > 0.0) ? make_double2(s.x / den, s.y / den) : make_double2(0.0, 0.0);
    }
  }
  if (threadIdx.x == 0 && s_bad) status[0] = 1;
}

// Hermitian eigensolve H = Q diag(w) Q^H by cyclic Jacobi with the
// round-robin (tournament) ordering: B/2 disjoint rotations per step.
// H row-major B x B (overwritten), Q row-major B x B (columns = vectors,
// kept in global memory), w descending on return (vectors permuted).
__global__ void __launch_bounds__(256) k_jacobi(double2* __restrict__ Hg, int B,
                                                double2* __restrict__ Q, double* __restrict__ w,
                                                int max_sweeps, int* __restrict__ sweeps_out) {
  extern __shared__ double2 sm[];
  const int Bp = B + (B & 1);
  double2* H = sm;                                        // Bp x Bp
  int* pr = reinterpret_cast<int*>(H + (size_t)Bp * Bp);  // Bp ring
  double* pc = reinterpret_cast<double*>(pr + Bp + (Bp & 1));  // per pair: c, s, phase re, im
  __shared__ double s_off, s_diag;
  __shared__ int s_done;
  for (int t = threadIdx.x; t < Bp * Bp; t += blockDim.x) {
    const int i = t / Bp, j = t % Bp;
    H[t] = (i < B && j < B) ? Hg[(size_t)i * B + j] : make_double2(0.0, 0.0);
  }
  for (int t = threadIdx.x; t < Bp * Bp; t += blockDim.x) {
    const int i = t / Bp, j = t % Bp;
    if (i < B && j < B) Q[(size_t)i * B + j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
  }
  for (int i = threadIdx.x; i < Bp; i += blockDim.x) pr[i] = i;
  __syncthreads();
  const int npairs = Bp / 2;
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    if (threadIdx.x == 0) {
      double off = 0.0, dg = 0.0;
      for (int i = 0; i < B; ++i)
        for (int j = 0; j < B; ++j) {
          const double2 h = H[i * Bp + j];
          if (i == j) dg += h.x * h.x; else off += h.x * h.x + h.y * h.y;
        }
      s_off = off;
      s_diag = dg;
      s_done = !(off > 1e-30 * dg) || dg == 0.0;
    }
    __syncthreads();
    if (s_done) break;
    for (int step = 0; step < Bp - 1; ++step) {
      // rotation parameters for pair (pr[t], pr[Bp-1-t])
      for (int t = threadIdx.x; t < npairs; t += blockDim.x) {
        int p = pr[t], q = pr[Bp - 1 - t];
        if (p > q) { const int tmp = p; p = q; q = tmp; }
        double c = 1.0, s = 0.0, er = 1.0, ei = 0.0;
        if (q < B) {
          const double2 b = H[p * Bp + q];
          const double ab = sqrt(b.x * b.x + b.y * b.y);
          const double a = H[p * Bp + p].x, d = H[q * Bp + q].x;
          if (ab > 1e-300 && ab > 1e-18 * sqrt(fabs(a * d))) {
            const double th = (d - a) / (2.0 * ab);
            const double tt = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
            c = 1.0 / sqrt(tt * tt + 1.0);
            s = tt * c;
            er = b.x / ab;
            ei = b.y / ab;  // e^{i phi} = b/|b|
          }
        }
        pc[4 * t] = c;
        pc[4 * t + 1] = s;
        pc[4 * t + 2] = er;
        pc[4 * t + 3] = ei;
      }
      __syncthreads();
      // columns: H <- H U with U = [[c, s],[-s e^{-i phi}, c e^{-i phi}]] on (p, q)
      for (int idx = threadIdx.x; idx < npairs * Bp; idx += blockDim.x) {
        const int t = idx / Bp, k = idx % Bp;
        int p = pr[t], q = pr[Bp - 1 - t];
        if (p > q) { const int tmp = p; p = q; q = tmp; }
        if (q >= B) continue;
        const double c = pc[4 * t], s = pc[4 * t + 1];
        const double2 em = make_double2(pc[4 * t + 2], -pc[4 * t + 3]);  // e^{-i phi}
        const double2 hp = H[k * Bp + p], hq = H[k * Bp + q];
        const double2 hqe = zmul(hq, em);
        H[k * Bp + p] = make_double2(c * hp.x - s * hqe.x, c * hp.y - s * hqe.y);
        H[k * Bp + q] = make_double2(s * hp.x + c * hqe.x, s * hp.y + c * hqe.y);
        if (k < B) {
          const double2 qp = Q[(size_t)k * B + p], qq = Q[(size_t)k * B + q];
          const double2 qqe = zmul(qq, em);
          Q[(size_t)k * B + p] = make_double2(c * qp.x - s * qqe.x, c * qp.y - s * qqe.y);
          Q[(size_t)k * B + q] = make_double2(s * qp.x + c * qqe.x, s * qp.y + c * qqe.y);
        }
      }
      __syncthreads();
      // rows: H <- U^H H
      for (int idx = threadIdx.x; idx < npairs * Bp; idx += blockDim.x) {
        const int t = idx / Bp, k = idx % Bp;
        int p = pr[t], q = pr[Bp - 1 - t];
        if (p > q) { const int tmp = p; p = q; q = tmp; }
        if (q >= B) continue;
        const double c = pc[4 * t], s = pc[4 * t + 1];
        const double2 ep = make_double2(pc[4 * t + 2], pc[4 * t + 3]);  // e^{+i phi}
        const double2 hp = H[p * Bp + k], hq = H[q * Bp + k];
        const double2 hqe = zmul(hq, ep);
        H[p * Bp + k] = make_double2(c * hp.x - s * hqe.x, c * hp.y - s * hqe.y);
        H[q * Bp + k] = make_double2(s * hp.x + c * hqe.x, s * hp.y + c * hqe.y);
      }
      __syncthreads();
      // advance the tournament: keep pr[0], rotate the rest
      if (threadIdx.x == 0) {
        const int last = pr[Bp - 1];
        for (int i = Bp - 1; i > 1; --i) pr[i] = pr[i - 1];
        pr[1] = last;
      }
      __syncthreads();
    }
  }
  // eigenvalues, sorted descending (selection by rank; B is small)
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    const double vi = H[i * Bp + i].x;
    int rank = 0;
    for (int j = 0; j < B; ++j) {
      const double vj = H[j * Bp + j].x;
      rank += (vj > vi) || (vj == vi && j < i);
    }
    w[rank] = vi;
    pr[i] = rank;  // reuse: destination column of vector i
  }
  __syncthreads();
  // permute the vectors through shared memory, one row of Q at a time
  double2* row = H;  // reuse
  for (int r = 0; r < B; ++r) {
    for (int i = threadIdx.x; i < B; i += blockDim.x) row[pr[i]] = Q[(size_t)r * B + i];
    __syncthreads();
    for (int i = threadIdx.x; i < B; i += blockDim.x) Q[(size_t)r * B + i] = row[i];
    __syncthreads();
  }
  if (threadIdx.x == 0 && sweeps_out) sweeps_out[0] = sweep;
}

// krn[k][j] = U[N-1-j][k] as float planes (klitho_tcc.cpp:358-362)
__global__ void k_to_kernels(const double2* __restrict__ U, int N, int ldu, int K,
                             float* __restrict__ re, float* __restrict__ im) {
  const size_t n = (size_t)N * K;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i / N), j = (int)(i % N);
    const double2 v = U[(size_t)(N - 1 - j) * ldu + k];
    re[i] = (float)v.x;
    im[i] = (float)v.y;
  }
}

struct Workspace {
  double2 *X = nullptr, *W = nullptr, *Z = nullptr, *G = nullptr, *Rinv = nullptr, *Q = nullptr;
  double* w = nullptr;
  int* status = nullptr;
  ~Workspace() {
    cudaFree(X);
    cudaFree(W);
    cudaFree(Z);
    cudaFree(G);
    cudaFree(Rinv);
    cudaFree(Q);
    cudaFree(w);
    cudaFree(status);
  }
};

size_t jacobi_smem(int B) {
  const int Bp = B + (B & 1);
  return sizeof(double2) * (size_t)Bp * Bp + sizeof(int) * (Bp + 1) + sizeof(double) * 4 * (Bp / 2 + 1) + 64;
}

// X (N x B) <- orth(X) by CholeskyQR2; the first pass shifted for safety
int cholqr2(double2* X, int N, int B, Workspace& ws, cudaStream_t st) {
  for (int pass = 0; pass < 2; ++pass) {
    int rc = zgemm<G_HH>(X, B, X, B, ws.G, B, B, B, N, st);
    if (rc) return rc;
    k_chol_inv<<<1, 256, sizeof(double2) * (size_t)B * B, st>>>(ws.G, B, pass == 0 ? 1e-14 : 0.0,
                                                                ws.Rinv, ws.status);
    KL_CUDA_TRY(cudaGetLastError());
    rc = zgemm<G_NN>(X, B, ws.Rinv, B, ws.W, B, N, B, B, st);
    if (rc) return rc;
    KL_CUDA_TRY(cudaMemcpyAsync(X, ws.W, sizeof(double2) * (size_t)N * B, cudaMemcpyDeviceToDevice, st));
  }
  return KL_OK;
}

int jacobi(double2* H, int B, Workspace& ws, cudaStream_t st) {
  const size_t sm = jacobi_smem(B);
  if (sm > 48 * 1024) KL_CUDA_TRY(cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_jacobi<<<1, 256, sm, st>>>(H, B, ws.Q, ws.w, 60, nullptr);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

// Generic driver.  apply(X, W): W = TCC X (N x B); project(X, H): H = X^H TCC X (B x B).
template <typename Apply, typename Project>
int subspace_iteration(int N, const EigenOptions& opt, int B, Apply apply, Project project,
                       double2* U, double* evals, EigenResult* res, cudaStream_t st) {
  Workspace ws;
  const int K = opt.K;
  if (cudaMalloc(&ws.X, sizeof(double2) * (size_t)N * B) || cudaMalloc(&ws.W, sizeof(double2) * (size_t)N * B) ||
      cudaMalloc(&ws.G, sizeof(double2) * (size_t)B * B) || cudaMalloc(&ws.Rinv, sizeof(double2) * (size_t)B * B) ||
      cudaMalloc(&ws.Q, sizeof(double2) * (size_t)B * B) || cudaMalloc(&ws.w, sizeof(double) * B) ||
      cudaMalloc(&ws.status, sizeof(int))) {
    cudaGetLastError();
    set_error("subspace iteration: device allocation failed");
    return KL_ERR_NOMEM;
  }
  const size_t sm_chol = sizeof(double2) * (size_t)B * B;
  if (sm_chol > 48 * 1024)
    KL_CUDA_TRY(cudaFuncSetAttribute(k_chol_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_chol));
  KL_CUDA_TRY(cudaMemsetAsync(ws.status, 0, sizeof(int), st));
  k_rand_block<<<256, 256, 0, st>>>(ws.X, N, B, opt.seed);
  KL_CUDA_TRY(cudaGetLastError());
  int rc;
  // one power step on the random block, then orthonormalise
  if ((rc = apply(ws.X, ws.W))) return rc;
  KL_CUDA_TRY(cudaMemcpyAsync(ws.X, ws.W, sizeof(double2) * (size_t)N * B, cudaMemcpyDeviceToDevice, st));
  if ((rc = cholqr2(ws.X, N, B, ws, st))) return rc;

  std::vector<double> prev(K, 0.0), cur(B, 0.0);
  int it = 0;
  double change = 1.0;
  const int check_every = 2;
  bool converged = false;
  for (it = 1; it <= opt.max_iter; ++it) {
    if (it % check_every == 0) {
      if ((rc = project(ws.X, ws.G))) return rc;
      if ((rc = jacobi(ws.G, B, ws, st))) return rc;
      KL_CUDA_TRY(cudaMemcpyAsync(cur.data(), ws.w, sizeof(double) * B, cudaMemcpyDeviceToHost, st));
      KL_CUDA_TRY(cudaStreamSynchronize(st));
      change = 0.0;
      for (int k = 0; k < K; ++k) {
        const double den = std::max(std::fabs(cur[k]), 1e-300 + std::fabs(cur[0]) * 1e-16);
        change = std::max(change, std::fabs(cur[k] - prev[k]) / den);
        prev[k] = cur[k];
      }
      if (change < opt.tol) {
        converged = true;
        break;
      }
    }
    if ((rc = apply(ws.X, ws.W))) return rc;
    KL_CUDA_TRY(cudaMemcpyAsync(ws.X, ws.W, sizeof(double2) * (size_t)N * B, cudaMemcpyDeviceToDevice, st));
    if ((rc = cholqr2(ws.X, N, B, ws, st))) return rc;
  }
  // final Rayleigh-Ritz on the current block (G holds the eigvecs in Q)
  if (!converged) {
    if ((rc = project(ws.X, ws.G))) return rc;
    if ((rc = jacobi(ws.G, B, ws, st))) return rc;
  }
  // U = X Q[:, :K] (N x K, row-major), eigenvalues
  if ((rc = zgemm<G_NN>(ws.X, B, ws.Q, B, ws.W, B, N, B, B, st))) return rc;
  KL_CUDA_TRY(cudaMemcpy2DAsync(U, sizeof(double2) * K, ws.W, sizeof(double2) * B, sizeof(double2) * K, N,
                                cudaMemcpyDeviceToDevice, st));
  KL_CUDA_TRY(cudaMemcpyAsync(evals, ws.w, sizeof(double) * K, cudaMemcpyDeviceToDevice, st));
  int status = 0;
  KL_CUDA_TRY(cudaMemcpyAsync(&status, ws.status, sizeof(int), cudaMemcpyDeviceToHost, st));
  KL_CUDA_TRY(cudaStreamSynchronize(st));
  if (res) {
    res->iterations = std::min(it, opt.max_iter);
    res->residual = change;
  }
  if (!converged && change >= opt.tol) {
    set_error("subspace iteration did not converge: relative Ritz change " + std::to_string(change) +
              " after " + std::to_string(opt.max_iter) + " iterations");
    return KL_ERR_NOT_CONVERGED;
  }
  (void)status;
  return KL_OK;
}

int block_size(const EigenOptions& opt, int N, int rank_bound) {
  int B = std::max(opt.B, opt.K);
  B = std::min(B, N);
  B = std::min(B, std::max(rank_bound, opt.K));
  B = std::min(B, 128);
  return B;
}

}  // namespace

int eig_topk_factor(const float2* A, int N, int S, const EigenOptions& opt, double2* U,
                    double* evals, EigenResult* res, cudaStream_t st) {
  KL_CHECK_ARG(opt.K > 0 && opt.K <= N, "eig_topk_factor: K out of range");
  const int B = block_size(opt, N, S);
  KL_CHECK_ARG(opt.K <= B, "eig_topk_factor: K exceeds the block size");
  double2* Z = nullptr;
  if (cudaMalloc(&Z, sizeof(double2) * (size_t)S * B)) {
    cudaGetLastError();
    set_error("eig_topk_factor: device allocation failed");
    return KL_ERR_NOMEM;
  }
  auto apply = [&](double2* X, double2* W) -> int {
    int rc = zgemm<G_AHX>(A, S, X, B, Z, B, S, B, N, st);  // Z = A^H X
    if (rc) return rc;
    return zgemm<G_AY>(A, S, Z, B, W, B, N, B, S, st);      // W = A Z
  };
  auto project = [&](double2* X, double2* H) -> int {
    int rc = zgemm<G_AHX>(A, S, X, B, Z, B, S, B, N, st);  // Z = A^H X
    if (rc) return rc;
    return zgemm<G_HH>(Z, B, Z, B, H, B, B, B, S, st);      // H = Z^H Z
  };
  int rc = subspace_iteration(N, opt, B, apply, project, U, evals, res, st);
  cudaFree(Z);
  return rc;
}

int eig_topk_dense(const double2* tcc, int N, const EigenOptions& opt, double2* U, double* evals,
                   EigenResult* res, cudaStream_t st) {
  KL_CHECK_ARG(opt.K > 0 && opt.K <= N, "eig_topk_dense: K out of range");
  const int B = block_size(opt, N, N);
  double2* Wt = nullptr;
  if (cudaMalloc(&Wt, sizeof(double2) * (size_t)N * B)) {
    cudaGetLastError();
    set_error("eig_topk_dense: device allocation failed");
    return KL_ERR_NOMEM;
  }
  auto apply = [&](double2* X, double2* W) -> int {
    return zgemm<G_DX>(tcc, N, X, B, W, B, N, B, N, st);
  };
  auto project = [&](double2* X, double2* H) -> int {
    int rc = zgemm<G_DX>(tcc, N, X, B, Wt, B, N, B, N, st);
    if (rc) return rc;
    return zgemm<G_HH>(X, B, Wt, B, H, B, B, B, N, st);
  };
  int rc = subspace_iteration(N, opt, B, apply, project, U, evals, res, st);
  cudaFree(Wt);
  return rc;
}

int eig_topk_dense_c64(const float2* tcc, int N, const EigenOptions& opt, double2* U,
                       double* evals, EigenResult* res, cudaStream_t st) {
  KL_CHECK_ARG(opt.K > 0 && opt.K <= N, "eig_topk_dense_c64: K out of range");
  const int B = block_size(opt, N, N);
  double2* Wt = nullptr;
  if (cudaMalloc(&Wt, sizeof(double2) * (size_t)N * B)) {
    cudaGetLastError();
    set_error("eig_topk_dense_c64: device allocation failed");
    return KL_ERR_NOMEM;
  }
  auto apply = [&](double2* X, double2* W) -> int {
    return zgemm<G_FX>(tcc, N, X, B, W, B, N, B, N, st);
  };
  auto project = [&](double2* X, double2* H) -> int {
    int rc = zgemm<G_FX>(tcc, N, X, B, Wt, B, N, B, N, st);
    if (rc) return rc;
    return zgemm<G_HH>(X, B, Wt, B, H, B, B, B, N, st);
  };
  int rc = subspace_iteration(N, opt, B, apply, project, U, evals, res, st);
  cudaFree(Wt);
  return rc;
}

int eig_to_kernels(const double2* U, int N, int K, float* re, float* im, cudaStream_t st) {
  k_to_kernels<<<256, 256, 0, st>>>(U, N, K, K, re, im);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

}  // namespace kl
