// eigen.cu -- top-K eigenpairs of the TCC by blocked subspace iteration with
// FP64 CholeskyQR2 re-orthogonalisation and FP64 Rayleigh-Ritz (replaces the
// LAPACK zheevr call of K-Litho-TCC/klitho_tcc.cpp:300-377).
//
// The operator is either the TCC's FP32 factor A (TCC = A A^H, matvecs
// A (A^H X) at cost 2 N S B) or a materialised TCC (N^2 B).  All block
// arithmetic is complex FP64 on the CUDA cores; products of the FP32 factor
// are formed exactly in FP64.  The B x B problems (Cholesky, triangular
// inverse, Hermitian eigensolve by cyclic Jacobi) run in one CTA each, except
// Jacobi eigensolves of order 64..256, which run on a thread-block cluster of
// eight CTAs holding the matrix in their shared memory (k_jacobi_cluster).
#include <cooperative_groups.h>
#include <cuda_pipeline.h>

#include <mutex>

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
  G_NN = 5,    // a = W[m][k],                               b = R[k][n]
  G_AHA = 6    // a = conj(A32[k][m]),                       b = A32[k][n] (FP64 Gram of A)
};

template <int MODE>
__device__ __forceinline__ double2 load_b(const void* B, int ldb, int k, int n) {
  if (MODE == G_AHA) {
    const float2 v = reinterpret_cast<const float2*>(B)[(size_t)k * ldb + n];
    return make_double2(v.x, v.y);
  }
  return reinterpret_cast<const double2*>(B)[(size_t)k * ldb + n];
}

template <int MODE>
__device__ __forceinline__ double2 load_a(const void* A, int lda, int m, int k) {
  if (MODE == G_AHX || MODE == G_AHA) {
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
                                               const void* __restrict__ Bm, int ldb,
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
      sb[kk][nn] = (n < N && k < kend) ? load_b<MODE>(Bm, ldb, k, n) : make_double2(0.0, 0.0);
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
int zgemm(const void* A, int lda, const void* Bm, int ldb, double2* C, int ldc, int M, int N,
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
// round-robin (circle) ordering: Bp/2 disjoint rotations per step, pairs in
// closed form.  One CTA per matrix keeps H in shared memory (or works on it in
// place in global memory when it is too large) and applies each step as
// independent two-sided 2 x 2 block updates U_a^H H[a, b] U_b over all pairs
// of pairs, writing the rotations to a log.  The eigenvectors Q = prod U are
// formed afterwards from the log by k_jacobi_vectors, one warp per row of Q,
// so the sequential sweep loop touches only H.  A launch takes a batch of
// independent matrices (one CTA each), e.g. the TCCs of several focus values.
constexpr int kJacobiThreads = 1024;
constexpr int kJacobiMaxSweeps = 40;
constexpr int kJacobiMaxJobs = 16;
constexpr int kGramMaxS = 256;  // factor widths solved by one Gram eigensolve (pair tables hold bytes)

struct JacobiJob {
  double2* H;    // B x B Hermitian input (overwritten when worked in place)
  double4* rot;  // rotation log (cluster solver: block log), jacobi_log_elems(B)
  double2* Q;    // B x B output, column j = eigenvector j
  double* w;     // B eigenvalues, descending
  int* jst;      // [0] steps applied, [1 + i] rank of diagonal entry i
  int B;
};
struct JacobiJobs {
  JacobiJob j[kJacobiMaxJobs];
};

__host__ __device__ inline void jacobi_pair(int t, int i, int Bp, int& p, int& q) {
  const int m = Bp - 1;
  if (i == 0) {
    p = 0;
    q = 1 + t % m;
  } else {
    p = 1 + (t + i) % m;
    q = 1 + (t - i + m) % m;
  }
  if (p > q) {
    const int x = p;
    p = q;
    q = x;
  }
}

// the (p, q) of pair t at step i of a sweep, for all steps (bytes: B <= 128)
__device__ void jacobi_pair_table(uchar2* tab, int Bp) {
  const int npairs = Bp / 2;
  for (int i = threadIdx.x; i < (Bp - 1) * npairs; i += blockDim.x) {
    const int step = i / npairs, t = i - step * npairs;
    int p, q;
    jacobi_pair(step, t, Bp, p, q);
    tab[i] = make_uchar2((unsigned char)p, (unsigned char)q);
  }
}

struct JacobiSmem {
  int npairs, nblocks;
  size_t pc, pt, bt, h, total_no_h;
  __host__ __device__ explicit JacobiSmem(int B) {
    const int Bp = B + (B & 1);
    npairs = Bp / 2;
    nblocks = npairs * (npairs + 1) / 2;
    pc = 0;                                                   // npairs double4
    pt = pc + sizeof(double4) * npairs;                       // (Bp - 1) x npairs uchar2
    bt = pt + sizeof(uchar2) * (Bp - 1) * npairs;             // nblocks ushort
    h = (bt + sizeof(unsigned short) * nblocks + 15) & ~size_t(15);
    total_no_h = h;
  }
};

// rotation zeroing b = H[p][q] given a = H[p][p], d = H[q][q]:
// (c, s, Re e, Im e) with e = b / |b|, t = s / c = sgn(th) / (|th| + sqrt(th^2 + 1)),
// th = (d - a) / (2 |b|); *tb = t |b| moves the diagonal (a - t|b|, d + t|b|)
__device__ __forceinline__ double4 jacobi_rotation(double a, double d, double2 b, double* tb) {
  const double b2 = b.x * b.x + b.y * b.y;
  if (b2 > 1e-300 && b2 > 1e-36 * fabs(a * d)) {
    const double r = rsqrt(b2);
    const double th = 0.5 * (d - a) * r;
    const double tt = copysign(1.0, th) / (fabs(th) + sqrt(fma(th, th, 1.0)));
    const double c = rsqrt(fma(tt, tt, 1.0));
    *tb = tt * (b2 * r);
    return make_double4(c, tt * c, b.x * r, b.y * r);
  }
  *tb = 0.0;
  return make_double4(1.0, 0.0, 1.0, 0.0);
}

// rows (p1, q1) rotated by u1 from the left (U1^H .), columns (p2, q2) by u2
__device__ __forceinline__ void rot_block(double2& x00, double2& x01, double2& x10, double2& x11, double4 u1,
                                          double4 u2) {
  // right: Y[:,0] = c2 X[:,0] - s2 conj(e2) X[:,1];  Y[:,1] = s2 X[:,0] + c2 conj(e2) X[:,1]
  const double2 e2c = make_double2(u2.z, -u2.w);
  const double2 a1 = zmul(x01, e2c), b1 = zmul(x11, e2c);
  const double2 y00 = make_double2(u2.x * x00.x - u2.y * a1.x, u2.x * x00.y - u2.y * a1.y);
  const double2 y01 = make_double2(u2.y * x00.x + u2.x * a1.x, u2.y * x00.y + u2.x * a1.y);
  const double2 y10 = make_double2(u2.x * x10.x - u2.y * b1.x, u2.x * x10.y - u2.y * b1.y);
  const double2 y11 = make_double2(u2.y * x10.x + u2.x * b1.x, u2.y * x10.y + u2.x * b1.y);
  // left: Z[0,:] = c1 Y[0,:] - s1 e1 Y[1,:];  Z[1,:] = s1 Y[0,:] + c1 e1 Y[1,:]
  const double2 e1 = make_double2(u1.z, u1.w);
  const double2 g0 = zmul(y10, e1), g1 = zmul(y11, e1);
  x00 = make_double2(u1.x * y00.x - u1.y * g0.x, u1.x * y00.y - u1.y * g0.y);
  x01 = make_double2(u1.x * y01.x - u1.y * g1.x, u1.x * y01.y - u1.y * g1.y);
  x10 = make_double2(u1.y * y00.x + u1.x * g0.x, u1.y * y00.y + u1.x * g0.y);
  x11 = make_double2(u1.y * y01.x + u1.x * g1.x, u1.y * y01.y + u1.x * g1.y);
}

// one 2 x 2 block (pair t1 rows, pair t2 columns, t1 <= t2) of a step; the
// rotated entries are left in x.. for the caller
__device__ __forceinline__ void jacobi_block(double2* H, int B, uchar2 pr, uchar2 pcl, bool diag, double4 u1,
                                             double4 u2, double2& x00, double2& x01, double2& x10,
                                             double2& x11) {
  const int rx = pr.x, ry = pr.y, cx = pcl.x, cy = pcl.y;
  const bool rq = ry < B, cq = cy < B;
  const double2 z = make_double2(0.0, 0.0);
  x00 = H[rx * B + cx];
  x01 = cq ? H[rx * B + cy] : z;
  x10 = rq ? H[ry * B + cx] : z;
  x11 = (rq && cq) ? H[ry * B + cy] : z;
  rot_block(x00, x01, x10, x11, u1, u2);
  if (diag) {
    H[rx * B + rx] = make_double2(x00.x, 0.0);
    if (rq) {
      H[rx * B + ry] = z;
      H[ry * B + rx] = z;
      H[ry * B + ry] = make_double2(x11.x, 0.0);
    }
  } else {
    H[rx * B + cx] = x00;
    H[cx * B + rx] = zconj(x00);
    if (cq) {
      H[rx * B + cy] = x01;
      H[cy * B + rx] = zconj(x01);
    }
    if (rq) {
      H[ry * B + cx] = x10;
      H[cx * B + ry] = zconj(x10);
    }
    if (rq && cq) {
      H[ry * B + cy] = x11;
      H[cy * B + ry] = zconj(x11);
    }
  }
}

__global__ void __launch_bounds__(kJacobiThreads) k_jacobi(JacobiJobs jobs, int h_in_smem, int max_sweeps) {
  extern __shared__ __align__(16) unsigned char jsm[];
  const JacobiJob job = jobs.j[blockIdx.x];
  const int B = job.B;
  double4* __restrict__ rot = job.rot;
  const JacobiSmem L(B);
  const int Bp = B + (B & 1), npairs = L.npairs, nblocks = L.nblocks;
  double4* pc = reinterpret_cast<double4*>(jsm + L.pc);
  const uchar2* ptab = reinterpret_cast<const uchar2*>(jsm + L.pt);
  unsigned short* bt = reinterpret_cast<unsigned short*>(jsm + L.bt);
  double2* H = h_in_smem ? reinterpret_cast<double2*>(jsm + L.h) : job.H;
  __shared__ double s_red[2][kJacobiThreads / 32];
  __shared__ int s_done;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (h_in_smem)
    for (int t = threadIdx.x; t < B * B; t += blockDim.x) H[t] = job.H[t];
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    // b -> (t1 <= t2) over the upper triangle of the npairs x npairs block grid
    int t1 = 0, rem = b;
    while (rem >= npairs - t1) {
      rem -= npairs - t1;
      ++t1;
    }
    bt[b] = (unsigned short)(t1 | ((t1 + rem) << 8));
  }
  jacobi_pair_table(reinterpret_cast<uchar2*>(jsm + L.pt), Bp);
  __syncthreads();
  int sweep = 0, nsteps = 0;
  for (; sweep < max_sweeps; ++sweep) {
    double off = 0.0, dg = 0.0;
    for (int t = threadIdx.x; t < B * B; t += blockDim.x) {
      const double2 h = H[t];
      if ((t / B) == (t % B)) dg += h.x * h.x; else off += h.x * h.x + h.y * h.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
      off += __shfl_xor_sync(0xffffffffu, off, o);
      dg += __shfl_xor_sync(0xffffffffu, dg, o);
    }
    if (lane == 0) {
      s_red[0][warp] = off;
      s_red[1][warp] = dg;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0.0, b = 0.0;
      for (int k = 0; k < nw; ++k) {
        a += s_red[0][k];
        b += s_red[1][k];
      }
      s_done = !(a > 1e-28 * b) || b == 0.0;
    }
    __syncthreads();
    if (s_done) break;
    for (int step = 0; step < Bp - 1; ++step, ++nsteps) {
      const uchar2* pairs = ptab + step * npairs;
      for (int t = threadIdx.x; t < npairs; t += blockDim.x) {
        const int p = pairs[t].x, q = pairs[t].y;
        double4 u = make_double4(1.0, 0.0, 1.0, 0.0);
        if (q < B) {
          double tb;
          u = jacobi_rotation(H[p * B + p].x, H[q * B + q].x, H[p * B + q], &tb);
        }
        pc[t] = u;
        rot[(size_t)nsteps * npairs + t] = u;
      }
      __syncthreads();
      for (int bi = threadIdx.x; bi < nblocks; bi += blockDim.x) {
        const int t1 = bt[bi] & 0xff, t2 = bt[bi] >> 8;
        double2 x00, x01, x10, x11;
        jacobi_block(H, B, pairs[t1], pairs[t2], t1 == t2, pc[t1], pc[t2], x00, x01, x10, x11);
      }
      __syncthreads();
    }
  }
  // eigenvalues sorted descending (rank by comparison; B is small)
  for (int i = threadIdx.x; i < B; i += blockDim.x) {
    const double vi = H[i * B + i].x;
    int r = 0;
    for (int j = 0; j < B; ++j) {
      const double vj = H[j * B + j].x;
      r += (vj > vi) || (vj == vi && j < i);
    }
    job.w[r] = vi;
    job.jst[1 + i] = r;
  }
  if (threadIdx.x == 0) job.jst[0] = nsteps;
}

// ---------------------------------------------------------------------------
// Cluster Jacobi for matrices too large for one CTA's shared memory
// (116 < B <= 256).  The padded order Bp (a multiple of 2 kCl) is cut into
// 2 kCl groups of g = Bp / (2 kCl) consecutive indices; a round gives each of
// the kCl CTAs of a thread-block cluster one pair of groups (a perfect
// matching of the groups by the circle method), and the CTA keeps those 2g
// rows of H (all B columns) in its shared memory.  Within a round every
// rotation pairs two rows of one CTA: round 0 runs a circle-method sweep over
// the CTA's 2g indices (its pairs inside and across its two groups), the
// other rounds pair index j of the lower group with index (j + k) mod g of the
// upper one at step k.  The 2 kCl - 1 rounds visit every pair once in Bp - 1
// steps, the minimum.  A step: each CTA computes its g rotations from its own
// rows and stores them into every CTA's shared memory, one cluster barrier,
// then each CTA applies all rotations to its own rows (two-sided 2 x 2
// updates; row p and q of a pair are local, the columns are all there).
// Between rounds each CTA keeps one of its groups and pulls the other new one
// from the CTA that held it (walking the alternating cycles of the two
// matchings makes such an assignment exist for any two matchings).
// The rotations of a round only mix the 2g indices of each CTA, so their
// product is block diagonal: each CTA accumulates its 2g x 2g block W (the
// rotations applied to W's columns) and logs it at the end of the round;
// k_jacobi_vectors_blocks forms the eigenvectors from these blocks.
// ---------------------------------------------------------------------------
constexpr int kCl = 8;            // CTAs per matrix (portable cluster size)
constexpr int kClUpdThreads = 480;                // warps that update H
constexpr int kClThreads = kClUpdThreads + 32;     // + one warp for the rotations
constexpr int kClRotBufs = 3;                      // rotation slots: steps s, s + 1 and s + 2 in flight
constexpr unsigned long long kClWaitNs = 2000000000ull;  // bound on one rotation wait
constexpr int kClMaxG = kGramMaxS / (2 * kCl);  // largest group

__host__ __device__ inline int jacobi_cluster_bp(int B) { return (B + 2 * kCl - 1) / (2 * kCl) * (2 * kCl); }

struct ClusterSmem {
  int g, npairs;
  size_t rows, rot, pq, w, r0, part, diag, total;
  __host__ __device__ explicit ClusterSmem(int B) {
    const int Bp = jacobi_cluster_bp(B);
    g = Bp / (2 * kCl);
    npairs = Bp / 2;
    rows = 0;                                                      // 3 slots x g rows x B
    rot = sizeof(double2) * 3 * (size_t)g * B;                     // kClRotBufs x npairs double4
    pq = rot + sizeof(double4) * kClRotBufs * npairs;              // kClRotBufs x npairs (p | q << 16)
    w = (pq + sizeof(uint32_t) * kClRotBufs * npairs + 15) & ~size_t(15);  // 2g x 2g double2
    r0 = w + sizeof(double2) * 4 * (size_t)g * g;                  // (2g - 1) x g uchar2
    part = (r0 + sizeof(uchar2) * (2 * g - 1) * g + 15) & ~size_t(15);  // kCl x 2 double
    diag = part + sizeof(double) * 2 * kCl;                        // Bp double (rank 0)
    total = diag + sizeof(double) * Bp;
  }
};

// Round transitions of the cluster, the same for every matrix size: entry
// [t * kCl + c] describes CTA c after the t-th round of the run (bits: lower
// group 0-3, upper group 4-7, matching edge 8-10, slot of the lower group
// 11-12, of the upper 13-14, CTA to pull the new group from 15-17, its slot
// there 18-19, slot it lands in 20-21, pull needed 22); filled by the host.
__constant__ uint32_t c_cluster_sched[kJacobiMaxSweeps * (2 * kCl - 1) * kCl];

// double2 elements of the block log: one 2g x 2g block per CTA and round
__host__ __device__ inline size_t cluster_log_elems(int B, int max_sweeps) {
  const int g2 = jacobi_cluster_bp(B) / kCl;
  return (size_t)max_sweeps * (2 * kCl - 1) * kCl * g2 * g2;
}

// local position l < 2g of the CTA holding groups ga < gb -> logical index
__device__ __forceinline__ int cluster_index(int l, int ga, int gb, int g) {
  return l < g ? ga * g + l : gb * g + l - g;
}

// local positions of pair j at step k of a round
__device__ __forceinline__ void cluster_local_pair(const uchar2* r0, int round, int k, int j, int g, int& lp, int& lq) {
  if (round == 0) {
    const uchar2 v = r0[k * g + j];
    lp = v.x;
    lq = v.y;
  } else {
    lp = j;
    lq = j + k < g ? g + j + k : j + k;  // g + (j + k) mod g
  }
}

// row[p], row[q] <- the pair's columns of row . U (U as in rot_block's right factor)
__device__ __forceinline__ void rot_cols(double2& vp, double2& vq, double4 u) {
  const double2 e = zmul(vq, make_double2(u.z, -u.w)), a = vp;
  vp = make_double2(u.x * a.x - u.y * e.x, u.x * a.y - u.y * e.y);
  vq = make_double2(u.y * a.x + u.x * e.x, u.y * a.y + u.x * e.y);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// address of `p`'s counterpart in the shared memory of CTA `cta` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(const void* p, uint32_t cta) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(cta));
  return r;
}
// bytes one step's rotations deliver to every CTA: npairs x (double4 + packed pair)
__host__ __device__ inline uint32_t cluster_step_bytes(int npairs) {
  return (uint32_t)npairs * (uint32_t)(sizeof(double4) + sizeof(uint32_t));
}
// rotation t (and its pair p | q << 16) into slot (rbuf, pbuf) of CTA `cta`;
// each store completes its bytes on that CTA's barrier `bar`
__device__ __forceinline__ void push_rotation(double4* rbuf, uint32_t* pbuf, uint64_t* bar, int t, double4 u,
                                              uint32_t pq, uint32_t cta) {
  const uint32_t rr = cluster_addr(&rbuf[t], cta), rp = cluster_addr(&pbuf[t], cta), rbar = cluster_addr(bar, cta);
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(rr),
               "d"(u.x), "d"(u.y), "r"(rbar)
               : "memory");
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(rr + 16),
               "d"(u.z), "d"(u.w), "r"(rbar)
               : "memory");
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(rp), "r"(pq),
               "r"(rbar)
               : "memory");
}
// this CTA expects `bytes` on its barrier in the barrier's current phase
__device__ __forceinline__ void mbar_arm(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_cluster(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for a barrier phase; false if it did not complete in kClWaitNs
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar, uint32_t parity) {
  if (mbar_try_cluster(bar, parity)) return true;
  unsigned long long t0, t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  while (!mbar_try_cluster(bar, parity)) {
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > kClWaitNs) return false;
  }
  return true;
}

__global__ void __cluster_dims__(kCl, 1, 1) __launch_bounds__(kClThreads, 1)
    k_jacobi_cluster(JacobiJobs jobs, int max_sweeps) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char csm[];
  const int me = (int)cl.block_rank();
  const JacobiJob job = jobs.j[blockIdx.x / kCl];
  const int B = job.B;
  const ClusterSmem L(B);
  const int g = L.g, g2 = 2 * g, npairs = L.npairs, ngroups = 2 * kCl;
  const int slot_elems = g * B;
  double2* slots = reinterpret_cast<double2*>(csm + L.rows);
  double4* rotx = reinterpret_cast<double4*>(csm + L.rot);
  uint32_t* pqx = reinterpret_cast<uint32_t*>(csm + L.pq);
  double2* W = reinterpret_cast<double2*>(csm + L.w);
  uchar2* r0 = reinterpret_cast<uchar2*>(csm + L.r0);
  double* part = reinterpret_cast<double*>(csm + L.part);
  double* diag = reinterpret_cast<double*>(csm + L.diag);
  double2* wlog = reinterpret_cast<double2*>(job.rot);
  __shared__ int s_rowoff[2 * kClMaxG];  // element offset of local position l's row, -1: padding
  __shared__ int4 s_own[2][kClMaxG];     // own pair j of the step: row offsets of p, q (-1: padding), lp, lq
  __shared__ double s_newdiag[2 * kClMaxG];  // diagonal at local position l after the last rotations
  __shared__ int s_pairof[2 * kClMaxG];      // own pair holding local position l (+256: second index)
  __shared__ double s_red[2][kClThreads / 32];
  // rotation slot b: its phase completes when the step's rotations from every
  // CTA have landed (st.async completes their bytes; this CTA arms each use)
  __shared__ __align__(8) uint64_t s_bar[kClRotBufs];
  __shared__ int s_fail, s_anyfail;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nthr = blockDim.x;
  const double2 zero = make_double2(0.0, 0.0), one = make_double2(1.0, 0.0);
  if (tid == 0) {
    for (int b = 0; b < kClRotBufs; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&s_bar[b])), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int b = 0; b < kClRotBufs; ++b) mbar_arm(&s_bar[b], cluster_step_bytes(npairs));
    s_fail = 0;
    s_anyfail = 0;
  }
  // this CTA's groups (ga < gb), their slots and its matching edge; round 0 starts with edge me
  int ga, gb, sa = 0, sb = 1, e = me;
  jacobi_pair(0, me, ngroups, ga, gb);

  for (int i = tid; i < (g2 - 1) * g; i += nthr) {
    int lp, lq;
    jacobi_pair(i / g, i % g, g2, lp, lq);
    r0[i] = make_uchar2((unsigned char)lp, (unsigned char)lq);
  }
  for (int i = tid; i < g2 * g2; i += nthr) W[i] = (i / g2 == i % g2) ? one : zero;
  for (int i = tid; i < 2 * slot_elems; i += nthr) {
    const int sl = i / slot_elems, rem = i - sl * slot_elems, rr = rem / B, col = rem - rr * B;
    const int l = (sl ? gb : ga) * g + rr;
    slots[i] = l < B ? job.H[(size_t)l * B + col] : zero;
  }
  if (tid < g2) {
    const int l = tid % g, gl = (tid < g ? ga : gb) * g + l;
    s_rowoff[tid] = gl < B ? ((tid < g ? sa : sb) * g + l) * B : -1;
  }
  __syncthreads();
  // the H update: thread (jg, t2) applies column pair t2 to own row pairs jg, jg + ngrp, ...;
  // the last warp computes the rotations
  const int rwarp = kClUpdThreads / 32, ngrp = kClUpdThreads / npairs, t2 = tid % npairs, jg = tid / npairs;

  int nsteps = 0, sweep = 0, round = 0, nrounds = 0;
  while (true) {
    if (round == 0) {
      // convergence: off-diagonal vs diagonal mass over the rows of all CTAs
      double off = 0.0, dg = 0.0;
      for (int i = tid; i < g2 * B; i += nthr) {
        const int l = i / B, col = i - l * B, o = s_rowoff[l];
        if (o < 0) continue;
        const double2 h = slots[o + col];
        if (col == cluster_index(l, ga, gb, g)) dg += h.x * h.x; else off += h.x * h.x + h.y * h.y;
      }
      for (int o = 16; o > 0; o >>= 1) {
        off += __shfl_xor_sync(0xffffffffu, off, o);
        dg += __shfl_xor_sync(0xffffffffu, dg, o);
      }
      if (lane == 0) {
        s_red[0][warp] = off;
        s_red[1][warp] = dg;
      }
      __syncthreads();
      if (tid < kCl) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < nthr / 32; ++w) {
          a += s_red[0][w];
          b += s_red[1][w];
        }
        double* dst = cl.map_shared_rank(part, tid);
        dst[2 * me] = a;
        dst[2 * me + 1] = b;
      }
      cl.sync();
      double a = 0.0, b = 0.0;
      for (int c = 0; c < kCl; ++c) {
        a += part[2 * c];
        b += part[2 * c + 1];
      }
      if (!(a > 1e-28 * b) || b == 0.0 || sweep == max_sweeps) break;  // uniform over the cluster
    }
    const int nk = round == 0 ? g2 - 1 : g;
    for (int k = 0; k < nk; ++k, ++nsteps) {
      const int par = nsteps & 1, bsel = nsteps % kClRotBufs, bnext = bsel + 1 == kClRotBufs ? 0 : bsel + 1;
      double4* rb = rotx + bsel * npairs;
      uint32_t* pb = pqx + bsel * npairs;
      const int4* own = s_own[par];
      // rotation warp: lane L handles own pair j = L % 16 and pushes it to CTAs
      // 4 (L / 16) .. 4 (L / 16) + 3 (every slot entry has one writer; the
      // receiving barrier counts the bytes of all npairs entries)
      const int j = lane & 15, c0 = (lane >> 4) * (kCl / 2);
      const bool rlane = warp == rwarp && j < g;
      // before the wait: the step's own rotations at a round start, then the
      // entries (of the not yet updated H) that fix the next step's rotations:
      // pair j of step k + 1 joins position lpn of own pair ja with lqn of own
      // pair jb, and H'[p'][q'] is one entry of the rotated block (ja, jb)
      int ja = 0, jb = 0, lpn = 0, lqn = 0;
      double2 X00 = zero, X01 = zero, X10 = zero, X11 = zero;
      if (warp == rwarp) {
        if (k == 0 && rlane) {
          int lp, lq;
          cluster_local_pair(r0, round, 0, j, g, lp, lq);
          const int p = cluster_index(lp, ga, gb, g), q = cluster_index(lq, ga, gb, g);
          const int op = s_rowoff[lp], oq = s_rowoff[lq];
          double4 u = make_double4(1.0, 0.0, 1.0, 0.0);
          double na = 0.0, nd = 0.0;
          if (q < B) {
            double tb;
            const double a = slots[op + p].x, d = slots[oq + q].x;
            u = jacobi_rotation(a, d, slots[op + q], &tb);
            na = a - tb;
            nd = d + tb;
          } else if (p < B) {
            na = slots[op + p].x;
          }
          if (lane < 16) {
            if (p < B) s_newdiag[lp] = na;
            if (q < B) s_newdiag[lq] = nd;
            s_own[par][j] = make_int4(op, q < B ? oq : -1, lp, lq);
          }
          if (!*(volatile int*)&s_fail)  // after a timeout no bytes go to barriers that may be unarmed
            for (int c = c0; c < c0 + kCl / 2; ++c)
              push_rotation(rb, pb, &s_bar[bsel], e * g + j, u, (uint32_t)p | (uint32_t)q << 16, c);
        }
        __syncwarp();
        if (k + 1 < nk) {
          if (lane < g) {
            const int4 o = own[lane];
            s_pairof[o.z] = lane;
            s_pairof[o.w] = lane | 256;
          }
          __syncwarp();
          if (rlane) {
            cluster_local_pair(r0, round, k + 1, j, g, lpn, lqn);
            ja = s_pairof[lpn];
            jb = s_pairof[lqn];
            const int4 oa = own[ja & 255], ob = own[jb & 255];
            const int pc = cluster_index(ob.z, ga, gb, g), qc = cluster_index(ob.w, ga, gb, g);
            if (oa.x >= 0 && pc < B) {
              const double2* rp = slots + oa.x;
              X00 = rp[pc];
              if (qc < B) X01 = rp[qc];
              if (oa.y >= 0) {
                const double2* rw = slots + oa.y;
                X10 = rw[pc];
                if (qc < B) X11 = rw[qc];
              }
            }
          }
        }
      }
      // this step's rotations from every CTA (the slot's phase: uses of the slot so far);
      // after one timeout the CTA stops waiting, finishes quickly and reports it
      if (!*(volatile int*)&s_fail && !mbar_wait_cluster(&s_bar[bsel], (uint32_t)((nsteps / kClRotBufs) & 1)))
        s_fail = 1;
      // the slot's next use (three steps on) is armed before this CTA's next
      // rotations leave, so no sender can complete bytes of an unarmed phase
      // (not once this CTA has timed out: the slot's phase may not have completed,
      // and a second arrival in one phase of a count-1 barrier is undefined)
      if (tid == 0 && !*(volatile int*)&s_fail) mbar_arm(&s_bar[bsel], cluster_step_bytes(npairs));
      // W <- W U over the own pairs (row r, columns lp and lq; W is kept
      // column-major so that consecutive rows are consecutive words).  The own
      // pairs of a round's first step are written by the rotation warp just
      // before the barrier below; later steps' were written a step earlier.
      auto update_w = [&]() {
        for (int i = tid; i < g * g2; i += kClUpdThreads) {
          const int jj = i / g2, r = i - jj * g2;
          const int4 o = own[jj];
          double2 vp = W[o.z * g2 + r], vq = W[o.w * g2 + r];
          rot_cols(vp, vq, rb[e * g + jj]);
          W[o.z * g2 + r] = vp;
          W[o.w * g2 + r] = vq;
        }
      };
      if (warp != rwarp && k > 0) update_w();
      // the rotation warp has read its entries of H (and, at a round start,
      // written the step's own pairs): the update may begin
      asm volatile("bar.sync 1, %0;" ::"r"(kClThreads) : "memory");
      if (warp == rwarp) {
        if (k + 1 < nk && rlane) {
          // the next step's rotation and diagonal, pushed while the other warps update H
          const int pn = cluster_index(lpn, ga, gb, g), qn = cluster_index(lqn, ga, gb, g);
          const int opn = s_rowoff[lpn], oqn = s_rowoff[lqn];
          double4 u = make_double4(1.0, 0.0, 1.0, 0.0);
          double na = 0.0, nd = 0.0;
          if (qn < B) {
            rot_block(X00, X01, X10, X11, rb[e * g + (ja & 255)], rb[e * g + (jb & 255)]);
            const double2 x = (ja & 256) ? ((jb & 256) ? X11 : X10) : ((jb & 256) ? X01 : X00);
            const double a = s_newdiag[lpn], d = s_newdiag[lqn];
            double tb;
            u = jacobi_rotation(a, d, x, &tb);
            na = a - tb;
            nd = d + tb;
          }
          // both half-warps have read s_newdiag before the lower half rewrites it
          const unsigned rmask = (1u << g) - 1u;
          __syncwarp(rmask | rmask << 16);
          if (lane < 16) {
            if (qn < B) {
              s_newdiag[lpn] = na;
              s_newdiag[lqn] = nd;
            }
            s_own[par ^ 1][j] = make_int4(opn, qn < B ? oqn : -1, lpn, lqn);
          }
          double4* rn = rotx + bnext * npairs;
          uint32_t* pn_ = pqx + bnext * npairs;
          if (!*(volatile int*)&s_fail)
            for (int c = c0; c < c0 + kCl / 2; ++c)
              push_rotation(rn, pn_, &s_bar[bnext], e * g + j, u, (uint32_t)pn | (uint32_t)qn << 16, c);
        }
      } else if (k == 0) {
        update_w();
      }
      if (warp != rwarp && jg < ngrp) {
        // U_j^H H[rows of own pair j, columns of pair t2] U_t2
        const uint32_t pc = pb[t2];
        const int p2 = (int)(pc & 0xffffu), q2 = (int)(pc >> 16);
        const bool cq = q2 < B;
        const double4 u2 = rb[t2];
        if (p2 < B)
          for (int jr = jg; jr < g; jr += ngrp) {
            const int t1 = e * g + jr;
            const int4 o = own[jr];
            if (o.x < 0) continue;
            const bool rq = o.y >= 0;
            double2* rp = slots + o.x;
            double2* rw = slots + (rq ? o.y : o.x);
            double2 x00 = rp[p2], x01 = cq ? rp[q2] : zero, x10 = rq ? rw[p2] : zero,
                    x11 = (rq && cq) ? rw[q2] : zero;
            rot_block(x00, x01, x10, x11, rb[t1], u2);
            if (t2 == t1) {  // (p2, q2) = (p, q)
              rp[p2] = make_double2(x00.x, 0.0);
              if (rq) {
                rp[q2] = zero;
                rw[p2] = zero;
                rw[q2] = make_double2(x11.x, 0.0);
              }
            } else {
              rp[p2] = x00;
              if (cq) rp[q2] = x01;
              if (rq) {
                rw[p2] = x10;
                if (cq) rw[q2] = x11;
              }
            }
          }
      }
      __syncthreads();
    }
    // log this round's block and restart it from the identity
    {
      double2* out = wlog + ((size_t)nrounds * kCl + e) * g2 * g2;  // row-major
      for (int i = tid; i < g2 * g2; i += nthr) {
        const int l = i / g2, m = i - l * g2;
        out[i] = W[m * g2 + l];
      }
      __syncthreads();
      for (int i = tid; i < g2 * g2; i += nthr) W[i] = (i / g2 == i % g2) ? one : zero;
    }
    ++nrounds;
    // next round: every CTA keeps one group and pulls the other from its holder
    const int nr = round + 1 == ngroups - 1 ? 0 : round + 1;
    const uint32_t tr = c_cluster_sched[(nrounds - 1) * kCl + me];
    ga = tr & 15;
    gb = (tr >> 4) & 15;
    e = (tr >> 8) & 7;
    sa = (tr >> 11) & 3;
    sb = (tr >> 13) & 3;
    cl.sync();  // every CTA's updates of the finished round are visible
    if ((tr >> 22) & 1) {
      const double2* from = cl.map_shared_rank(slots, (int)((tr >> 15) & 7)) + (size_t)((tr >> 18) & 3) * slot_elems;
      double2* to = slots + (size_t)((tr >> 20) & 3) * slot_elems;
      constexpr int U = 4;  // independent remote loads in flight per thread
      for (int i0 = tid; i0 < slot_elems; i0 += U * nthr) {
        double2 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (i0 + u * nthr < slot_elems) v[u] = from[i0 + u * nthr];
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (i0 + u * nthr < slot_elems) to[i0 + u * nthr] = v[u];
      }
    }
    if (tid < g2) {
      const int l = tid % g, gl = (tid < g ? ga : gb) * g + l;
      s_rowoff[tid] = gl < B ? ((tid < g ? sa : sb) * g + l) * B : -1;
    }
    __syncthreads();
    round = nr;
    if (round == 0) ++sweep;
  }
  // eigenvalues: every CTA sends its diagonal to rank 0, which ranks them
  if (tid == 0 && s_fail) *cl.map_shared_rank(&s_anyfail, 0) = 1;
  {
    for (int l = tid; l < g2; l += nthr) {
      const int gl = cluster_index(l, ga, gb, g), o = s_rowoff[l];
      if (o >= 0) cl.map_shared_rank(diag, 0)[gl] = slots[o + gl].x;
    }
  }
  cl.sync();
  if (me == 0) {
    for (int i = tid; i < B; i += nthr) {
      const double vi = diag[i];
      int r = 0;
      for (int j = 0; j < B; ++j) {
        const double vj = diag[j];
        r += (vj > vi) || (vj == vi && j < i);
      }
      job.w[r] = vi;
      job.jst[1 + i] = r;
    }
    if (tid == 0) job.jst[0] = s_anyfail ? -1 : nsteps;  // -1: a rotation exchange timed out
  }
}

// Q[k][rank[c]] = (e_k^T W_1 W_2 ... )[c] for the logged block-diagonal
// round products of k_jacobi_cluster: each CTA keeps kVbRows rows of Q in
// shared memory and, per round, stages the round's kCl blocks and replaces
// each row's 2g entries of every block by their product with the block.
constexpr int kVbRows = 2;
constexpr int kVbThreads = 256;
constexpr int kVbItems = (kVbRows * kCl * 2 * kClMaxG + kVbThreads - 1) / kVbThreads;

// shared memory of k_jacobi_vectors_blocks with nbuf staging buffers for the round's blocks
size_t jacobi_vectors_blocks_smem(int B, int nbuf) {
  const int Bp = jacobi_cluster_bp(B), g2 = Bp / kCl;
  return sizeof(double2) * ((size_t)nbuf * kCl * g2 * g2 + (size_t)kVbRows * Bp + (size_t)kVbRows * kCl * g2);
}
// two buffers (the next round's blocks load while this round's are applied) when they fit
int jacobi_vectors_blocks_nbuf(int B) { return jacobi_vectors_blocks_smem(B, 2) <= 220 * 1024 ? 2 : 1; }

__global__ void __launch_bounds__(kVbThreads) k_jacobi_vectors_blocks(JacobiJobs jobs, int nbuf) {
  extern __shared__ __align__(16) unsigned char vsm[];
  const JacobiJob job = jobs.j[blockIdx.y];
  const int B = job.B, Bp = jacobi_cluster_bp(B), g = Bp / (2 * kCl), g2 = 2 * g, ngroups = 2 * kCl;
  const int k0 = blockIdx.x * kVbRows;
  if (k0 >= B) return;  // uniform over the CTA
  const int bsz = g2 * g2;
  double2* Wsm = reinterpret_cast<double2*>(vsm);  // nbuf x kCl blocks of a round
  double2* rows = Wsm + nbuf * kCl * bsz;           // kVbRows x Bp
  double2* xg = rows + kVbRows * Bp;                // kVbRows x kCl x 2g: the round's entries of each block
  const double2* __restrict__ wlog = reinterpret_cast<const double2*>(job.rot);
  for (int i = threadIdx.x; i < kVbRows * Bp; i += blockDim.x) {
    const int r = i / Bp, c = i - r * Bp;
    rows[i] = make_double2(k0 + r == c ? 1.0 : 0.0, 0.0);
  }
  const int rounds = job.jst[0] / (Bp - 1) * (ngroups - 1);
  const int items = kVbRows * kCl * g2;
  // logical index of position l of block e in round r
  auto index_of = [&](int r, int e, int l) {
    int ga, gb;
    jacobi_pair(r, e, ngroups, ga, gb);
    return cluster_index(l, ga, gb, g);
  };
  auto stage = [&](int rd) {  // the round's blocks into buffer rd % nbuf
    const double2* src = wlog + (size_t)rd * kCl * bsz;
    double2* dst = Wsm + (rd % nbuf) * kCl * bsz;
    for (int i = threadIdx.x; i < kCl * bsz; i += blockDim.x) __pipeline_memcpy_async(dst + i, src + i, sizeof(double2));
    __pipeline_commit();
  };
  if (rounds > 0) stage(0);
  for (int rd = 0; rd < rounds; ++rd) {
    const int r = rd % (ngroups - 1);
    __syncthreads();  // the previous round's rows are written, its buffer is free
    if (nbuf > 1 && rd + 1 < rounds) {
      stage(rd + 1);
      __pipeline_wait_prior(1);  // this round's blocks have landed
    } else {
      if (nbuf == 1 && rd > 0) stage(rd);
      __pipeline_wait_prior(0);
    }
    // each row's entries of each block, gathered contiguously
    for (int i = threadIdx.x; i < items; i += blockDim.x) {
      const int l = i % g2, e = (i / g2) % kCl, rr = i / (g2 * kCl);
      xg[i] = rows[rr * Bp + index_of(r, e, l)];
    }
    __syncthreads();
    const double2* Wr = Wsm + (rd % nbuf) * kCl * bsz;
    double2 y[kVbItems];
#pragma unroll
    for (int it = 0; it < kVbItems; ++it) {
      const int item = threadIdx.x + it * kVbThreads;
      y[it] = make_double2(0.0, 0.0);
      if (item < items) {
        const int m = item % g2, e = (item / g2) % kCl, rr = item / (g2 * kCl);
        const double2* x = xg + (rr * kCl + e) * g2;
        const double2* w = Wr + e * bsz + m;
        double2 a0 = make_double2(0.0, 0.0), a1 = make_double2(0.0, 0.0);
#pragma unroll 2
        for (int l = 0; l < g2; l += 2) {
          a0 = zfma(x[l], w[l * g2], a0);
          a1 = zfma(x[l + 1], w[(l + 1) * g2], a1);
        }
        y[it] = zadd(a0, a1);
      }
    }
    // rows are read only by the gather, so each thread writes its outputs back at once
#pragma unroll
    for (int it = 0; it < kVbItems; ++it) {
      const int item = threadIdx.x + it * kVbThreads;
      if (item < items) {
        const int m = item % g2, e = (item / g2) % kCl, rr = item / (g2 * kCl);
        rows[rr * Bp + index_of(r, e, m)] = y[it];
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kVbRows * B; i += blockDim.x) {
    const int rr = i / B, c = i - rr * B, k = k0 + rr;
    if (k < B) job.Q[(size_t)k * B + job.jst[1 + c]] = rows[rr * Bp + c];
  }
}

// Q[k][rank[p]] = (prod of the logged rotations)[k][p]: row k of Q evolves
// independently (entries p, q of the row mix under pair (p, q)), so each warp
// replays the log on one row held in shared memory, two pairs per lane.
constexpr int kVecWarps = 8;
constexpr int kVecChunkMax = 32;  // logged steps staged per pass (fewer for large B)

int jacobi_vectors_chunk(int B, int Bp) {
  const int npairs = Bp / 2;
  const size_t fixed = sizeof(double2) * kVecWarps * B + sizeof(uchar2) * (Bp - 1) * npairs + 16;
  const size_t budget = 200 * 1024;
  const int c = (int)((budget - std::min(budget, fixed)) / (sizeof(double4) * npairs));
  return std::max(1, std::min(kVecChunkMax, c));
}

size_t jacobi_vectors_smem(int B, int Bp) {
  const int npairs = Bp / 2;
  return sizeof(double4) * jacobi_vectors_chunk(B, Bp) * npairs + sizeof(double2) * kVecWarps * B +
         ((sizeof(uchar2) * (Bp - 1) * npairs + 15) & ~size_t(15));
}

__device__ __forceinline__ void replay_pair(double2* row, int B, uchar2 pq, double4 u) {
  const int p = pq.x, q = pq.y;
  if (q >= B) return;
  const double2 vp = row[p], e = zmul(row[q], make_double2(u.z, -u.w));
  row[p] = make_double2(u.x * vp.x - u.y * e.x, u.x * vp.y - u.y * e.y);
  row[q] = make_double2(u.y * vp.x + u.x * e.x, u.y * vp.y + u.x * e.y);
}

__global__ void __launch_bounds__(32 * kVecWarps) k_jacobi_vectors(JacobiJobs jobs, int chunk) {
  extern __shared__ __align__(16) unsigned char vsm[];
  const JacobiJob job = jobs.j[blockIdx.y];
  const int B = job.B;
  if (blockIdx.x * kVecWarps >= B) return;  // uniform over the CTA
  const double4* __restrict__ rot = job.rot;
  const int* __restrict__ jst = job.jst;
  double2* __restrict__ Q = job.Q;
  const int Bp = B + (B & 1), npairs = Bp / 2;
  double4* lg = reinterpret_cast<double4*>(vsm);                   // chunk x npairs
  double2* rows = reinterpret_cast<double2*>(lg + chunk * npairs);  // kVecWarps x B
  uchar2* ptab = reinterpret_cast<uchar2*>(rows + kVecWarps * B);   // (Bp - 1) x npairs
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int k = blockIdx.x * kVecWarps + warp;
  double2* row = rows + warp * B;
  for (int p = lane; p < B; p += 32) row[p] = make_double2(p == k ? 1.0 : 0.0, 0.0);
  jacobi_pair_table(ptab, Bp);
  const int nsteps = jst[0];
  int step = 0;
  for (int s0 = 0; s0 < nsteps; s0 += chunk) {
    const int ns = min(chunk, nsteps - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < ns * npairs; i += blockDim.x) lg[i] = rot[(size_t)s0 * npairs + i];
    __syncthreads();
    if (k >= B) continue;
    for (int j = 0; j < ns; ++j) {
      const uchar2* pr = ptab + step * npairs;
      const double4* uj = lg + j * npairs;
      // disjoint pairs: each lane takes pairs lane, lane + 32, ... (two at a time)
      for (int t = lane; t < npairs; t += 64) {
        const bool two = t + 32 < npairs;
        const uchar2 a = pr[t], b = two ? pr[t + 32] : make_uchar2(0, 255);
        const double4 ua = uj[t], ub = two ? uj[t + 32] : ua;
        replay_pair(row, B, a, ua);
        if (two) replay_pair(row, B, b, ub);
      }
      __syncwarp();
      if (++step == Bp - 1) step = 0;
    }
  }
  if (k < B)
    for (int p = lane; p < B; p += 32) Q[(size_t)k * B + jst[1 + p]] = row[p];
}

// krn[k][j] = U[N-1-j][k] as float planes (klitho_tcc.cpp:358-362), or as
// interleaved complex64 in re when im is null
__global__ void k_to_kernels(const double2* __restrict__ U, int N, int ldu, int K,
                             float* __restrict__ re, float* __restrict__ im) {
  const size_t n = (size_t)N * K;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i / N), j = (int)(i % N);
    const double2 v = U[(size_t)(N - 1 - j) * ldu + k];
    if (im) {
      re[i] = (float)v.x;
      im[i] = (float)v.y;
    } else {
      reinterpret_cast<float2*>(re)[i] = make_float2((float)v.x, (float)v.y);
    }
  }
}

struct Workspace {
  double2 *X = nullptr, *W = nullptr, *Z = nullptr, *G = nullptr, *Rinv = nullptr, *Q = nullptr;
  double4* rot = nullptr;
  double* w = nullptr;
  int *status = nullptr, *jst = nullptr;
  cudaStream_t st = nullptr;
  std::vector<void*> owned;
  template <typename T>
  int get(T** p, size_t count) {
    void* v = nullptr;
    const int rc = scratch_alloc(&v, sizeof(T) * count, st, "eigen workspace");
    if (rc) return rc;
    owned.push_back(v);
    *p = static_cast<T*>(v);
    return KL_OK;
  }
  ~Workspace() {
    for (void* v : owned) scratch_free(v, st);
  }
};

// k_jacobi keeps H in shared memory up to this size, else works in place
constexpr size_t kJacobiSmemCap = 220 * 1024;
bool jacobi_h_in_smem(int B) { return JacobiSmem(B).total_no_h + sizeof(double2) * (size_t)B * B <= kJacobiSmemCap; }

// matrices of kClusterMinB .. kGramMaxS go to the cluster solver when the
// device can co-schedule a cluster of kCl CTAs of its size (eight SMs beat one
// from about 64 up); otherwise k_jacobi keeps H in shared memory or works on
// it in place in global memory
constexpr int kClusterMinB = 64;
std::mutex g_cluster_mu;  // guards the per-device answers below (host threads may share the library)

bool jacobi_use_cluster(int B) {
  if (B < kClusterMinB || B > kGramMaxS) return false;
  static std::vector<int> known;  // per device: -1 unknown, 0 no, 1 yes
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  std::lock_guard<std::mutex> lock(g_cluster_mu);
  if ((int)known.size() <= dev) known.resize(dev + 1, -1);
  int& ok = known[dev];
  if (ok < 0) {
    ok = 0;
    const size_t sm = ClusterSmem(kGramMaxS).total;
    if (cudaFuncSetAttribute(k_jacobi_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) ==
        cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(kCl);
      cfg.blockDim = dim3(kClThreads);
      cfg.dynamicSmemBytes = sm;
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, k_jacobi_cluster, &cfg) == cudaSuccess && n > 0) ok = 1;
    }
    (void)cudaGetLastError();
  }
  return ok == 1;
}
// c_cluster_sched: the host walks the same state the kernel's groups move
// through.  After each round every CTA keeps one of its groups and takes the
// other group of its next edge from the CTA holding it; following the
// alternating cycles of the two matchings (edge of CTA c -> the next-round
// edge at the group c keeps -> the CTA holding that edge's other group ...)
// gives every CTA exactly one group to send and one to receive.
std::vector<uint32_t> cluster_schedule() {
  const int ng = 2 * kCl, rounds = ng - 1;
  std::vector<uint32_t> tab((size_t)kJacobiMaxSweeps * rounds * kCl);
  int grp[kCl][2], gcta[2 * kCl], gslot[2 * kCl], fre[kCl];
  for (int c = 0; c < kCl; ++c) {
    int a, b;
    jacobi_pair(0, c, ng, a, b);
    grp[c][0] = a;
    grp[c][1] = b;
    gcta[a] = gcta[b] = c;
    gslot[a] = 0;
    gslot[b] = 1;
    fre[c] = 2;
  }
  for (int t = 0; t < kJacobiMaxSweeps * rounds; ++t) {
    const int nr = (t + 1) % rounds;
    int np[2 * kCl], ne[2 * kCl], keep[kCl], recv[kCl], src[kCl], srcslot[kCl], dst[kCl], nfree[kCl];
    bool seen[kCl];
    for (int x = 0; x < kCl; ++x) {
      int a, b;
      jacobi_pair(nr, x, ng, a, b);
      np[a] = b;
      np[b] = a;
      ne[a] = ne[b] = x;
      seen[x] = false;
    }
    for (int c0 = 0; c0 < kCl; ++c0) {
      if (seen[c0]) continue;
      int c = c0, kp = grp[c0][0];
      for (int guard = 0; guard < kCl; ++guard) {
        const int rv = np[kp];
        keep[c] = kp;
        recv[c] = rv;
        seen[c] = true;
        const int c2 = gcta[rv];
        if (seen[c2]) break;
        kp = grp[c2][0] == rv ? grp[c2][1] : grp[c2][0];
        c = c2;
      }
    }
    for (int c = 0; c < kCl; ++c) {
      src[c] = gcta[recv[c]];
      srcslot[c] = gslot[recv[c]];
      if (src[c] == c) {
        dst[c] = srcslot[c];
        nfree[c] = fre[c];
      } else {
        const int sent = grp[c][0] == keep[c] ? grp[c][1] : grp[c][0];
        dst[c] = fre[c];
        nfree[c] = gslot[sent];
      }
    }
    for (int c = 0; c < kCl; ++c) {
      gcta[recv[c]] = c;
      gslot[recv[c]] = dst[c];
      fre[c] = nfree[c];
      grp[c][0] = std::min(keep[c], recv[c]);
      grp[c][1] = std::max(keep[c], recv[c]);
    }
    for (int c = 0; c < kCl; ++c) {
      const int a = grp[c][0], b = grp[c][1];
      tab[(size_t)t * kCl + c] = (uint32_t)a | (uint32_t)b << 4 | (uint32_t)ne[keep[c]] << 8 |
                                 (uint32_t)gslot[a] << 11 | (uint32_t)gslot[b] << 13 | (uint32_t)src[c] << 15 |
                                 (uint32_t)srcslot[c] << 18 | (uint32_t)dst[c] << 20 | (uint32_t)(src[c] != c) << 22;
    }
  }
  return tab;
}

// uploads c_cluster_sched once per device, ordered before work later queued on st
int ensure_cluster_schedule(cudaStream_t st) {
  static const std::vector<uint32_t> tab = cluster_schedule();
  static std::vector<char> done;  // per device
  int dev = 0;
  KL_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_cluster_mu);
  if ((int)done.size() > dev && done[dev]) return KL_OK;
  KL_CUDA_TRY(cudaMemcpyToSymbolAsync(c_cluster_sched, tab.data(), sizeof(uint32_t) * tab.size(), 0,
                                      cudaMemcpyHostToDevice, st));
  KL_CUDA_TRY(cudaStreamSynchronize(st));
  if ((int)done.size() <= dev) done.resize(dev + 1, 0);
  done[dev] = 1;
  return KL_OK;
}

// padded order of the sweep (pairs per step = order / 2, steps per sweep = order - 1)
int jacobi_order(int B) { return jacobi_use_cluster(B) ? jacobi_cluster_bp(B) : B + (B & 1); }
size_t jacobi_log_elems(int B) {  // double4 units
  if (jacobi_use_cluster(B)) return (cluster_log_elems(B, kJacobiMaxSweeps) + 1) / 2;
  const int Bp = jacobi_order(B);
  return (size_t)kJacobiMaxSweeps * (Bp - 1) * (Bp / 2) + 1;
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

// Eigen-decompositions of a batch of Hermitian matrices (see JacobiJob): one
// CTA each, or one cluster each for the sizes jacobi_use_cluster picks; H is
// overwritten when one CTA works on it in global memory.
int jacobi_batch(const std::vector<JacobiJob>& all, cudaStream_t st) {
  std::vector<JacobiJob> by_path[2];
  for (const JacobiJob& j : all) by_path[jacobi_use_cluster(j.B) ? 1 : 0].push_back(j);
  for (int cluster = 0; cluster < 2; ++cluster) {
    const std::vector<JacobiJob>& v = by_path[cluster];
    for (size_t j0 = 0; j0 < v.size(); j0 += kJacobiMaxJobs) {
      const int nj = (int)std::min(v.size() - j0, (size_t)kJacobiMaxJobs);
      JacobiJobs jobs{};
      int bmax = 1, bpmax = 2;
      for (int j = 0; j < nj; ++j) {
        jobs.j[j] = v[j0 + j];
        bmax = std::max(bmax, jobs.j[j].B);
        bpmax = std::max(bpmax, jacobi_order(jobs.j[j].B));
      }
      if (cluster) {
        if (int rc = ensure_cluster_schedule(st)) return rc;
        const size_t sm = ClusterSmem(bmax).total;
        KL_CUDA_TRY(cudaFuncSetAttribute(k_jacobi_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k_jacobi_cluster<<<nj * kCl, kClThreads, sm, st>>>(jobs, kJacobiMaxSweeps);
        KL_CUDA_TRY(cudaGetLastError());
        const int nbuf = jacobi_vectors_blocks_nbuf(bmax);
        const size_t vsm = jacobi_vectors_blocks_smem(bmax, nbuf);
        KL_CUDA_TRY(cudaFuncSetAttribute(k_jacobi_vectors_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vsm));
        k_jacobi_vectors_blocks<<<dim3((bmax + kVbRows - 1) / kVbRows, nj), kVbThreads, vsm, st>>>(jobs, nbuf);
        KL_CUDA_TRY(cudaGetLastError());
        continue;
      }
      const bool in_smem = jacobi_h_in_smem(bmax);
      const size_t sm = JacobiSmem(bmax).total_no_h + (in_smem ? sizeof(double2) * (size_t)bmax * bmax : 0);
      if (sm > 48 * 1024)
        KL_CUDA_TRY(cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      k_jacobi<<<nj, kJacobiThreads, sm, st>>>(jobs, in_smem ? 1 : 0, kJacobiMaxSweeps);
      KL_CUDA_TRY(cudaGetLastError());
      const size_t vsm = jacobi_vectors_smem(bmax, bpmax);
      if (vsm > 48 * 1024)
        KL_CUDA_TRY(cudaFuncSetAttribute(k_jacobi_vectors, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)vsm));
      k_jacobi_vectors<<<dim3((bmax + kVecWarps - 1) / kVecWarps, nj), 32 * kVecWarps, vsm, st>>>(
          jobs, jacobi_vectors_chunk(bmax, bpmax));
      KL_CUDA_TRY(cudaGetLastError());
    }
  }
  return KL_OK;
}

// Q (B x B, column j = eigenvector j) and w (descending) of the Hermitian H
int jacobi(double2* H, int B, double4* rot, int* jst, double2* Q, double* w, cudaStream_t st) {
  return jacobi_batch({JacobiJob{H, rot, Q, w, jst, B}}, st);
}

// Generic driver.  apply(X, W): W = TCC X (N x B); project(X, H): H = X^H TCC X (B x B).
template <typename Apply, typename Project>
int subspace_iteration(int N, const EigenOptions& opt, int B, Apply apply, Project project,
                       double2* U, double* evals, EigenResult* res, cudaStream_t st) {
  Workspace ws;
  ws.st = st;
  const int K = opt.K;
  int arc;
  if ((arc = ws.get(&ws.X, (size_t)N * B)) || (arc = ws.get(&ws.W, (size_t)N * B)) ||
      (arc = ws.get(&ws.G, (size_t)B * B)) || (arc = ws.get(&ws.Rinv, (size_t)B * B)) ||
      (arc = ws.get(&ws.Q, (size_t)B * B)) || (arc = ws.get(&ws.rot, jacobi_log_elems(B))) ||
      (arc = ws.get(&ws.jst, (size_t)B + 1)) || (arc = ws.get(&ws.w, (size_t)B)) ||
      (arc = ws.get(&ws.status, 1)))
    return arc;
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
      if ((rc = jacobi(ws.G, B, ws.rot, ws.jst, ws.Q, ws.w, st))) return rc;
      int jsteps = 0;
      KL_CUDA_TRY(cudaMemcpyAsync(cur.data(), ws.w, sizeof(double) * B, cudaMemcpyDeviceToHost, st));
      KL_CUDA_TRY(cudaMemcpyAsync(&jsteps, ws.jst, sizeof(int), cudaMemcpyDeviceToHost, st));
      KL_CUDA_TRY(cudaStreamSynchronize(st));
      if (jsteps < 0) {
        set_error("subspace iteration: the cluster Jacobi eigensolve timed out exchanging rotations");
        return KL_ERR_CUDA;
      }
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
      // continue from the Ritz basis: the next projected matrix is then nearly
      // diagonal and its Jacobi solve takes a few sweeps
      if ((rc = zgemm<G_NN>(ws.X, B, ws.Q, B, ws.W, B, N, B, B, st))) return rc;
      KL_CUDA_TRY(cudaMemcpyAsync(ws.X, ws.W, sizeof(double2) * (size_t)N * B, cudaMemcpyDeviceToDevice, st));
    }
    if ((rc = apply(ws.X, ws.W))) return rc;
    KL_CUDA_TRY(cudaMemcpyAsync(ws.X, ws.W, sizeof(double2) * (size_t)N * B, cudaMemcpyDeviceToDevice, st));
    if ((rc = cholqr2(ws.X, N, B, ws, st))) return rc;
  }
  // final Rayleigh-Ritz on the current block (G holds the eigvecs in Q)
  if (!converged) {
    if ((rc = project(ws.X, ws.G))) return rc;
    if ((rc = jacobi(ws.G, B, ws.rot, ws.jst, ws.Q, ws.w, st))) return rc;
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

namespace {

// V[s][k] = Q[s][k] / sqrt(w[k]) for k < K (zero for a numerically null w[k])
__global__ void k_ritz_scale(const double2* __restrict__ Q, int ldq, const double* __restrict__ w,
                             int S, int K, double2* __restrict__ V) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S * K) return;
  const int s = i / K, k = i - s * K;
  const double wk = w[k];
  const double f = (wk > 1e-15 * fabs(w[0]) && wk > 0.0) ? 1.0 / sqrt(wk) : 0.0;
  const double2 q = Q[(size_t)s * ldq + k];
  V[i] = make_double2(q.x * f, q.y * f);
}

// TCC = A A^H with S <= kGramMaxS columns: the TCC's range is span(A), so the
// Rayleigh-Ritz step on that span is exact.  G = A^H A (S x S, exact FP64
// products of the FP32 factor: integer digits on the tensor cores, gram_i8.cu,
// or FP64 CUDA cores elsewhere), G = V diag(w) V^H, U = A V diag(w)^{-1/2}.  Orders the
// cluster reduction handles (64 .. 256) take the tridiagonal solver
// (eig_tridiag.cu), smaller ones Jacobi on one CTA; all problems of a path are
// solved in one batch of launches.
int eig_topk_gram(const std::vector<FactorProblem>& pr, cudaStream_t st) {
  const size_t n = pr.size();
  std::vector<Workspace> ws(n);
  std::vector<JacobiJob> jobs;
  std::vector<TridiagJob> tjobs;
  std::vector<char> tri(n, 0);
  for (size_t i = 0; i < n; ++i) {
    const int S = pr[i].S, K = pr[i].K;
    Workspace& w = ws[i];
    w.st = st;
    tri[i] = tridiag_eig_supported(S) ? 1 : 0;
    int arc;
    if ((arc = w.get(&w.G, (size_t)S * S)) || (arc = w.get(&w.Q, (size_t)S * S)) ||
        (arc = w.get(&w.jst, (size_t)S + 1)) || (arc = w.get(&w.W, (size_t)S * K)) || (arc = w.get(&w.w, (size_t)S)) ||
        (arc = w.get(&w.status, 1)))
      return arc;
    // one status word for the Gram product's and the reduction's bounded waits
    KL_CUDA_TRY(cudaMemsetAsync(w.status, 0, sizeof(int), st));
    if (tri[i]) {
      TridiagJob t{};
      double* lw = nullptr;
      double* y = nullptr;
      double* d = nullptr;
      double2* e = nullptr;
      double2* wyb = nullptr;
      if ((arc = w.get(&w.Z, (size_t)S * S)) || (arc = w.get(&d, (size_t)S)) || (arc = w.get(&e, (size_t)S)) ||
          (arc = w.get(&lw, (size_t)S * K)) || (arc = w.get(&y, (size_t)S * K)) ||
          (arc = w.get(&wyb, (size_t)tridiag_wy_blocks(S) * 64)))
        return arc;
      t.wy = wyb;
      t.H = w.G;
      t.refl = w.Z;
      t.d = d;
      t.e = e;
      t.w = w.w;
      t.lw = lw;
      t.Y = y;
      t.Q = w.Q;
      t.B = S;
      t.K = K;
      t.ldq = S;
      t.err = w.status;
      tjobs.push_back(t);
    } else {
      if ((arc = w.get(&w.rot, jacobi_log_elems(S)))) return arc;
      jobs.push_back(JacobiJob{w.G, w.rot, w.Q, w.w, w.jst, S});
    }
    if (int rc = gram_factor(pr[i].A, pr[i].N, S, w.G, w.status, st)) return rc;
  }
  int rc = jacobi_batch(jobs, st);
  if (rc) return rc;
  if ((rc = tridiag_eig_batch(tjobs, st))) return rc;
  std::vector<int> nsteps(n, 0), gerr(n, 0);
  for (size_t i = 0; i < n; ++i) {
    const int S = pr[i].S, K = pr[i].K;
    if (ws[i].status) KL_CUDA_TRY(cudaMemcpyAsync(&gerr[i], ws[i].status, sizeof(int), cudaMemcpyDeviceToHost, st));
    k_ritz_scale<<<(S * K + 255) / 256, 256, 0, st>>>(ws[i].Q, S, ws[i].w, S, K, ws[i].W);
    KL_CUDA_TRY(cudaGetLastError());
    if ((rc = zgemm<G_AY>(pr[i].A, S, ws[i].W, K, pr[i].U, K, pr[i].N, K, S, st))) return rc;
    KL_CUDA_TRY(cudaMemcpyAsync(pr[i].evals, ws[i].w, sizeof(double) * K, cudaMemcpyDeviceToDevice, st));
    if (!tri[i]) KL_CUDA_TRY(cudaMemcpyAsync(&nsteps[i], ws[i].jst, sizeof(int), cudaMemcpyDeviceToHost, st));
  }
  KL_CUDA_TRY(cudaStreamSynchronize(st));
  for (size_t i = 0; i < n; ++i) {
    const int S = pr[i].S;
    if (gerr[i]) {
      set_error("eig_topk_factor: a bounded wait gave up (code " + std::to_string(gerr[i]) +
                ": 31-35 the tensor-core Gram product, 41 the tridiagonal reduction's exchange)");
      return KL_ERR_CUDA;
    }
    if (tri[i]) {
      if (pr[i].res) {
        pr[i].res->iterations = 1;  // one direct solve
        pr[i].res->residual = 0.0;
      }
      continue;
    }
    if (nsteps[i] < 0) {
      set_error("eig_topk_factor: the cluster Jacobi eigensolve timed out exchanging rotations");
      return KL_ERR_CUDA;
    }
    const int sweeps = nsteps[i] / (jacobi_order(S) - 1);
    if (sweeps >= kJacobiMaxSweeps) {
      set_error("eig_topk_factor: Jacobi eigensolve of the Gram matrix did not converge in " +
                std::to_string(kJacobiMaxSweeps) + " sweeps");
      return KL_ERR_NOT_CONVERGED;
    }
    if (pr[i].res) {
      pr[i].res->iterations = sweeps;  // Jacobi sweeps of the single Rayleigh-Ritz step
      pr[i].res->residual = 0.0;
    }
  }
  return KL_OK;
}

}  // namespace

int gram_factor(const float2* A, int N, int S, double2* G, int* err_dev, cudaStream_t st) {
  if (gram_i8_supported(N, S)) return gram_i8(A, N, S, G, err_dev, st);  // tensor cores, integer digits
  return zgemm<G_AHA>(A, S, A, S, G, S, S, S, N, st);                    // FP64 CUDA cores
}

int eig_topk_factor(const float2* A, int N, int S, const EigenOptions& opt, double2* U,
                    double* evals, EigenResult* res, cudaStream_t st) {
  KL_CHECK_ARG(opt.K > 0 && opt.K <= N, "eig_topk_factor: K out of range");
  if (S <= kGramMaxS && opt.K <= S) return eig_topk_gram({FactorProblem{A, N, S, opt.K, U, evals, res}}, st);
  const int B = block_size(opt, N, S);
  KL_CHECK_ARG(opt.K <= B, "eig_topk_factor: K exceeds the block size");
  double2* Z = nullptr;
  if (int arc = scratch_alloc((void**)&Z, sizeof(double2) * (size_t)S * B, st, "eigen workspace")) return arc;
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
  scratch_free(Z, st);
  return rc;
}

int eig_topk_factor_batch(const std::vector<FactorProblem>& pr, const EigenOptions& opt, cudaStream_t st) {
  bool gram = true;
  for (const FactorProblem& f : pr) {
    KL_CHECK_ARG(f.K > 0 && f.K <= f.N, "eig_topk_factor: K out of range");
    gram = gram && f.S <= kGramMaxS && f.K <= f.S;
  }
  if (gram) return eig_topk_gram(pr, st);
  for (const FactorProblem& f : pr) {
    EigenOptions o = opt;
    o.K = f.K;
    const int rc = eig_topk_factor(f.A, f.N, f.S, o, f.U, f.evals, f.res, st);
    if (rc) return rc;
  }
  return KL_OK;
}

int eig_topk_dense(const double2* tcc, int N, const EigenOptions& opt, double2* U, double* evals,
                   EigenResult* res, cudaStream_t st) {
  KL_CHECK_ARG(opt.K > 0 && opt.K <= N, "eig_topk_dense: K out of range");
  const int B = block_size(opt, N, N);
  double2* Wt = nullptr;
  if (int arc = scratch_alloc((void**)&Wt, sizeof(double2) * (size_t)N * B, st, "eigen workspace")) return arc;
  auto apply = [&](double2* X, double2* W) -> int {
    return zgemm<G_DX>(tcc, N, X, B, W, B, N, B, N, st);
  };
  auto project = [&](double2* X, double2* H) -> int {
    int rc = zgemm<G_DX>(tcc, N, X, B, Wt, B, N, B, N, st);
    if (rc) return rc;
    return zgemm<G_HH>(X, B, Wt, B, H, B, B, B, N, st);
  };
  int rc = subspace_iteration(N, opt, B, apply, project, U, evals, res, st);
  scratch_free(Wt, st);
  return rc;
}

int eig_topk_dense_c64(const float2* tcc, int N, const EigenOptions& opt, double2* U,
                       double* evals, EigenResult* res, cudaStream_t st) {
  KL_CHECK_ARG(opt.K > 0 && opt.K <= N, "eig_topk_dense_c64: K out of range");
  const int B = block_size(opt, N, N);
  double2* Wt = nullptr;
  if (int arc = scratch_alloc((void**)&Wt, sizeof(double2) * (size_t)N * B, st, "eigen workspace")) return arc;
  auto apply = [&](double2* X, double2* W) -> int {
    return zgemm<G_FX>(tcc, N, X, B, W, B, N, B, N, st);
  };
  auto project = [&](double2* X, double2* H) -> int {
    int rc = zgemm<G_FX>(tcc, N, X, B, Wt, B, N, B, N, st);
    if (rc) return rc;
    return zgemm<G_HH>(X, B, Wt, B, H, B, B, B, N, st);
  };
  int rc = subspace_iteration(N, opt, B, apply, project, U, evals, res, st);
  scratch_free(Wt, st);
  return rc;
}

int eig_to_kernels(const double2* U, int N, int K, float* re, float* im, cudaStream_t st) {
  k_to_kernels<<<256, 256, 0, st>>>(U, N, K, K, re, im);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

}  // namespace kl
