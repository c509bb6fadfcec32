// gram_i8.cu -- the Gram matrix G = A^H A of the TCC's FP32 factor A (N x S)
// on the tensor cores, exactly: the FP64 product the Rayleigh-Ritz step on
// span(A) needs (the reduction of zheevr's N x N problem in
// K-Litho-TCC/klitho_tcc.cpp:300-377 to an S x S one).
//
// Each column s of A = X + iY is scaled by 2^(27 - E_s), E_s = ilogb(max |x|,
// |y| over the column) + 1, rounded to integers |x'| < 2^27 (exact for every
// entry within 2^4 of the column's largest; the others keep 2^-27 of it,
// finer than the FP32 rounding the factor already carries), and written as
// four balanced base-128 digits: x' = d0 2^21 + d1 2^14 + d2 2^7 + d3 with
// |d| <= 65 (the splitting of Ozaki, Ogita, Oishi and Rump's error-free
// matrix products, with integer slices).  The digit planes of X and Y form
// Z^T = [X_0 .. X_3 Y_0 .. Y_3]^T (8S rows of N int8), and one tcgen05.mma
// kind::i8 GEMM forms P = Z^T Z with 32-bit integer accumulation, exact since
// N 65^2 < 2^31 for N < 508,000.  G is then assembled in FP64:
//   Re G[s][s'] = sum_{t,u} 2^(E_s + E_s' - 12 - 7(t+u)) (P[X_t s][X_u s'] + P[Y_t s][Y_u s'])
//   Im G[s][s'] = sum_{t,u} 2^(E_s + E_s' - 12 - 7(t+u)) (P[X_t s][Y_u s'] - P[Y_t s][X_u s'])
// P is symmetric: only its upper 128 x 128 tiles are computed, one per CTA.
#include <algorithm>
#include <mutex>
#include <vector>

#include "kl_internal.h"
#include "kl_tc.cuh"
#include "kl_tcc.h"

namespace kl {

namespace {

using namespace tc;

constexpr int kGT = 128;        // P tile (rows and columns) and K block (int8 bytes per swizzled row)
constexpr int kGStages = 6;     // K blocks in flight
constexpr int kGTileBytes = kGT * kGT;          // one operand tile of a K block
constexpr int kGStageBytes = 2 * kGTileBytes;   // row tile + column tile
constexpr int kGThreads = 192;  // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int kGSmem = kGStages * kGStageBytes + 1024 + 256;
constexpr int kGMaxN = 500000;  // factor rows for which the 32-bit accumulation is exact

__device__ __forceinline__ void upper_tile_g(int t, int nt, int& ib, int& jb) {
  int rowlen = nt;
  ib = 0;
  while (t >= rowlen) {
    t -= rowlen;
    ++ib;
    --rowlen;
  }
  jb = ib + t;
}

// colmax[s] = max over the CTA's rows f of max(|Re A[f][s]|, |Im A[f][s]|)
// (float bits: non-negative floats order like their bit patterns)
__global__ void __launch_bounds__(256) k_gram_colmax(const float2* __restrict__ A, int N, int S, int rows,
                                                     unsigned* __restrict__ colmax) {
  const int f0 = blockIdx.x * rows, f1 = min(N, f0 + rows);
  for (int s = threadIdx.x; s < S; s += blockDim.x) {
    float m = 0.f;
    for (int f = f0; f < f1; ++f) {
      const float2 a = A[(size_t)f * S + s];
      m = fmaxf(m, fmaxf(fabsf(a.x), fabsf(a.y)));
    }
    atomicMax(&colmax[s], __float_as_uint(m));
  }
}

// the four base-128 digits of round(v 2^sh) (|result| < 2^27), most significant first
__device__ __forceinline__ void gram_digits(float v, int sh, int (&d)[4]) {
  int x = __double2int_rn(ldexp((double)v, sh));
#pragma unroll
  for (int t = 3; t > 0; --t) {
    d[t] = ((x + 64) & 127) - 64;
    x = (x - d[t]) >> 7;
  }
  d[0] = x;
}

// Z^T rows (part * 4 + t) * S + s, columns f: digit t of the scaled real
// (part 0) or imaginary (part 1) part of A[f][s]; a thread writes 16
// consecutive f of one s into each of its 8 rows.  E[s] = E_s.
__global__ void __launch_bounds__(256) k_gram_digits(const float2* __restrict__ A, int N, int S, int Kp,
                                                     const unsigned* __restrict__ colmax, int8_t* __restrict__ Z,
                                                     int* __restrict__ E) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = gid % S, g = gid / S, f0 = 16 * g;
  if (f0 >= N) return;
  const float m = __uint_as_float(colmax[s]);
  const int e = m > 0.f ? ilogbf(m) + 1 : 0;
  if (g == 0) E[s] = e;
  uint32_t w[8][4];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int q = 0; q < 4; ++q) w[r][q] = 0u;
#pragma unroll
  for (int u = 0; u < 16; ++u) {
    const int f = f0 + u;
    const float2 a = f < N ? A[(size_t)f * S + s] : make_float2(0.f, 0.f);
    int dx[4], dy[4];
    gram_digits(a.x, 27 - e, dx);
    gram_digits(a.y, 27 - e, dy);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      w[t][u >> 2] |= (uint32_t)(dx[t] & 0xff) << (8 * (u & 3));
      w[4 + t][u >> 2] |= (uint32_t)(dy[t] & 0xff) << (8 * (u & 3));
    }
  }
#pragma unroll
  for (int r = 0; r < 8; ++r)
    *reinterpret_cast<uint4*>(Z + ((size_t)r * S + s) * Kp + f0) = make_uint4(w[r][0], w[r][1], w[r][2], w[r][3]);
}

// P tile (ib, jb), ib <= jb, of P = Z^T Z: one CTA each
__global__ void __launch_bounds__(kGThreads, 1)
    k_gram_i8_gemm(const __grid_constant__ CUtensorMap tmZ, int nkb, int nt, int ldp, int* __restrict__ P,
                   int* __restrict__ err) {
  extern __shared__ uint8_t gsm_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(gsm_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kGStages * kGStageBytes);
  uint64_t* empty = full + kGStages;
  uint64_t* tfull = empty + kGStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tfull + 1);
  __shared__ int s_abort;
  volatile int* abort = &s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int ib, jb;
  upper_tile_g(blockIdx.x, nt, ib, jb);
  if (threadIdx.x == 0) {
    for (int s = 0; s < kGStages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    mbar_init(smem_u32(tfull), 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(kGT)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // TMA producer: K block kb of the row tile ib and the column tile jb into stage kb % kGStages
    int armed[kGStages];
    for (int s = 0; s < kGStages; ++s) armed[s] = -1;
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % kGStages, use = kb / kGStages;
      if (use > 0 && !mbar_wait_ab(smem_u32(&empty[s]), (uint32_t)((use - 1) & 1), err, 31, abort)) break;
      const uint32_t bar = smem_u32(&full[s]);
      mbar_expect_tx(bar, kGStageBytes);
      uint8_t* st = smem + s * kGStageBytes;
      tma_load_2d(smem_u32(st), &tmZ, kb * kGT, ib * kGT, bar);
      tma_load_2d(smem_u32(st + kGTileBytes), &tmZ, kb * kGT, jb * kGT, bar);
      armed[s] = use;
    }
    // every issued copy lands before the CTA can retire
    for (int s = 0; s < kGStages; ++s)
      if (armed[s] >= 0) mbar_wait(smem_u32(&full[s]), (uint32_t)(armed[s] & 1), err, 32);
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: four K = 32 steps per K block (32 bytes along the swizzled row)
    constexpr uint32_t idesc = idesc_s8(kGT, kGT);
    for (int kb = 0; kb < nkb; ++kb) {
      const int s = kb % kGStages, use = kb / kGStages;
      if (!mbar_wait_ab(smem_u32(&full[s]), (uint32_t)(use & 1), err, 33, abort)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a = smem_u32(smem + s * kGStageBytes), b = a + kGTileBytes;
#pragma unroll
      for (int k = 0; k < kGT / 32; ++k)
        mma_i8(tmem, smem_desc(a + 32 * k), smem_desc(b + 32 * k), idesc, (kb > 0 || k > 0) ? 1u : 0u);
      mma_commit(smem_u32(&empty[s]));
    }
    // tfull completes when every MMA issued above has; waiting for it here too
    // keeps TMEM from being released under a running MMA on any path
    mma_commit(smem_u32(tfull));
    mbar_wait(smem_u32(tfull), 0u, err, 34);
  } else if (warp >= 2) {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 = tile rows; each
    // thread stores its row's 128 columns
    const int q = warp & 3;
    const bool ready = mbar_wait_ab(smem_u32(tfull), 0u, err, 35, abort);
    __syncwarp();
    if (__all_sync(0xffffffffu, ready)) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int row = ib * kGT + q * 32 + lane;
      int* prow = P + (size_t)row * ldp + jb * kGT;
#pragma unroll 1
      for (int c0 = 0; c0 < kGT; c0 += 32) {
        uint32_t r[32];
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c0, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int c = 0; c < 32; c += 4)
          *reinterpret_cast<int4*>(prow + c0 + c) = make_int4((int)r[c], (int)r[c + 1], (int)r[c + 2], (int)r[c + 3]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kGT) : "memory");
  }
}

// G[s][s'] from the digit products (see the file header); one thread each
__global__ void __launch_bounds__(256) k_gram_combine(const int* __restrict__ P, int ldp, const int* __restrict__ E,
                                                      int S, double2* __restrict__ G) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= S * S) return;
  const int s = i / S, s2 = i - s * S;
  auto p = [&](int r, int c) -> double {  // P is stored in its upper tiles only
    return (double)((r / kGT <= c / kGT) ? P[(size_t)r * ldp + c] : P[(size_t)c * ldp + r]);
  };
  double re = 0.0, im = 0.0;
#pragma unroll
  for (int tu = 6; tu >= 0; --tu) {  // smallest weights first
    double pr = 0.0, pi = 0.0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int u = tu - t;
      if (u < 0 || u > 3) continue;
      const int rx = t * S + s, ry = (4 + t) * S + s, cx = u * S + s2, cy = (4 + u) * S + s2;
      pr += p(rx, cx) + p(ry, cy);
      pi += p(rx, cy) - p(ry, cx);
    }
    re += ldexp(pr, -7 * tu);
    im += ldexp(pi, -7 * tu);
  }
  const int sh = E[s] + E[s2] - 12;
  G[i] = make_double2(ldexp(re, sh), s == s2 ? 0.0 : ldexp(im, sh));
}

}  // namespace

bool gram_i8_supported(int N, int S) {
  if (N < 1 || N > kGMaxN || S < 1 || S > kGramI8MaxS) return false;
  int dev = 0, major = 0, minor = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) ||
      cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev)) {
    (void)cudaGetLastError();
    return false;
  }
  return major == 10 && minor == 0;
}

int gram_i8(const float2* A, int N, int S, double2* G, int* err_dev, cudaStream_t st) {
  KL_CHECK_ARG(A && G && err_dev && N >= 1 && N <= kGMaxN && S >= 1 && S <= kGramI8MaxS, "gram_i8: bad arguments");
  const int R = 8 * S, nt = (R + kGT - 1) / kGT, Rp = nt * kGT;
  const int Kp = (N + kGT - 1) / kGT * kGT;
  const size_t zbytes = (size_t)Rp * Kp, pbytes = sizeof(int) * (size_t)Rp * Rp;
  const size_t bytes = zbytes + pbytes + sizeof(unsigned) * S + sizeof(int) * S + 256;
  void* buf = nullptr;
  if (int rc = scratch_alloc(&buf, bytes, st, "Gram work")) return rc;
  int8_t* Z = static_cast<int8_t*>(buf);
  int* P = reinterpret_cast<int*>(static_cast<char*>(buf) + zbytes);
  unsigned* colmax = reinterpret_cast<unsigned*>(static_cast<char*>(buf) + zbytes + pbytes);
  int* E = reinterpret_cast<int*>(colmax + S);
  int rc = KL_OK;
  CUtensorMap mz;
  do {
    if (cudaMemsetAsync(Z, 0, zbytes, st) != cudaSuccess || cudaMemsetAsync(colmax, 0, sizeof(unsigned) * S, st)) {
      set_error("gram_i8: cudaMemsetAsync failed");
      rc = KL_ERR_CUDA;
      break;
    }
    constexpr int kRows = 64;
    k_gram_colmax<<<(N + kRows - 1) / kRows, 256, 0, st>>>(A, N, S, kRows, colmax);
    const int nthreads = S * ((N + 15) / 16);
    k_gram_digits<<<(nthreads + 255) / 256, 256, 0, st>>>(A, N, S, Kp, colmax, Z, E);
    if ((rc = make_map_1b(&mz, Z, Rp, Kp, kGT, kGT))) break;
    if (cudaFuncSetAttribute(k_gram_i8_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kGSmem) != cudaSuccess) {
      set_error("gram_i8: shared memory attribute refused");
      rc = KL_ERR_CUDA;
      break;
    }
    k_gram_i8_gemm<<<nt * (nt + 1) / 2, kGThreads, kGSmem, st>>>(mz, Kp / kGT, nt, Rp, P, err_dev);
    k_gram_combine<<<(S * S + 255) / 256, 256, 0, st>>>(P, Rp, E, S, G);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error(std::string("gram_i8: ") + cudaGetErrorString(e));
      rc = KL_ERR_CUDA;
    }
  } while (false);
  scratch_free(buf, st);
  return rc;
}

}  // namespace kl
