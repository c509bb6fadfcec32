// tcc.cu -- TCC assembly (K-Litho-TCC/klitho_tcc.cpp:186-267 calcTCC).
//
// The reference accumulates TCC[f1][f2] += J(s) P(f1,s) conj P(f2,s) over
// source points.  That is the Hermitian product TCC = A A^H with
// A[f][s] = sqrt(J_s) P(f, s).  Fast path: A is sampled in FP32 on the GPU and
// the product runs on the 5th-generation tensor cores as real GEMMs on a
// 3-term BF16 split (hi*hi + hi*lo + lo*hi), FP32 accumulation in TMEM:
//     TCC_re = [Ar Ai](hi,hi,lo) . [Ar Ai](hi,lo,hi)^T
//     TCC_im = [Ai -Ar](hi,hi,lo) . [Ar Ai](hi,lo,hi)^T
// 128 x 128 upper tiles on persistent CTAs (one per SM): a TMA producer
// thread streams 128 x 64 bf16 tiles (128-byte swizzle) through a 4-stage
// mbarrier pipeline, one thread issues tcgen05.mma into one of two TMEM
// accumulator sets (each re, im), and four warps drain the other set with
// tcgen05.ld, writing the tile and its conjugate transpose (coalesced) so the
// result is exactly Hermitian.
// FP64 path: the same sum accumulated in FP64 on the CUDA cores from the
// reference-identical pupil table.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kl_internal.h"
#include "kl_tc.cuh"
#include "kl_tcc.h"

namespace kl {

// ---------------------------------------------------------------------------
// host: source points and the reference pupil table
// ---------------------------------------------------------------------------
void tcc_source_points(const float* src, int srcSize, float outerSigma, float lambda, float NA,
                       float defocus, double n_medium, int Lx, int Ly, int Nx, int Ny,
                       std::vector<SrcPoint>& pts, PupilParams& pp) {
  // float arithmetic of klitho_tcc.cpp:189-197 and :202-211
  const int sh = (int)((srcSize - 1) / 2.0);
  const float sig = outerSigma > 1.0f ? 1.0f : outerSigma;
  const int oSgm = (int)std::ceil((float)sh * sig);
  const float dz = defocus / (NA * NA / lambda);
  const float k = (float)(2 * M_PI / lambda);
  const float Lxn = (float)Lx * NA / lambda, Lyn = (float)Ly * NA / lambda;
  pts.clear();
  for (int q = -oSgm; q <= oSgm; ++q)
    for (int p = -oSgm; p <= oSgm; ++p) {
      const int id = (q + sh) * srcSize + p + sh;
      if (src[id] != 0.0f && p * p + q * q <= sh * sh) {
        SrcPoint t;
        t.sx = (float)p / (float)sh;
        t.sy = (float)q / (float)sh;
        t.J = src[id];
        t.nxmin = (int)((-1.0f - t.sx) * Lxn);
        t.nxmax = (int)((1.0f - t.sx) * Lxn);
        t.nymin = (int)((-1.0f - t.sy) * Lyn);
        t.nymax = (int)((1.0f - t.sy) * Lyn);
        t.src_id = id;
        pts.push_back(t);
      }
    }
  pp.Nx = Nx;
  pp.Ny = Ny;
  pp.N = (2 * Nx + 1) * (2 * Ny + 1);
  pp.S = (int)pts.size();
  pp.Lx_norm = Lxn;
  pp.Ly_norm = Lyn;
  pp.dzk = dz * k;
  pp.NA = NA;
  pp.n_medium2 = n_medium * n_medium;
}

void tcc_pupil_host(const std::vector<SrcPoint>& pts, const PupilParams& pp, double* P) {
  const int N = pp.N, S = pp.S, bw = 2 * pp.Nx + 1;
  std::memset(P, 0, sizeof(double) * 2 * (size_t)N * S);
  for (int s = 0; s < S; ++s) {
    const SrcPoint& t = pts[s];
    for (int ny = t.nymin; ny <= t.nymax; ++ny) {
      const float fy = (float)ny / pp.Ly_norm + t.sy;
      if (!(fy * fy <= 1.0f)) continue;
      for (int nx = t.nxmin; nx <= t.nxmax; ++nx) {
        const float fx = (float)nx / pp.Lx_norm + t.sx;
        const float rho2 = fx * fx + fy * fy;
        if (!(rho2 <= 1.0f)) continue;
        if (ny < -pp.Ny || ny > pp.Ny || nx < -pp.Nx || nx > pp.Nx) continue;
        const float ph = (float)((double)pp.dzk * std::sqrt(pp.n_medium2 - (double)(rho2 * pp.NA * pp.NA)));
        const size_t f = (size_t)((ny + pp.Ny) * bw + nx + pp.Nx);
        P[2 * (f * S + s)] = (double)cosf(ph);
        P[2 * (f * S + s) + 1] = (double)sinf(ph);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// device: A = sqrt(J) P in FP32, same float roundings as the reference
// ---------------------------------------------------------------------------
__global__ void k_build_A(const SrcPoint* __restrict__ pts, const PupilParams pp,
                          float2* __restrict__ A) {
  const int bw = 2 * pp.Nx + 1;
  const size_t n = (size_t)pp.N * pp.S;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(i / pp.S), s = (int)(i % pp.S);
    const int ny = f / bw - pp.Ny, nx = f % bw - pp.Nx;
    const SrcPoint t = pts[s];
    float2 v = make_float2(0.f, 0.f);
    if (ny >= t.nymin && ny <= t.nymax && nx >= t.nxmin && nx <= t.nxmax) {
      const float fy = __fadd_rn(__fdiv_rn((float)ny, pp.Ly_norm), t.sy);
      const float fx = __fadd_rn(__fdiv_rn((float)nx, pp.Lx_norm), t.sx);
      const float rho2 = __fadd_rn(__fmul_rn(fx, fx), __fmul_rn(fy, fy));
      if (__fmul_rn(fy, fy) <= 1.0f && rho2 <= 1.0f) {
        const float r2na = __fmul_rn(__fmul_rn(rho2, pp.NA), pp.NA);
        const double arg = __dsub_rn(pp.n_medium2, (double)r2na);
        const float ph = __double2float_rn(__dmul_rn((double)pp.dzk, sqrt(arg)));
        float sn, cs;
        sincosf(ph, &sn, &cs);
        const float a = sqrtf(t.J);
        v = make_float2(a * cs, a * sn);
      }
    }
    A[i] = v;
  }
}

int tcc_build_A(const SrcPoint* pts_dev, const PupilParams& pp, float2* A, cudaStream_t st) {
  const size_t n = (size_t)pp.N * pp.S;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_build_A<<<blocks > 0 ? blocks : 1, 256, 0, st>>>(pts_dev, pp, A);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

// ---------------------------------------------------------------------------
// bf16 split operands
// ---------------------------------------------------------------------------
// Four planes of N x K2p bf16, K2p = round_up(2 S, 32), one after another in
// one buffer: X1h, X2h, X1l, X2l.  With a = A[f][s] split as
// a = ah + al (ah = bf16(a), al = bf16(a - ah)), the K index k < S holds the
// real part of source point s = k, S <= k < 2S the imaginary part of s = k - S:
//   X1 = (ar, ai), X2 = (ai, -ar), each as hi and lo planes, and Y = X1, so
//   Re TCC = X1h Yh^T + X1h Yl^T + X1l Yh^T, Im TCC = the same with X2
// (the three split terms; the lo x lo term is dropped), Y's tiles being X1's
// rows of the other tile index.  Each hi tile is loaded once per k block and
// used by two MMAs.
int tcc_kp(int S) { return ((2 * S + 31) / 32) * 32; }

__global__ void k_tcc_split(const float2* __restrict__ A, int N, int S, int K2p, __nv_bfloat16* __restrict__ ops) {
  const size_t n = (size_t)N * K2p, plane = n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(i / K2p), k = (int)(i % K2p);
    float x1h = 0.f, x2h = 0.f, x1l = 0.f, x2l = 0.f;
    if (k < 2 * S) {
      const int s = k < S ? k : k - S;
      const float2 a = A[(size_t)f * S + s];
      const float rh = __bfloat162float(__float2bfloat16_rn(a.x)), ih = __bfloat162float(__float2bfloat16_rn(a.y));
      const float rl = __bfloat162float(__float2bfloat16_rn(a.x - rh));
      const float il = __bfloat162float(__float2bfloat16_rn(a.y - ih));
      if (k < S) {
        x1h = rh; x2h = ih; x1l = rl; x2l = il;
      } else {
        x1h = ih; x2h = -rh; x1l = il; x2l = -rl;
      }
    }
    ops[i] = __float2bfloat16_rn(x1h);              // X1h
    ops[plane + i] = __float2bfloat16_rn(x2h);      // X2h
    ops[2 * plane + i] = __float2bfloat16_rn(x1l);  // X1l
    ops[3 * plane + i] = __float2bfloat16_rn(x2l);  // X2l
  }
}

int tcc_split_operands(const float2* A, int N, int S, int K2p, void* ops, cudaStream_t st) {
  const size_t n = (size_t)N * K2p;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  k_tcc_split<<<blocks > 0 ? blocks : 1, 256, 0, st>>>(A, N, S, K2p, (__nv_bfloat16*)ops);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

// ---------------------------------------------------------------------------
// tcgen05 Hermitian GEMM
// ---------------------------------------------------------------------------
namespace {
// K blocks of 32 bf16: rows of 64 bytes in the 64-byte swizzle, so that four
// stages fit in shared memory and three K blocks are in flight while one is
// multiplied
constexpr int TM = 128, TN = 128, TK = 32;
constexpr int TILE_BYTES = TM * TK * 2;         // 8 KB, one 128 x 32 bf16 tile
constexpr int STAGE_BYTES = 6 * TILE_BYTES;     // X1h X2h | X1l X2l | Yh | Yl
// One MMA computes re and im of a tile: A = the Y tile (128 rows j), B = the X1
// and X2 tiles stacked (256 rows: X1 then X2, adjacent in shared memory), so
// the accumulator holds re[i][j] in columns i and im[i][j] in columns 128 + i
// of lane j, and each k step reads Y once instead of twice.
// Instruction descriptor: dense, f32 accumulate, bf16 A/B, both K-major, M=128, N=256.
constexpr uint32_t IDESC = tc::idesc_f16(TM, 2 * TN, true);

using tc::mbar_arrive;
using tc::mbar_expect_tx;
using tc::mbar_init;
using tc::mbar_wait;
using tc::mbar_wait_ab;
using tc::mma_commit;
using tc::smem_desc_sw64;
using tc::smem_u32;
using tc::tma_load_2d;
using tc::tmem_ld32;
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accum) {
  tc::mma_f16(tmem_d, da, db, IDESC, accum);
}
}  // namespace

// Persistent, warp-specialised: one CTA per SM walks the upper tiles
// blockIdx.x, blockIdx.x + gridDim.x, ...  Warp 0 (one thread) streams the
// operand tiles through kStages shared-memory stages with TMA; warp 1 (one
// thread) issues the MMAs of a tile into one of two TMEM accumulator sets
// while warps 2..5 drain the other set (tcgen05.ld, then the tile and its
// conjugate transpose to global memory through their own staging buffers), so
// loads, MMAs and stores of consecutive tiles overlap.  Every wait is bounded:
// a timeout records `err`, raises the CTA's abort flag and every role stops.
namespace {
constexpr int kStages = 4;
constexpr int kEpiWarps = 4;
constexpr int kGemmThreads = 32 * (2 + kEpiWarps);
constexpr int EPI_BYTES = kEpiWarps * 32 * 33 * 8;  // per epilogue warp a 32 x 33 float2 tile
constexpr int PSMEM_BYTES = kStages * STAGE_BYTES + EPI_BYTES + 1024 + 128;
constexpr uint32_t PTMEM_COLS = 512;  // two accumulator sets of (re 128 | im 128)

__device__ __forceinline__ void upper_tile(int t, int nt, int& ib, int& jb) {
  int rowlen = nt;
  ib = 0;
  while (t >= rowlen) {
    t -= rowlen;
    ++ib;
    --rowlen;
  }
  jb = ib + t;
}
}  // namespace

__global__ void __launch_bounds__(kGemmThreads, 1)
    k_tcc_gemm(const __grid_constant__ CUtensorMap tmO, int N, int nkb, int nt, float2* __restrict__ tcc,
               int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  float2* epi = reinterpret_cast<float2*>(smem + kStages * STAGE_BYTES);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * STAGE_BYTES + EPI_BYTES);
  uint64_t* empty = full + kStages;
  uint64_t* tfull = empty + kStages;   // accumulator set ready for the epilogue
  uint64_t* tempty = tfull + 2;        // accumulator set drained
  uint64_t* drain = tempty + 2;        // the MMA thread's last MMAs (abort path)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  __shared__ int s_abort;
  volatile int* abort = &s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tiles = nt * (nt + 1) / 2;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&tfull[a]), 1);
      mbar_init(smem_u32(&tempty[a]), kEpiWarps);
    }
    mbar_init(smem_u32(drain), 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(PTMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // TMA producer: k-block `it` of the CTA's run goes to stage it % kStages
    int armed[kStages];
    for (int s = 0; s < kStages; ++s) armed[s] = -1;
    bool ok = true;
    int it = 0;
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
      int ib, jb;
      upper_tile(t, nt, ib, jb);
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int s = it % kStages, use = it / kStages;
        if (use > 0 && !(ok = mbar_wait_ab(smem_u32(&empty[s]), (uint32_t)((use - 1) & 1), err, 1, abort))) break;
        const uint32_t bar = smem_u32(&full[s]);
        mbar_expect_tx(bar, STAGE_BYTES);
        // planes of the operand buffer: X1h rows 0.., X2h rows N.., X1l rows
        // 2N.., X2l rows 3N..; Y's tiles are X1's rows of tile jb
        uint8_t* st = smem + s * STAGE_BYTES;
        tma_load_2d(smem_u32(st), &tmO, kb * TK, ib * TM, bar);
        tma_load_2d(smem_u32(st + TILE_BYTES), &tmO, kb * TK, N + ib * TM, bar);
        tma_load_2d(smem_u32(st + 2 * TILE_BYTES), &tmO, kb * TK, 2 * N + ib * TM, bar);
        tma_load_2d(smem_u32(st + 3 * TILE_BYTES), &tmO, kb * TK, 3 * N + ib * TM, bar);
        tma_load_2d(smem_u32(st + 4 * TILE_BYTES), &tmO, kb * TK, jb * TN, bar);
        tma_load_2d(smem_u32(st + 5 * TILE_BYTES), &tmO, kb * TK, 2 * N + jb * TN, bar);
        armed[s] = use;
      }
    }
    // every issued copy lands before the CTA can retire (its stage parity is known)
    for (int s = 0; s < kStages; ++s)
      if (armed[s] >= 0) mbar_wait(smem_u32(&full[s]), (uint32_t)(armed[s] & 1), err, 4);
  } else if (warp == 1 && lane == 0) {
    // MMA issuer: tile number `tl` of the run accumulates into set tl & 1
    bool ok = true;
    int it = 0, tl = 0;
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x, ++tl) {
      const int a = tl & 1, ause = tl >> 1;
      if (ause > 0 && !(ok = mbar_wait_ab(smem_u32(&tempty[a]), (uint32_t)((ause - 1) & 1), err, 5, abort))) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t acc = tmem + (uint32_t)(a * 256);
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int s = it % kStages, use = it / kStages;
        if (!(ok = mbar_wait_ab(smem_u32(&full[s]), (uint32_t)(use & 1), err, 2, abort))) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t xh = smem_u32(smem + s * STAGE_BYTES), xl = xh + 2 * TILE_BYTES;
        const uint32_t yh = xh + 4 * TILE_BYTES, yl = xh + 5 * TILE_BYTES;
#pragma unroll
        for (int k = 0; k < TK / 16; ++k) {
          const uint32_t accum = (kb > 0 || k > 0) ? 1u : 0u;
          const uint32_t off = (uint32_t)(k * 32);  // 16 bf16 along K inside the swizzle atom
          mma_bf16(acc, smem_desc_sw64(yh + off), smem_desc_sw64(xh + off), accum);
          mma_bf16(acc, smem_desc_sw64(yl + off), smem_desc_sw64(xh + off), 1u);
          mma_bf16(acc, smem_desc_sw64(yh + off), smem_desc_sw64(xl + off), 1u);
        }
        mma_commit(smem_u32(&empty[s]));
      }
      if (ok) mma_commit(smem_u32(&tfull[a]));
    }
    // the MMAs issued so far complete before TMEM can be released
    mma_commit(smem_u32(drain));
    mbar_wait(smem_u32(drain), 0u, err, 6);
  } else if (warp >= 2) {
    // epilogue: warp w drains TMEM lanes 32 (w % 4) .. + 31, i.e. tile columns
    // j = jb TN + 32 (w % 4) + lane; each lane holds re and im of TCC[i][j] for
    // the tile's i in its TMEM columns
    const int q = warp & 3;
    float2* stage = epi + (warp - 2) * 32 * 33;
    int tl = 0;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++tl) {
      const int a = tl & 1, ause = tl >> 1;
      const bool ready = mbar_wait_ab(smem_u32(&tfull[a]), (uint32_t)(ause & 1), err, 3, abort);
      __syncwarp();
      if (!__all_sync(0xffffffffu, ready)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      int ib, jb;
      upper_tile(t, nt, ib, jb);
      const int r = q * 32 + lane;  // tile column of this lane
      const int j = jb * TN + r;
      const bool diag = ib == jb;
      const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * 256);
#pragma unroll 1
      for (int c0 = 0; c0 < TM; c0 += 32) {
        uint32_t re[32], im[32];
        tmem_ld32(base + (uint32_t)c0, re);
        tmem_ld32(base + 128u + (uint32_t)c0, im);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        // TCC[i][j] (i <= j): consecutive lanes write consecutive j
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int i = ib * TM + c0 + c;
          if (i < N && j < N && (!diag || r >= c0 + c)) {
            float2 v = make_float2(__uint_as_float(re[c]), __uint_as_float(im[c]));
            if (diag && r == c0 + c) v.y = 0.f;
            tcc[(size_t)i * N + j] = v;
          }
        }
        // TCC[j][i] = conj TCC[i][j] (i < j, the lower triangle of a diagonal
        // tile): the warp's 32 x 32 block goes through its staging buffer so
        // that each store writes 32 consecutive i of one row j
#pragma unroll
        for (int c = 0; c < 32; ++c) stage[lane * 33 + c] = make_float2(__uint_as_float(re[c]), -__uint_as_float(im[c]));
        __syncwarp();
        {
          const int i = ib * TM + c0 + lane;
#pragma unroll 4
          for (int rr = 0; rr < 32; ++rr) {
            const int col = q * 32 + rr, jj = jb * TN + col;
            if (jj < N && i < N && (!diag || c0 + lane < col)) tcc[(size_t)jj * N + i] = stage[rr * 33 + lane];
          }
        }
        __syncwarp();
      }
      // this set's TMEM is read: the MMAs of tile tl + 2 may overwrite it
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&tempty[a]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(PTMEM_COLS)
                 : "memory");
  }
}

namespace {
int make_map(CUtensorMap* m, const void* base, int rows, int Kp) {
  return tc::make_map_2b(m, base, rows, Kp, TK, TM, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, CU_TENSOR_MAP_SWIZZLE_64B);
}
}  // namespace

int tcc_gemm_tc(const void* ops, int N, int K2p, float2* tcc, int* err_dev, cudaStream_t st) {
  KL_CHECK_ARG(N > 0 && K2p > 0 && K2p % TK == 0, "tcc_gemm_tc: bad sizes");
  KL_CHECK_ARG((uintptr_t)ops % 16 == 0, "tcc_gemm_tc: operands must be 16-byte aligned");
  CUtensorMap mo;
  int rc;
  if ((rc = make_map(&mo, ops, 4 * N, K2p))) return rc;
  const int nt = (N + TM - 1) / TM;
  const int tiles = nt * (nt + 1) / 2;
  int dev = 0, sms = 0;
  KL_CUDA_TRY(cudaGetDevice(&dev));
  KL_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  KL_CUDA_TRY(cudaFuncSetAttribute(k_tcc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, PSMEM_BYTES));
  k_tcc_gemm<<<std::min(tiles, std::max(1, sms)), kGemmThreads, PSMEM_BYTES, st>>>(mo, N, K2p / TK, nt, tcc, err_dev);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

// ---------------------------------------------------------------------------
// FP64 direct TCC: tcc[i][j] = sum_s J_s P[i][s] conj P[j][s], upper tiles + mirror
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_tcc_direct(const double2* __restrict__ P,
                                                    const float* __restrict__ J, int N, int S,
                                                    int nt, double2* __restrict__ tcc) {
  constexpr int T = 32, TKS = 16;
  __shared__ double2 sa[TKS][T + 1];
  __shared__ double2 sb[TKS][T + 1];
  int t = blockIdx.x, ib = 0, rowlen = nt;
  while (t >= rowlen) {
    t -= rowlen;
    ++ib;
    --rowlen;
  }
  const int jb = ib + t;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double2 acc[2][2] = {};
  for (int s0 = 0; s0 < S; s0 += TKS) {
    for (int i = threadIdx.x; i < TKS * T; i += 256) {
      const int kk = i / T, r = i - kk * T, s = s0 + kk;
      const int gi = ib * T + r, gj = jb * T + r;
      double2 a = make_double2(0, 0), b = make_double2(0, 0);
      if (s < S && gi < N) {
        const double2 p = P[(size_t)gi * S + s];
        const double w = (double)J[s];
        a = make_double2(p.x * w, p.y * w);
      }
      if (s < S && gj < N) {
        const double2 p = P[(size_t)gj * S + s];
        b = make_double2(p.x, -p.y);
      }
      sa[kk][r] = a;
      sb[kk][r] = b;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < TKS; ++kk) {
      const double2 a0 = sa[kk][ty], a1 = sa[kk][ty + 16], b0 = sb[kk][tx], b1 = sb[kk][tx + 16];
      acc[0][0] = make_double2(fma(a0.x, b0.x, fma(-a0.y, b0.y, acc[0][0].x)), fma(a0.x, b0.y, fma(a0.y, b0.x, acc[0][0].y)));
      acc[0][1] = make_double2(fma(a0.x, b1.x, fma(-a0.y, b1.y, acc[0][1].x)), fma(a0.x, b1.y, fma(a0.y, b1.x, acc[0][1].y)));
      acc[1][0] = make_double2(fma(a1.x, b0.x, fma(-a1.y, b0.y, acc[1][0].x)), fma(a1.x, b0.y, fma(a1.y, b0.x, acc[1][0].y)));
      acc[1][1] = make_double2(fma(a1.x, b1.x, fma(-a1.y, b1.y, acc[1][1].x)), fma(a1.x, b1.y, fma(a1.y, b1.x, acc[1][1].y)));
    }
    __syncthreads();
  }
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b < 2; ++b) {
      const int i = ib * T + ty + 16 * a, j = jb * T + tx + 16 * b;
      if (i < N && j < N && j >= i) {
        double2 v = acc[a][b];
        if (i == j) v.y = 0.0;
        tcc[(size_t)i * N + j] = v;
        if (j > i) tcc[(size_t)j * N + i] = make_double2(v.x, -v.y);
      }
    }
}

int tcc_direct_fp64(const double2* P, const float* J, int N, int S, double2* tcc, cudaStream_t st) {
  const int nt = (N + 31) / 32;
  k_tcc_direct<<<nt * (nt + 1) / 2, 256, 0, st>>>(P, J, N, S, nt, tcc);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

// ---------------------------------------------------------------------------
// Hopkins image through the factor: H_s[f] = conj A[f][s], weight 1
// ---------------------------------------------------------------------------
__global__ void k_factor_kernels(const float2* __restrict__ A, int N, int S, float2* __restrict__ H,
                                 float* __restrict__ lam) {
  const size_t n = (size_t)N * S;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(i / N), f = (int)(i % N);
    const float2 a = A[(size_t)f * S + s];
    H[i] = make_float2(a.x, -a.y);
    if (f == 0) lam[s] = 1.0f;
  }
}

int tcc_factor_kernels(const float2* A, int N, int S, float2* H, float* lam, cudaStream_t st) {
  k_factor_kernels<<<296, 256, 0, st>>>(A, N, S, H, lam);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

// ---------------------------------------------------------------------------
// min / max of the real and imaginary parts
// ---------------------------------------------------------------------------
template <typename C>
__global__ void k_minmax(const C* __restrict__ m, size_t n, double* __restrict__ out) {
  double mxr = -1e300, mnr = 1e300, mxi = -1e300, mni = 1e300;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double r = (double)m[i].x, im = (double)m[i].y;
    mxr = fmax(mxr, r);
    mnr = fmin(mnr, r);
    mxi = fmax(mxi, im);
    mni = fmin(mni, im);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mxr = fmax(mxr, __shfl_xor_sync(0xffffffffu, mxr, o));
    mnr = fmin(mnr, __shfl_xor_sync(0xffffffffu, mnr, o));
    mxi = fmax(mxi, __shfl_xor_sync(0xffffffffu, mxi, o));
    mni = fmin(mni, __shfl_xor_sync(0xffffffffu, mni, o));
  }
  __shared__ double sm[4][32];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sm[0][w] = mxr;
    sm[1][w] = mnr;
    sm[2][w] = mxi;
    sm[3][w] = mni;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
      mxr = fmax(mxr, sm[0][k]);
      mnr = fmin(mnr, sm[1][k]);
      mxi = fmax(mxi, sm[2][k]);
      mni = fmin(mni, sm[3][k]);
    }
    out[4 * blockIdx.x + 0] = fmax(mxr, sm[0][0]);
    out[4 * blockIdx.x + 1] = fmin(mnr, sm[1][0]);
    out[4 * blockIdx.x + 2] = fmax(mxi, sm[2][0]);
    out[4 * blockIdx.x + 3] = fmin(mni, sm[3][0]);
  }
}

template <typename C>
int minmax(const C* m, size_t n, double* out4, cudaStream_t st) {
  const int blocks = 296;
  void* d = nullptr;
  int rc = scratch_alloc(&d, sizeof(double) * 4 * blocks, st, "minmax partials");
  if (rc) return rc;
  k_minmax<C><<<blocks, 256, 0, st>>>(m, n, static_cast<double*>(d));
  std::vector<double> h(4 * blocks);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), d, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st);
  scratch_free(d, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_error(std::string("minmax: ") + cudaGetErrorString(e));
    return KL_ERR_CUDA;
  }
  out4[0] = -1e300;
  out4[1] = 1e300;
  out4[2] = -1e300;
  out4[3] = 1e300;
  for (int b = 0; b < blocks; ++b) {
    out4[0] = std::fmax(out4[0], h[4 * b]);
    out4[1] = std::fmin(out4[1], h[4 * b + 1]);
    out4[2] = std::fmax(out4[2], h[4 * b + 2]);
    out4[3] = std::fmin(out4[3], h[4 * b + 3]);
  }
  return KL_OK;
}

int tcc_minmax_c64(const float2* m, size_t n, double* out4, cudaStream_t st) { return minmax(m, n, out4, st); }
int tcc_minmax_c128(const double2* m, size_t n, double* out4, cudaStream_t st) { return minmax(m, n, out4, st); }

}  // namespace kl
