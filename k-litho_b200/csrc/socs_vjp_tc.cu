// socs_vjp_tc.cu -- the image, resist, loss and row transform of dL/dI of the
// SOCS adjoint (the work of k_vjp_inverse in socs_vjp.cu) on the tensor cores.
//
// For a tile of 128 image rows (128/J strips, y = s + nS j):
//   1. image[y][x] = sum_k A[y][k] B[k][x] as in k_socs_synth_tc: the
//      coefficient warps build A = [Re Q, -Im Q] (FP16 hi/lo, scaled per
//      image) in TMEM from the image's intensity spectrum, the MMA multiplies
//      it with the plan's cos/sin basis, 64 columns at a time;
//   2. the epilogue warps take each 32 x 32 block of the image, read the
//      matching targets (TMA loads, staged ahead), and form the resist
//      s = 1/(1 + e^{-a(I - c)}), the loss (s - t)^2 and G = dL/dI =
//      2 (s - t) s (1 - s) a; G (scaled by a power of two, FP16 hi/lo) goes to
//      TMEM with tcgen05.st;
//   3. a second MMA accumulates the row DFT of G, Gr[y][b] = sum_x G[y][x]
//      e^{-2 pi i b x / Lx} for b <= 2Nx, as G . B2 with B2 the transposed
//      basis (same 3-term FP16 split), over the tile's 64-column blocks;
//   4. at the end of the tile the epilogue warps read Gr, run the J-point
//      column FFTs of each strip and write its partial band spectrum of G
//      (|gy| <= 2Ny, the layout k_vjp_spectral reads), exactly as
//      k_vjp_inverse does on the CUDA cores.
// The model is the adjoint of K-Litho-SOCS/klitho_socs.cpp:158-241 (calcSOCS +
// FI) under the sigmoid resist at the reference's TARGET_INTENSITY
// (K-Litho-TCC/klitho_tcc.cpp:442); no counterpart in the reference.
//
// Roles (448 threads, one CTA per SM): warps 0-3 coefficient warps, warps
// 4-11 epilogue warps (two per TMEM lane quarter, the per-pixel resist math
// needs the latency hiding), warp 12 TMA producer of the basis units (image
// basis and transposed basis, one ring), warp 13 MMA issuer.  TMEM: three 64-column
// image accumulators, two A buffers, two G buffers, the 64-column Gr
// accumulator.  Every wait is bounded; a timeout sets the plan's status word
// and stops every role.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <climits>
#include <cstdint>

#include "kl_device.cuh"
#include "kl_internal.h"
#include "kl_tc.cuh"

namespace kl {
namespace {
constexpr int vRows = 128;        // tile rows (MMA M, TMEM lanes)
constexpr int vCW = 4;            // coefficient warps
constexpr int vEW = 8;            // epilogue warps: two per TMEM lane quarter, one per 32-column half
constexpr int vThreads = 32 * (vCW + vEW + 2);
constexpr int vProdWarp = vCW + vEW, vMmaWarp = vCW + vEW + 1;
constexpr int vNT = 64;           // image N tile = one 64-column K atom of the second MMA
constexpr int vUnit = 64 * 128;   // basis unit: 64 rows x 128 bytes
constexpr int vStages = 6;        // basis unit ring
constexpr int vTgtBufs = 2;       // target tiles in flight per epilogue warp
constexpr int vImgBufs = 1;       // image staging tiles per epilogue warp
constexpr int vSets = 3;          // image accumulators
constexpr int vScaleRing = 8;
// TMEM columns
constexpr int vAcc = 0;                     // [vSets][64] image accumulators
constexpr int vA1 = vSets * vNT;            // [2][64] A buffers (hi 32 | lo 32)
constexpr int vA2 = vA1 + 2 * 64;           // [2][64] G buffers (hi 32 | lo 32)
constexpr int vD2 = vA2 + 2 * 64;           // 64 columns: Gr accumulator
constexpr int vTmemCols = 512;
static_assert(vD2 + 64 == vTmemCols, "TMEM layout");

__host__ __device__ constexpr int v_ntx8(int ntx) { return (ntx + 7) & ~7; }
__host__ __device__ constexpr int v_tstride(int ntx) { return v_ntx8(ntx) + 2; }
constexpr int vGrStride = 33;  // float2 per row of the staged Gr (32 bins + 1 against bank conflicts)

struct VjpSmem {
  size_t b, tgt, img, gr, ts, ph, bars, total;
};
__host__ __device__ inline VjpSmem vjp_smem(int nty, int ntx, int nst) {
  VjpSmem s{};
  s.b = 0;                                                     // [vStages] basis units
  s.tgt = s.b + (size_t)vStages * vUnit;                       // [vEW][vTgtBufs] 4 KB target tiles
  s.img = s.tgt + (size_t)vEW * vTgtBufs * 4096;               // [vEW][vImgBufs] 4 KB image tiles
  s.gr = s.img + (size_t)vEW * vImgBufs * 4096;                // [128][vGrStride] float2 row bins of G
  s.ts = s.gr + sizeof(float2) * 128 * vGrStride;              // T [nty][tstride] float2
  s.ph = s.ts + sizeof(float2) * (size_t)nty * v_tstride(ntx);  // phases [nst][nty] float2
  s.bars = (s.ph + sizeof(float2) * (size_t)nst * nty + 15) & ~(size_t)15;
  s.total = s.bars + 8 * (2 * vStages + 4 + 2 * vSets + 4 + 2 + vEW * vTgtBufs + 1) + 64;
  return s;
}
constexpr size_t vSmemMax = 227 * 1024 - 1024;
}  // namespace

// plan-time transposed basis of the row DFT: BT[k][x] = cos(2 pi b x / Lx) for
// K index k of (b, part 0), sin(2 pi b x / Lx) for (b, part 1) (b = 8 (k / 16)
// + k % 8, part = (k / 8) % 2), 0 for b >= ntx; FP16 hi and lo halves, [64][Lx]
__global__ void k_vjp_basis_t(int Lx, int ntx, __half* __restrict__ bhi, __half* __restrict__ blo) {
  const size_t n = (size_t)64 * Lx;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i / Lx), x = (int)(i % Lx);
    const int b = 8 * (k >> 4) + (k & 7), part = (k >> 3) & 1;
    float v = 0.f;
    if (b < ntx) {
      const float2 e = expi2pi_frac((long long)b * x, Lx);
      v = part ? e.y : e.x;
    }
    const __half h = __float2half_rn(v);
    bhi[i] = h;
    blo[i] = __float2half_rn(v - __half2float(h));
  }
}

template <int RJ>
__global__ void __launch_bounds__(vThreads, 1)
    k_vjp_synth_tc(const float2* __restrict__ T, const SocsGeom g, const float2* __restrict__ ty, int nsplit,
                   int nsets, const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
                   const __grid_constant__ CUtensorMap tm_thi, const __grid_constant__ CUtensorMap tm_tlo,
                   const __grid_constant__ CUtensorMap tm_img, const __grid_constant__ CUtensorMap tm_tgt,
                   int write_images, float alpha, float thr, float gscale, int nimg, double* __restrict__ loss,
                   float2* __restrict__ gpart, int* __restrict__ err) {
  constexpr int J = 32 * RJ;
  constexpr int NST = vRows / J;  // strips per tile
  constexpr int PHR = 2;          // strip phases per coefficient thread (nst * nty <= 256)
  constexpr uint32_t IDESC = tc::idesc_f16(vRows, 64, false);
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const VjpSmem L = vjp_smem(g.nty, g.ntx, NST);
  uint8_t* bst = smem + L.b;
  uint8_t* tgs = smem + L.tgt;
  uint8_t* ims = smem + L.img;
  float2* grs = reinterpret_cast<float2*>(smem + L.gr);
  float2* Ts = reinterpret_cast<float2*>(smem + L.ts);
  float2* ph = reinterpret_cast<float2*>(smem + L.ph);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars);  // basis unit loaded
  uint64_t* empty = full + vStages;                              // basis unit consumed
  uint64_t* afull = empty + vStages;                             // A buffer written
  uint64_t* aempty = afull + 2;                                  // A buffer consumed
  uint64_t* tfull = aempty + 2;                                  // image accumulator ready
  uint64_t* tempty = tfull + vSets;                              // image accumulator drained
  uint64_t* gfull = tempty + vSets;                              // G buffer written
  uint64_t* gempty = gfull + 2;                                  // G buffer consumed
  uint64_t* dfull = gempty + 2;                                  // Gr of the tile complete
  uint64_t* dempty = dfull + 1;                                  // Gr read
  uint64_t* tgtb = dempty + 1;                                   // [vEW][vTgtBufs] target tile landed
  uint64_t* drain = tgtb + vEW * vTgtBufs;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  __shared__ int s_abort;
  __shared__ float s_scale[2];
  __shared__ float s_inv[vScaleRing];
  __shared__ volatile int s_seq[vScaleRing];
  __shared__ unsigned s_bound;
  volatile int* abort = &s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
  const int ntx = g.ntx, nty = g.nty, A2 = 2 * g.Ny;
  const int tiles_img = g.Ly / vRows, ntile = g.Lx / vNT;
  const int total = nimg * tiles_img;
  const int per = (total + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per, t1 = min(total, t0 + per);
  const size_t tsz = (size_t)nty * ntx;

  if (tid == 0) {
    for (int s = 0; s < vStages; ++s) {
      tc::mbar_init(tc::smem_u32(&full[s]), 1);
      tc::mbar_init(tc::smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(tc::smem_u32(&afull[b]), 1);
      tc::mbar_init(tc::smem_u32(&aempty[b]), 1);
      tc::mbar_init(tc::smem_u32(&gfull[b]), vEW);
      tc::mbar_init(tc::smem_u32(&gempty[b]), 1);
    }
    for (int a = 0; a < vSets; ++a) {
      tc::mbar_init(tc::smem_u32(&tfull[a]), 1);
      tc::mbar_init(tc::smem_u32(&tempty[a]), vEW);
    }
    tc::mbar_init(tc::smem_u32(dfull), 1);
    tc::mbar_init(tc::smem_u32(dempty), vEW);
    for (int i = 0; i < vEW * vTgtBufs; ++i) tc::mbar_init(tc::smem_u32(&tgtb[i]), 1);
    tc::mbar_init(tc::smem_u32(drain), 1);
    for (int i = 0; i < vScaleRing; ++i) s_seq[i] = -1;
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(tmem_slot)),
                 "r"(vTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == vProdWarp) {
    // TMA producer (one lane): the basis units in the order the MMA issuer
    // consumes them: per 64-column block n of a tile the image basis (hi, lo),
    // then the transposed basis of block n - 1 (hi, lo), and after the last
    // block the transposed basis of that block
    if (lane == 0) {
      int u = 0, armed[vStages];
      for (int s = 0; s < vStages; ++s) armed[s] = -1;
      bool ok = true;
      auto put = [&](const CUtensorMap* m, int x, int y) {
        const int s = u % vStages, use = u / vStages;
        if (use > 0 && !(ok = tc::mbar_wait_ab(tc::smem_u32(&empty[s]), (uint32_t)((use - 1) & 1), err, 31, abort)))
          return;
        const uint32_t bar = tc::smem_u32(&full[s]);
        tc::mbar_expect_tx(bar, vUnit);
        tc::tma_load_2d(tc::smem_u32(bst + (size_t)s * vUnit), m, x, y, bar);
        armed[s] = use;
        ++u;
      };
      for (int t = t0; t < t1 && ok; ++t)
        for (int n = 0; n <= ntile && ok; ++n) {
          if (n < ntile) {
            put(&tm_hi, 0, n * vNT);
            if (ok) put(&tm_lo, 0, n * vNT);
          }
          if (n > 0 && ok) {
            put(&tm_thi, (n - 1) * vNT, 0);
            if (ok) put(&tm_tlo, (n - 1) * vNT, 0);
          }
        }
      // no copy may still be writing shared memory when the CTA exits
      for (int s = 0; s < vStages; ++s)
        if (armed[s] >= 0) tc::mbar_wait(tc::smem_u32(&full[s]), (uint32_t)(armed[s] & 1), err, 34);
    }
    __syncwarp();
  } else if (warp == vMmaWarp) {
    // MMA issuer (one lane).  Per tile: image block n into accumulator
    // it % vSets (A from TMEM against the basis units), then the row DFT of G
    // for block n - 1 into the Gr accumulator (G from TMEM against the
    // transposed basis); the A buffer is released after the tile's last image
    // block, Gr is reported complete after its last block.
    if (lane == 0) {
      int it = 0, ti = 0, u = 0, gb = 0;
      bool ok = true;
      auto unit = [&](uint32_t& addr) -> bool {
        const int s = u % vStages, use = u / vStages;
        if (!(ok = tc::mbar_wait_ab(tc::smem_u32(&full[s]), (uint32_t)(use & 1), err, 35, abort))) return false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        addr = tc::smem_u32(bst + (size_t)s * vUnit);
        return true;
      };
      auto release = [&]() {
        tc::mma_commit(tc::smem_u32(&empty[u % vStages]));
        ++u;
      };
      for (int t = t0; t < t1 && ok; ++t, ++ti) {
        const int buf = ti & 1, ause = ti >> 1;
        if (!(ok = tc::mbar_wait_ab(tc::smem_u32(&afull[buf]), (uint32_t)(ause & 1), err, 36, abort))) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t ah = tmem + (uint32_t)(vA1 + 64 * buf), al = ah + 32;
        for (int n = 0; n <= ntile && ok; ++n) {
          if (n < ntile) {
            const int a = it % vSets, tuse = it / vSets;
            if (tuse > 0 &&
                !(ok = tc::mbar_wait_ab(tc::smem_u32(&tempty[a]), (uint32_t)((tuse - 1) & 1), err, 37, abort)))
              break;
            const uint32_t acc = tmem + (uint32_t)(vAcc + a * vNT);
            uint32_t bh, bl;
            if (!unit(bh)) break;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const uint64_t db = tc::smem_desc(bh + k * 32);
              tc::mma_f16_ts(acc, ah + 8 * k, db, IDESC, k ? 1u : 0u);
              tc::mma_f16_ts(acc, al + 8 * k, db, IDESC, 1u);
            }
            release();
            if (!unit(bl)) break;
#pragma unroll
            for (int k = 0; k < 4; ++k) tc::mma_f16_ts(acc, ah + 8 * k, tc::smem_desc(bl + k * 32), IDESC, 1u);
            release();
            tc::mma_commit(tc::smem_u32(&tfull[a]));
            ++it;
            if (n == ntile - 1) tc::mma_commit(tc::smem_u32(&aempty[buf]));
          }
          if (n > 0) {
            // row DFT of G for block m = n - 1
            const int m = n - 1, gbuf = gb & 1, guse = gb >> 1;
            if (!(ok = tc::mbar_wait_ab(tc::smem_u32(&gfull[gbuf]), (uint32_t)(guse & 1), err, 38, abort))) break;
            if (m == 0 && ti > 0 &&
                !(ok = tc::mbar_wait_ab(tc::smem_u32(dempty), (uint32_t)((ti - 1) & 1), err, 39, abort)))
              break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t gh = tmem + (uint32_t)(vA2 + 64 * gbuf), gl = gh + 32, d2 = tmem + (uint32_t)vD2;
            uint32_t th, tl;
            if (!unit(th)) break;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const uint64_t db = tc::smem_desc(th + k * 32);
              tc::mma_f16_ts(d2, gh + 8 * k, db, IDESC, (m | k) ? 1u : 0u);
              tc::mma_f16_ts(d2, gl + 8 * k, db, IDESC, 1u);
            }
            release();
            if (!unit(tl)) break;
#pragma unroll
            for (int k = 0; k < 4; ++k) tc::mma_f16_ts(d2, gh + 8 * k, tc::smem_desc(tl + k * 32), IDESC, 1u);
            release();
            tc::mma_commit(tc::smem_u32(&gempty[gbuf]));
            ++gb;
            if (m == ntile - 1) tc::mma_commit(tc::smem_u32(dfull));
          }
        }
      }
      tc::mma_commit(tc::smem_u32(drain));
      tc::mbar_wait(tc::smem_u32(drain), 0u, err, 40);
    }
    __syncwarp();
  } else if (warp >= vCW) {
    // epilogue warps: warp ew reads TMEM lanes 32 (ew % 4) .. + 31, rows j0 ..
    // j0 + 31 of strip st of the tile (y = s + nS j), and columns 32 hc0 ..
    // 32 hc0 + 31 of every 64-column block
    const int ew = warp - vCW, hc0 = ew >> 2;
    const int r0 = 32 * (warp & 3), st = r0 / J, j0 = r0 - st * J;
    uint8_t* mytg = tgs + (size_t)ew * vTgtBufs * 4096;
    uint8_t* myim = ims + (size_t)ew * vImgBufs * 4096;
    const uint64_t policy = tc::policy_evict_first();
    const uint32_t lanebase = tmem + ((uint32_t)r0 << 16);
    const int ng = 2 * g.Nx + 1, A = 2 * g.Ny;
    const int nchunk = (t1 - t0) * ntile;  // 32 x 32 blocks of this warp
    // target block of chunk q: tile t0 + q / ntile, columns 64 (q % ntile) + 32 hc0
    auto issue_tgt = [&](int q) {
      const int tq = t0 + q / ntile, c32 = 2 * (q % ntile) + hc0;
      const int img = tq / tiles_img, s0 = (tq - img * tiles_img) * NST;
      const int b = q % vTgtBufs;
      const uint32_t bar = tc::smem_u32(&tgtb[ew * vTgtBufs + b]);
      tc::mbar_expect_tx(bar, 4096);
      tc::tma_load_4d(tc::smem_u32(mytg + b * 4096), &tm_tgt, 32 * c32, s0 + st, j0, img / nsets, bar);
    };
    int qi = 0;  // next chunk whose targets are requested (lane 0)
    if (lane == 0)
      for (; qi < min(vTgtBufs, nchunk); ++qi) issue_tgt(qi);
    int it = 0, ti = 0, q = 0, gbk = 0, sb = 0;
    bool ok = true;
    WarpFFT<RJ, -1> wc;
    wc.init(lane);
    const int br = (int)(__brev((unsigned)lane) >> 27);
    for (int t = t0; t < t1; ++t, ++ti) {
      const int img = t / tiles_img, s0 = (t - img * tiles_img) * NST;
      // the tile's inverse scale, published with its tile number
      const int slot = ti % vScaleRing;
      bool seen = true;
      if (lane == 0 && s_seq[slot] != ti) {
        const unsigned long long w0 = tc::now_ns();
        while (s_seq[slot] != ti) {
          if (*abort) {
            seen = false;
            break;
          }
          if (tc::now_ns() - w0 > tc::kWaitNs) {
            atomicExch(err, 41);
            *abort = 1;
            seen = false;
            break;
          }
          __nanosleep(64);
        }
      }
      ok = ok && __shfl_sync(0xffffffffu, seen, 0);
      __threadfence_block();
      const float inv = s_inv[slot];
      double lacc = 0.0;
      for (int n = 0; n < ntile && ok; ++n, ++it) {
        const int a = it % vSets, tuse = it / vSets;
        const bool ready = tc::mbar_wait_ab(tc::smem_u32(&tfull[a]), (uint32_t)(tuse & 1), err, 42, abort);
        if (!__all_sync(0xffffffffu, ready)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int gbuf = gbk & 1, guse = gbk >> 1;
#pragma unroll 1
        for (int hc = hc0; hc < hc0 + 1 && ok; ++hc, ++q) {
          uint32_t v[32];
          tc::tmem_ld32(lanebase + (uint32_t)(vAcc + a * vNT + 32 * hc), v);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          {
            // the warp's half of the accumulator is in registers: hand it back
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(tc::smem_u32(&tempty[a]));
          }
          // the targets of the block (TMA, requested vTgtBufs blocks ahead)
          const int b = q % vTgtBufs;
          const bool landed = tc::mbar_wait_ab(tc::smem_u32(&tgtb[ew * vTgtBufs + b]), (uint32_t)((q / vTgtBufs) & 1),
                                               err, 43, abort);
          if (!__all_sync(0xffffffffu, landed)) {
            ok = false;
            break;
          }
          float tv[32];
#pragma unroll
          for (int c = 0; c < 8; ++c) {
            const float4 f = *reinterpret_cast<const float4*>(mytg + b * 4096 + lane * 128 + ((c ^ (lane & 7)) << 4));
            tv[4 * c] = f.x;
            tv[4 * c + 1] = f.y;
            tv[4 * c + 2] = f.z;
            tv[4 * c + 3] = f.w;
          }
          __syncwarp();  // every lane has read target tile b: request the block vTgtBufs ahead into it
          if (lane == 0 && qi < nchunk && qi == q + vTgtBufs) issue_tgt(qi++);
          // resist, loss and G = dL/dI on the lane's 32 pixels (four partial
          // loss sums keep the dependency chains short)
          float rs[4] = {0.f, 0.f, 0.f, 0.f};
          const float ga = 2.0f * alpha * gscale;
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            const float I = __uint_as_float(v[c]) * inv;
            v[c] = __float_as_uint(I);
            const float sg = __fdividef(1.0f, 1.0f + __expf(-alpha * (I - thr)));
            const float d = sg - tv[c];
            rs[c & 3] = fmaf(d, d, rs[c & 3]);
            tv[c] = ga * d * sg * (1.0f - sg);
          }
          lacc += (double)((rs[0] + rs[1]) + (rs[2] + rs[3]));
          if (write_images) {
            if (lane == 0) tc::bulk_wait_read<vImgBufs - 1>();
            __syncwarp();
            uint8_t* tile = myim + sb * 4096;
#pragma unroll
            for (int c = 0; c < 8; ++c)
              *reinterpret_cast<float4*>(tile + lane * 128 + ((c ^ (lane & 7)) << 4)) =
                  make_float4(__uint_as_float(v[4 * c]), __uint_as_float(v[4 * c + 1]), __uint_as_float(v[4 * c + 2]),
                              __uint_as_float(v[4 * c + 3]));
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) {
              tc::tma_store_4d(&tm_img, tc::smem_u32(tile), n * vNT + 32 * hc, s0 + st, j0, img, policy);
              tc::bulk_commit();
            }
            sb = sb + 1 == vImgBufs ? 0 : sb + 1;
          }
          // G of the block, FP16 hi and lo, into TMEM buffer gbuf
          if (guse > 0) {
            const bool freed =
                tc::mbar_wait_ab(tc::smem_u32(&gempty[gbuf]), (uint32_t)((guse - 1) & 1), err, 44, abort);
            if (!__all_sync(0xffffffffu, freed)) {
              ok = false;
              break;
            }
          }
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          uint32_t hi[16], lo[16];
#pragma unroll
          for (int p = 0; p < 16; ++p) {
            const __half2 h2 = __floats2half2_rn(tv[2 * p], tv[2 * p + 1]);
            const float2 hf = __half22float2(h2);
            const __half2 l2 = __floats2half2_rn(tv[2 * p] - hf.x, tv[2 * p + 1] - hf.y);
            hi[p] = *reinterpret_cast<const uint32_t*>(&h2);
            lo[p] = *reinterpret_cast<const uint32_t*>(&l2);
          }
          tc::tmem_st16(lanebase + (uint32_t)(vA2 + 64 * gbuf + 16 * hc), hi);
          tc::tmem_st16(lanebase + (uint32_t)(vA2 + 64 * gbuf + 32 + 16 * hc), lo);
        }
        if (!ok) break;
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(tc::smem_u32(&gfull[gbuf]));
        ++gbk;
      }
      // the tile's loss
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) lacc += __shfl_xor_sync(0xffffffffu, lacc, o);
      if (ok && lane == 0) atomicAdd(loss + img, lacc);
      // row bins of G for the tile's rows
      if (ok) {
        const bool done = tc::mbar_wait_ab(tc::smem_u32(dfull), (uint32_t)(ti & 1), err, 45, abort);
        ok = __all_sync(0xffffffffu, done);
      }
      if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t d0[32];
        tc::tmem_ld32(lanebase + (uint32_t)(vD2 + 32 * hc0), d0);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(tc::smem_u32(dempty));
        // Gr[b] = sum_x G e^{-2 pi i b x / Lx}: Re from the cos columns, Im =
        // -(sin columns); K index of (b, part) is 16 (b / 8) + 8 part + b % 8,
        // so the warp's 32 columns hold bins 16 hc0 .. 16 hc0 + 15
        const float ig = 1.0f / gscale;
        float2* row = grs + (r0 + lane) * vGrStride;
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int b = 16 * hc0 + 8 * (c >> 4) + (c & 7);
          if (!(c & 8)) row[b] = make_float2(__uint_as_float(d0[c]) * ig, -__uint_as_float(d0[c + 8]) * ig);
        }
      }
      // the epilogue warps go on or leave together (a named-barrier OR)
      int stop;
      asm volatile(
          "{\n\t.reg .pred p, q;\n\t"
          "setp.ne.s32 p, %1, 0;\n\t"
          "bar.red.or.pred q, 2, %2, p;\n\t"
          "selp.s32 %0, 1, 0, q;\n\t}"
          : "=r"(stop)
          : "r"((!ok || *abort) ? 1 : 0), "r"(32 * vEW)
          : "memory");
      if (stop) {
        ok = false;
        break;
      }
      // column DFT of each strip: bins gy in [-2Ny, 2Ny] (J >= 4Ny+1), times
      // e^{-2 pi i gy s / Ly}: the strip's partial band spectrum of G
      for (int task = ew; task < NST * ng; task += vEW) {
        const int s2 = task / ng, gx = task - s2 * ng;
        float2 vv[RJ];
#pragma unroll
        for (int j = 0; j < RJ; ++j) vv[j] = grs[(s2 * J + lane + 32 * j) * vGrStride + gx];
        wc.run(vv, lane);
        const int s = s0 + s2;
#pragma unroll
        for (int q1 = 0; q1 < RJ; ++q1) {
          const int bin = q1 + RJ * br;
          const int gy = bin <= J / 2 ? bin : bin - J;
          if (gy >= -A && gy <= A)
            gpart[(((size_t)img * g.nS + s) * nty + (gy + A)) * ng + gx] =
                cmulc(vv[q1], __ldg(ty + (size_t)s * nty + gy + A));
        }
      }
      asm volatile("bar.sync 2, %0;" ::"r"(32 * vEW) : "memory");  // the staged bins are read
    }
    // no TMA copy may still be writing or reading this warp's tiles at exit
    if (lane == 0) {
      for (int qq = q; qq < qi; ++qq)
        tc::mbar_wait(tc::smem_u32(&tgtb[ew * vTgtBufs + qq % vTgtBufs]), (uint32_t)((qq / vTgtBufs) & 1), err, 46);
      tc::bulk_wait_all();
    }
    __syncwarp();
  } else {
    // coefficient warps: warp w writes TMEM lanes 32w .. 32w + 31, rows
    // jw .. jw + 31 of strip sw of the tile (all 8-column groups)
    const int sw = (32 * warp) / J, jw = 32 * warp - sw * J;
    const int br = (int)(__brev((unsigned)lane) >> 27);
    // lane of the FFT output that holds row jw + lane, and its register
    const int R = jw + lane, qsel = R % RJ, src = (int)(__brev((unsigned)(R / RJ)) >> 27);
    const uint32_t lanebase = tmem + ((uint32_t)(32 * warp) << 16);
    const int nph = NST * nty;
    const int ng = v_ntx8(ntx) / 8;  // 8-column groups
    const int tstr = v_tstride(ntx);
    (void)br;
    int cur_img = -1, ti = 0;
    WarpFFT<RJ, +1> wf;
    wf.init(lane);
    // the K padding (columns 8 ng .. 32 of each half) is zero once for both buffers
    {
      uint32_t z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int c = 8 * ng; c < 32; c += 8)
        for (int hb = 0; hb < 4; ++hb) tc::tmem_st8(lanebase + (uint32_t)(vA1 + hb * 32 + c), z);
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    // phases e^{2 pi i a s / Ly} of the next tile's strips, held in registers
    float2 phn[PHR];
    auto load_ph = [&](int t) {
      const int img = t / tiles_img, s0 = (t - img * tiles_img) * NST;
#pragma unroll
      for (int k = 0; k < PHR; ++k) {
        const int i = tid + 32 * vCW * k;
        if (i < nph) {
          const int st = i / nty;
          phn[k] = __ldg(ty + (size_t)(s0 + st) * nty + (i - st * nty));
        }
      }
    };
    if (t0 < t1) load_ph(t0);
    for (int t = t0; t < t1; ++t, ++ti) {
      const int img = t / tiles_img;
      const int buf = ti & 1, ause = ti >> 1;
      bool ok = true;
      if (ause > 0) ok = tc::mbar_wait_ab(tc::smem_u32(&aempty[buf]), (uint32_t)((ause - 1) & 1), err, 47, abort);
      // the four warps go on or leave together (a named-barrier OR)
      int stop;
      asm volatile(
          "{\n\t.reg .pred p, q;\n\t"
          "setp.ne.s32 p, %1, 0;\n\t"
          "bar.red.or.pred q, 1, %2, p;\n\t"
          "selp.s32 %0, 1, 0, q;\n\t}"
          : "=r"(stop)
          : "r"((!ok || *abort) ? 1 : 0), "r"(32 * vCW)
          : "memory");
      if (stop) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      // the image's spectrum (slices summed, rows padded with zeros) and the
      // power-of-two scale of A
      if (img != cur_img) {
        cur_img = img;
        if (tid == 0) s_bound = 0u;
        const float2* Ti = T + (size_t)img * nsplit * tsz;
        // eight independent loads in flight per thread (the first tile of a
        // run waits on them)
        for (int i0 = tid; i0 < nty * tstr; i0 += 8 * 32 * vCW) {
          float2 v[8];
          size_t o[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * 32 * vCW, ar = i / tstr, b = i - ar * tstr;
            o[u] = (i < nty * tstr && b < ntx) ? (size_t)ar * ntx + b : SIZE_MAX;
            v[u] = o[u] != SIZE_MAX ? __ldg(Ti + o[u]) : make_float2(0.f, 0.f);
          }
          for (int p = 1; p < nsplit; ++p)
#pragma unroll
            for (int u = 0; u < 8; ++u)
              if (o[u] != SIZE_MAX) v[u] = cadd(v[u], __ldg(Ti + p * tsz + o[u]));
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * 32 * vCW;
            if (i < nty * tstr) Ts[i] = v[u];
          }
        }
        asm volatile("bar.sync 1, %0;" ::"r"(32 * vCW) : "memory");
        // |Q[y][b]| <= w_b sum_a |T[a][b]|: the largest bound fixes the exponent
        for (int b = tid; b < ntx; b += 32 * vCW) {
          float sum = 0.f;
          for (int ar = 0; ar < nty; ++ar) sum += fabsf(Ts[ar * tstr + b].x) + fabsf(Ts[ar * tstr + b].y);
          atomicMax(&s_bound, __float_as_uint(sum * (b == 0 ? 1.f : 2.f)));
        }
        asm volatile("bar.sync 1, %0;" ::"r"(32 * vCW) : "memory");
        if (tid == 0) {
          const float bnd = __uint_as_float(s_bound);
          int e = 0;
          if (bnd > 0.f) {
            int x;
            frexpf(bnd, &x);  // bnd < 2^x
            e = min(max(14 - x, -100), 100);
          }
          s_scale[0] = ldexpf(1.f, e);
          s_scale[1] = ldexpf(1.f, -e);
        }
      }
#pragma unroll
      for (int k = 0; k < PHR; ++k) {
        const int i = tid + 32 * vCW * k;
        if (i < nph) ph[i] = phn[k];
      }
      if (t + 1 < t1) load_ph(t + 1);
      asm volatile("bar.sync 1, %0;" ::"r"(32 * vCW) : "memory");
      const float sc = s_scale[0];
      if (tid == 0) {
        s_inv[ti % vScaleRing] = s_scale[1];
        __threadfence_block();
        s_seq[ti % vScaleRing] = ti;
      }
      const uint32_t ahi = lanebase + (uint32_t)(vA1 + buf * 64), alo = ahi + 32;
      const float2* phs = ph + sw * nty;
      // per group of 8 columns: eight independent J-point FFTs along y, each
      // lane then fetches the values of its own row and writes 8 columns of
      // A_hi and A_lo (16 K entries) to TMEM
      for (int g8 = 0; g8 < ng; ++g8) {
        float2 v[8][RJ];
#pragma unroll
        for (int j = 0; j < RJ; ++j) {
          const int n = lane + 32 * j;
#pragma unroll
          for (int i = 0; i < 8; ++i) v[i][j] = make_float2(0.f, 0.f);
          for (int ar = n - J * ((n + A2) / J); ar <= A2; ar += J) {
            const float2 p = phs[ar + A2];
            const float4* trow = reinterpret_cast<const float4*>(Ts + (ar + A2) * tstr + 8 * g8);
#pragma unroll
            for (int h = 0; h < 4; ++h) {
              const float4 tt = trow[h];
              v[2 * h][j] = cfma(make_float2(tt.x, tt.y), p, v[2 * h][j]);
              v[2 * h + 1][j] = cfma(make_float2(tt.z, tt.w), p, v[2 * h + 1][j]);
            }
          }
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) wf.run(v[i], lane);
        uint32_t hi[8], lo[8];
#pragma unroll
        for (int i = 0; i < 8; i += 2) {
          float2 s0v = make_float2(0.f, 0.f), s1v = make_float2(0.f, 0.f);
#pragma unroll
          for (int q = 0; q < RJ; ++q) {
            const float ax = __shfl_sync(0xffffffffu, v[i][q].x, src), ay = __shfl_sync(0xffffffffu, v[i][q].y, src);
            const float bx = __shfl_sync(0xffffffffu, v[i + 1][q].x, src);
            const float by = __shfl_sync(0xffffffffu, v[i + 1][q].y, src);
            if (q == qsel) {
              s0v = make_float2(ax, ay);
              s1v = make_float2(bx, by);
            }
          }
          // weight 2 folds the conjugate half plane in, except at b = 0
          const float w0 = (g8 == 0 && i == 0 ? 1.f : 2.f) * sc, w1 = 2.f * sc;
          const float re0 = s0v.x * w0, re1 = s1v.x * w1, im0 = -s0v.y * w0, im1 = -s1v.y * w1;
          const __half2 hr = __floats2half2_rn(re0, re1), hm = __floats2half2_rn(im0, im1);
          const float2 fr = __half22float2(hr), fm = __half22float2(hm);
          const __half2 lr = __floats2half2_rn(re0 - fr.x, re1 - fr.y), lm = __floats2half2_rn(im0 - fm.x, im1 - fm.y);
          hi[i / 2] = *reinterpret_cast<const uint32_t*>(&hr);
          hi[4 + i / 2] = *reinterpret_cast<const uint32_t*>(&hm);
          lo[i / 2] = *reinterpret_cast<const uint32_t*>(&lr);
          lo[4 + i / 2] = *reinterpret_cast<const uint32_t*>(&lm);
        }
        tc::tmem_st8(ahi + (uint32_t)(8 * g8), hi);
        tc::tmem_st8(alo + (uint32_t)(8 * g8), lo);
      }
      // A complete in TMEM before the MMA issuer is told
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      asm volatile("bar.sync 1, %0;" ::"r"(32 * vCW) : "memory");
      if (tid == 0) tc::mbar_arrive(tc::smem_u32(&afull[buf]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(vTmemCols) : "memory");
  }
}
// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
bool vjp_tc_supported(const SocsGeom& g) {
  if (g.Ly % vRows != 0 || g.Lx % vNT != 0 || 2 * v_ntx8(g.ntx) > 64) return false;
  if (g.J != 32 && g.J != 64) return false;
  const int nst = vRows / g.J;
  if (nst * g.nty > 2 * 32 * vCW) return false;  // strip phases held two per coefficient thread
  return vjp_smem(g.nty, g.ntx, nst).total <= vSmemMax;
}

int vjp_tc_build_basis_t(const SocsGeom& g, void* thi, void* tlo, cudaStream_t st) {
  const size_t n = (size_t)64 * g.Lx;
  k_vjp_basis_t<<<(int)std::min<size_t>((n + 255) / 256, 4096), 256, 0, st>>>(g.Lx, g.ntx, static_cast<__half*>(thi),
                                                                               static_cast<__half*>(tlo));
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

namespace {
template <int RJ>
int launch_vjp_tc(const SocsGeom& g, const float2* T, const float2* ty, int nclips, int nsets, int nsplit,
                  const void* bhi, const void* blo, const void* thi, const void* tlo, const float* targets,
                  float alpha, float thr, float* images, double* loss, float2* gpart, int* err, cudaStream_t st) {
  const int nimg = nclips * nsets;
  CUtensorMap mh, ml, mth, mtl, mi, mt;
  const unsigned long long dimi[4] = {(unsigned long long)g.Lx, (unsigned long long)g.nS, (unsigned long long)g.J,
                                      (unsigned long long)nimg};
  const unsigned long long dimt[4] = {(unsigned long long)g.Lx, (unsigned long long)g.nS, (unsigned long long)g.J,
                                      (unsigned long long)nclips};
  const unsigned long long strides[3] = {4ull * g.Lx, 4ull * g.Lx * g.nS, 4ull * g.Lx * g.Ly};
  int rc;
  // (without an image output the image map is never used; it is made on the targets)
  if ((rc = tc::make_map_2b(&mh, bhi, g.Lx, 64, 64, 64, CU_TENSOR_MAP_DATA_TYPE_FLOAT16)) ||
      (rc = tc::make_map_2b(&ml, blo, g.Lx, 64, 64, 64, CU_TENSOR_MAP_DATA_TYPE_FLOAT16)) ||
      (rc = tc::make_map_2b(&mth, thi, 64, g.Lx, 64, 64, CU_TENSOR_MAP_DATA_TYPE_FLOAT16)) ||
      (rc = tc::make_map_2b(&mtl, tlo, 64, g.Lx, 64, 64, CU_TENSOR_MAP_DATA_TYPE_FLOAT16)) ||
      (rc = tc::make_map_f32_rows(&mi, images ? images : const_cast<float*>(targets), images ? dimi : dimt, strides)) ||
      (rc = tc::make_map_f32_rows(&mt, const_cast<float*>(targets), dimt, strides)))
    return rc;
  // G = dL/dI is bounded by alpha / 2: a power of two keeps G scale <= 2^15
  float gscale = 1.0f;
  const float gmax = 0.5f * std::fabs(alpha);
  if (gmax > 0.f) {
    int e;
    std::frexp(gmax, &e);  // gmax < 2^e
    gscale = std::ldexp(1.0f, std::min(std::max(15 - e, -60), 60));
  }
  const VjpSmem L = vjp_smem(g.nty, g.ntx, vRows / (32 * RJ));
  const size_t sm = std::max<size_t>(L.total, 120 * 1024) + 1024;  // one CTA per SM
  auto kern = k_vjp_synth_tc<RJ>;
  KL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int dev = 0, sms = 148;
  KL_CUDA_TRY(cudaGetDevice(&dev));
  KL_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int tiles = nimg * (g.Ly / vRows);
  const int per = (tiles + sms - 1) / sms;
  const int grid = (tiles + per - 1) / per;
  kern<<<grid, vThreads, sm, st>>>(T, g, ty, nsplit, nsets, mh, ml, mth, mtl, mi, mt, images ? 1 : 0, alpha, thr,
                                   gscale, nimg, loss, gpart, err);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}
}  // namespace

int vjp_tc_launch(const SocsGeom& g, const float2* T, const float2* ty, int nclips, int nsets, int nsplit,
                  const void* bhi, const void* blo, const void* thi, const void* tlo, const float* targets,
                  float alpha, float thr, float* images, double* loss, float2* gpart, int* err, cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  if (!vjp_tc_supported(g) || ((reinterpret_cast<uintptr_t>(targets) | reinterpret_cast<uintptr_t>(images)) & 15)) {
    set_error("vjp_tc_launch: geometry or alignment outside the tensor-core adjoint");
    return KL_ERR_UNSUPPORTED;
  }
  if (g.J == 32)
    return launch_vjp_tc<1>(g, T, ty, nclips, nsets, nsplit, bhi, blo, thi, tlo, targets, alpha, thr, images, loss,
                            gpart, err, st);
  return launch_vjp_tc<2>(g, T, ty, nclips, nsets, nsplit, bhi, blo, thi, tlo, targets, alpha, thr, images, loss,
                          gpart, err, st);
}

}  // namespace kl
