// socs_fwd_tc.cu -- the mask transform of the specialised SOCS pipeline (the
// work of k_socs_forward in socs_fast.cu) on the tensor cores.
//
// FT_r2c of K-Litho-SOCS/klitho_socs.cpp:70-121 restricted to the band: for
// each strip s of J rows (y = s + nS j) the partial band spectrum
//     D_s[fy][fx] = sum_j e^{-2 pi i fy (s + nS j)/Ly} R[s + nS j][fx],
//     R[y][fx]    = sum_x m[y][x] e^{-2 pi i fx x / Lx},   0 <= fx <= Nx,
// of which k_socs_spectral sums the strips.  The row DFT R is a matrix
// product per tile of 128 rows (128/J strips): R = M . BT with the mask block
// M (FP16 hi/lo halves in TMEM: mask values must lie within +-2^15) and the
// plan's transposed cos/sin basis BT (FP16 hi/lo, L2-resident), accumulated
// over the tile's 64-column blocks as M_hi BT_hi + M_lo BT_hi + M_hi BT_lo in
// FP32 in TMEM.  At the end of a tile the warps read R, run the J-point column
// FFTs of each strip and write its partial spectrum, as k_socs_forward does.
//
// Roles (320 threads, one CTA per SM): warps 0-7 conversion warps (warp w
// reads the 32 x 32 mask blocks of TMEM lane quarter w % 4 and column half
// w / 4 by TMA, splits them and writes them to TMEM), warp 8 TMA producer of
// the basis units, warp 9 MMA issuer.  Every wait is bounded; a timeout, or a
// mask value outside the FP16 range, sets the plan's status word.
#include <cuda_fp16.h>

#include <algorithm>
#include <climits>
#include <cstdint>

#include "kl_device.cuh"
#include "kl_internal.h"
#include "kl_tc.cuh"

namespace kl {
namespace {
constexpr int fRows = 128;        // tile rows (MMA M, TMEM lanes)
constexpr int fCW = 8;            // conversion warps: two per TMEM lane quarter
constexpr int fThreads = 32 * (fCW + 2);
constexpr int fProdWarp = fCW, fMmaWarp = fCW + 1;
constexpr int fNT = 64;           // mask columns per block (one K atom)
constexpr int fUnit = 64 * 128;   // basis unit: 64 rows x 128 bytes
constexpr int fStages = 4;        // basis unit ring
constexpr int fMaskBufs = 3;      // mask blocks in flight per conversion warp
constexpr int fRStride = 33;      // float2 per row of the staged row bins
// TMEM columns: fABufs mask buffers (hi 32 | lo 32), then the 64-column R accumulator
constexpr int fABufs = 4;
constexpr int fA = 0, fD = 64 * fABufs, fTmemCols = 512;

struct FwdSmem {
  size_t b, msk, r, bars, total;
};
__host__ __device__ inline FwdSmem fwd_smem() {
  FwdSmem s{};
  s.b = 0;                                             // [fStages] basis units
  s.msk = s.b + (size_t)fStages * fUnit;               // [fCW][fMaskBufs] 4 KB mask blocks
  s.r = s.msk + (size_t)fCW * fMaskBufs * 4096;        // [128][fRStride] float2 row bins
  s.bars = (s.r + sizeof(float2) * 128 * fRStride + 15) & ~(size_t)15;
  s.total = s.bars + 8 * (2 * fStages + 2 * fABufs + 2 + fCW * fMaskBufs + 1) + 64;
  return s;
}
}  // namespace

template <int RJ>
__global__ void __launch_bounds__(fThreads, 1)
    k_socs_fwd_tc(const __grid_constant__ CUtensorMap tm_msk, const SocsGeom g, const float2* __restrict__ ty,
                  const __grid_constant__ CUtensorMap tm_thi, const __grid_constant__ CUtensorMap tm_tlo, int nclips,
                  float2* __restrict__ partial, int* __restrict__ err) {
  constexpr int J = 32 * RJ;
  constexpr int NST = fRows / J;  // strips per tile
  constexpr uint32_t IDESC = tc::idesc_f16(fRows, 64, false);
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const FwdSmem L = fwd_smem();
  uint8_t* bst = smem + L.b;
  uint8_t* mks = smem + L.msk;
  float2* rs = reinterpret_cast<float2*>(smem + L.r);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars);  // basis unit loaded
  uint64_t* empty = full + fStages;                              // basis unit consumed
  uint64_t* afull = empty + fStages;                             // mask buffer written
  uint64_t* aempty = afull + fABufs;                             // mask buffer consumed
  uint64_t* dfull = aempty + fABufs;                             // R of the tile complete
  uint64_t* dempty = dfull + 1;                                  // R read
  uint64_t* mskb = dempty + 1;                                   // [fCW][fMaskBufs] mask block landed
  uint64_t* drain = mskb + fCW * fMaskBufs;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  __shared__ int s_abort;
  volatile int* abort = &s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
  const int tiles_img = g.Ly / fRows, ntile = g.Lx / fNT;
  const int total = nclips * tiles_img;
  const int per = (total + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per, t1 = min(total, t0 + per);

  if (tid == 0) {
    for (int s = 0; s < fStages; ++s) {
      tc::mbar_init(tc::smem_u32(&full[s]), 1);
      tc::mbar_init(tc::smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < fABufs; ++b) {
      tc::mbar_init(tc::smem_u32(&afull[b]), fCW);
      tc::mbar_init(tc::smem_u32(&aempty[b]), 1);
    }
    tc::mbar_init(tc::smem_u32(dfull), 1);
    tc::mbar_init(tc::smem_u32(dempty), fCW);
    for (int i = 0; i < fCW * fMaskBufs; ++i) tc::mbar_init(tc::smem_u32(&mskb[i]), 1);
    tc::mbar_init(tc::smem_u32(drain), 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(tmem_slot)),
                 "r"(fTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == fProdWarp) {
    // TMA producer (one lane): per 64-column block the transposed basis, hi then lo
    if (lane == 0) {
      int u = 0, armed[fStages];
      for (int s = 0; s < fStages; ++s) armed[s] = -1;
      bool ok = true;
      for (int t = t0; t < t1 && ok; ++t)
        for (int n = 0; n < ntile && ok; ++n)
          for (int h = 0; h < 2; ++h, ++u) {
            const int s = u % fStages, use = u / fStages;
            if (use > 0 &&
                !(ok = tc::mbar_wait_ab(tc::smem_u32(&empty[s]), (uint32_t)((use - 1) & 1), err, 51, abort)))
              break;
            const uint32_t bar = tc::smem_u32(&full[s]);
            tc::mbar_expect_tx(bar, fUnit);
            tc::tma_load_2d(tc::smem_u32(bst + (size_t)s * fUnit), h ? &tm_tlo : &tm_thi, n * fNT, 0, bar);
            armed[s] = use;
          }
      // no copy may still be writing shared memory when the CTA exits
      for (int s = 0; s < fStages; ++s)
        if (armed[s] >= 0) tc::mbar_wait(tc::smem_u32(&full[s]), (uint32_t)(armed[s] & 1), err, 52);
    }
    __syncwarp();
  } else if (warp == fMmaWarp) {
    // MMA issuer (one lane): R += M_hi BT_hi + M_lo BT_hi (hi unit), M_hi BT_lo
    // (lo unit) for each block of the tile; R is reported after the last block
    if (lane == 0) {
      int ab = 0, ti = 0, u = 0;
      bool ok = true;
      const uint32_t d = tmem + (uint32_t)fD;
      for (int t = t0; t < t1 && ok; ++t, ++ti) {
        for (int n = 0; n < ntile && ok; ++n, ++ab) {
          const int buf = ab % fABufs;
          if (!(ok = tc::mbar_wait_ab(tc::smem_u32(&afull[buf]), (uint32_t)((ab / fABufs) & 1), err, 53, abort)))
            break;
          if (n == 0 && ti > 0 &&
              !(ok = tc::mbar_wait_ab(tc::smem_u32(dempty), (uint32_t)((ti - 1) & 1), err, 54, abort)))
            break;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          const uint32_t mh = tmem + (uint32_t)(fA + 64 * buf), ml = mh + 32;
          for (int h = 0; h < 2 && ok; ++h, ++u) {
            const int s = u % fStages, use = u / fStages;
            if (!(ok = tc::mbar_wait_ab(tc::smem_u32(&full[s]), (uint32_t)(use & 1), err, 55, abort))) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t bb = tc::smem_u32(bst + (size_t)s * fUnit);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const uint64_t db = tc::smem_desc(bb + k * 32);
              if (h == 0) {
                tc::mma_f16_ts(d, mh + 8 * k, db, IDESC, (n | k) ? 1u : 0u);
                tc::mma_f16_ts(d, ml + 8 * k, db, IDESC, 1u);
              } else {
                tc::mma_f16_ts(d, mh + 8 * k, db, IDESC, 1u);
              }
            }
            tc::mma_commit(tc::smem_u32(&empty[s]));
          }
          if (!ok) break;
          tc::mma_commit(tc::smem_u32(&aempty[buf]));
          if (n == ntile - 1) tc::mma_commit(tc::smem_u32(dfull));
        }
      }
      tc::mma_commit(tc::smem_u32(drain));
      tc::mbar_wait(tc::smem_u32(drain), 0u, err, 56);
    }
    __syncwarp();
  } else {
    // conversion warps: warp w holds TMEM lanes 32 (w % 4) .. + 31, rows j0 ..
    // j0 + 31 of strip st of the tile, and columns 32 hc0 .. + 31 of each block
    const int cw = warp, hc0 = cw >> 2;
    const int r0 = 32 * (cw & 3), st = r0 / J, j0 = r0 - st * J;
    uint8_t* mym = mks + (size_t)cw * fMaskBufs * 4096;
    const uint32_t lanebase = tmem + ((uint32_t)r0 << 16);
    const int nf = g.nf, nby = g.nby, Ny = g.Ny;
    const int nchunk = (t1 - t0) * ntile;
    auto issue = [&](int q) {
      const int tq = t0 + q / ntile, n = q % ntile;
      const int clip = tq / tiles_img, s0 = (tq - clip * tiles_img) * NST;
      const int b = q % fMaskBufs;
      const uint32_t bar = tc::smem_u32(&mskb[cw * fMaskBufs + b]);
      tc::mbar_expect_tx(bar, 4096);
      tc::tma_load_4d(tc::smem_u32(mym + b * 4096), &tm_msk, n * fNT + 32 * hc0, s0 + st, j0, clip, bar);
    };
    int qi = 0;  // next block whose mask is requested (lane 0)
    if (lane == 0)
      for (; qi < min(fMaskBufs, nchunk); ++qi) issue(qi);
    int q = 0, ab = 0, ti = 0;
    bool ok = true;
    WarpFFT<RJ, -1> wf;
    wf.init(lane);
    const int br = (int)(__brev((unsigned)lane) >> 27);
    for (int t = t0; t < t1; ++t, ++ti) {
      const int clip = t / tiles_img, s0 = (t - clip * tiles_img) * NST;
      for (int n = 0; n < ntile && ok; ++n, ++q, ++ab) {
        const int b = q % fMaskBufs, buf = ab % fABufs;
        const bool landed =
            tc::mbar_wait_ab(tc::smem_u32(&mskb[cw * fMaskBufs + b]), (uint32_t)((q / fMaskBufs) & 1), err, 57, abort);
        if (!__all_sync(0xffffffffu, landed)) {
          ok = false;
          break;
        }
        float mv[32];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const float4 f = *reinterpret_cast<const float4*>(mym + b * 4096 + lane * 128 + ((c ^ (lane & 7)) << 4));
          mv[4 * c] = f.x;
          mv[4 * c + 1] = f.y;
          mv[4 * c + 2] = f.z;
          mv[4 * c + 3] = f.w;
        }
        __syncwarp();  // every lane has read block b: request the block fMaskBufs ahead into it
        if (lane == 0 && qi < nchunk && qi == q + fMaskBufs) issue(qi++);
        // FP16 hi and lo halves of the lane's 32 mask values
        uint32_t hi[16], lo[16];
        bool range = true;
#pragma unroll
        for (int p = 0; p < 16; ++p) {
          range = range && fabsf(mv[2 * p]) < 32768.f && fabsf(mv[2 * p + 1]) < 32768.f;
          const __half2 h2 = __floats2half2_rn(mv[2 * p], mv[2 * p + 1]);
          const float2 hf = __half22float2(h2);
          const __half2 l2 = __floats2half2_rn(mv[2 * p] - hf.x, mv[2 * p + 1] - hf.y);
          hi[p] = *reinterpret_cast<const uint32_t*>(&h2);
          lo[p] = *reinterpret_cast<const uint32_t*>(&l2);
        }
        if (!__all_sync(0xffffffffu, range) && lane == 0) atomicExch(err, 50);  // mask value outside +-2^15
        if (ab >= fABufs) {
          const bool freed =
              tc::mbar_wait_ab(tc::smem_u32(&aempty[buf]), (uint32_t)((ab / fABufs - 1) & 1), err, 58, abort);
          if (!__all_sync(0xffffffffu, freed)) {
            ok = false;
            break;
          }
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        tc::tmem_st16(lanebase + (uint32_t)(fA + 64 * buf + 16 * hc0), hi);
        tc::tmem_st16(lanebase + (uint32_t)(fA + 64 * buf + 32 + 16 * hc0), lo);
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(tc::smem_u32(&afull[buf]));
      }
      // row bins of the tile's rows
      if (ok) {
        const bool done = tc::mbar_wait_ab(tc::smem_u32(dfull), (uint32_t)(ti & 1), err, 59, abort);
        ok = __all_sync(0xffffffffu, done);
      }
      if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        uint32_t d0[32];
        tc::tmem_ld32(lanebase + (uint32_t)(fD + 32 * hc0), d0);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(tc::smem_u32(dempty));
        // R[fx] = sum_x m e^{-2 pi i fx x / Lx}: Re from the cos columns, Im =
        // -(sin columns); K index of (fx, part) is 16 (fx / 8) + 8 part + fx % 8,
        // so the warp's 32 columns hold bins 16 hc0 .. 16 hc0 + 15
        float2* row = rs + (r0 + lane) * fRStride;
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int fx = 16 * hc0 + 8 * (c >> 4) + (c & 7);
          if (!(c & 8)) row[fx] = make_float2(__uint_as_float(d0[c]), -__uint_as_float(d0[c + 8]));
        }
      }
      // the conversion warps go on or leave together (a named-barrier OR)
      int stop;
      asm volatile(
          "{\n\t.reg .pred p, q;\n\t"
          "setp.ne.s32 p, %1, 0;\n\t"
          "bar.red.or.pred q, 1, %2, p;\n\t"
          "selp.s32 %0, 1, 0, q;\n\t}"
          : "=r"(stop)
          : "r"((!ok || *abort) ? 1 : 0), "r"(32 * fCW)
          : "memory");
      if (stop) {
        ok = false;
        break;
      }
      // column DFT of each strip: bins fy in [-Ny, Ny] (J >= 2Ny+1), times
      // e^{-2 pi i fy s / Ly}: the strip's partial band spectrum
      for (int task = cw; task < NST * nf; task += fCW) {
        const int s2 = task / nf, fx = task - s2 * nf;
        float2 vv[RJ];
#pragma unroll
        for (int j = 0; j < RJ; ++j) vv[j] = rs[(s2 * J + lane + 32 * j) * fRStride + fx];
        wf.run(vv, lane);
        const int s = s0 + s2;
#pragma unroll
        for (int q1 = 0; q1 < RJ; ++q1) {
          const int bin = q1 + RJ * br;
          const int fy = bin <= J / 2 ? bin : bin - J;
          if (fy >= -Ny && fy <= Ny)
            partial[(((size_t)clip * g.nS + s) * nby + (fy + Ny)) * nf + fx] =
                cmulc(vv[q1], __ldg(ty + (size_t)s * g.nty + 2 * Ny + fy));
        }
      }
      asm volatile("bar.sync 1, %0;" ::"r"(32 * fCW) : "memory");  // the staged bins are read
    }
    // no TMA copy may still be writing this warp's blocks at exit
    if (lane == 0)
      for (int qq = q; qq < qi; ++qq)
        tc::mbar_wait(tc::smem_u32(&mskb[cw * fMaskBufs + qq % fMaskBufs]), (uint32_t)((qq / fMaskBufs) & 1), err, 60);
    __syncwarp();
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(fTmemCols) : "memory");
  }
}
// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
bool fwd_tc_supported(const SocsGeom& g) {
  if (g.Ly % fRows != 0 || g.Lx % fNT != 0 || g.nf > 32) return false;
  if (g.J != 32 && g.J != 64 && g.J != 128) return false;
  return fwd_smem().total <= 227 * 1024 - 1024;
}

namespace {
template <int RJ>
int launch_fwd_tc(const SocsGeom& g, const float* masks, int nclips, const float2* ty, const void* thi,
                  const void* tlo, float2* partial, int* err, cudaStream_t st) {
  CUtensorMap mm, mth, mtl;
  const unsigned long long dims[4] = {(unsigned long long)g.Lx, (unsigned long long)g.nS, (unsigned long long)g.J,
                                      (unsigned long long)nclips};
  const unsigned long long strides[3] = {4ull * g.Lx, 4ull * g.Lx * g.nS, 4ull * g.Lx * g.Ly};
  int rc;
  if ((rc = tc::make_map_f32_rows(&mm, const_cast<float*>(masks), dims, strides)) ||
      (rc = tc::make_map_2b(&mth, thi, 64, g.Lx, 64, 64, CU_TENSOR_MAP_DATA_TYPE_FLOAT16)) ||
      (rc = tc::make_map_2b(&mtl, tlo, 64, g.Lx, 64, 64, CU_TENSOR_MAP_DATA_TYPE_FLOAT16)))
    return rc;
  const size_t sm = fwd_smem().total + 1024;
  auto kern = k_socs_fwd_tc<RJ>;
  KL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int dev = 0, sms = 148;
  KL_CUDA_TRY(cudaGetDevice(&dev));
  KL_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int tiles = nclips * (g.Ly / fRows);
  const int per = (tiles + sms - 1) / sms;
  const int grid = (tiles + per - 1) / per;
  kern<<<grid, fThreads, sm, st>>>(mm, g, ty, mth, mtl, nclips, partial, err);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}
}  // namespace

int fwd_tc_launch(const SocsGeom& g, const float* masks, int nclips, const float2* ty, const void* thi,
                  const void* tlo, float2* partial, int* err, cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  if (!fwd_tc_supported(g) || (reinterpret_cast<uintptr_t>(masks) & 15)) {
    set_error("fwd_tc_launch: geometry or alignment outside the tensor-core mask transform");
    return KL_ERR_UNSUPPORTED;
  }
  if (g.J == 32) return launch_fwd_tc<1>(g, masks, nclips, ty, thi, tlo, partial, err, st);
  if (g.J == 64) return launch_fwd_tc<2>(g, masks, nclips, ty, thi, tlo, partial, err, st);
  return launch_fwd_tc<4>(g, masks, nclips, ty, thi, tlo, partial, err, st);
}

}  // namespace kl
