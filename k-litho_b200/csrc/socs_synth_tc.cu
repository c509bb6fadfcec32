// socs_synth_tc.cu -- the image synthesis of the specialised SOCS pipeline on
// the 5th-generation tensor cores (sm_100a).
//
// k_socs_inverse (socs_fast.cu) synthesises each image row from its 2Nx+1
// row coefficients Q[b] (the FI step of K-Litho-SOCS/klitho_socs.cpp:158-194
// restricted to the band) with a per-lane DFT on the CUDA cores.  The same
// step is a real matrix product per tile of 128 rows:
//     image[y][x] = sum_b Re(Q[y][b] e^{2 pi i b x / Lx})
//                 = sum_k A[y][k] B[k][x],  A = [Re Q, -Im Q],  B = [cos; sin],
// with K = 2 ntx8 <= 128 (ntx = 2Nx+1 columns rounded up to groups of 8).  It
// runs as tcgen05.mma kind::f16 on a 3-term FP16 split, A_hi B_hi + A_lo B_hi
// + A_hi B_lo, accumulated in FP32 in TMEM: each split operand keeps 22
// significant bits and the dropped A_lo B_lo term is 2^-22 of a product, far
// below the 1e-5-of-clear-field bar.  A is scaled per image by a power of two
// so that FP16's range holds it (the bound |Q[b]| <= w_b sum_a |T[a][b]| fixes
// the exponent); the epilogue undoes it.
//
// The kernel is bound by shared-memory bandwidth long before the tensor
// cores are busy, so A lives in TMEM (the MMA reads it from there, not from
// shared memory) and shared memory carries only the basis tiles and the
// output staging.  One persistent CTA per SM handles a contiguous run of
// 128-row tiles (rows of 128/J strips, y = s + nS j as in k_socs_inverse):
//   warps 0-3  coefficient warps: warp w owns TMEM lanes 32w..32w+31, i.e.
//              rows 32w.. of the tile (strip 32w/J).  It loads the image's
//              band-limited intensity spectrum T into shared memory (when the
//              image changes, shared by the four warps), runs J-point warp
//              FFTs along y for 8 columns at a time, moves each row's values
//              to its lane and writes the FP16 halves of A into TMEM
//              (double-buffered: the next tile's A is built while the tensor
//              cores work on this one);
//   warps 4-7  epilogue warps: TMEM accumulator tiles -> registers -> (scale)
//              -> a swizzled 32 x 32 staging tile per warp -> TMA bulk store of
//              32 image rows (whole 128-byte lines);
//   warp 8     TMA producer of the basis units (plan-time, L2-resident);
//   warp 9     MMA issuer, into a ring of TMEM accumulators.
// Every wait is bounded; a timeout sets the plan's status word and stops
// every role.
#include <cuda_fp16.h>

#include <algorithm>
#include <climits>
#include <cstdint>

#include "kl_device.cuh"
#include "kl_internal.h"
#include "kl_tc.cuh"

namespace kl {
namespace {
constexpr int kRows = 128;       // tile rows (MMA M, TMEM lanes)
constexpr int kCW = 4;           // coefficient warps
constexpr int kEW = 4;           // epilogue warps
constexpr int kSThreads = 32 * (kCW + kEW + 2);
constexpr int kProdWarp = kCW + kEW, kMmaWarp = kCW + kEW + 1;
constexpr int kStages = 6;       // basis unit stages (16 KB each)
constexpr int kStageBufs = 2;    // staging tiles per epilogue warp
constexpr int kTmemCols = 512;
constexpr int kScaleRing = 8;
constexpr int kMaxSets = 4;      // TMEM accumulator ring slots
constexpr int kNT = 128;         // N tile (MMA N): accumulator columns per slot

// columns b of the row coefficients come in groups of 8: K index of column b,
// part 0 (Re, against cos) or 1 (-Im, against sin) is 16 (b / 8) + 8 part + b % 8
__host__ __device__ constexpr int synth_ntx8(int ntx) { return (ntx + 7) & ~7; }
// row stride of the staged spectrum (float2): 8-column groups stay 16-byte
// aligned and consecutive rows fall on different banks
__host__ __device__ constexpr int synth_tstride(int ntx) { return synth_ntx8(ntx) + 2; }
// TMEM columns: accumulator slots first, then two A buffers of K columns each
// (hi halves in the first K/2, lo halves in the next K/2)
__host__ __device__ constexpr int synth_nset(int KA) { return (kTmemCols - 2 * 64 * KA) / kNT; }

struct SynthSmem {
  size_t b, stg, ts, ph, bars, total;
};
__host__ __device__ inline SynthSmem synth_smem(int nty, int ntx, int nst) {
  SynthSmem s{};
  s.b = 0;                                                     // [kStages] units of kNT x 128 B
  s.stg = s.b + (size_t)kStages * kNT * 128;                   // [kEW][kStageBufs] 4 KB tiles
  s.ts = s.stg + (size_t)kEW * kStageBufs * 4096;              // T [nty][tstride] float2
  s.ph = s.ts + sizeof(float2) * (size_t)nty * synth_tstride(ntx);  // phases [nst][nty] float2
  s.bars = (s.ph + sizeof(float2) * (size_t)nst * nty + 15) & ~(size_t)15;
  s.total = s.bars + 8 * (2 * kStages + 4 + 2 * kMaxSets + 1) + 64;
  return s;
}
constexpr size_t kSmemMax = 227 * 1024 - 1024;  // dynamic bytes usable after the 1 KB alignment pad
}  // namespace

// plan-time basis: B[x][k] = cos(2 pi b x / Lx) for K index k of (b, part 0),
// sin(2 pi b x / Lx) for (b, part 1), 0 for b >= ntx and the padding; FP16 hi
// and lo halves, [Lx][Kp]
__global__ void k_synth_basis(int Lx, int ntx, int Kp, __half* __restrict__ bhi, __half* __restrict__ blo) {
  const size_t n = (size_t)Lx * Kp;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i / Kp), k = (int)(i % Kp);
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

template <int RJ, int KA>
__global__ void __launch_bounds__(kSThreads, 1)
    k_socs_synth_tc(const float2* __restrict__ T, const SocsGeom g, const float2* __restrict__ ty, int nsplit,
                    const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
                    const __grid_constant__ CUtensorMap tm_img, int nimg, int* __restrict__ err) {
  constexpr int J = 32 * RJ;
  constexpr int NST = kRows / J;       // strips per tile
  constexpr int UNIT = kNT * 128;      // one K atom of one half of a basis tile
  constexpr int KC = 32 * KA;          // TMEM columns of one half of A
  constexpr int NSET = synth_nset(KA);
  constexpr int ACOL = NSET * kNT;     // first A column
  constexpr int PHR = 2;               // strip phases per coefficient thread (nst * nty <= 256)
  constexpr uint32_t IDESC = tc::idesc_f16(kRows, kNT, false);
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  const SynthSmem L = synth_smem(g.nty, g.ntx, NST);
  uint8_t* bst = smem + L.b;
  uint8_t* stg = smem + L.stg;
  float2* Ts = reinterpret_cast<float2*>(smem + L.ts);
  float2* ph = reinterpret_cast<float2*>(smem + L.ph);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars);  // basis unit loaded
  uint64_t* empty = full + kStages;                              // basis unit consumed
  uint64_t* afull = empty + kStages;                             // A buffer written
  uint64_t* aempty = afull + 2;                                  // A buffer consumed
  uint64_t* tfull = aempty + 2;                                  // accumulator ready
  uint64_t* tempty = tfull + kMaxSets;                           // accumulator drained
  uint64_t* drain = tempty + kMaxSets;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain + 1);
  __shared__ int s_abort;
  __shared__ float s_scale[2];                // scale of A and its inverse for the current image
  __shared__ float s_inv[kScaleRing];         // inverse scale per tile, read by the epilogue
  __shared__ volatile int s_seq[kScaleRing];  // tile number whose scale a slot holds
  __shared__ unsigned s_bound;
  volatile int* abort = &s_abort;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
  const int ntx = g.ntx, nty = g.nty, A2 = 2 * g.Ny;
  const int tiles_img = g.Ly / kRows, ntile = g.Lx / kNT;
  const int total = nimg * tiles_img;
  const int per = (total + gridDim.x - 1) / gridDim.x;
  const int t0 = blockIdx.x * per, t1 = min(total, t0 + per);
  const size_t tsz = (size_t)nty * ntx;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      tc::mbar_init(tc::smem_u32(&full[s]), 1);
      tc::mbar_init(tc::smem_u32(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(tc::smem_u32(&afull[b]), 1);
      tc::mbar_init(tc::smem_u32(&aempty[b]), 1);
    }
    for (int a = 0; a < kMaxSets; ++a) {
      tc::mbar_init(tc::smem_u32(&tfull[a]), 1);
      tc::mbar_init(tc::smem_u32(&tempty[a]), kEW);
    }
    tc::mbar_init(tc::smem_u32(drain), 1);
    for (int i = 0; i < kScaleRing; ++i) s_seq[i] = -1;
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == kProdWarp) {
    // TMA producer (one lane): per N tile, for each K atom the hi unit then
    // the lo unit of the basis, tile after tile
    if (lane == 0) {
      int u = 0, armed[kStages];
      for (int s = 0; s < kStages; ++s) armed[s] = -1;
      bool ok = true;
      for (int t = t0; t < t1 && ok; ++t)
        for (int n = 0; n < ntile && ok; ++n)
          for (int h = 0; h < 2 * KA; ++h, ++u) {
            const int s = u % kStages, use = u / kStages;
            if (use > 0 &&
                !(ok = tc::mbar_wait_ab(tc::smem_u32(&empty[s]), (uint32_t)((use - 1) & 1), err, 11, abort)))
              break;
            const uint32_t bar = tc::smem_u32(&full[s]);
            tc::mbar_expect_tx(bar, UNIT);
            tc::tma_load_2d(tc::smem_u32(bst + (size_t)s * UNIT), (h & 1) ? &tm_lo : &tm_hi, 64 * (h >> 1), n * kNT,
                            bar);
            armed[s] = use;
          }
      // no copy may still be writing shared memory when the CTA exits
      for (int s = 0; s < kStages; ++s)
        if (armed[s] >= 0) tc::mbar_wait(tc::smem_u32(&full[s]), (uint32_t)(armed[s] & 1), err, 14);
    }
    __syncwarp();
  } else if (warp == kMmaWarp) {
    // MMA issuer (one lane): N tile number `it` of the run accumulates into
    // ring slot it % NSET; per K atom, the hi unit of the basis serves
    // A_hi B_hi and A_lo B_hi, the lo unit A_hi B_lo (A from TMEM).  The A
    // buffer is released after the tile's last MMA.
    if (lane == 0) {
      int it = 0, ti = 0, u = 0;
      bool ok = true;
      for (int t = t0; t < t1 && ok; ++t, ++ti) {
        const int buf = ti & 1, ause = ti >> 1;
        if (!(ok = tc::mbar_wait_ab(tc::smem_u32(&afull[buf]), (uint32_t)(ause & 1), err, 12, abort))) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t ah = tmem + (uint32_t)(ACOL + buf * 2 * KC), al = ah + KC;
        for (int n = 0; n < ntile && ok; ++n, ++it) {
          const int a = it % NSET, tuse = it / NSET;
          if (tuse > 0 && !(ok = tc::mbar_wait_ab(tc::smem_u32(&tempty[a]), (uint32_t)((tuse - 1) & 1), err, 13, abort)))
            break;
          const uint32_t acc = tmem + (uint32_t)(a * kNT);
          for (int h = 0; h < 2 * KA && ok; ++h, ++u) {
            const int s = u % kStages, use = u / kStages;
            if (!(ok = tc::mbar_wait_ab(tc::smem_u32(&full[s]), (uint32_t)(use & 1), err, 15, abort))) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t bb = tc::smem_u32(bst + (size_t)s * UNIT);
            const uint32_t ac0 = (uint32_t)(32 * (h >> 1));  // A column of the atom's first k step
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const uint64_t db = tc::smem_desc(bb + k * 32);
              const uint32_t ac = ac0 + 8 * k;  // 16 K elements = 8 columns
              if ((h & 1) == 0) {
                tc::mma_f16_ts(acc, ah + ac, db, IDESC, (h | k) ? 1u : 0u);
                tc::mma_f16_ts(acc, al + ac, db, IDESC, 1u);
              } else {
                tc::mma_f16_ts(acc, ah + ac, db, IDESC, 1u);
              }
            }
            tc::mma_commit(tc::smem_u32(&empty[s]));
          }
          if (ok) tc::mma_commit(tc::smem_u32(&tfull[a]));
        }
        if (ok) tc::mma_commit(tc::smem_u32(&aempty[buf]));
      }
      tc::mma_commit(tc::smem_u32(drain));
      tc::mbar_wait(tc::smem_u32(drain), 0u, err, 16);
    }
    __syncwarp();
  } else if (warp >= kCW) {
    // epilogue warps: TMEM lanes 32 ew .. 32 ew + 31 are rows of one strip,
    // j = j0 .. j0 + 31 (y = s + nS j), written as 32 x 32 boxes by TMA
    const int ew = warp & 3;
    const int r0 = 32 * ew, st = r0 / J, j0 = r0 - st * J;
    uint8_t* mystg = stg + (size_t)ew * kStageBufs * 4096;
    const uint64_t policy = tc::policy_evict_first();
    int it = 0, ti = 0, sb = 0;
    bool ok = true;
    for (int t = t0; t < t1 && ok; ++t, ++ti) {
      const int img = t / tiles_img, s0 = (t - img * tiles_img) * NST;
      // the tile's inverse scale, published with its tile number
      const int slot = ti % kScaleRing;
      bool seen = true;
      if (lane == 0 && s_seq[slot] != ti) {
        const unsigned long long w0 = tc::now_ns();
        while (s_seq[slot] != ti) {
          if (*abort) {
            seen = false;
            break;
          }
          if (tc::now_ns() - w0 > tc::kWaitNs) {
            atomicExch(err, 18);
            *abort = 1;
            seen = false;
            break;
          }
          __nanosleep(64);
        }
      }
      if (!__shfl_sync(0xffffffffu, seen, 0)) break;
      __threadfence_block();
      const float inv = s_inv[slot];
      for (int n = 0; n < ntile; ++n, ++it) {
        const int a = it % NSET, tuse = it / NSET;
        const bool ready = tc::mbar_wait_ab(tc::smem_u32(&tfull[a]), (uint32_t)(tuse & 1), err, 17, abort);
        if (!__all_sync(0xffffffffu, ready)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t base = tmem + ((uint32_t)r0 << 16) + (uint32_t)(a * kNT);
#pragma unroll 1
        for (int c0 = 0; c0 < kNT; c0 += 32) {
          uint32_t v[32];
          tc::tmem_ld32(base + (uint32_t)c0, v);
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          if (c0 + 32 == kNT) {
            // the accumulator is in registers: hand it back to the MMA
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(tc::smem_u32(&tempty[a]));
          }
          // staging tile sb is free once its previous store has read it
          if (lane == 0) tc::bulk_wait_read<kStageBufs - 1>();
          __syncwarp();
          uint8_t* tile = mystg + sb * 4096;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float4 o = make_float4(__uint_as_float(v[4 * q]) * inv, __uint_as_float(v[4 * q + 1]) * inv,
                                         __uint_as_float(v[4 * q + 2]) * inv, __uint_as_float(v[4 * q + 3]) * inv);
            *reinterpret_cast<float4*>(tile + lane * 128 + ((q ^ (lane & 7)) << 4)) = o;
          }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) {
            tc::tma_store_4d(&tm_img, tc::smem_u32(tile), n * kNT + c0, s0 + st, j0, img, policy);
            tc::bulk_commit();
          }
          sb = sb + 1 == kStageBufs ? 0 : sb + 1;
        }
      }
    }
    if (lane == 0) tc::bulk_wait_all();
    __syncwarp();
  } else {
    // coefficient warps: warp w writes TMEM lanes 32w .. 32w + 31, rows
    // jw .. jw + 31 of strip sw of the tile (all 8-column groups)
    const int sw = (32 * warp) / J, jw = 32 * warp - sw * J;
    // lane of the FFT output that holds row jw + lane, and its register
    const int R = jw + lane, qsel = R % RJ, src = (int)(__brev((unsigned)(R / RJ)) >> 27);
    const uint32_t lanebase = tmem + ((uint32_t)(32 * warp) << 16);
    const int nph = NST * nty;
    const int ng = synth_ntx8(ntx) / 8;  // 8-column groups
    const int tstr = synth_tstride(ntx);
    int cur_img = -1, ti = 0;
    WarpFFT<RJ, +1> wf;
    wf.init(lane);
    // the K padding (columns 8 ng .. KC of each half) is zero once for both buffers
    {
      uint32_t z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int c = 8 * ng; c < KC; c += 8)
        for (int hb = 0; hb < 4; ++hb) tc::tmem_st8(lanebase + (uint32_t)(ACOL + hb * KC + c), z);
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    // phases e^{2 pi i a s / Ly} of the next tile's strips, held in registers
    float2 phn[PHR];
    auto load_ph = [&](int t) {
      const int img = t / tiles_img, s0 = (t - img * tiles_img) * NST;
#pragma unroll
      for (int k = 0; k < PHR; ++k) {
        const int i = tid + 32 * kCW * k;
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
      if (ause > 0) ok = tc::mbar_wait_ab(tc::smem_u32(&aempty[buf]), (uint32_t)((ause - 1) & 1), err, 19, abort);
      // the four warps go on or leave together (a named-barrier OR)
      int stop;
      asm volatile(
          "{\n\t.reg .pred p, q;\n\t"
          "setp.ne.s32 p, %1, 0;\n\t"
          "bar.red.or.pred q, 1, %2, p;\n\t"
          "selp.s32 %0, 1, 0, q;\n\t}"
          : "=r"(stop)
          : "r"((!ok || *abort) ? 1 : 0), "r"(32 * kCW)
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
        for (int i0 = tid; i0 < nty * tstr; i0 += 8 * 32 * kCW) {
          float2 v[8];
          size_t o[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * 32 * kCW, ar = i / tstr, b = i - ar * tstr;
            o[u] = (i < nty * tstr && b < ntx) ? (size_t)ar * ntx + b : SIZE_MAX;
            v[u] = o[u] != SIZE_MAX ? __ldg(Ti + o[u]) : make_float2(0.f, 0.f);
          }
          for (int p = 1; p < nsplit; ++p)
#pragma unroll
            for (int u = 0; u < 8; ++u)
              if (o[u] != SIZE_MAX) v[u] = cadd(v[u], __ldg(Ti + p * tsz + o[u]));
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * 32 * kCW;
            if (i < nty * tstr) Ts[i] = v[u];
          }
        }
        asm volatile("bar.sync 1, %0;" ::"r"(32 * kCW) : "memory");
        // |Q[y][b]| <= w_b sum_a |T[a][b]|: the largest bound fixes the exponent
        for (int b = tid; b < ntx; b += 32 * kCW) {
          float sum = 0.f;
          for (int ar = 0; ar < nty; ++ar) sum += fabsf(Ts[ar * tstr + b].x) + fabsf(Ts[ar * tstr + b].y);
          atomicMax(&s_bound, __float_as_uint(sum * (b == 0 ? 1.f : 2.f)));
        }
        asm volatile("bar.sync 1, %0;" ::"r"(32 * kCW) : "memory");
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
        const int i = tid + 32 * kCW * k;
        if (i < nph) ph[i] = phn[k];
      }
      if (t + 1 < t1) load_ph(t + 1);
      asm volatile("bar.sync 1, %0;" ::"r"(32 * kCW) : "memory");
      const float sc = s_scale[0];
      if (tid == 0) {
        s_inv[ti % kScaleRing] = s_scale[1];
        __threadfence_block();
        s_seq[ti % kScaleRing] = ti;
      }
      const uint32_t ahi = lanebase + (uint32_t)(ACOL + buf * 2 * KC), alo = ahi + KC;
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
      asm volatile("bar.sync 1, %0;" ::"r"(32 * kCW) : "memory");
      if (tid == 0) tc::mbar_arrive(tc::smem_u32(&afull[buf]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {
int synth_ka(const SocsGeom& g) { return 2 * synth_ntx8(g.ntx) <= 64 ? 1 : 2; }
}  // namespace

bool synth_tc_supported(const SocsGeom& g) {
  if (g.Ly % kRows != 0 || g.Lx % kNT != 0 || 2 * synth_ntx8(g.ntx) > 128) return false;
  if (g.J != 32 && g.J != 64 && g.J != 128) return false;
  const int nst = kRows / g.J;
  if (nst * g.nty > 2 * 32 * kCW) return false;  // strip phases held two per coefficient thread
  return synth_smem(g.nty, g.ntx, nst).total <= kSmemMax;
}

int synth_tc_kp(const SocsGeom& g) { return 64 * synth_ka(g); }

int synth_tc_build_basis(const SocsGeom& g, void* bhi, void* blo, cudaStream_t st) {
  const int Kp = synth_tc_kp(g);
  const size_t n = (size_t)g.Lx * Kp;
  k_synth_basis<<<(int)std::min<size_t>((n + 255) / 256, 4096), 256, 0, st>>>(
      g.Lx, g.ntx, Kp, static_cast<__half*>(bhi), static_cast<__half*>(blo));
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

namespace {
template <int RJ, int KA>
int launch_synth(const SocsGeom& g, const float2* T, const float2* ty, int nsplit, const void* bhi, const void* blo,
                 int nimg, float* images, int* err, cudaStream_t st) {
  const int Kp = 64 * KA;
  CUtensorMap mh, ml, mi;
  // images as [nimg][J][nS][Lx]: row y = s + nS j of image i
  const unsigned long long dims[4] = {(unsigned long long)g.Lx, (unsigned long long)g.nS, (unsigned long long)g.J,
                                      (unsigned long long)nimg};
  const unsigned long long strides[3] = {4ull * g.Lx, 4ull * g.Lx * g.nS, 4ull * g.Lx * g.Ly};
  int rc;
  if ((rc = tc::make_map_2b(&mh, bhi, g.Lx, Kp, 64, kNT, CU_TENSOR_MAP_DATA_TYPE_FLOAT16)) ||
      (rc = tc::make_map_2b(&ml, blo, g.Lx, Kp, 64, kNT, CU_TENSOR_MAP_DATA_TYPE_FLOAT16)) ||
      (rc = tc::make_map_f32_rows(&mi, images, dims, strides)))
    return rc;
  const SynthSmem L = synth_smem(g.nty, g.ntx, kRows / (32 * RJ));
  // one CTA per SM: the kernel allocates all 512 TMEM columns, and the shared
  // memory request keeps a second CTA off the SM
  const size_t sm = std::max<size_t>(L.total, 120 * 1024) + 1024;
  auto kern = k_socs_synth_tc<RJ, KA>;
  KL_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int dev = 0, sms = 148;
  KL_CUDA_TRY(cudaGetDevice(&dev));
  KL_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // runs of equal length: every CTA but possibly the last takes `per` tiles
  const int tiles = nimg * (g.Ly / kRows);
  const int per = (tiles + sms - 1) / sms;
  const int grid = (tiles + per - 1) / per;
  kern<<<grid, kSThreads, sm, st>>>(T, g, ty, nsplit, mh, ml, mi, nimg, err);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}
}  // namespace

bool synth_tc_aligned(const float* images) { return (reinterpret_cast<uintptr_t>(images) & 15) == 0; }

int synth_tc_launch(const SocsGeom& g, const float2* T, const float2* ty, int nsplit, const void* bhi,
                    const void* blo, int nimg, float* images, int* err, cudaStream_t st) {
  if (nimg <= 0) return KL_OK;
  if (!synth_tc_supported(g) || !synth_tc_aligned(images)) {
    set_error("synth_tc_launch: geometry or image alignment outside the tensor-core synthesis");
    return KL_ERR_UNSUPPORTED;
  }
  const int RJ = g.J / 32, KA = synth_ka(g);
  if (RJ == 1 && KA == 1) return launch_synth<1, 1>(g, T, ty, nsplit, bhi, blo, nimg, images, err, st);
  if (RJ == 1 && KA == 2) return launch_synth<1, 2>(g, T, ty, nsplit, bhi, blo, nimg, images, err, st);
  if (RJ == 2 && KA == 1) return launch_synth<2, 1>(g, T, ty, nsplit, bhi, blo, nimg, images, err, st);
  if (RJ == 2 && KA == 2) return launch_synth<2, 2>(g, T, ty, nsplit, bhi, blo, nimg, images, err, st);
  if (RJ == 4 && KA == 1) return launch_synth<4, 1>(g, T, ty, nsplit, bhi, blo, nimg, images, err, st);
  return launch_synth<4, 2>(g, T, ty, nsplit, bhi, blo, nimg, images, err, st);
}

}  // namespace kl
