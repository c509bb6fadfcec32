// socs_vjp.cu -- hand-written adjoint (vector-Jacobian product) of the SOCS
// image under a sigmoid resist model and an L2 loss.  No counterpart in the
// reference; the forward model is K-Litho-SOCS/klitho_socs.cpp:196-241.
//
//   I(x)  = sum_k lam_k |E_k(x)|^2 ,  E_k(x) = sum_f H_k[f] M[f] e^{2 pi i f.(x-d)/L}
//   L     = sum_x (s(x) - t(x))^2 ,   s = 1 / (1 + exp(-a (I - c)))
//   G(x)  = dL/dI = 2 (s - t) s (1 - s) a
//   dL/dm[y] = (2/(LxLy)) Re sum_f Gam[f] e^{-2 pi i f.y/L},
//   Gam[f]   = sum_k lam_k H_k[f] B_k[f],
//   B_k[f]   = sum_x G(x) conj(E_k(x)) e^{2 pi i f.(x-d)/L}
//            = coefficient of e^{-2 pi i f.s} in conj(e_k(s)) gam(s),
//   gam(s)   = sum_{|g|<=2N} Gb[g] e^{-2 pi i g.s},  Gb[g] = sum_x G(x) e^{2 pi i g.(x-d)/L}
// Both factors are band-limited, so B_k is exact from samples on the same
// G x G grid the forward pass uses (G >= 4N+1): the K coherent fields are
// recomputed on chip and never stored.
//
// Source weights (through the TCC factor A = sqrt(J) P, the Hopkins model):
//   dL/dJ_s = sum_x G(x) |E_s(x)|^2 = (1/G^2) sum_p gam(p) |e_s(p)|^2 / J_s
// with e_s built from the kernel conj(A[:, s]).
//
// Kernels: k_vjp_inverse (image rows + loss + row DFT of G, fused; HBM-bound),
// k_vjp_spectral (per clip and kernel slice: Gam), k_vjp_gradT (Gam -> the
// half-plane spectrum of the gradient, synthesised by k_socs_inverse), and
// k_vjp_source (per clip and source slice: dL/dJ).
#include <cuda_pipeline.h>

#include <algorithm>
#include <climits>

#include "kl_device.cuh"
#include "kl_internal.h"

namespace kl {

namespace {
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
}  // namespace

// ---------------------------------------------------------------------------
// image rows + loss + forward row DFT of G (bins gx in [0, 2Nx])
// ---------------------------------------------------------------------------
template <int P, int V, int NBM, int RJ>
__global__ void __launch_bounds__(kThreads, 2) k_vjp_inverse(const float2* __restrict__ T,
                                                          const SocsGeom g,
                                                          const float2* __restrict__ tx,
                                                          const float2* __restrict__ ty,
                                                          int nsplit, int nsets,
                                                          const float* __restrict__ targets,
                                                          float alpha, float thr,
                                                          float* __restrict__ images,
                                                          double* __restrict__ loss,
                                                          float2* __restrict__ gpart) {
  constexpr int J = 32 * RJ;
  constexpr int QP = NBM + 1;
  extern __shared__ float4 smem4[];
  float2* tw = reinterpret_cast<float2*>(smem4);  // [NBM][V] e^{-2 pi i b l'/Lx}
  float2* Qs = tw + NBM * V;                       // [J][QP]
  float2* Gr = Qs + J * QP;                        // [J][NBM]  row bins of G
  float2* Ts = Gr + J * NBM;                       // [nty][ntx]
  float2* ph = Ts + g.nty * g.ntx;                 // [nty]
  // [kWarps][V P] target rows, on a 16-byte boundary (an even float2 offset)
  const int toff = NBM * V + J * QP + J * NBM + g.nty * g.ntx + g.nty;
  float* trows = reinterpret_cast<float*>(reinterpret_cast<float2*>(smem4) + toff + (toff & 1));
  __shared__ double s_loss[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int s = blockIdx.x, img = blockIdx.y, clip = img / nsets;
  const size_t tsz = (size_t)g.nty * g.ntx;
  const float2* Ti = T + (size_t)img * nsplit * tsz;

  for (int i = threadIdx.x; i < (int)tsz; i += kThreads) {
    float2 v = __ldg(Ti + i);
    for (int p = 1; p < nsplit; ++p) v = cadd(v, __ldg(Ti + p * tsz + i));
    Ts[i] = v;
  }
  for (int i = threadIdx.x; i < NBM * V; i += kThreads) tw[i] = __ldg(tx + i);
  for (int i = threadIdx.x; i < g.nty; i += kThreads) ph[i] = __ldg(ty + (size_t)s * g.nty + i);
  for (int i = threadIdx.x; i < J * QP; i += kThreads) Qs[i] = make_float2(0.f, 0.f);
  __syncthreads();

  const int br = (int)(__brev((unsigned)lane) >> 27);
  const int A = 2 * g.Ny;
  {
    WarpFFT<RJ, +1> wf;
    wf.init(lane);
    for (int b = warp; b < g.ntx; b += kWarps) {
      float2 vv[RJ];
#pragma unroll
      for (int j = 0; j < RJ; ++j) {
        const int n = lane + 32 * j;
        float2 f = make_float2(0.f, 0.f);
        for (int a = n - J * ((n + A) / J); a <= A; a += J) f = cfma(Ts[(a + A) * g.ntx + b], ph[a + A], f);
        vv[j] = f;
      }
      wf.run(vv, lane);
      const float w = b == 0 ? 1.f : 2.f;
#pragma unroll
      for (int q1 = 0; q1 < RJ; ++q1) Qs[(q1 + RJ * br) * QP + b] = cscale(vv[q1], w);
    }
  }
  __syncthreads();

  const size_t px = (size_t)g.Lx * g.Ly;
  float* out = images ? images + (size_t)img * px : nullptr;
  const float* tgt = targets + (size_t)clip * px;
  double lsum = 0.0;
  float* trow = trows + warp * (V * P);
  for (int jj = warp; jj < J; jj += kWarps) {
    const size_t roff = (size_t)(s + g.nS * jj) * (V * P);
    const float2* q = Qs + jj * QP;
    // the row's targets go to shared memory asynchronously while the row is
    // synthesised (16-byte pieces; rows start on 16-byte boundaries)
    for (int m = lane; m < V * P / 4; m += 32) __pipeline_memcpy_async(trow + 4 * m, tgt + roff + 4 * m, 16);
    __pipeline_commit();
    // row DFT of G, bins gx in [0, NBM): reduce-scattered over the warp in two
    // halves of NBM floats, each lane keeping NBM/32 sums per half
    constexpr int PER = NBM / 32;
    float red[2][PER];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int i = 0; i < PER; ++i) red[h][i] = 0.f;
#pragma unroll 1
    for (int c = 0; c < V / 32; ++c) {
      const int lp = lane + 32 * c;
      float o[P];
      {
        // the Hermitian fold of the lane's sub-bins, accumulated in the order of
        // k_socs_inverse so that the image equals the forward pass's bit for bit
        float2 Y[P / 2 + 1];
#pragma unroll
        for (int i = 0; i <= P / 2; ++i) Y[i] = make_float2(0.f, 0.f);
#pragma unroll
        for (int b = 0; b < NBM; ++b) {
          const float2 qb = q[b], w = tw[b * V + lp];
          const int k = b % P;
          if (2 * k <= P) {
            Y[k] = make_float2(fmaf(qb.x, w.x, fmaf(qb.y, w.y, Y[k].x)),
                               fmaf(qb.y, w.x, fmaf(-qb.x, w.y, Y[k].y)));
          } else {
            Y[P - k] = make_float2(fmaf(qb.x, w.x, fmaf(qb.y, w.y, Y[P - k].x)),
                                   fmaf(-qb.y, w.x, fmaf(qb.x, w.y, Y[P - k].y)));
          }
        }
        c2r_half<P>(Y, o);
      }
      // resist model, loss and dL/dI on the lane's pixels
      __pipeline_wait_prior(0);
      __syncwarp();
      float rsum = 0.f;  // the lane's P pixels; added to the double total once per row
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const size_t x = roff + lp + V * i;
        if (out) out[x] = o[i];
        const float sg = __frcp_rn(1.0f + __expf(-alpha * (o[i] - thr)));
        const float d = sg - trow[lp + V * i];
        rsum = fmaf(d, d, rsum);
        o[i] = 2.0f * d * sg * (1.0f - sg) * alpha;
      }
      lsum += (double)rsum;
      float2 S[P / 2 + 1];
      rdft_reg<P>(o, S);
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float acc[NBM];
#pragma unroll
        for (int j = 0; j < NBM / 2; ++j) {
          const int gx = h * (NBM / 2) + j;
          const int k = gx % P;
          const float2 sv = (k <= P / 2) ? S[k] : cconj(S[P - k]);
          const float2 w = tw[gx * V + lp];
          acc[2 * j] = fmaf(sv.x, w.x, -sv.y * w.y);
          acc[2 * j + 1] = fmaf(sv.x, w.y, sv.y * w.x);
        }
        warp_reduce_scatter<NBM>(acc, lane);
#pragma unroll
        for (int i = 0; i < PER; ++i) red[h][i] += acc[i];
      }
    }
    float* rb = reinterpret_cast<float*>(Gr + jj * NBM);
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int i = 0; i < PER; ++i) rb[h * NBM + lane * PER + i] = red[h][i];
    __syncwarp();  // every lane has read trow before the next row's copy
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) s_loss[warp] = lsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kWarps; ++w) t += s_loss[w];
    atomicAdd(loss + img, t);
  }
  // column DFT of the strip: bins gy in [-2Ny, 2Ny] (J >= 4Ny+1)
  WarpFFT<RJ, -1> wc;
  wc.init(lane);
  const int ng = 2 * g.Nx + 1;
  for (int gx = warp; gx < ng; gx += kWarps) {
    float2 vv[RJ];
#pragma unroll
    for (int j = 0; j < RJ; ++j) vv[j] = Gr[(lane + 32 * j) * NBM + gx];
    wc.run(vv, lane);
#pragma unroll
    for (int q1 = 0; q1 < RJ; ++q1) {
      const int bin = q1 + RJ * br;
      const int gy = bin <= J / 2 ? bin : bin - J;
      if (gy >= -A && gy <= A)
        gpart[(((size_t)img * g.nS + s) * g.nty + (gy + A)) * ng + gx] = cmulc(vv[q1], ph[gy + A]);
    }
  }
}

// ---------------------------------------------------------------------------
// shared helpers of the spectral adjoint kernels
// ---------------------------------------------------------------------------
// Gb[g] on the full band |gy| <= 2Ny, |gx| <= 2Nx ([4Ny+1][4Nx+1]) from the strip
// partials of G's spectrum, conjugated and shifted as the forward model's d.
__device__ void load_gbar(const float2* __restrict__ gpart, const SocsGeom& g, int img,
                          float2* Gb) {
  const int ng = 2 * g.Nx + 1, W = 4 * g.Nx + 1, A = 2 * g.Ny;
  const size_t per = (size_t)g.nty * ng;
  const float2* p0 = gpart + (size_t)img * g.nS * per;
  for (int i = threadIdx.x; i < g.nty * ng; i += blockDim.x) {
    const int r = i / ng, gx = i - r * ng, gy = r - A;
    float2 v = make_float2(0.f, 0.f);
    for (int s = 0; s < g.nS; ++s) v = cadd(v, __ldg(p0 + (size_t)s * per + i));
    // Gb = e^{-2 pi i g.d/L} conj(Ghat)
    float2 gb = cconj(v);
    if (g.dx | g.dy) {
      const float2 e = cmul(expi2pi_frac(-(long long)gy * g.dy, g.Ly), expi2pi_frac(-(long long)gx * g.dx, g.Lx));
      gb = cmul(gb, e);
    }
    Gb[r * W + 2 * g.Nx + gx] = gb;
    if (gx > 0) Gb[(2 * A - r) * W + 2 * g.Nx - gx] = cconj(gb);
  }
}

// gam(p) = Re sum_g Gb[g] e^{-2 pi i g.p/G} on the G x G grid (gam: [G][GP])
template <int RG>
__device__ void make_gamma(const SocsGeom& g, const float2* Gb, float2* scratch, float* gam,
                           int lane, int warp) {
  constexpr int G = 32 * RG, GP = G + 1;
  const int W = 4 * g.Nx + 1, A = 2 * g.Ny, Bx = 2 * g.Nx;
  const int br = (int)(__brev((unsigned)lane) >> 27);
  WarpFFT<RG, -1> wf;
  wf.init(lane);
  for (int r = warp; r < g.nty; r += kWarps) {
    float2 vv[RG];
#pragma unroll
    for (int j = 0; j < RG; ++j) {
      const int n = lane + 32 * j;
      const int gx = n <= Bx ? n : (n >= G - Bx ? n - G : INT_MIN);
      vv[j] = gx != INT_MIN ? Gb[r * W + Bx + gx] : make_float2(0.f, 0.f);
    }
    wf.run(vv, lane);
#pragma unroll
    for (int q1 = 0; q1 < RG; ++q1) scratch[r * GP + q1 + RG * br] = vv[q1];
  }
  __syncthreads();
  for (int q = warp; q < G; q += kWarps) {
    float2 vv[RG];
#pragma unroll
    for (int j = 0; j < RG; ++j) {
      const int n = lane + 32 * j;
      const int gy = n <= A ? n : (n >= G - A ? n - G : INT_MIN);
      vv[j] = gy != INT_MIN ? scratch[(gy + A) * GP + q] : make_float2(0.f, 0.f);
    }
    wf.run(vv, lane);
#pragma unroll
    for (int q1 = 0; q1 < RG; ++q1) gam[(q1 + RG * br) * GP + q] = vv[q1].x;
  }
  __syncthreads();
}

__device__ __forceinline__ void load_band_v(const float2* __restrict__ partial, const SocsGeom& g,
                                            int clip, float2* Cm) {
  const float inv = 1.0f / ((float)g.Lx * (float)g.Ly);
  const size_t per = (size_t)g.nby * g.nf;
  const float2* p0 = partial + (size_t)clip * g.nS * per;
  for (int i = threadIdx.x; i < g.nby * g.nf; i += blockDim.x) {
    const int r = i / g.nf, fx = i - r * g.nf;
    float2 sum = make_float2(0.f, 0.f);
    for (int s = 0; s < g.nS; ++s) sum = cadd(sum, __ldg(p0 + (size_t)s * per + i));
    sum = cscale(sum, inv);
    Cm[r * g.nbx + g.Nx + fx] = sum;
    if (fx > 0) Cm[(2 * g.Ny - r) * g.nbx + g.Nx - fx] = cconj(sum);
  }
}

// e_k on the grid: stage 1 (rows fy, along x) into E1 [nby][GP], then the
// caller's stage 2 reads columns.  Sign +1.
template <int RG>
__device__ __forceinline__ void field_rows(const SocsGeom& g, const float2* __restrict__ Hk,
                                           const float2* Cm, float2* E1, const WarpFFT<RG, +1>& wi,
                                           int lane, int warp) {
  constexpr int G = 32 * RG, GP = G + 1;
  const int br = (int)(__brev((unsigned)lane) >> 27);
  for (int r = warp; r < g.nby; r += kWarps) {
    float2 vv[RG];
#pragma unroll
    for (int j = 0; j < RG; ++j) {
      const int n = lane + 32 * j;
      const int fx = n <= g.Nx ? n : (n >= G - g.Nx ? n - G : INT_MIN);
      vv[j] = make_float2(0.f, 0.f);
      if (fx != INT_MIN) {
        const int o = r * g.nbx + fx + g.Nx;
        vv[j] = cmul(__ldg(Hk + o), Cm[o]);
      }
    }
    wi.run(vv, lane);
#pragma unroll
    for (int q1 = 0; q1 < RG; ++q1) E1[r * GP + q1 + RG * br] = vv[q1];
  }
}

// ---------------------------------------------------------------------------
// Gam partial per (clip, set, kernel slice)
// ---------------------------------------------------------------------------
template <int RG>
__global__ void __launch_bounds__(kThreads) k_vjp_spectral(const float2* __restrict__ partial,
                                                           const float2* __restrict__ gpart,
                                                           const SocsGeom g,
                                                           const float2* __restrict__ H,
                                                           const float* __restrict__ lam, int K,
                                                           float2* __restrict__ gam_out) {
  constexpr int G = 32 * RG, GP = G + 1;
  extern __shared__ float4 smem4[];
  const int nb2 = g.nby * g.nbx;
  float2* Cm = reinterpret_cast<float2*>(smem4);    // [nby][nbx]
  float2* Gacc = Cm + nb2;                           // [nby][nbx]
  float2* E1 = Gacc + nb2;                           // [G][GP]  (G >= nby, nty)
  float* gam = reinterpret_cast<float*>(E1 + G * GP);  // [G][GP]
  // the band of dL/dI is read only while gam is made; the per-kernel stages
  // then reuse its space (two CTAs per SM at 1024^2)
  float2* Gb = reinterpret_cast<float2*>(gam + G * GP);  // [nty][W]
  float2* Wg = Gb;                                        // [G][GP]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int clip = blockIdx.x, set = blockIdx.y, split = blockIdx.z;
  const int nsets = gridDim.y, nsplit = gridDim.z;
  const int img = clip * nsets + set;
  const int k0 = (int)(((long long)K * split) / nsplit), k1 = (int)(((long long)K * (split + 1)) / nsplit);
  const int br = (int)(__brev((unsigned)lane) >> 27);

  load_band_v(partial, g, clip, Cm);
  load_gbar(gpart, g, img, Gb);
  for (int i = threadIdx.x; i < nb2; i += kThreads) Gacc[i] = make_float2(0.f, 0.f);
  __syncthreads();
  make_gamma<RG>(g, Gb, E1, gam, lane, warp);

  WarpFFT<RG, +1> wi;
  wi.init(lane);
  const float invg2 = 1.0f / ((float)G * (float)G);
  const size_t nbs = (size_t)nb2;
  const float2* Hs = H + (size_t)set * K * nbs;
  for (int k = k0; k < k1; ++k) {
    const float2* Hk = Hs + (size_t)k * nbs;
    const float lk = __ldg(lam + set * K + k) * invg2;
    field_rows<RG>(g, Hk, Cm, E1, wi, lane, warp);
    __syncthreads();
    // stage 2: columns q -> e(p, q); w = conj(e) gam
    for (int q = warp; q < G; q += kWarps) {
      float2 vv[RG];
#pragma unroll
      for (int j = 0; j < RG; ++j) {
        const int n = lane + 32 * j;
        const int fy = n <= g.Ny ? n : (n >= G - g.Ny ? n - G : INT_MIN);
        vv[j] = (fy != INT_MIN) ? E1[(fy + g.Ny) * GP + q] : make_float2(0.f, 0.f);
      }
      wi.run(vv, lane);
#pragma unroll
      for (int q1 = 0; q1 < RG; ++q1) {
        const int p = q1 + RG * br;
        Wg[p * GP + q] = cscale(cconj(vv[q1]), gam[p * GP + q]);
      }
    }
    __syncthreads();
    // stage 3: rows p, transform along x (sign +1), keep |fx| <= Nx -> E1[p][fx+Nx]
    for (int p = warp; p < G; p += kWarps) {
      float2 vv[RG];
#pragma unroll
      for (int j = 0; j < RG; ++j) vv[j] = Wg[p * GP + lane + 32 * j];
      wi.run(vv, lane);
#pragma unroll
      for (int q1 = 0; q1 < RG; ++q1) {
        const int bin = q1 + RG * br;
        const int fx = bin <= G / 2 ? bin : bin - G;
        if (fx >= -g.Nx && fx <= g.Nx) E1[p * GP + fx + g.Nx] = vv[q1];
      }
    }
    __syncthreads();
    // stage 4: columns fx, transform along y (sign +1), keep |fy| <= Ny -> B
    for (int c = warp; c < g.nbx; c += kWarps) {
      float2 vv[RG];
#pragma unroll
      for (int j = 0; j < RG; ++j) vv[j] = E1[(lane + 32 * j) * GP + c];
      wi.run(vv, lane);
#pragma unroll
      for (int q1 = 0; q1 < RG; ++q1) {
        const int bin = q1 + RG * br;
        const int fy = bin <= G / 2 ? bin : bin - G;
        if (fy >= -g.Ny && fy <= g.Ny) {
          const int o = (fy + g.Ny) * g.nbx + c;
          Gacc[o] = cfma(cscale(__ldg(Hk + o), lk), vv[q1], Gacc[o]);
        }
      }
    }
    __syncthreads();
  }
  float2* out = gam_out + (((size_t)clip * nsets + set) * nsplit + split) * nbs;
  for (int i = threadIdx.x; i < nb2; i += kThreads) out[i] = Gacc[i];
}

// ---------------------------------------------------------------------------
// Gam partials -> half-plane spectrum of dL/dm (for k_socs_inverse)
// T[a][b] = (conj Gam[f] + Gam[-f]) / (Lx Ly), f = (a, b), |a| <= Ny, b <= Nx
// ---------------------------------------------------------------------------
__global__ void k_vjp_gradT(const float2* __restrict__ gam, const SocsGeom g, int nparts,
                            float2* __restrict__ T) {
  const int clip = blockIdx.x;
  const size_t nbs = (size_t)g.nby * g.nbx;
  const float2* p0 = gam + (size_t)clip * nparts * nbs;
  const float s = 1.0f / ((float)g.Lx * (float)g.Ly);
  float2* To = T + (size_t)clip * g.nty * g.ntx;
  for (int i = threadIdx.x; i < g.nty * g.ntx; i += blockDim.x) {
    const int r = i / g.ntx, b = i - r * g.ntx, a = r - 2 * g.Ny;
    float2 v = make_float2(0.f, 0.f);
    if (a >= -g.Ny && a <= g.Ny && b <= g.Nx) {
      const size_t o1 = (size_t)(a + g.Ny) * g.nbx + (b + g.Nx);
      const size_t o2 = (size_t)(-a + g.Ny) * g.nbx + (-b + g.Nx);
      float2 f1 = make_float2(0.f, 0.f), f2 = make_float2(0.f, 0.f);
      for (int p = 0; p < nparts; ++p) {
        f1 = cadd(f1, p0[p * nbs + o1]);
        f2 = cadd(f2, p0[p * nbs + o2]);
      }
      v = cscale(cadd(cconj(f1), f2), s);
    }
    To[i] = v;
  }
}

// ---------------------------------------------------------------------------
// dL/dJ per (image, source slice): (1/G^2) sum_p gam |e_s|^2 / J_s
// ---------------------------------------------------------------------------
template <int RG>
__global__ void __launch_bounds__(kThreads) k_vjp_source(const float2* __restrict__ partial,
                                                         const float2* __restrict__ gpart,
                                                         const SocsGeom g,
                                                         const float2* __restrict__ Hs,  // S x band: conj A
                                                         const float* __restrict__ Jw,
                                                         const int* __restrict__ src_id, int S,
                                                         int nsets, float* __restrict__ grad_src) {
  constexpr int G = 32 * RG, GP = G + 1;
  extern __shared__ float4 smem4[];
  const int nb2 = g.nby * g.nbx;
  const int W = 4 * g.Nx + 1;
  float2* Cm = reinterpret_cast<float2*>(smem4);
  float2* Gb = Cm + nb2;
  float2* E1 = Gb + g.nty * W;                      // [G][GP]
  float* gam = reinterpret_cast<float*>(E1 + G * GP);
  __shared__ float s_red[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int img = blockIdx.x, split = blockIdx.y, nsplit = gridDim.y;
  const int clip = img / nsets;
  const int s0 = (int)(((long long)S * split) / nsplit), s1 = (int)(((long long)S * (split + 1)) / nsplit);
  const int br = (int)(__brev((unsigned)lane) >> 27);

  load_band_v(partial, g, clip, Cm);
  load_gbar(gpart, g, img, Gb);
  __syncthreads();
  make_gamma<RG>(g, Gb, E1, gam, lane, warp);
  WarpFFT<RG, +1> wi;
  wi.init(lane);
  const float invg2 = 1.0f / ((float)G * (float)G);
  for (int s = s0; s < s1; ++s) {
    field_rows<RG>(g, Hs + (size_t)s * nb2, Cm, E1, wi, lane, warp);
    __syncthreads();
    float part = 0.f;
    for (int q = warp; q < G; q += kWarps) {
      float2 vv[RG];
#pragma unroll
      for (int j = 0; j < RG; ++j) {
        const int n = lane + 32 * j;
        const int fy = n <= g.Ny ? n : (n >= G - g.Ny ? n - G : INT_MIN);
        vv[j] = (fy != INT_MIN) ? E1[(fy + g.Ny) * GP + q] : make_float2(0.f, 0.f);
      }
      wi.run(vv, lane);
#pragma unroll
      for (int q1 = 0; q1 < RG; ++q1) part = fmaf(gam[(q1 + RG * br) * GP + q], cabs2(vv[q1]), part);
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) s_red[warp] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      float t = 0.f;
      for (int w = 0; w < kWarps; ++w) t += s_red[w];
      atomicAdd(grad_src + src_id[s], t * invg2 / Jw[s]);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
namespace {
template <typename Kern>
int set_smem(Kern k, size_t bytes) {
  if (bytes > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) {
      set_error(std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
      return KL_ERR_CUDA;
    }
  }
  return KL_OK;
}
int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return KL_ERR_CUDA;
  }
  return KL_OK;
}

template <int P, int V, int NBM, int RJ>
int launch_vinv(const SocsGeom& g, const float2* tx, const float2* ty, const float2* T, int nimg,
                int nsplit, int nsets, const float* targets, float alpha, float thr, float* images,
                double* loss, float2* gpart, cudaStream_t st) {
  constexpr int J = 32 * RJ;
  const size_t toff = (size_t)NBM * V + (size_t)J * (NBM + 1) + (size_t)J * NBM + (size_t)g.nty * g.ntx + g.nty;
  size_t sm = sizeof(float2) * (toff + (toff & 1)) + sizeof(float) * (size_t)kWarps * V * P;
  auto kern = k_vjp_inverse<P, V, NBM, RJ>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  kern<<<dim3(g.nS, nimg), kThreads, sm, st>>>(T, g, tx, ty, nsplit, nsets, targets, alpha, thr,
                                                 images, loss, gpart);
  return check_launch("k_vjp_inverse");
}

size_t vjp_spectral_smem(const SocsGeom& g) {
  const int G = g.G, GP = G + 1, nb2 = g.nby * g.nbx, W = 4 * g.Nx + 1;
  const size_t shared = std::max((size_t)g.nty * W, (size_t)G * GP);  // dL/dI band, then Wg
  return sizeof(float2) * ((size_t)2 * nb2 + (size_t)G * GP + shared) + sizeof(float) * (size_t)G * GP;
}
size_t vjp_source_smem(const SocsGeom& g) {
  const int G = g.G, GP = G + 1, nb2 = g.nby * g.nbx, W = 4 * g.Nx + 1;
  return sizeof(float2) * ((size_t)nb2 + (size_t)g.nty * W + (size_t)G * GP) +
         sizeof(float) * (size_t)G * GP;
}
}  // namespace

int vjp_supported(const SocsGeom& g) {
  if (g.NBM != 32 || g.J < g.nty || (g.J != 32 && g.J != 64) || g.G > 64) {
    set_error("the adjoint supports 2Nx+1 <= 32, 4Ny+1 <= 64 (clips up to 1024^2 at NA 1.35)");
    return KL_ERR_UNSUPPORTED;
  }
  return KL_OK;
}

size_t vjp_gpart_bytes(const SocsGeom& g, int nimg) {
  return sizeof(float2) * (size_t)nimg * g.nS * g.nty * (2 * g.Nx + 1);
}

int vjp_launch_inverse(const SocsGeom& g, const float2* tx, const float2* ty, const float2* T,
                       int nclips, int nsets, int nsplit, const float* targets, float alpha,
                       float thr, float* images, double* loss, float2* gpart, cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  const int RJ = g.J / 32, nimg = nclips * nsets;
#define KL_VINV(P_, V_, R_)                               \
  if (g.P == P_ && g.V == V_ && RJ == R_)               \
    return launch_vinv<P_, V_, 32, R_>(g, tx, ty, T, nimg, nsplit, nsets, targets, alpha, thr, images, loss, gpart, st);
  KL_VINV(8, 32, 1) KL_VINV(8, 32, 2) KL_VINV(16, 32, 1) KL_VINV(16, 32, 2)
  KL_VINV(32, 32, 1) KL_VINV(32, 32, 2) KL_VINV(32, 64, 1) KL_VINV(32, 64, 2)
  KL_VINV(8, 96, 1) KL_VINV(8, 96, 2) KL_VINV(16, 96, 1) KL_VINV(16, 96, 2)
#undef KL_VINV
  set_error("vjp_launch_inverse: no kernel for this geometry");
  return KL_ERR_UNSUPPORTED;
}

int vjp_launch_spectral(const SocsGeom& g, const float2* partial, const float2* gpart, int nclips,
                        const float2* H, const float* lam, int K, int nsets, int nsplit,
                        float2* gam_out, cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  const size_t sm = vjp_spectral_smem(g);
  if (g.G == 32) {
    int rc = set_smem(k_vjp_spectral<1>, sm);
    if (rc) return rc;
    k_vjp_spectral<1><<<dim3(nclips, nsets, nsplit), kThreads, sm, st>>>(partial, gpart, g, H, lam, K, gam_out);
  } else {
    int rc = set_smem(k_vjp_spectral<2>, sm);
    if (rc) return rc;
    k_vjp_spectral<2><<<dim3(nclips, nsets, nsplit), kThreads, sm, st>>>(partial, gpart, g, H, lam, K, gam_out);
  }
  return check_launch("k_vjp_spectral");
}

int vjp_launch_gradT(const SocsGeom& g, const float2* gam, int nclips, int nparts, float2* T,
                     cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  k_vjp_gradT<<<nclips, kThreads, 0, st>>>(gam, g, nparts, T);
  return check_launch("k_vjp_gradT");
}

int vjp_launch_source(const SocsGeom& g, const float2* partial, const float2* gpart, int nimg,
                      int nsets, const float2* Hs, const float* Jw, const int* src_id, int S,
                      int nsplit, float* grad_src, cudaStream_t st) {
  if (nimg <= 0) return KL_OK;
  const size_t sm = vjp_source_smem(g);
  if (g.G == 32) {
    int rc = set_smem(k_vjp_source<1>, sm);
    if (rc) return rc;
    k_vjp_source<1><<<dim3(nimg, nsplit), kThreads, sm, st>>>(partial, gpart, g, Hs, Jw, src_id, S, nsets, grad_src);
  } else {
    int rc = set_smem(k_vjp_source<2>, sm);
    if (rc) return rc;
    k_vjp_source<2><<<dim3(nimg, nsplit), kThreads, sm, st>>>(partial, gpart, g, Hs, Jw, src_id, S, nsets, grad_src);
  }
  return check_launch("k_vjp_source");
}

}  // namespace kl
