// socs_fast.cu -- fused single-precision SOCS imaging for sm_100a.
//
// Computes, for every mask clip m (Ly x Lx, 1 nm pixels) and kernel set
// {H_k, lambda_k}, the K-Litho SOCS image
//     image = sum_k lambda_k |IFFT(H_k . FT(m))|^2 , Fourier-interpolated to Lx x Ly
// (K-Litho-SOCS/klitho_socs.cpp:196-241 calcSOCS + :158-194 FI, fed by
// FT_r2c :70-121), without ever materialising the K coherent fields or a
// full-size spectrum in HBM.  Three stream-ordered kernels:
//
//  1. k_socs_forward  (HBM-bound; reads the mask once)
//     One CTA per (clip, strip of J rows spaced Ly/J apart).  Each warp turns
//     a row into its Nx+1 non-negative x-frequency bins: lane l' holds
//     pixels x = l' + V*i, does an in-register real DFT of length P over i,
//     multiplies by e^{-2 pi i fx l'/Lx} and the warp reduce-scatters the
//     bins.  The strip's J rows then go through a J-point warp FFT along y
//     (rows are J-periodic in the strip), giving the strip's partial band
//     spectrum D_s[fy][fx], |fy| <= Ny.
//  2. k_socs_spectral (on-chip; CTAs per clip, kernel set and kernel slice)
//     Sums the strip partials into the band spectrum, then for each kernel
//     of its slice forms H_k . M, runs a pruned 2-D inverse FFT on a G x G
//     grid (G >= 4N+1, so |E_k|^2 is sampled without aliasing) with warp FFTs
//     in shared memory and accumulates lambda_k |E_k|^2 in registers.  A
//     forward 2-D FFT of that intensity gives the slice's share of the exact
//     band-limited intensity spectrum T[a][b], |a| <= 2Ny, 0 <= b <= 2Nx.
//  3. k_socs_inverse  (HBM-bound; writes the image once)
//     One CTA per (image, strip).  Sums the slices of T, forms the strip's
//     rows by a J-point warp FFT along y, and each warp synthesises a row of
//     Lx real pixels from its 2Nx+1 bins with a real-output length-P inverse
//     DFT per lane.
//
// Twiddle factors that depend on the clip size are made once per plan
// (k_socs_tables, exact double-precision arguments) and read from L2.
// Only the strip partials, T and the tables pass through global memory.
#include <climits>

#include "kl_device.cuh"
#include "kl_internal.h"

namespace kl {

namespace {
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__host__ __device__ inline int pow2_at_least(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}
}  // namespace

int socs_geometry(int Lx, int Ly, int Nx, int Ny, SocsGeom* g, bool adjoint) {
  if (Lx <= 0 || Ly <= 0 || Nx < 0 || Ny < 0) {
    set_error("socs_geometry: invalid sizes");
    return KL_ERR_INVALID;
  }
  SocsGeom r{};
  r.Lx = Lx;
  r.Ly = Ly;
  r.Nx = Nx;
  r.Ny = Ny;
  r.nbx = 2 * Nx + 1;
  r.nby = 2 * Ny + 1;
  r.nf = Nx + 1;
  r.ntx = 2 * Nx + 1;
  r.nty = 4 * Ny + 1;
  if (Lx % 1024 == 0)
    r.P = 32;
  else if (Lx % 512 == 0)
    r.P = 16;
  else if (Lx % 256 == 0)
    r.P = 8;
  else {
    set_error("fast SOCS path needs Lx to be a multiple of 256 (got " + std::to_string(Lx) + ")");
    return KL_ERR_UNSUPPORTED;
  }
  r.V = Lx / r.P;
  if (r.V != 32 && r.V != 64 && r.V != 96) {
    set_error("fast SOCS path supports Lx in {256, 512, 768, 1024, 1536, 2048, 3072} (got " +
              std::to_string(Lx) + ")");
    return KL_ERR_UNSUPPORTED;
  }
  if (r.nf <= 16)
    r.NFM = 16;
  else if (r.nf <= 32)
    r.NFM = 32;
  else {
    set_error("fast SOCS path supports Nx <= 31 (got " + std::to_string(Nx) + ")");
    return KL_ERR_UNSUPPORTED;
  }
  r.NBM = r.ntx <= 32 ? 32 : 64;
  r.KX = r.NBM > r.NFM ? r.NBM : r.NFM;
  r.J = pow2_at_least(adjoint ? r.nty : r.nby);
  if (r.J < 32) r.J = 32;
  if (r.J > (adjoint ? 128 : 64) || Ly % r.J != 0) {
    set_error("fast SOCS path needs Ly divisible by " + std::to_string(r.J) +
              (adjoint ? " and 4Ny+1 <= 128" : " and Ny <= 31"));
    return KL_ERR_UNSUPPORTED;
  }
  r.nS = Ly / r.J;
  int gmin = 4 * (Nx > Ny ? Nx : Ny) + 1;
  r.G = pow2_at_least(gmin);
  if (r.G < 32) r.G = 32;
  if (r.G > 128) {
    set_error("fast SOCS path needs 4N+1 <= 128");
    return KL_ERR_UNSUPPORTED;
  }
  // a band reaching the Nyquist bin would change the reference's half-spectrum
  // bookkeeping; never the case for physical optics (2N << L/2)
  if (4 * Nx + 1 > Lx / 2 || 4 * Ny + 1 > Ly / 2) {
    set_error("band too wide for the clip size");
    return KL_ERR_UNSUPPORTED;
  }
  r.dx = 2 * ((Lx + 1) / 2) - Lx;
  r.dy = 2 * ((Ly + 1) / 2) - Ly;
  *g = r;
  return KL_OK;
}

size_t socs_partial_bytes(const SocsGeom& g, int nclips) {
  return sizeof(float2) * (size_t)nclips * g.nS * g.nby * g.nf;
}
size_t socs_spectrum_bytes(const SocsGeom& g, int nclips, int nsets, int nsplit) {
  return sizeof(float2) * (size_t)nclips * nsets * nsplit * g.nty * g.ntx;
}
size_t socs_table_x_elems(const SocsGeom& g) { return (size_t)g.KX * g.V; }
size_t socs_table_y_elems(const SocsGeom& g) { return (size_t)g.nS * g.nty; }

int socs_choose_split(const SocsGeom& g, int nclips, int nsets, int K) {
  // enough CTAs to cover the GPU about twice; slices of at least 3 kernels
  const int ctas = nclips * nsets;
  int ns = 1;
  while (ns < kSocsMaxSplit && ctas * ns < 2 * 148 && K / (2 * ns) >= 3) ns *= 2;
  (void)g;
  return ns;
}

// ---------------------------------------------------------------------------
// plan-time tables: tx[k][l'] = e^{-2 pi i k l'/Lx}, ty[s][a+2Ny] = e^{+2 pi i a s/Ly}
// ---------------------------------------------------------------------------
__global__ void k_socs_tables(const SocsGeom g, float2* __restrict__ tx, float2* __restrict__ ty) {
  const int nx = g.KX * g.V, ny = g.nS * g.nty;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nx + ny; i += gridDim.x * blockDim.x) {
    if (i < nx) {
      const int k = i / g.V, lp = i - k * g.V;
      tx[i] = expi2pi_frac(-(long long)k * lp, g.Lx);
    } else {
      const int j = i - nx, s = j / g.nty, a = j - s * g.nty - 2 * g.Ny;
      ty[j] = expi2pi_frac((long long)a * s, g.Ly);
    }
  }
}

int socs_build_tables(const SocsGeom& g, float2* tx, float2* ty, cudaStream_t st) {
  const int n = (int)(socs_table_x_elems(g) + socs_table_y_elems(g));
  k_socs_tables<<<(n + 255) / 256, 256, 0, st>>>(g, tx, ty);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("k_socs_tables: ") + cudaGetErrorString(e));
    return KL_ERR_CUDA;
  }
  return KL_OK;
}

// ---------------------------------------------------------------------------
// 1. forward: mask rows -> per-strip partial band spectra
// ---------------------------------------------------------------------------
template <int P, int V, int NFM, int RJ>
__global__ void __launch_bounds__(kThreads) k_socs_forward(const float* __restrict__ masks,
                                                           const SocsGeom g,
                                                           const float2* __restrict__ tx,
                                                           const float2* __restrict__ ty,
                                                           float2* __restrict__ partial) {
  constexpr int J = 32 * RJ;
  extern __shared__ float4 smem4[];
  float2* twf = reinterpret_cast<float2*>(smem4);  // [NFM][V]   e^{-2 pi i fx l'/Lx}
  float2* rowbuf = twf + NFM * V;                  // [J][NFM]   row bins of the strip
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int s = blockIdx.x, clip = blockIdx.y;
  const float* mask = masks + (size_t)clip * g.Lx * g.Ly;

  for (int i = threadIdx.x; i < NFM * V; i += kThreads) twf[i] = __ldg(tx + i);
  __syncthreads();

  for (int jj = warp; jj < J; jj += kWarps) {
    const float* row = mask + (size_t)(s + g.nS * jj) * (V * P);
    float acc[2 * NFM];
#pragma unroll
    for (int i = 0; i < 2 * NFM; ++i) acc[i] = 0.f;
#pragma unroll 1
    for (int c = 0; c < V / 32; ++c) {
      const int lp = lane + 32 * c;
      float val[P];
#pragma unroll
      for (int i = 0; i < P; ++i) val[i] = __ldcs(row + lp + V * i);
      float2 S[P / 2 + 1];
      rdft_reg<P>(val, S);
#pragma unroll
      for (int fx = 0; fx < NFM; ++fx) {
        const int k = fx % P;
        const float2 sv = (k <= P / 2) ? S[k] : cconj(S[P - k]);
        const float2 w = twf[fx * V + lp];
        acc[2 * fx] = fmaf(sv.x, w.x, fmaf(-sv.y, w.y, acc[2 * fx]));
        acc[2 * fx + 1] = fmaf(sv.x, w.y, fmaf(sv.y, w.x, acc[2 * fx + 1]));
      }
    }
    warp_reduce_scatter<2 * NFM>(acc, lane);
    constexpr int PER = 2 * NFM / 32;
    float* rb = reinterpret_cast<float*>(rowbuf + jj * NFM);
#pragma unroll
    for (int i = 0; i < PER; ++i) rb[lane * PER + i] = acc[i];
  }
  __syncthreads();

  // y-direction: J-point FFT of each fx column of the strip
  WarpFFT<RJ, -1> wf;
  wf.init(lane);
  const int br = (int)(__brev((unsigned)lane) >> 27);
  const float2* tys = ty + (size_t)s * g.nty + 2 * g.Ny;  // e^{+2 pi i a s/Ly} at [a]
  for (int fx = warp; fx < g.nf; fx += kWarps) {
    float2 vv[RJ];
#pragma unroll
    for (int j = 0; j < RJ; ++j) vv[j] = rowbuf[(lane + 32 * j) * NFM + fx];
    wf.run(vv, lane);
#pragma unroll
    for (int q1 = 0; q1 < RJ; ++q1) {
      const int bin = q1 + RJ * br;
      const int fy = bin <= J / 2 ? bin : bin - J;
      if (fy >= -g.Ny && fy <= g.Ny)
        partial[(((size_t)clip * g.nS + s) * g.nby + (fy + g.Ny)) * g.nf + fx] =
            cmulc(vv[q1], __ldg(tys + fy));
    }
  }
}

// ---------------------------------------------------------------------------
// 2. spectral core: band spectrum -> sum_k lambda_k |E_k|^2 -> its spectrum T
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_band(const float2* __restrict__ partial, const SocsGeom& g,
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

template <int RG>
__global__ void __launch_bounds__(kThreads) k_socs_spectral(const float2* __restrict__ partial,
                                                            const SocsGeom g,
                                                            const float2* __restrict__ H,
                                                            const float* __restrict__ lam, int K,
                                                            float2* __restrict__ Tout) {
  constexpr int G = 32 * RG;
  constexpr int GP = G + 1;  // padded row pitch (bank-conflict free columns)
  constexpr int CW = G / kWarps;  // columns owned by each warp
  extern __shared__ float4 smem4[];
  float2* Cm = reinterpret_cast<float2*>(smem4);  // [nby][nbx] band spectrum / (Lx Ly)
  float2* E1 = Cm + g.nby * g.nbx;                // [nby][GP] stage-1 rows; later T1 [G][ntx]
  const int e1n = g.nby * GP > G * g.ntx ? g.nby * GP : G * g.ntx;
  float* Is = reinterpret_cast<float*>(E1 + e1n);  // [G][GP] intensity
  float2* Zs = reinterpret_cast<float2*>(Is + G * GP);  // [warps][G]

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int clip = blockIdx.x, set = blockIdx.y, split = blockIdx.z;
  const int nsets = gridDim.y, nsplit = gridDim.z;
  const int k0 = (int)(((long long)K * split) / nsplit), k1 = (int)(((long long)K * (split + 1)) / nsplit);
  const int br = (int)(__brev((unsigned)lane) >> 27);

  load_band(partial, g, clip, Cm);
  __syncthreads();

  WarpFFT<RG, +1> wi;
  wi.init(lane);
  float acc[CW][RG];
#pragma unroll
  for (int t = 0; t < CW; ++t)
#pragma unroll
    for (int q = 0; q < RG; ++q) acc[t][q] = 0.f;

  const size_t nb2 = (size_t)g.nby * g.nbx;
  const float2* Hs = H + (size_t)set * K * nb2;
  for (int k = k0; k < k1; ++k) {
    const float2* Hk = Hs + (size_t)k * nb2;
    const float lk = __ldg(lam + set * K + k);
    // stage 1: rows fy, inverse FFT along x of H_k . M (two rows per pass)
    for (int r0 = warp; r0 < g.nby; r0 += 2 * kWarps) {
      float2 va[RG], vb[RG];
      const int r1 = r0 + kWarps;
      const bool has1 = r1 < g.nby;
#pragma unroll
      for (int j = 0; j < RG; ++j) {
        const int n = lane + 32 * j;
        const int fx = n <= g.Nx ? n : (n >= G - g.Nx ? n - G : INT_MIN);
        va[j] = make_float2(0.f, 0.f);
        vb[j] = make_float2(0.f, 0.f);
        if (fx != INT_MIN) {
          const int o0 = r0 * g.nbx + fx + g.Nx;
          va[j] = cmul(__ldg(Hk + o0), Cm[o0]);
          if (has1) {
            const int o1 = r1 * g.nbx + fx + g.Nx;
            vb[j] = cmul(__ldg(Hk + o1), Cm[o1]);
          }
        }
      }
      wi.run(va, lane);
      wi.run(vb, lane);
#pragma unroll
      for (int q1 = 0; q1 < RG; ++q1) {
        E1[r0 * GP + q1 + RG * br] = va[q1];
        if (has1) E1[r1 * GP + q1 + RG * br] = vb[q1];
      }
    }
    __syncthreads();
    // stage 2: columns q, inverse FFT along y; accumulate lambda |E|^2
#pragma unroll
    for (int t = 0; t < CW; ++t) {
      const int q = warp + kWarps * t;
      float2 vv[RG];
#pragma unroll
      for (int j = 0; j < RG; ++j) {
        const int n = lane + 32 * j;
        const int fy = n <= g.Ny ? n : (n >= G - g.Ny ? n - G : INT_MIN);
        vv[j] = (fy != INT_MIN) ? E1[(fy + g.Ny) * GP + q] : make_float2(0.f, 0.f);
      }
      wi.run(vv, lane);
#pragma unroll
      for (int q1 = 0; q1 < RG; ++q1) acc[t][q1] = fmaf(lk, cabs2(vv[q1]), acc[t][q1]);
    }
    __syncthreads();
  }

  // intensity to shared memory: I[p][q], p = q1 + RG*brev(lane), q = warp + 8t
#pragma unroll
  for (int t = 0; t < CW; ++t)
#pragma unroll
    for (int q1 = 0; q1 < RG; ++q1) Is[(q1 + RG * br) * GP + warp + kWarps * t] = acc[t][q1];
  __syncthreads();

  // stage A: forward FFT along x of row pairs packed as one complex row
  WarpFFT<RG, -1> wfw;
  wfw.init(lane);
  float2* T1 = E1;  // [G][ntx]
  float2* Zw = Zs + warp * G;
  for (int pp = warp; pp < G / 2; pp += kWarps) {
    const int p1 = 2 * pp, p2 = 2 * pp + 1;
    float2 vv[RG];
#pragma unroll
    for (int j = 0; j < RG; ++j) {
      const int q = lane + 32 * j;
      vv[j] = make_float2(Is[p1 * GP + q], Is[p2 * GP + q]);
    }
    wfw.run(vv, lane);
#pragma unroll
    for (int q1 = 0; q1 < RG; ++q1) Zw[q1 + RG * br] = vv[q1];
    __syncwarp();
    for (int b = lane; b < g.ntx; b += 32) {
      const float2 za = Zw[b];
      const float2 zb = cconj(Zw[(G - b) & (G - 1)]);
      const float2 x1 = cscale(cadd(za, zb), 0.5f);
      const float2 d = cscale(csub(za, zb), 0.5f);  // x2 = d / i
      T1[p1 * g.ntx + b] = x1;
      T1[p2 * g.ntx + b] = make_float2(d.y, -d.x);
    }
    __syncwarp();
  }
  __syncthreads();

  // stage B: forward FFT along y of each kept column b; scale and shift phase
  const float invg = 1.0f / ((float)G * (float)G);
  float2* To = Tout + (((size_t)clip * nsets + set) * nsplit + split) * g.nty * g.ntx;
  for (int b = warp; b < g.ntx; b += kWarps) {
    float2 vv[RG];
#pragma unroll
    for (int j = 0; j < RG; ++j) vv[j] = T1[(lane + 32 * j) * g.ntx + b];
    wfw.run(vv, lane);
#pragma unroll
    for (int q1 = 0; q1 < RG; ++q1) {
      const int bin = q1 + RG * br;
      const int a = bin <= G / 2 ? bin : bin - G;
      if (a >= -2 * g.Ny && a <= 2 * g.Ny) {
        float2 v = cscale(vv[q1], invg);
        if (g.dx | g.dy) {
          // odd periods: the reference's shifts move the image by one pixel
          const float2 ph1 = expi2pi_frac(-(long long)a * g.dy, g.Ly);
          const float2 ph2 = expi2pi_frac(-(long long)b * g.dx, g.Lx);
          v = cmul(v, cmul(ph1, ph2));
        }
        To[(a + 2 * g.Ny) * g.ntx + b] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// 3. inverse: intensity spectrum -> image rows
// ---------------------------------------------------------------------------
template <int P, int V, int NBM, int RJ>
__global__ void __launch_bounds__(kThreads) k_socs_inverse(const float2* __restrict__ T,
                                                           const SocsGeom g,
                                                           const float2* __restrict__ tx,
                                                           const float2* __restrict__ ty,
                                                           int nsplit, int spc,
                                                           float* __restrict__ images) {
  constexpr int J = 32 * RJ;
  constexpr int QP = NBM + 1;
  extern __shared__ float4 smem4[];
  float2* twi = reinterpret_cast<float2*>(smem4);  // [NBM][V]  e^{-2 pi i b l'/Lx} (conj used)
  float2* Qs = twi + NBM * V;                       // [J][QP]   row coefficients
  float2* Ts = Qs + J * QP;                         // [nty][ntx]
  float2* ph = Ts + g.nty * g.ntx;                  // [nty]     e^{2 pi i a s / Ly}
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int img = blockIdx.y;
  const int s0 = blockIdx.x * spc, s1 = min(g.nS, s0 + spc);  // this CTA's strips
  const size_t tsz = (size_t)g.nty * g.ntx;
  const float2* Ti = T + (size_t)img * nsplit * tsz;

  // once per CTA: the image's band spectrum (slices summed), the x twiddles,
  // and the zero columns b >= ntx of the row coefficients
#pragma unroll 4
  for (int i = threadIdx.x; i < (int)tsz; i += kThreads) {
    float2 v = __ldg(Ti + i);
    for (int p = 1; p < nsplit; ++p) v = cadd(v, __ldg(Ti + p * tsz + i));
    Ts[i] = v;
  }
#pragma unroll 4
  for (int i = threadIdx.x; i < NBM * V; i += kThreads) twi[i] = __ldg(tx + i);
  for (int i = threadIdx.x; i < J * QP; i += kThreads) Qs[i] = make_float2(0.f, 0.f);
  float2 ph_next = make_float2(0.f, 0.f);
  if (threadIdx.x < g.nty) ph_next = __ldg(ty + (size_t)s0 * g.nty + threadIdx.x);
  __syncthreads();

  WarpFFT<RJ, +1> wf;
  wf.init(lane);
  const int br = (int)(__brev((unsigned)lane) >> 27);
  const int A = 2 * g.Ny;
  float* out = images + (size_t)img * g.Lx * g.Ly;
#pragma unroll 1
  for (int s = s0; s < s1; ++s) {
    if (threadIdx.x < g.nty) {
      ph[threadIdx.x] = ph_next;
      if (s + 1 < s1) ph_next = __ldg(ty + (size_t)(s + 1) * g.nty + threadIdx.x);
    }
    __syncthreads();
    // rows of the strip: Q[y = s + nS j][b] = sum_a T[a][b] e^{2 pi i a y / Ly}
    for (int b = warp; b < g.ntx; b += kWarps) {
      float2 vv[RJ];
#pragma unroll
      for (int j = 0; j < RJ; ++j) {
        const int n = lane + 32 * j;
        float2 f = make_float2(0.f, 0.f);
        for (int a = n - J * ((n + A) / J); a <= A; a += J)
          f = cfma(Ts[(a + A) * g.ntx + b], ph[a + A], f);
        vv[j] = f;
      }
      wf.run(vv, lane);
      const float w = b == 0 ? 1.f : 2.f;
#pragma unroll
      for (int q1 = 0; q1 < RJ; ++q1) Qs[(q1 + RJ * br) * QP + b] = cscale(vv[q1], w);
    }
    __syncthreads();

    for (int jj = warp; jj < J; jj += kWarps) {
      float* row = out + (size_t)(s + g.nS * jj) * (V * P);
      const float2* q = Qs + jj * QP;
#pragma unroll 1
      for (int c = 0; c < V / 32; ++c) {
        const int lp = lane + 32 * c;
        // Z[k] = sum over b = k (mod P) of q[b] conj(tw[b]).  With 32 bins it is
        // accumulated as its Hermitian fold Y[k] = Z[k] + conj Z[P-k] (k <= P/2),
        // half the registers of Z (measured faster for the 512^2 and 1024^2
        // classes); with 64 bins Z itself (measured faster for 2048^2)
        if constexpr (NBM > 32) {
          float2 Z[P];
#pragma unroll
          for (int i = 0; i < P; ++i) Z[i] = make_float2(0.f, 0.f);
          constexpr int KB = NBM < P ? NBM : P;
#pragma unroll 1
          for (int b0 = 0; b0 < NBM; b0 += KB) {
#pragma unroll
            for (int k = 0; k < KB; ++k) {
              const float2 qb = q[b0 + k], w = twi[(b0 + k) * V + lp];
              Z[k] = make_float2(fmaf(qb.x, w.x, fmaf(qb.y, w.y, Z[k].x)),
                                 fmaf(qb.y, w.x, fmaf(-qb.x, w.y, Z[k].y)));
            }
          }
          float o[P];
          re_idft_reg<P>(Z, o);
#pragma unroll
          for (int i = 0; i < P; ++i) row[lp + V * i] = o[i];
        } else {
        float2 Y[P / 2 + 1];
#pragma unroll
        for (int i = 0; i <= P / 2; ++i) Y[i] = make_float2(0.f, 0.f);
        constexpr int KB = NBM < P ? NBM : P;
#pragma unroll 1
        for (int b0 = 0; b0 < NBM; b0 += KB) {
#pragma unroll
          for (int k = 0; k < KB; ++k) {
            const float2 qb = q[b0 + k], w = twi[(b0 + k) * V + lp];
            // z = qb conj(w); b0 is a multiple of P when NBM > P
            if (2 * k <= P) {
              Y[k] = make_float2(fmaf(qb.x, w.x, fmaf(qb.y, w.y, Y[k].x)),
                                 fmaf(qb.y, w.x, fmaf(-qb.x, w.y, Y[k].y)));
            } else {
              Y[P - k] = make_float2(fmaf(qb.x, w.x, fmaf(qb.y, w.y, Y[P - k].x)),
                                     fmaf(-qb.y, w.x, fmaf(qb.x, w.y, Y[P - k].y)));
            }
          }
        }
        float o[P];
        c2r_half<P>(Y, o);
#pragma unroll
        for (int i = 0; i < P; ++i) row[lp + V * i] = o[i];
        }
      }
    }
    __syncthreads();  // Qs and ph are rewritten for the next strip
  }
}

// centred FT_r2c band: M(ky,kx) = D(ky,kx) e^{-2 pi i (ky yh/Ly + kx xh/Lx)} / (Lx Ly)
__global__ void k_socs_band(const float2* __restrict__ partial, const SocsGeom g,
                            float2* __restrict__ band) {
  extern __shared__ float4 smem4[];
  float2* Cm = reinterpret_cast<float2*>(smem4);
  const int clip = blockIdx.x;
  load_band(partial, g, clip, Cm);
  __syncthreads();
  const int yh = (g.Ly + 1) / 2, xh = (g.Lx + 1) / 2;
  for (int i = threadIdx.x; i < g.nby * g.nbx; i += blockDim.x) {
    const int r = i / g.nbx, c = i - r * g.nbx;
    const int ky = r - g.Ny, kx = c - g.Nx;
    const float2 p1 = expi2pi_frac(-(long long)ky * yh, g.Ly);
    const float2 p2 = expi2pi_frac(-(long long)kx * xh, g.Lx);
    band[(size_t)clip * g.nby * g.nbx + i] = cmul(Cm[i], cmul(p1, p2));
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

template <int P, int V, int NFM, int RJ>
int launch_fwd(const SocsGeom& g, const float2* tx, const float2* ty, const float* masks,
               int nclips, float2* partial, cudaStream_t st) {
  size_t sm = sizeof(float2) * ((size_t)NFM * V + (size_t)32 * RJ * NFM);
  auto kern = k_socs_forward<P, V, NFM, RJ>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  kern<<<dim3(g.nS, nclips), kThreads, sm, st>>>(masks, g, tx, ty, partial);
  return check_launch("k_socs_forward");
}

template <int P, int V, int NBM, int RJ>
int launch_inv(const SocsGeom& g, const float2* tx, const float2* ty, const float2* T, int nimg,
               int nsplit, float* images, cudaStream_t st, int spc) {
  size_t sm = sizeof(float2) * ((size_t)NBM * V + (size_t)32 * RJ * (NBM + 1) +
                                (size_t)g.nty * g.ntx + g.nty);
  auto kern = k_socs_inverse<P, V, NBM, RJ>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  // strips per CTA: the image's spectrum and the twiddle table are loaded once
  // per CTA, so give each CTA several strips while keeping >= 4 CTAs per SM
  if (spc <= 0) {
    spc = 1;
    while (spc < 8 && spc * 2 <= g.nS && (long long)nimg * ((g.nS + 2 * spc - 1) / (2 * spc)) >= 4 * 148) spc *= 2;
  }
  spc = spc < g.nS ? spc : g.nS;
  kern<<<dim3((g.nS + spc - 1) / spc, nimg), kThreads, sm, st>>>(T, g, tx, ty, nsplit, spc, images);
  return check_launch("k_socs_inverse");
}

template <int RG>
int launch_spec(const SocsGeom& g, const float2* partial, int nclips, const float2* H,
                const float* lam, int K, int nsets, int nsplit, float2* T, cudaStream_t st) {
  constexpr int G = 32 * RG, GP = G + 1;
  size_t e1n = (size_t)g.nby * GP > (size_t)G * g.ntx ? (size_t)g.nby * GP : (size_t)G * g.ntx;
  size_t sm = sizeof(float2) * ((size_t)g.nby * g.nbx + e1n) + sizeof(float) * (size_t)G * GP +
              sizeof(float2) * (size_t)kWarps * G;
  auto kern = k_socs_spectral<RG>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  kern<<<dim3(nclips, nsets, nsplit), kThreads, sm, st>>>(partial, g, H, lam, K, T);
  return check_launch("k_socs_spectral");
}
}  // namespace

#define KL_PV_LIST(X, A, B) \
  X(8, 32, A, B) X(8, 96, A, B) X(16, 32, A, B) X(16, 96, A, B) X(32, 32, A, B) X(32, 64, A, B) X(32, 96, A, B)

int socs_launch_forward(const SocsGeom& g, const float2* tx, const float2* ty, const float* masks,
                        int nclips, float2* partial, cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  const int RJ = g.J / 32;
#define KL_FWD(P_, V_, N_, R_)                               \
  if (g.P == P_ && g.V == V_ && g.NFM == N_ && RJ == R_) \
    return launch_fwd<P_, V_, N_, R_>(g, tx, ty, masks, nclips, partial, st);
  KL_PV_LIST(KL_FWD, 16, 1)
  KL_PV_LIST(KL_FWD, 16, 2)
  KL_PV_LIST(KL_FWD, 32, 1)
  KL_PV_LIST(KL_FWD, 32, 2)
#undef KL_FWD
  set_error("socs_launch_forward: no kernel for this geometry");
  return KL_ERR_UNSUPPORTED;
}

int socs_launch_spectral(const SocsGeom& g, const float2* partial, int nclips, const float2* H,
                         const float* lam, int K, int nsets, int nsplit, float2* T,
                         cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  switch (g.G) {
    case 32: return launch_spec<1>(g, partial, nclips, H, lam, K, nsets, nsplit, T, st);
    case 64: return launch_spec<2>(g, partial, nclips, H, lam, K, nsets, nsplit, T, st);
    case 128: return launch_spec<4>(g, partial, nclips, H, lam, K, nsets, nsplit, T, st);
  }
  set_error("socs_launch_spectral: unsupported spectral grid");
  return KL_ERR_UNSUPPORTED;
}

int socs_launch_inverse(const SocsGeom& g, const float2* tx, const float2* ty, const float2* T,
                        int nclips, int nsets, int nsplit, float* images, cudaStream_t st, int spc) {
  if (nclips <= 0) return KL_OK;
  const int RJ = g.J / 32, nimg = nclips * nsets;
#define KL_INV(P_, V_, N_, R_)                               \
  if (g.P == P_ && g.V == V_ && g.NBM == N_ && RJ == R_) \
    return launch_inv<P_, V_, N_, R_>(g, tx, ty, T, nimg, nsplit, images, st, spc);
  KL_PV_LIST(KL_INV, 32, 1)
  KL_PV_LIST(KL_INV, 32, 2)
  KL_PV_LIST(KL_INV, 64, 1)
  KL_PV_LIST(KL_INV, 64, 2)
#undef KL_INV
  set_error("socs_launch_inverse: no kernel for this geometry");
  return KL_ERR_UNSUPPORTED;
}

int socs_launch_band(const SocsGeom& g, const float2* partial, int nclips, float2* band,
                     cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  size_t sm = sizeof(float2) * (size_t)g.nby * g.nbx;
  int rc = set_smem(k_socs_band, sm);
  if (rc) return rc;
  k_socs_band<<<nclips, kThreads, sm, st>>>(partial, g, band);
  return check_launch("k_socs_band");
}

}  // namespace kl
