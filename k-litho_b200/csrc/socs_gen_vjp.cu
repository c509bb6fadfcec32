// socs_gen_vjp.cu -- adjoint (vector-Jacobian product) of the general-geometry
// SOCS pipeline of socs_gen.cu under a sigmoid resist and an L2 loss.  No
// counterpart in the reference; the forward model is
// K-Litho-SOCS/klitho_socs.cpp:196-241.  The mathematics is that of
// socs_vjp.cu:
//
//   G(x)   = dL/dI = 2 (s - t) s (1 - s) a ,  s = sigmoid(a (I - c))
//   dL/dm  = (2/(LxLy)) Re sum_f Gam[f] e^{-2 pi i f.y/L}
//   Gam[f] = sum_k lam_k H_k[f] B_k[f],  B_k = coefficient of e^{-2 pi i f.s}
//            in conj(e_k(s)) gam(s),  gam(s) = Re sum_{|g|<=2N} Gb[g] e^{-2 pi i g.s}
//
// with the band-limited products sampled exactly on the G x G grid.  Stages:
//   row_vjp       image rows from Q (as row_inv), resist, loss, dL/dI, and the
//                 row DFT of dL/dI for gx in [0, 2Nx], written over Q in place
//   col_fwd       (socs_gen.cu) those rows' DFT along y, |gy| <= 2Ny
//   vjp_spectral  per (image, kernel slice) a cluster of G/32 CTAs, each owning
//                 the grid columns x = c + (G/32) j: gam at its columns, the
//                 fields recomputed, w = conj(e) gam transformed back (y by the
//                 transposed warp FFT from registers, x by a 32-point FFT) and
//                 accumulated against H_k; the CTAs sum Gam through
//                 distributed shared memory
//   gradT         Gam -> half-plane spectrum of dL/dm
//   col_inv, row_inv (socs_gen.cu) the gradient image
//   vjp_source    dL/dJ through the TCC factor A (one pass per source point)
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>

#include "kl_device.cuh"
#include "kl_internal.h"

namespace cg = cooperative_groups;

namespace kl {

namespace {
constexpr int kT = 256;
constexpr int kW = kT / 32;
constexpr int kSMs = 148;
__device__ __forceinline__ int brev5(int lane) { return (int)(__brev((unsigned)lane) >> 27); }
__host__ __device__ inline size_t off_tw2(const GenGeom& g) { return (size_t)g.NBX * 64; }

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
}  // namespace

// ---------------------------------------------------------------------------
// row_vjp: Q rows -> image rows, resist, loss, dL/dI row DFT (written over Q)
// ---------------------------------------------------------------------------
template <int PF>
__global__ void __launch_bounds__(kT, 2) k_gen_rowvjp(float2* __restrict__ Q, const GenGeom g,
                                                   const float2* __restrict__ tables, int nsets,
                                                   const float* __restrict__ targets, float alpha, float thr,
                                                   float* __restrict__ images, double* __restrict__ loss) {
  constexpr int HS = PF / 2 + 1;
  extern __shared__ float4 smem4[];
  __shared__ double s_loss[kW];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int NBX = g.NBX, ntx = g.ntx;
  float2* tb = reinterpret_cast<float2*>(smem4);  // [NBX][32] e^{+2 pi i b l / Lx}
  float2* tl = tb + NBX * 32;                      // [32][NBX] the same, transposed
  float2* qc = tl + NBX * 32 + warp * NBX;         // [NBX]
  float2* sb = tl + NBX * 32 + kW * NBX + warp * HS * 33;  // [HS][33]
  float2* t2s = tl + NBX * 32 + kW * NBX + kW * HS * 33;   // [nC][NBX] chunk twiddles, when they fit
  const int Lx = g.Lx, Ly = g.Ly, V = g.Vf, nch = (V + 31) / 32;
  const bool t2_shared = gen_t2_in_smem(g);
  const float2* tw2 = t2_shared ? t2s : tables + off_tw2(g);
  for (int i = threadIdx.x; i < 64 * NBX; i += kT) tb[i] = __ldg(tables + i);
  if (t2_shared)
    for (int i = threadIdx.x; i < nch * NBX; i += kT) t2s[i] = __ldg(tables + off_tw2(g) + i);
  __syncthreads();
  const int img = blockIdx.y, clip = img / nsets;
  const int nbp = (ntx + PF - 1) / PF * PF;
  const int nt = (ntx + 31) / 32;
  double lsum = 0.0;
  // each lane holds the coefficients b = lane + 32 t of its warp's row (the
  // next row's are loaded while the current one is worked on)
  const int y0 = blockIdx.x * kW + warp, ystep = gridDim.x * kW;
  float2 qn[4];
  if (y0 < Ly) gen_load_qrow(Q + ((size_t)img * Ly + y0) * ntx, ntx, lane, qn);
  for (int y = y0; y < Ly; y += ystep) {
    const size_t row = (size_t)img * Ly + y;
    float2* qr = Q + row * ntx;
    float2 q[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) q[t] = qn[t];
    if (y + ystep < Ly) gen_load_qrow(Q + (row + ystep) * ntx, ntx, lane, qn);
    float* orow = images ? images + row * Lx : nullptr;
    const float* trow = targets + ((size_t)clip * Ly + y) * Lx;
    float2 acc[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) acc[t] = make_float2(0.f, 0.f);
    float rsum = 0.f;
#pragma unroll 1
    for (int c = 0; c < nch; ++c) {
      const int lp = lane + 32 * c;
      // the chunk's targets are loaded first, so that they arrive during the synthesis
      float tg[PF];
#pragma unroll
      for (int i = 0; i < PF; ++i) tg[i] = lp < V ? __ldcs(trow + lp + V * i) : 0.f;
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int b = lane + 32 * t;
        if (b < nbp) qc[b] = b < ntx ? cmul(q[t], tw2[(size_t)c * NBX + b]) : make_float2(0.f, 0.f);
      }
      __syncwarp();
      float2 Y[HS];
#pragma unroll
      for (int k = 0; k < HS; ++k) Y[k] = make_float2(0.f, 0.f);
#pragma unroll 1
      for (int b0 = 0; b0 < nbp; b0 += PF) {
#pragma unroll
        for (int k = 0; k < PF; ++k) {
          const float2 q = qc[b0 + k];
          const float2 w = tb[(b0 + k) * 32 + lane];
          if (2 * k <= PF) {
            Y[k] = cfma(q, w, Y[k]);
          } else {
            Y[PF - k].x = fmaf(q.x, w.x, fmaf(-q.y, w.y, Y[PF - k].x));
            Y[PF - k].y = fmaf(-q.x, w.y, fmaf(-q.y, w.x, Y[PF - k].y));
          }
        }
      }
      float o[PF];
      c2r_half<PF>(Y, o);
      if (lp < V) {
#pragma unroll
        for (int i = 0; i < PF; ++i) {
          const int x = lp + V * i;
          if (orow) __stcs(orow + x, o[i]);
          const float sg = __frcp_rn(1.0f + __expf(-alpha * (o[i] - thr)));
          const float d = sg - tg[i];
          rsum = fmaf(d, d, rsum);
          o[i] = 2.0f * d * sg * (1.0f - sg) * alpha;
        }
      } else {
#pragma unroll
        for (int i = 0; i < PF; ++i) o[i] = 0.f;
      }
      float2 S[HS];
      rdft_any<PF>(o, S);
#pragma unroll
      for (int k = 0; k < HS; ++k) sb[k * 33 + lane] = S[k];
      __syncwarp();
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int gx = lane + 32 * t;
        if (t < nt && gx < ntx) {
          const int k = gx % PF;
          const bool cj = 2 * k > PF;
          const int kk = cj ? PF - k : k;
          const float sgn = cj ? -1.f : 1.f;
          float2 s = make_float2(0.f, 0.f);
#pragma unroll 8
          for (int l = 0; l < 32; ++l) {
            const float2 sv = sb[kk * 33 + l];
            const float svy = sgn * sv.y;
            const float2 w = tl[l * NBX + gx];
            s.x = fmaf(sv.x, w.x, fmaf(svy, w.y, s.x));
            s.y = fmaf(svy, w.x, fmaf(-sv.x, w.y, s.y));
          }
          acc[t] = cfma(s, cconj(tw2[(size_t)c * NBX + gx]), acc[t]);
        }
      }
      __syncwarp();
    }
    lsum += (double)rsum;
    // the row's dL/dI bins replace its Q (every chunk has read Q above)
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int gx = lane + 32 * t;
      if (t < nt && gx < ntx) qr[gx] = acc[t];
    }
  }
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
  if (lane == 0) s_loss[warp] = lsum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kW; ++w) t += s_loss[w];
    atomicAdd(loss + img, t);
  }
}

// ---------------------------------------------------------------------------
// shared pieces of the column-decimated spectral adjoint kernels
// ---------------------------------------------------------------------------
// Mask band half [nby][nf] (parts summed) times e^{2 pi i fx c / G}.
__device__ void gv_load_mask_band(const float2* __restrict__ band, int nparts, const GenGeom& g, int clip, int c,
                                  const float2* rootG, float2* Mh) {
  const int G = g.G, nf = g.nf;
  const size_t per = (size_t)g.nby * nf;
  const float2* b0 = band + (size_t)clip * nparts * per;
  for (int i = threadIdx.x; i < g.nby * nf; i += kT) {
    const int fx = i % nf;
    float2 v = __ldg(b0 + i);
    for (int p = 1; p < nparts; ++p) v = cadd(v, __ldg(b0 + p * per + i));
    Mh[i] = cmul(v, rootG[(fx * c) & (G - 1)]);
  }
}

// gam(p, c + RG j) at the CTA's columns, in the registers' layout of a column
// FFT: gam[t][q] for column j = warp + kW t and row p = q + RG brev5(lane).
// G1 is scratch of [nty][33] float2.
template <int RG>
__device__ void gv_make_gamma(const float2* __restrict__ gband, int gparts, const GenGeom& g, int img, int c,
                              const float2* rootG, float2* G1, float (&gam)[32 / kW][RG]) {
  constexpr int G = 32 * RG;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int A = 2 * g.Ny, Bx = 2 * g.Nx, ntx = g.ntx, nty = g.nty;
  const size_t per = (size_t)nty * ntx;
  const float2* g0 = gband + (size_t)img * gparts * per;
  const int br = brev5(lane);
  WarpFFT<1, -1> w1;
  w1.init(lane);
  const int gxs = lane - 32 * ((lane + Bx) / 32);
  // rows gy: fold gx mod 32 with e^{-2 pi i gx c/G}, forward 32-point FFT over the lanes
  for (int r = warp; r < nty; r += kW) {
    const int gy = r - A;
    float2 v = make_float2(0.f, 0.f);
    for (int gx = gxs; gx <= Bx; gx += 32) {
      // Ghat[gy][gx] from the half plane (gx >= 0); Gb = e^{-2 pi i g.d/L} conj(Ghat)
      const int rr = gx >= 0 ? r : nty - 1 - r, cc = gx >= 0 ? gx : -gx;
      float2 h = __ldg(g0 + (size_t)rr * ntx + cc);
      for (int p = 1; p < gparts; ++p) h = cadd(h, __ldg(g0 + p * per + (size_t)rr * ntx + cc));
      if (gx < 0) h = cconj(h);
      float2 gb = cconj(h);
      if (g.dx | g.dy) {
        const float2 e = cmul(expi2pi_frac(-(long long)gy * g.dy, g.Ly), expi2pi_frac(-(long long)gx * g.dx, g.Lx));
        gb = cmul(gb, e);
      }
      v = cfma(gb, cconj(rootG[(gx * c) & (G - 1)]), v);
    }
    float2 vv[1] = {v};
    w1.run(vv, lane);
    G1[r * 33 + br] = vv[0];
  }
  __syncthreads();
  WarpFFT<RG, -1> wf;
  wf.init(lane);
#pragma unroll
  for (int t = 0; t < 32 / kW; ++t) {
    const int j = warp + kW * t;
    float2 vv[RG];
#pragma unroll
    for (int i = 0; i < RG; ++i) {
      const int n = lane + 32 * i;
      const int gy = n <= A ? n : (n >= G - A ? n - G : INT_MIN);
      vv[i] = gy != INT_MIN ? G1[(gy + A) * 33 + j] : make_float2(0.f, 0.f);
    }
    wf.run(vv, lane);
#pragma unroll
    for (int q = 0; q < RG; ++q) gam[t][q] = vv[q].x;
  }
  __syncthreads();
}

// stage 1 of a field: band rows of Hk . M' folded mod 32, inverse 32-point FFT
// over the lanes -> E1[r][j].  hn holds the loads of the warp's first row of
// Hk on entry and, on exit, those of the first row of Hnext (when not NULL):
// each row's successor is in flight while the row is worked on.
__device__ __forceinline__ void gv_field_rows(const GenGeom& g, const float2* __restrict__ Hk,
                                              const float2* __restrict__ Hnext, const float2* Mh, float2* E1,
                                              const WarpFFT<1, +1>& w1, int lane, int warp,
                                              float2 (&hn)[kGenMaxFold]) {
  const int nf = g.nf, nby = g.nby, nbx = g.nbx, Nx = g.Nx;
  const int fxs = lane - 32 * ((lane + Nx) / 32);
  const int br = brev5(lane);
  for (int r = warp; r < nby; r += kW) {
    float2 h[kGenMaxFold];
#pragma unroll
    for (int t = 0; t < kGenMaxFold; ++t) h[t] = hn[t];
    if (r + kW < nby) gen_load_hrow(Hk, r + kW, nbx, Nx, fxs, hn);
    else if (Hnext) gen_load_hrow(Hnext, warp, nbx, Nx, fxs, hn);
    float2 v = make_float2(0.f, 0.f);
#pragma unroll
    for (int t = 0; t < kGenMaxFold; ++t) {
      const int fx = fxs + 32 * t;
      if (fx <= Nx) {
        const float2 m = fx >= 0 ? Mh[r * nf + fx] : cconj(Mh[(nby - 1 - r) * nf - fx]);
        v = cfma(h[t], m, v);
      }
    }
    float2 vv[1] = {v};
    w1.run(vv, lane);
    E1[r * 33 + br] = vv[0];
  }
}

// column j of the field: G-point inverse FFT along y of E1[.][j]
template <int RG>
__device__ __forceinline__ void gv_field_column(const GenGeom& g, const float2* E1, int j,
                                                const WarpFFT<RG, +1>& wi, int lane, float2 (&vv)[RG]) {
  constexpr int G = 32 * RG;
  const int Ny = g.Ny;
#pragma unroll
  for (int i = 0; i < RG; ++i) {
    const int n = lane + 32 * i;
    const int fy = n <= Ny ? n : (n >= G - Ny ? n - G : INT_MIN);
    vv[i] = fy != INT_MIN ? E1[(fy + Ny) * 33 + j] : make_float2(0.f, 0.f);
  }
  wi.run(vv, lane);
}

__host__ __device__ inline size_t gv_spec_smem_elems(const GenGeom& g) {
  const size_t acc = std::max((size_t)g.nby * g.nbx, (size_t)g.nty * 33);
  return (size_t)g.nby * g.nf + 2 * (size_t)g.nby * 33 + acc + g.G;
}

// ---------------------------------------------------------------------------
// vjp_spectral: Gam[img][split][fy][fx] (full band) per (image, kernel slice)
// ---------------------------------------------------------------------------
template <int RG>
__global__ void __launch_bounds__(kT, 1) k_gen_vjp_spectral(const float2* __restrict__ band, int nparts,
                                                            const float2* __restrict__ gband, int gparts,
                                                            const GenGeom g, const float2* __restrict__ H,
                                                            const float* __restrict__ lam, int K, int nsets,
                                                            float2* __restrict__ gam_out) {
  constexpr int G = 32 * RG;
  constexpr int CW = 32 / kW;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ float4 smem4[];
  const int nby = g.nby, nbx = g.nbx, nf = g.nf, Nx = g.Nx, Ny = g.Ny;
  float2* Mh = reinterpret_cast<float2*>(smem4);  // [nby][nf]
  float2* E1 = Mh + nby * nf;                      // [nby][33] field stage-1 rows
  float2* Ws = E1 + nby * 33;                      // [nby][33] y-transformed w, |fy| <= Ny
  float2* Acc = Ws + nby * 33;                     // [nby][nbx]; the gamma prologue's scratch first
  const size_t accn = std::max((size_t)nby * nbx, (size_t)g.nty * 33);
  float2* rootG = Acc + accn;                      // [G]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = blockIdx.x, img = blockIdx.y, split = blockIdx.z, nsplit = gridDim.z;
  const int clip = img / nsets, set = img - clip * nsets;
  const int k0 = (int)(((long long)K * split) / nsplit), k1 = (int)(((long long)K * (split + 1)) / nsplit);
  const int br = brev5(lane);

  for (int i = threadIdx.x; i < G; i += kT) rootG[i] = expi2pi_frac(i, G);
  __syncthreads();
  gv_load_mask_band(band, nparts, g, clip, c, rootG, Mh);
  float gam[CW][RG];
  gv_make_gamma<RG>(gband, gparts, g, img, c, rootG, Acc, gam);
  for (int i = threadIdx.x; i < nby * nbx; i += kT) Acc[i] = make_float2(0.f, 0.f);
  __syncthreads();

  WarpFFT<1, +1> w1;
  w1.init(lane);
  WarpFFT<RG, +1> wi;
  wi.init(lane);
  const float invg2 = 1.0f / ((float)G * (float)G);
  const size_t nb2 = (size_t)nby * nbx;
  const float2* Hs = H + (size_t)set * K * nb2;
  const int fxm = br - 32 * ((br + Nx) / 32);  // smallest fx >= -Nx with fx = brev5(lane) (mod 32)
  const int fxs = lane - 32 * ((lane + Nx) / 32);
  float2 hn[kGenMaxFold];
  if (k0 < k1 && warp < nby) gen_load_hrow(Hs + (size_t)k0 * nb2, warp, nbx, Nx, fxs, hn);
  for (int k = k0; k < k1; ++k) {
    const float2* Hk = Hs + (size_t)k * nb2;
    const float lk = __ldg(lam + set * K + k) * invg2;
    gv_field_rows(g, Hk, k + 1 < k1 ? Hk + nb2 : nullptr, Mh, E1, w1, lane, warp, hn);
    __syncthreads();
    // per column: field e(p), w = conj(e) gam lk, then W1[fy] = sum_p w e^{+2 pi i fy p/G}
#pragma unroll
    for (int t = 0; t < CW; ++t) {
      const int j = warp + kW * t;
      float2 vv[RG];
      gv_field_column<RG>(g, E1, j, wi, lane, vv);
#pragma unroll
      for (int q = 0; q < RG; ++q) vv[q] = cscale(cconj(vv[q]), gam[t][q] * lk);
      wi.run_rev(vv, lane);
#pragma unroll
      for (int i = 0; i < RG; ++i) {
        const int n = lane + 32 * i;
        const int fy = n <= Ny ? n : (n >= G - Ny ? n - G : INT_MIN);
        if (fy != INT_MIN) Ws[(fy + Ny) * 33 + j] = vv[i];
      }
    }
    __syncthreads();
    // rows fy: F[m] = sum_j W1[fy][j] e^{+2 pi i m j / 32}; Acc[fy][fx] += H_k F[fx mod 32]
    for (int r = warp; r < nby; r += kW) {
      // the row's kernel values are loaded before the FFT so the loads overlap it
      float2 hh[kGenMaxFold];
      gen_load_hrow(Hk, r, nbx, Nx, fxm, hh);
      float2 vv[1] = {Ws[r * 33 + lane]};
      w1.run(vv, lane);
      // lane holds F[m], m = brev5(lane): the bins fx = m (mod 32)
      float2* ar = Acc + (size_t)r * nbx + Nx;
#pragma unroll
      for (int t = 0; t < kGenMaxFold; ++t) {
        const int fx = fxm + 32 * t;
        if (fx <= Nx) ar[fx] = cfma(hh[t], vv[0], ar[fx]);
      }
    }
    __syncthreads();
  }
  cl.sync();
  // Gam[f] = sum_c e^{+2 pi i fx c / G} Acc_c[f]; this CTA writes rows [r0, r1)
  {
    const int per = (nby + RG - 1) / RG;
    const int r0 = c * per, r1 = min(nby, r0 + per);
    float2* out = gam_out + ((size_t)img * nsplit + split) * nb2;
    const float2* peers[RG];
#pragma unroll
    for (int cc = 0; cc < RG; ++cc) peers[cc] = cl.map_shared_rank(Acc, cc);
    for (int i = r0 * nbx + threadIdx.x; i < r1 * nbx; i += kT) {
      const int fx = i % nbx - Nx;
      float2 s = make_float2(0.f, 0.f);
#pragma unroll
      for (int cc = 0; cc < RG; ++cc) s = cfma(peers[cc][i], rootG[(fx * cc) & (G - 1)], s);
      out[i] = s;
    }
  }
  cl.sync();
}

// ---------------------------------------------------------------------------
// gradT: Tg[clip][b][a + Ny] = sum_parts (conj Gam[a][b] + Gam[-a][-b]) / (Lx Ly),
// |a| <= Ny, b in [0, Nx] (the layout col_inv reads)
// ---------------------------------------------------------------------------
__global__ void k_gen_gradT(const float2* __restrict__ gam, const GenGeom g, int nparts, float2* __restrict__ Tg) {
  const int clip = blockIdx.x;
  const size_t nb2 = (size_t)g.nby * g.nbx;
  const float2* p0 = gam + (size_t)clip * nparts * nb2;
  const float s = 1.0f / ((float)g.Lx * (float)g.Ly);
  float2* To = Tg + (size_t)clip * g.nf * g.nby;
  for (int i = threadIdx.x; i < g.nf * g.nby; i += blockDim.x) {
    const int b = i / g.nby, r = i - b * g.nby, a = r - g.Ny;
    const size_t o1 = (size_t)(a + g.Ny) * g.nbx + (b + g.Nx);
    const size_t o2 = (size_t)(-a + g.Ny) * g.nbx + (-b + g.Nx);
    float2 f1 = make_float2(0.f, 0.f), f2 = make_float2(0.f, 0.f);
    for (int p = 0; p < nparts; ++p) {
      f1 = cadd(f1, __ldg(p0 + p * nb2 + o1));
      f2 = cadd(f2, __ldg(p0 + p * nb2 + o2));
    }
    To[i] = cscale(cadd(cconj(f1), f2), s);
  }
}

// ---------------------------------------------------------------------------
// vjp_source: dL/dJ_s = (1/G^2) sum_p gam(p) |e_s(p)|^2 / J_s, per (image, slice)
// ---------------------------------------------------------------------------
__host__ __device__ inline size_t gv_src_smem_elems(const GenGeom& g) {
  return (size_t)g.nby * g.nf + std::max((size_t)g.nby * 33, (size_t)g.nty * 33) + g.G;
}

template <int RG>
__global__ void __launch_bounds__(kT) k_gen_vjp_source(const float2* __restrict__ band, int nparts,
                                                       const float2* __restrict__ gband, int gparts,
                                                       const GenGeom g, const float2* __restrict__ Hs, int S,
                                                       const float* __restrict__ Jw, const int* __restrict__ src_id,
                                                       int nsets, float* __restrict__ grad_src) {
  constexpr int G = 32 * RG;
  constexpr int CW = 32 / kW;
  extern __shared__ float4 smem4[];
  __shared__ float s_red[kW];
  const int nby = g.nby, nf = g.nf;
  float2* Mh = reinterpret_cast<float2*>(smem4);  // [nby][nf]
  float2* E1 = Mh + nby * nf;                      // [max(nby, nty)][33]: gamma scratch, then field rows
  float2* rootG = E1 + std::max((size_t)nby * 33, (size_t)g.nty * 33);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = blockIdx.x, img = blockIdx.y, split = blockIdx.z, nsplit = gridDim.z;
  const int clip = img / nsets;
  const int s0 = (int)(((long long)S * split) / nsplit), s1 = (int)(((long long)S * (split + 1)) / nsplit);
  for (int i = threadIdx.x; i < G; i += kT) rootG[i] = expi2pi_frac(i, G);
  __syncthreads();
  gv_load_mask_band(band, nparts, g, clip, c, rootG, Mh);
  float gam[CW][RG];
  gv_make_gamma<RG>(gband, gparts, g, img, c, rootG, E1, gam);
  WarpFFT<1, +1> w1;
  w1.init(lane);
  WarpFFT<RG, +1> wi;
  wi.init(lane);
  const float invg2 = 1.0f / ((float)G * (float)G);
  const size_t nb2 = (size_t)nby * g.nbx;
  const int fxs = lane - 32 * ((lane + g.Nx) / 32);
  float2 hn[kGenMaxFold];
  if (s0 < s1 && warp < nby) gen_load_hrow(Hs + (size_t)s0 * nb2, warp, g.nbx, g.Nx, fxs, hn);
  for (int s = s0; s < s1; ++s) {
    gv_field_rows(g, Hs + (size_t)s * nb2, s + 1 < s1 ? Hs + (size_t)(s + 1) * nb2 : nullptr, Mh, E1, w1, lane, warp,
                  hn);
    __syncthreads();
    float part = 0.f;
#pragma unroll
    for (int t = 0; t < CW; ++t) {
      float2 vv[RG];
      gv_field_column<RG>(g, E1, warp + kW * t, wi, lane, vv);
#pragma unroll
      for (int q = 0; q < RG; ++q) part = fmaf(gam[t][q], cabs2(vv[q]), part);
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) s_red[warp] = part;
    __syncthreads();
    if (threadIdx.x == 0) {
      float t = 0.f;
      for (int w = 0; w < kW; ++w) t += s_red[w];
      atomicAdd(grad_src + src_id[s], t * invg2 / Jw[s]);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
namespace {
template <int PF>
int launch_rowvjp_t(const GenGeom& g, const float2* tables, float2* Q, int nimg, int nsets, const float* targets,
                    float alpha, float thr, float* images, double* loss, cudaStream_t st) {
  const size_t sm = sizeof(float2) * ((size_t)64 * g.NBX + (size_t)kW * g.NBX + (size_t)kW * (PF / 2 + 1) * 33 +
                                      (gen_t2_in_smem(g) ? (size_t)g.nC * g.NBX : 0));
  auto kern = k_gen_rowvjp<PF>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  // about four CTAs per SM over the whole batch, each on rows of one image
  int bx = (4 * kSMs + nimg - 1) / nimg;
  bx = std::max(1, std::min(bx, (g.Ly + kW - 1) / kW));
  kern<<<dim3(bx, nimg), kT, sm, st>>>(Q, g, tables, nsets, targets, alpha, thr, images, loss);
  return check_launch("k_gen_rowvjp");
}

template <typename Kern, typename... Args>
int launch_cluster(Kern kern, int RG, dim3 grid, size_t sm, cudaStream_t st, const char* what, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(kT);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = RG;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&cfg, kern, args...);
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return KL_ERR_CUDA;
  }
  return check_launch(what);
}

template <int RG>
int launch_vspec_t(const GenGeom& g, const float2* band, int nparts, const float2* gband, int gparts, int nclips,
                   const float2* H, const float* lam, int K, int nsets, int nsplit, float2* gam, cudaStream_t st) {
  const size_t sm = sizeof(float2) * gv_spec_smem_elems(g);
  auto kern = k_gen_vjp_spectral<RG>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  return launch_cluster(kern, RG, dim3(RG, nclips * nsets, nsplit), sm, st, "k_gen_vjp_spectral", band, nparts,
                        gband, gparts, g, H, lam, K, nsets, gam);
}

template <int RG>
int launch_vsrc_t(const GenGeom& g, const float2* band, int nparts, const float2* gband, int gparts, int nimg,
                  int nsets, const float2* Hs, int S, const float* Jw, const int* src_id, int nsplit,
                  float* grad_src, cudaStream_t st) {
  const size_t sm = sizeof(float2) * gv_src_smem_elems(g);
  auto kern = k_gen_vjp_source<RG>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  kern<<<dim3(RG, nimg, nsplit), kT, sm, st>>>(band, nparts, gband, gparts, g, Hs, S, Jw, src_id, nsets, grad_src);
  return check_launch("k_gen_vjp_source");
}
}  // namespace

int gen_launch_rowvjp(const GenGeom& g, const float2* tables, float2* Q, int nimg, int nsets, const float* targets,
                      float alpha, float thr, float* images, double* loss, cudaStream_t st) {
  if (nimg <= 0) return KL_OK;
  switch (g.Pf) {
    case 1: return launch_rowvjp_t<1>(g, tables, Q, nimg, nsets, targets, alpha, thr, images, loss, st);
    case 2: return launch_rowvjp_t<2>(g, tables, Q, nimg, nsets, targets, alpha, thr, images, loss, st);
    case 4: return launch_rowvjp_t<4>(g, tables, Q, nimg, nsets, targets, alpha, thr, images, loss, st);
    case 8: return launch_rowvjp_t<8>(g, tables, Q, nimg, nsets, targets, alpha, thr, images, loss, st);
    case 16: return launch_rowvjp_t<16>(g, tables, Q, nimg, nsets, targets, alpha, thr, images, loss, st);
    case 32: return launch_rowvjp_t<32>(g, tables, Q, nimg, nsets, targets, alpha, thr, images, loss, st);
  }
  set_error("gen_launch_rowvjp: unsupported row transform length");
  return KL_ERR_UNSUPPORTED;
}

int gen_launch_vjp_spectral(const GenGeom& g, const float2* band, int nparts, const float2* gband, int gparts,
                            int nclips, const float2* H, const float* lam, int K, int nsets, int nsplit, float2* gam,
                            cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  switch (g.RG) {
    case 1: return launch_vspec_t<1>(g, band, nparts, gband, gparts, nclips, H, lam, K, nsets, nsplit, gam, st);
    case 2: return launch_vspec_t<2>(g, band, nparts, gband, gparts, nclips, H, lam, K, nsets, nsplit, gam, st);
    case 4: return launch_vspec_t<4>(g, band, nparts, gband, gparts, nclips, H, lam, K, nsets, nsplit, gam, st);
    case 8: return launch_vspec_t<8>(g, band, nparts, gband, gparts, nclips, H, lam, K, nsets, nsplit, gam, st);
  }
  set_error("gen_launch_vjp_spectral: unsupported spectral grid");
  return KL_ERR_UNSUPPORTED;
}

int gen_launch_gradT(const GenGeom& g, const float2* gam, int nclips, int nparts, float2* Tg, cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  k_gen_gradT<<<nclips, kT, 0, st>>>(gam, g, nparts, Tg);
  return check_launch("k_gen_gradT");
}

int gen_launch_vjp_source(const GenGeom& g, const float2* band, int nparts, const float2* gband, int gparts,
                          int nimg, int nsets, const float2* Hs, int S, const float* Jw, const int* src_id,
                          int nsplit, float* grad_src, cudaStream_t st) {
  if (nimg <= 0) return KL_OK;
  switch (g.RG) {
    case 1: return launch_vsrc_t<1>(g, band, nparts, gband, gparts, nimg, nsets, Hs, S, Jw, src_id, nsplit, grad_src, st);
    case 2: return launch_vsrc_t<2>(g, band, nparts, gband, gparts, nimg, nsets, Hs, S, Jw, src_id, nsplit, grad_src, st);
    case 4: return launch_vsrc_t<4>(g, band, nparts, gband, gparts, nimg, nsets, Hs, S, Jw, src_id, nsplit, grad_src, st);
    case 8: return launch_vsrc_t<8>(g, band, nparts, gband, gparts, nimg, nsets, Hs, S, Jw, src_id, nsplit, grad_src, st);
  }
  set_error("gen_launch_vjp_source: unsupported spectral grid");
  return KL_ERR_UNSUPPORTED;
}

}  // namespace kl
