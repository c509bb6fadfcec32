// socs_gen.cu -- fused single-precision SOCS imaging for any clip period and
// bands up to a 256-point spectral grid (sm_100a).
//
// Same model as socs_fast.cu -- the K-Litho SOCS image
//     image = sum_k lambda_k |IFFT(H_k . FT(m))|^2 , Fourier-interpolated to Lx x Ly
// (K-Litho-SOCS/klitho_socs.cpp:196-241 calcSOCS, :158-194 FI, fed by
// FT_r2c :70-121) -- but with no restriction on Lx, Ly (the reference takes
// any period, klitho_socs.cpp:256-270) and with spectral grids up to G = 256
// (4N+1 <= 256: 4096^2 clips at NA 1.35 have N = 53, 4N+1 = 213).  The K
// coherent fields and the full-size spectrum never reach HBM.  Stages:
//
//  row_fwd   (HBM-bound) each warp turns mask rows into their Nx+1 row bins:
//            lane l' holds pixels x = l' + Vf i, a real DFT of length Pf over i
//            in registers, then the bins are gathered by the lanes that own
//            them through a per-warp shared buffer (no warp reduce-scatter, so
//            the register count does not grow with the band).
//  col_fwd   the row bins' DFT along y, kept for |fy| <= Ny: 32-point warp FFTs
//            over strips of 32 rows spaced Ly/32 apart when 32 divides Ly,
//            otherwise a direct sum; strips are split over `nparts` partial bands.
//  spectral  per (image, kernel slice) a cluster of RG = G/32 CTAs; CTA c holds
//            the grid columns x = c + RG j (j < 32): the band rows are folded
//            mod 32 with the twiddle e^{2 pi i fx c/G} and inverse transformed by
//            a 32-point warp FFT, the columns by G-point warp FFTs; the K fields'
//            lambda |E|^2 stay in registers.  The intensity is transformed back
//            (y by the transposed warp FFT straight from registers, x by a
//            32-point FFT) and the RG CTAs sum their contributions to the
//            intensity spectrum T through distributed shared memory.
//  col_inv   T's columns synthesised along y for every image row (strip FFTs
//            or a direct sum), giving the rows' coefficients Q[y][b], b <= 2Nx.
//  row_inv   (HBM-bound) each warp synthesises image rows from Q: lane l'
//            accumulates the Hermitian half of its P sub-bins and runs one
//            length-P complex-to-real transform in registers.
//
// Twiddle tables that depend on the period are made once per plan with exact
// double-precision arguments.  Only row bins (Nx+1 or 2Nx+1 per row), band
// partials and T pass through global memory.
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

__host__ __device__ inline int pow2_ge(int v) {
  int p = 1;
  while (p < v) p <<= 1;
  return p;
}
__device__ __forceinline__ int brev5(int lane) { return (int)(__brev((unsigned)lane) >> 27); }
__device__ __forceinline__ int mod_pos(int a, int m) {
  int r = a % m;
  return r < 0 ? r + m : r;
}

// table offsets inside one float2 buffer
__host__ __device__ inline size_t off_twl(const GenGeom& g) { return (size_t)g.NBX * 32; }
__host__ __device__ inline size_t off_tw2(const GenGeom& g) { return (size_t)g.NBX * 64; }
__host__ __device__ inline size_t off_rly(const GenGeom& g) { return (size_t)g.NBX * 64 + (size_t)g.nC * g.NBX; }
}  // namespace

// ---------------------------------------------------------------------------
// geometry and plan-time tables
// ---------------------------------------------------------------------------
int gen_geometry(int Lx, int Ly, int Nx, int Ny, GenGeom* out) {
  if (Lx <= 0 || Ly <= 0 || Nx < 0 || Ny < 0) {
    set_error("gen_geometry: invalid sizes");
    return KL_ERR_INVALID;
  }
  GenGeom g{};
  g.Lx = Lx;
  g.Ly = Ly;
  g.Nx = Nx;
  g.Ny = Ny;
  g.nbx = 2 * Nx + 1;
  g.nby = 2 * Ny + 1;
  g.nf = Nx + 1;
  g.ntx = 2 * Nx + 1;
  g.nty = 4 * Ny + 1;
  const int gmin = 4 * std::max(Nx, Ny) + 1;
  g.G = std::max(32, pow2_ge(gmin));
  if (g.G > 256) {
    set_error("SOCS path supports 4*max(Nx,Ny)+1 <= 256 (got " + std::to_string(gmin) + ")");
    return KL_ERR_UNSUPPORTED;
  }
  g.RG = g.G / 32;
  // the reference's half-spectrum bookkeeping in FI assumes the SOCS grid
  // 4N+1 fits in half the period; physical optics always satisfies it
  if (4 * Nx + 1 > Lx / 2 || 4 * Ny + 1 > Ly / 2) {
    set_error("band too wide for the clip size (4N+1 must not exceed half the period)");
    return KL_ERR_UNSUPPORTED;
  }
  // synthesis: the largest power of two P <= 64 dividing Lx that leaves at
  // least 32 lanes of work per row
  int P = 1;
  while (P < 64 && Lx % (2 * P) == 0 && Lx / (2 * P) >= 32) P *= 2;
  g.P = P;
  g.V = Lx / P;
  g.Pf = std::min(P, 32);
  g.Vf = Lx / g.Pf;
  g.nC = (std::max(g.V, g.Vf) + 31) / 32;
  const int q = std::max(32, P);
  g.NBX = (g.ntx + q - 1) / q * q;
  g.ystrip = (Ly % 32 == 0) ? 1 : 0;
  g.nS = g.ystrip ? Ly / 32 : (Ly + 31) / 32;
  g.dx = 2 * ((Lx + 1) / 2) - Lx;
  g.dy = 2 * ((Ly + 1) / 2) - Ly;
  *out = g;
  return KL_OK;
}

size_t gen_rowbins_bytes(const GenGeom& g, int nimg, int nbins) {
  return sizeof(float2) * (size_t)nimg * g.Ly * nbins;
}
size_t gen_band_bytes(const GenGeom& g, int n, int nparts, int nrows, int ncols) {
  (void)g;
  return sizeof(float2) * (size_t)n * nparts * nrows * ncols;
}
size_t gen_T_bytes(const GenGeom& g, int nimg, int nsplit) {
  return sizeof(float2) * (size_t)nimg * nsplit * g.ntx * g.nty;
}
size_t gen_table_elems(const GenGeom& g) { return off_rly(g) + (size_t)g.Ly; }

int gen_choose_split(const GenGeom& g, int nimg, int K, int per_sm) {
  // kernel slices per image: the count whose CTAs fill the GPU's resident
  // slots most evenly (waves x work per CTA), with slices of at least 3 kernels
  const long long slots = (long long)kSMs * per_sm, ctas = (long long)g.RG * nimg;
  int best = 1;
  double best_t = 1e30;
  for (int ns = 1; ns <= kGenMaxSplit && (ns == 1 || K / ns >= 3); ns *= 2) {
    const double t = (double)((ctas * ns + slots - 1) / slots) / ns;
    if (t < best_t * 0.98) {
      best_t = t;
      best = ns;
    }
  }
  return best;
}

int gen_choose_parts(const GenGeom& g, int n, int ncols) {
  // enough CTAs of the column transform to cover the GPU, at least 4 strips each
  const int groups = (ncols + kW - 1) / kW;
  int np = 1;
  while (groups * n * np < 2 * kSMs && g.nS / (2 * np) >= 4) np *= 2;
  return np;
}

// twb[b][l] = twl[l][b] = e^{+2 pi i b l / Lx}; tw2[c][b] = e^{+2 pi i b 32 c / Lx};
// rly[m] = e^{+2 pi i m / Ly}
__global__ void k_gen_tables(const GenGeom g, float2* __restrict__ t) {
  const size_t n1 = (size_t)g.NBX * 32, n2 = (size_t)g.nC * g.NBX;
  const size_t n = off_rly(g) + g.Ly;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float2 v;
    if (i < n1) {
      const int b = (int)(i / 32), l = (int)(i % 32);
      v = expi2pi_frac((long long)b * l, g.Lx);
    } else if (i < 2 * n1) {
      const size_t j = i - n1;
      const int l = (int)(j / g.NBX), b = (int)(j % g.NBX);
      v = expi2pi_frac((long long)b * l, g.Lx);
    } else if (i < 2 * n1 + n2) {
      const size_t j = i - 2 * n1;
      const int c = (int)(j / g.NBX), b = (int)(j % g.NBX);
      v = expi2pi_frac((long long)b * 32 * c, g.Lx);
    } else {
      v = expi2pi_frac((long long)(i - off_rly(g)), g.Ly);
    }
    t[i] = v;
  }
}

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
}  // namespace

int gen_build_tables(const GenGeom& g, float2* tables, cudaStream_t st) {
  const size_t n = gen_table_elems(g);
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 4096);
  k_gen_tables<<<blocks, 256, 0, st>>>(g, tables);
  return check_launch("k_gen_tables");
}

// ---------------------------------------------------------------------------
// 1. row_fwd: rows of `src` (Lx floats each) -> R[row][fx], fx < nbins
// ---------------------------------------------------------------------------
template <int PF>
__global__ void __launch_bounds__(kT) k_gen_rowfwd(const float* __restrict__ src, int nrows, const GenGeom g,
                                                   const float2* __restrict__ tables, int nbins,
                                                   float2* __restrict__ R) {
  constexpr int HS = PF / 2 + 1;
  extern __shared__ float4 smem4[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float2* tl = reinterpret_cast<float2*>(smem4);  // [32][NBX]  e^{+2 pi i b l / Lx}
  float2* sb = tl + 32 * g.NBX + warp * HS * 33;  // [HS][33]   the lanes' real-DFT outputs
  const float2* twl = tables + off_twl(g);
  const float2* tw2 = tables + off_tw2(g);
  for (int i = threadIdx.x; i < 32 * g.NBX; i += kT) tl[i] = __ldg(twl + i);
  __syncthreads();
  const int V = g.Vf, nch = (V + 31) / 32, nt = (nbins + 31) / 32;
  for (int row = blockIdx.x * kW + warp; row < nrows; row += gridDim.x * kW) {
    const float* rp = src + (size_t)row * g.Lx;
    float2 acc[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) acc[t] = make_float2(0.f, 0.f);
#pragma unroll 1
    for (int c = 0; c < nch; ++c) {
      const int lp = lane + 32 * c;
      float val[PF];
      if (lp < V) {
#pragma unroll
        for (int i = 0; i < PF; ++i) val[i] = __ldcs(rp + lp + V * i);
      } else {
#pragma unroll
        for (int i = 0; i < PF; ++i) val[i] = 0.f;
      }
      float2 S[HS];
      rdft_any<PF>(val, S);
#pragma unroll
      for (int k = 0; k < HS; ++k) sb[k * 33 + lane] = S[k];
      __syncwarp();
      // bin fx = sum over the chunk's lanes l of S_l[fx mod PF] e^{-2 pi i fx (l + 32c)/Lx}
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int fx = lane + 32 * t;
        if (t < nt && fx < nbins) {
          const int k = fx % PF;
          const bool cj = 2 * k > PF;
          const int kk = cj ? PF - k : k;
          const float sg = cj ? -1.f : 1.f;
          float2 s = make_float2(0.f, 0.f);
#pragma unroll 8
          for (int l = 0; l < 32; ++l) {
            const float2 sv = sb[kk * 33 + l];
            const float svy = sg * sv.y;
            const float2 w = tl[l * g.NBX + fx];
            s.x = fmaf(sv.x, w.x, fmaf(svy, w.y, s.x));
            s.y = fmaf(svy, w.x, fmaf(-sv.x, w.y, s.y));
          }
          acc[t] = cfma(s, cconj(__ldg(tw2 + (size_t)c * g.NBX + fx)), acc[t]);
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int fx = lane + 32 * t;
      if (t < nt && fx < nbins) R[(size_t)row * nbins + fx] = acc[t];
    }
  }
}

// ---------------------------------------------------------------------------
// 2. col_fwd: R[n][y][fx] -> band[n][part][fy + Yb][fx], |fy| <= Yb, times scale
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kT) k_gen_colfwd(const float2* __restrict__ R, int ncols, int Yb,
                                                   const GenGeom g, const float2* __restrict__ rly,
                                                   float scale, float2* __restrict__ band) {
  constexpr int MT = 8;  // 2 Yb + 1 <= 256
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int fx = blockIdx.x * kW + warp;
  const int n = blockIdx.y, part = blockIdx.z, nparts = gridDim.z;
  if (fx >= ncols) return;  // whole warp; no block-wide barrier below
  const int nyo = 2 * Yb + 1, Ly = g.Ly;
  const float2* Rn = R + (size_t)n * Ly * ncols;
  float2* out = band + ((size_t)n * nparts + part) * nyo * ncols;
  float2 acc[MT];
#pragma unroll
  for (int t = 0; t < MT; ++t) acc[t] = make_float2(0.f, 0.f);
  if (g.ystrip) {
    const int nS = g.nS;
    const int s0 = (int)((long long)nS * part / nparts), s1 = (int)((long long)nS * (part + 1) / nparts);
    WarpFFT<1, -1> wf;
    wf.init(lane);
    const int q = brev5(lane);
    const int fy0 = q - 32 * ((q + Yb) / 32);  // smallest fy >= -Yb with fy = q (mod 32)
    // the next strip's row bin and phases are loaded while this strip is transformed
    float2 rn = make_float2(0.f, 0.f), pn[MT];
    auto fetch = [&](int s) {
      rn = __ldg(Rn + (size_t)(s + nS * lane) * ncols + fx);
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        const int fy = fy0 + 32 * t;
        pn[t] = fy <= Yb ? __ldg(rly + mod_pos(fy * s, Ly)) : make_float2(1.f, 0.f);
      }
    };
    if (s0 < s1) fetch(s0);
    for (int s = s0; s < s1; ++s) {
      float2 v[1] = {rn};
      float2 p[MT];
#pragma unroll
      for (int t = 0; t < MT; ++t) p[t] = pn[t];
      if (s + 1 < s1) fetch(s + 1);
      wf.run(v, lane);
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        const int fy = fy0 + 32 * t;
        if (fy <= Yb) acc[t] = cfma(v[0], cconj(p[t]), acc[t]);
      }
    }
#pragma unroll
    for (int t = 0; t < MT; ++t) {
      const int fy = fy0 + 32 * t;
      if (fy <= Yb) out[(size_t)(fy + Yb) * ncols + fx] = cscale(acc[t], scale);
    }
  } else {
    const int y0 = (int)((long long)Ly * part / nparts), y1 = (int)((long long)Ly * (part + 1) / nparts);
    int m[MT];
#pragma unroll
    for (int t = 0; t < MT; ++t) m[t] = mod_pos((-Yb + lane + 32 * t) * y0, Ly);
    for (int y = y0; y < y1; ++y) {
      const float2 v = __ldg(Rn + (size_t)y * ncols + fx);
#pragma unroll
      for (int t = 0; t < MT; ++t) {
        const int fy = -Yb + lane + 32 * t;
        if (fy <= Yb) {
          acc[t] = cfma(v, cconj(__ldg(rly + m[t])), acc[t]);
          m[t] += fy;
          if (m[t] >= Ly) m[t] -= Ly;
          else if (m[t] < 0) m[t] += Ly;
        }
      }
    }
#pragma unroll
    for (int t = 0; t < MT; ++t) {
      const int fy = -Yb + lane + 32 * t;
      if (fy <= Yb) out[(size_t)(fy + Yb) * ncols + fx] = cscale(acc[t], scale);
    }
  }
}

// ---------------------------------------------------------------------------
// 3. spectral core: band -> sum_k lambda_k |E_k|^2 -> T[img][split][b][a]
// ---------------------------------------------------------------------------
// Shared memory (float2 units): the band half Mh [nby][nf] and stage-1 rows
// E1 [nby][33] during the kernel loop; afterwards, over the same space, the
// per-warp FFT rows Zw [8][G] and the y-transformed intensity Ys [nty][33];
// then the G roots of unity.
__host__ __device__ inline size_t gen_spec_smem_elems(const GenGeom& g) {
  const size_t r0 = (size_t)g.nby * g.nf + (size_t)g.nby * 33;
  const size_t r1 = (size_t)kW * g.G + (size_t)g.nty * 33;
  return (r0 > r1 ? r0 : r1) + g.G;
}

template <int RG>
__global__ void __launch_bounds__(kT, 2) k_gen_spectral(const float2* __restrict__ band, int nparts,
                                                        const GenGeom g, const float2* __restrict__ H,
                                                        const float* __restrict__ lam, int K, int nsets,
                                                        float2* __restrict__ Tout) {
  constexpr int G = 32 * RG;
  constexpr int CW = 32 / kW;  // columns per warp
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ float4 smem4[];
  float2* base = reinterpret_cast<float2*>(smem4);
  float2* Mh = base;                    // [nby][nf]
  float2* E1 = Mh + g.nby * g.nf;       // [nby][33]
  float2* Zw = base;                    // [kW][G]   (after the kernel loop)
  float2* Ys = Zw + kW * G;             // [nty][33] (after the kernel loop)
  const size_t r0 = (size_t)g.nby * g.nf + (size_t)g.nby * 33;
  const size_t r1 = (size_t)kW * G + (size_t)g.nty * 33;
  float2* rootG = base + (r0 > r1 ? r0 : r1);  // [G] e^{+2 pi i m / G}

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = blockIdx.x;  // grid column class = rank in the cluster
  const int img = blockIdx.y, split = blockIdx.z, nsplit = gridDim.z;
  const int clip = img / nsets, set = img - clip * nsets;
  const int k0 = (int)(((long long)K * split) / nsplit), k1 = (int)(((long long)K * (split + 1)) / nsplit);
  const int br = brev5(lane);
  const int nf = g.nf, nby = g.nby, nbx = g.nbx, Nx = g.Nx, Ny = g.Ny;

  for (int i = threadIdx.x; i < G; i += kT) rootG[i] = expi2pi_frac(i, G);
  __syncthreads();
  // band half, parts summed, times e^{2 pi i fx c / G} (keeps the conjugate
  // symmetry M'[fy][-fx] = conj M'[-fy][fx])
  {
    const size_t per = (size_t)nby * nf;
    const float2* b0 = band + (size_t)clip * nparts * per;
    for (int i = threadIdx.x; i < nby * nf; i += kT) {
      const int fx = i % nf;
      float2 v = __ldg(b0 + i);
      for (int p = 1; p < nparts; ++p) v = cadd(v, __ldg(b0 + p * per + i));
      Mh[i] = cmul(v, rootG[(fx * c) & (G - 1)]);
    }
  }
  __syncthreads();

  WarpFFT<1, +1> w1;
  w1.init(lane);
  WarpFFT<RG, +1> wi;
  wi.init(lane);
  float acc[CW][RG];
#pragma unroll
  for (int t = 0; t < CW; ++t)
#pragma unroll
    for (int q = 0; q < RG; ++q) acc[t][q] = 0.f;

  const size_t nb2 = (size_t)nby * nbx;
  const float2* Hs = H + (size_t)set * K * nb2;
  const int fxs = lane - 32 * ((lane + Nx) / 32);  // smallest fx >= -Nx with fx = lane (mod 32)
  // the kernel rows come from L2: each warp keeps the loads of its next row in
  // flight while it folds and transforms the current one (the next kernel's
  // first row after its last), so their latency overlaps the work
  float2 hn[kGenMaxFold];
  if (k0 < k1 && warp < nby) gen_load_hrow(Hs + (size_t)k0 * nb2, warp, nbx, Nx, fxs, hn);
  for (int k = k0; k < k1; ++k) {
    const float2* Hk = Hs + (size_t)k * nb2;
    const float lk = __ldg(lam + set * K + k);
    // stage 1: band rows folded mod 32, then a 32-point inverse FFT over the lanes
    for (int r = warp; r < nby; r += kW) {
      float2 h[kGenMaxFold];
#pragma unroll
      for (int t = 0; t < kGenMaxFold; ++t) h[t] = hn[t];
      if (r + kW < nby) gen_load_hrow(Hk, r + kW, nbx, Nx, fxs, hn);
      else if (k + 1 < k1) gen_load_hrow(Hk + nb2, warp, nbx, Nx, fxs, hn);
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
    __syncthreads();
    // stage 2: the CTA's 32 columns, G-point inverse FFT along y
#pragma unroll
    for (int t = 0; t < CW; ++t) {
      const int j = warp + kW * t;
      float2 vv[RG];
#pragma unroll
      for (int i = 0; i < RG; ++i) {
        const int n = lane + 32 * i;
        const int fy = n <= Ny ? n : (n >= G - Ny ? n - G : INT_MIN);
        vv[i] = fy != INT_MIN ? E1[(fy + Ny) * 33 + j] : make_float2(0.f, 0.f);
      }
      wi.run(vv, lane);
#pragma unroll
      for (int q = 0; q < RG; ++q) acc[t][q] = fmaf(lk, cabs2(vv[q]), acc[t][q]);
    }
    __syncthreads();
  }

  // y transform of the intensity columns, two real columns per complex FFT,
  // straight from the registers' bit-reversed layout
  WarpFFT<RG, -1> wf;
  wf.init(lane);
  float2* zw = Zw + warp * G;
  const int A = 2 * Ny;
#pragma unroll
  for (int pr = 0; pr < CW / 2; ++pr) {
    const int j0 = warp + kW * (2 * pr), j1 = warp + kW * (2 * pr + 1);
    float2 vv[RG];
#pragma unroll
    for (int q = 0; q < RG; ++q) vv[q] = make_float2(acc[2 * pr][q], acc[2 * pr + 1][q]);
    wf.run_rev(vv, lane);
#pragma unroll
    for (int i = 0; i < RG; ++i) zw[lane + 32 * i] = vv[i];
    __syncwarp();
    for (int a = -A + lane; a <= A; a += 32) {
      const float2 za = zw[a & (G - 1)], zb = cconj(zw[(-a) & (G - 1)]);
      const float2 y0 = cscale(cadd(za, zb), 0.5f);
      const float2 d = cscale(csub(za, zb), 0.5f);
      Ys[(a + A) * 33 + j0] = y0;
      Ys[(a + A) * 33 + j1] = make_float2(d.y, -d.x);
    }
    __syncwarp();
  }
  __syncthreads();
  // x transform over the CTA's 32 columns: F[a][m] = sum_j Ys[a][j] e^{-2 pi i m j/32}
  {
    WarpFFT<1, -1> wx;
    wx.init(lane);
    for (int r = warp; r < g.nty; r += kW) {
      float2 vv[1] = {Ys[r * 33 + lane]};
      wx.run(vv, lane);
      __syncwarp();
      Ys[r * 33 + br] = vv[0];
    }
  }
  cl.sync();
  // T[b][a] = (1/G^2) sum_c e^{-2 pi i b c / G} F_c[a][b mod 32]; this CTA
  // writes rows a in [a0, a1)
  {
    const int per = (g.nty + RG - 1) / RG;
    const int a0 = c * per, a1 = min(g.nty, a0 + per), na = a1 - a0;
    const float invg = 1.0f / ((float)G * (float)G);
    float2* To = Tout + ((size_t)img * nsplit + split) * g.ntx * g.nty;
    const float2* peers[RG];
#pragma unroll
    for (int cc = 0; cc < RG; ++cc) peers[cc] = cl.map_shared_rank(Ys, cc);
    for (int i = threadIdx.x; i < na * g.ntx; i += kT) {
      const int b = i / na, r = a0 + (i - b * na);
      const int m = b & 31;
      float2 s = make_float2(0.f, 0.f);
#pragma unroll
      for (int cc = 0; cc < RG; ++cc) s = cfma(peers[cc][r * 33 + m], cconj(rootG[(b * cc) & (G - 1)]), s);
      s = cscale(s, invg);
      if (g.dx | g.dy) {
        // odd periods: the reference's shifts move the image by one pixel
        const float2 ph1 = expi2pi_frac(-(long long)(r - A) * g.dy, g.Ly);
        const float2 ph2 = expi2pi_frac(-(long long)b * g.dx, g.Lx);
        s = cmul(s, cmul(ph1, ph2));
      }
      To[(size_t)b * g.nty + r] = s;
    }
  }
  cl.sync();  // peers' shared memory stays valid until every CTA has read it
}

// ---------------------------------------------------------------------------
// 4. col_inv: T[img][split][b][a + A] -> Q[img][y][b] = w_b sum_a T e^{2 pi i a y/Ly}
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kT) k_gen_colinv(const float2* __restrict__ T, int nsplit, int A, int nbins,
                                                   const GenGeom g, const float2* __restrict__ rly,
                                                   float2* __restrict__ Q, int spc) {
  extern __shared__ float4 smem4[];
  float2* Qs = reinterpret_cast<float2*>(smem4);  // [32][nbins + 1]
  float2* ph = Qs + 32 * (nbins + 1);             // [2A + 1] e^{2 pi i a s / Ly} of the strip
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lda = 2 * A + 1, qp = nbins + 1, Ly = g.Ly;
  const int img = blockIdx.y;
  const size_t tsz = (size_t)nbins * lda;
  const float2* Ti = T + (size_t)img * nsplit * tsz;
  float2* Qi = Q + (size_t)img * Ly * nbins;
  WarpFFT<1, +1> wf;
  wf.init(lane);
  const int br = brev5(lane);
  const int s0 = blockIdx.x * spc, s1 = min(g.nS, s0 + spc);
  for (int s = s0; s < s1; ++s) {
    int nr = 32;
    if (g.ystrip) {
      for (int i = threadIdx.x; i < lda; i += kT) ph[i] = __ldg(rly + mod_pos((i - A) * s, Ly));
      __syncthreads();
      const int a0 = lane - 32 * ((lane + A) / 32);  // smallest a >= -A with a = lane (mod 32)
      for (int b = warp; b < nbins; b += kW) {
        // the column's terms a = a0 + 32 t (at most 8: 2A + 1 <= 255), loads issued together
        float2 tv[8];
        const float2* tp = Ti + (size_t)b * lda + A;
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          const int a = a0 + 32 * t;
          tv[t] = a <= A ? __ldg(tp + a) : make_float2(0.f, 0.f);
        }
        float2 f = make_float2(0.f, 0.f);
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          const int a = a0 + 32 * t;
          if (a <= A) f = cfma(tv[t], ph[a + A], f);
        }
        float2 v[1] = {f};
        wf.run(v, lane);
        Qs[br * qp + b] = cscale(v[0], b == 0 ? 1.f : 2.f);
      }
    } else {
      const int y = s * 32 + lane;
      nr = min(32, Ly - s * 32);
      for (int b = warp; b < nbins; b += kW) {
        float2 f = make_float2(0.f, 0.f);
        if (y < Ly) {
          int m = mod_pos(-A * y, Ly);
          const float2* tp = Ti + (size_t)b * lda;
          for (int a = 0; a < lda; ++a) {
            f = cfma(__ldg(tp + a), __ldg(rly + m), f);
            m += y;
            if (m >= Ly) m -= Ly;
          }
        }
        Qs[lane * qp + b] = cscale(f, b == 0 ? 1.f : 2.f);
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nr * nbins; i += kT) {
      const int j = i / nbins, b = i - j * nbins;
      const int y = g.ystrip ? s + g.nS * j : s * 32 + j;
      Qi[(size_t)y * nbins + b] = Qs[j * qp + b];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// 5. row_inv: Q[row][b] (b < nbins) -> out[row][x] = Re sum_b Q[b] e^{2 pi i b x/Lx}
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(kT) k_gen_rowinv(const float2* __restrict__ Q, int nbins, int nrows,
                                                   const GenGeom g, const float2* __restrict__ tables,
                                                   float* __restrict__ out) {
  constexpr int HY = P / 2 + 1;
  extern __shared__ float4 smem4[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float2* tb = reinterpret_cast<float2*>(smem4);  // [NBX][32]  e^{+2 pi i b l / Lx}
  float2* qc = tb + g.NBX * 32 + warp * g.NBX;    // [NBX]      this warp's chunk coefficients
  float2* t2s = tb + g.NBX * 32 + kW * g.NBX;     // [nC][NBX]  chunk twiddles, when they fit
  const int V = g.V, nch = (V + 31) / 32;
  const bool t2_shared = gen_t2_in_smem(g);
  const float2* tw2 = t2_shared ? t2s : tables + off_tw2(g);
  for (int i = threadIdx.x; i < 32 * g.NBX; i += kT) tb[i] = __ldg(tables + i);
  if (t2_shared)
    for (int i = threadIdx.x; i < nch * g.NBX; i += kT) t2s[i] = __ldg(tables + off_tw2(g) + i);
  __syncthreads();
  const int nbp = (nbins + P - 1) / P * P;
  // each lane holds the coefficients b = lane + 32 t of its warp's row; the
  // next row's are loaded while the current one is synthesised
  float2 qn[4];
  const int row0 = blockIdx.x * kW + warp, rstep = gridDim.x * kW;
  if (row0 < nrows) gen_load_qrow(Q + (size_t)row0 * nbins, nbins, lane, qn);
  for (int row = row0; row < nrows; row += rstep) {
    float2 q[4];
#pragma unroll
    for (int t = 0; t < 4; ++t) q[t] = qn[t];
    if (row + rstep < nrows) gen_load_qrow(Q + (size_t)(row + rstep) * nbins, nbins, lane, qn);
    float* orow = out + (size_t)row * g.Lx;
#pragma unroll 1
    for (int c = 0; c < nch; ++c) {
      // q_c[b] = Q[b] e^{2 pi i b 32 c / Lx}: the lane twiddle then only depends on the lane
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int b = lane + 32 * t;
        if (b < nbp) qc[b] = b < nbins ? cmul(q[t], tw2[(size_t)c * g.NBX + b]) : make_float2(0.f, 0.f);
      }
      __syncwarp();
      float2 Y[HY];
#pragma unroll
      for (int k = 0; k < HY; ++k) Y[k] = make_float2(0.f, 0.f);
#pragma unroll 1
      for (int b0 = 0; b0 < nbp; b0 += P) {
#pragma unroll
        for (int k = 0; k < P; ++k) {
          const float2 q = qc[b0 + k];
          const float2 w = tb[(b0 + k) * 32 + lane];
          if (2 * k <= P) {
            Y[k] = cfma(q, w, Y[k]);
          } else {
            Y[P - k].x = fmaf(q.x, w.x, fmaf(-q.y, w.y, Y[P - k].x));
            Y[P - k].y = fmaf(-q.x, w.y, fmaf(-q.y, w.x, Y[P - k].y));
          }
        }
      }
      float o[P];
      c2r_half<P>(Y, o);
      const int lp = lane + 32 * c;
      if (lp < V) {
#pragma unroll
        for (int i = 0; i < P; ++i) __stcs(orow + lp + V * i, o[i]);
      }
      __syncwarp();
    }
  }
}

// slice partials of T summed into slice 0 (one pass over L2-resident data), so
// that the column synthesis reads one spectrum per image
__global__ void k_gen_sumT(float2* __restrict__ T, size_t tsz, int nsplit) {
  float2* Ti = T + (size_t)blockIdx.y * nsplit * tsz;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tsz; i += (size_t)gridDim.x * blockDim.x) {
    float2 v = Ti[i];
    for (int p = 1; p < nsplit; ++p) v = cadd(v, Ti[p * tsz + i]);
    Ti[i] = v;
  }
}

// centred FT_r2c band: M(ky,kx) = D(ky,kx) e^{-2 pi i (ky yh/Ly + kx xh/Lx)}
__global__ void k_gen_bandout(const float2* __restrict__ band, int nparts, const GenGeom g,
                              float2* __restrict__ out) {
  const int clip = blockIdx.x;
  const size_t per = (size_t)g.nby * g.nf;
  const float2* b0 = band + (size_t)clip * nparts * per;
  const int yh = (g.Ly + 1) / 2, xh = (g.Lx + 1) / 2;
  for (int i = threadIdx.x; i < g.nby * g.nbx; i += blockDim.x) {
    const int r = i / g.nbx, cidx = i - r * g.nbx;
    const int ky = r - g.Ny, kx = cidx - g.Nx;
    const size_t src = kx >= 0 ? (size_t)r * g.nf + kx : (size_t)(g.nby - 1 - r) * g.nf - kx;
    float2 v = __ldg(b0 + src);
    for (int p = 1; p < nparts; ++p) v = cadd(v, __ldg(b0 + p * per + src));
    if (kx < 0) v = cconj(v);
    const float2 p1 = expi2pi_frac(-(long long)ky * yh, g.Ly);
    const float2 p2 = expi2pi_frac(-(long long)kx * xh, g.Lx);
    out[(size_t)clip * g.nby * g.nbx + i] = cmul(v, cmul(p1, p2));
  }
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
namespace {
int row_grid(int nrows, int per_sm) {
  const int need = (nrows + kW - 1) / kW;
  return std::max(1, std::min(need, kSMs * per_sm));
}

template <int PF>
int launch_rowfwd_t(const GenGeom& g, const float2* tables, const float* src, int nrows, int nbins, float2* R,
                    cudaStream_t st) {
  const size_t sm = sizeof(float2) * ((size_t)32 * g.NBX + (size_t)kW * (PF / 2 + 1) * 33);
  auto kern = k_gen_rowfwd<PF>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  kern<<<row_grid(nrows, 8), kT, sm, st>>>(src, nrows, g, tables, nbins, R);
  return check_launch("k_gen_rowfwd");
}

template <int P>
int launch_rowinv_t(const GenGeom& g, const float2* tables, const float2* Q, int nrows, int nbins, float* out,
                    cudaStream_t st) {
  const size_t sm = sizeof(float2) * ((size_t)32 * g.NBX + (size_t)kW * g.NBX +
                                      (gen_t2_in_smem(g) ? (size_t)g.nC * g.NBX : 0));
  auto kern = k_gen_rowinv<P>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  kern<<<row_grid(nrows, 8), kT, sm, st>>>(Q, nbins, nrows, g, tables, out);
  return check_launch("k_gen_rowinv");
}

template <int RG>
int launch_spectral_t(const GenGeom& g, const float2* band, int nparts, int nclips, const float2* H,
                      const float* lam, int K, int nsets, int nsplit, float2* T, cudaStream_t st) {
  const size_t sm = sizeof(float2) * gen_spec_smem_elems(g);
  auto kern = k_gen_spectral<RG>;
  int rc = set_smem(kern, sm);
  if (rc) return rc;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(RG, nclips * nsets, nsplit);
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
  cudaError_t e = cudaLaunchKernelEx(&cfg, kern, band, nparts, g, H, lam, K, nsets, T);
  if (e != cudaSuccess) {
    set_error(std::string("k_gen_spectral: ") + cudaGetErrorString(e));
    return KL_ERR_CUDA;
  }
  return check_launch("k_gen_spectral");
}
}  // namespace

int gen_launch_rowfwd(const GenGeom& g, const float2* tables, const float* src, int nrows, float2* R,
                      cudaStream_t st) {
  if (nrows <= 0) return KL_OK;
  switch (g.Pf) {
    case 1: return launch_rowfwd_t<1>(g, tables, src, nrows, g.nf, R, st);
    case 2: return launch_rowfwd_t<2>(g, tables, src, nrows, g.nf, R, st);
    case 4: return launch_rowfwd_t<4>(g, tables, src, nrows, g.nf, R, st);
    case 8: return launch_rowfwd_t<8>(g, tables, src, nrows, g.nf, R, st);
    case 16: return launch_rowfwd_t<16>(g, tables, src, nrows, g.nf, R, st);
    case 32: return launch_rowfwd_t<32>(g, tables, src, nrows, g.nf, R, st);
  }
  set_error("gen_launch_rowfwd: unsupported row transform length");
  return KL_ERR_UNSUPPORTED;
}

int gen_launch_colfwd(const GenGeom& g, const float2* tables, const float2* R, int n, int ncols, int Yb,
                      float scale, int nparts, float2* band, cudaStream_t st) {
  if (n <= 0) return KL_OK;
  if (2 * Yb + 1 > 256) {
    set_error("gen_launch_colfwd: band taller than 256 rows");
    return KL_ERR_UNSUPPORTED;
  }
  dim3 grid((ncols + kW - 1) / kW, n, nparts);
  k_gen_colfwd<<<grid, kT, 0, st>>>(R, ncols, Yb, g, tables + off_rly(g), scale, band);
  return check_launch("k_gen_colfwd");
}

int gen_launch_spectral(const GenGeom& g, const float2* band, int nparts, int nclips, const float2* H,
                        const float* lam, int K, int nsets, int nsplit, float2* T, cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  switch (g.RG) {
    case 1: return launch_spectral_t<1>(g, band, nparts, nclips, H, lam, K, nsets, nsplit, T, st);
    case 2: return launch_spectral_t<2>(g, band, nparts, nclips, H, lam, K, nsets, nsplit, T, st);
    case 4: return launch_spectral_t<4>(g, band, nparts, nclips, H, lam, K, nsets, nsplit, T, st);
    case 8: return launch_spectral_t<8>(g, band, nparts, nclips, H, lam, K, nsets, nsplit, T, st);
  }
  set_error("gen_launch_spectral: unsupported spectral grid");
  return KL_ERR_UNSUPPORTED;
}

int gen_launch_colinv(const GenGeom& g, const float2* tables, const float2* T, int nimg, int nsplit, int A,
                      int nbins, float2* Q, cudaStream_t st) {
  if (nimg <= 0) return KL_OK;
  if (nsplit > 1) {
    // fold the slices into slice 0 first (T is the caller's spectra buffer)
    const size_t tsz = (size_t)nbins * (2 * A + 1);
    const int bx = (int)std::min<size_t>((tsz + 255) / 256, 64);
    k_gen_sumT<<<dim3(bx, nimg), 256, 0, st>>>(const_cast<float2*>(T), tsz, nsplit);
    int rc = check_launch("k_gen_sumT");
    if (rc) return rc;
  }
  // a few strips per CTA so the image's T is reused from L1, enough CTAs to fill the GPU
  int spc = 1;
  while (spc < 8 && (long long)nimg * ((g.nS + 2 * spc - 1) / (2 * spc)) >= 4 * kSMs) spc *= 2;
  const size_t sm = sizeof(float2) * ((size_t)32 * (nbins + 1) + (size_t)(2 * A + 1));
  int rc = set_smem(k_gen_colinv, sm);
  if (rc) return rc;
  dim3 grid((g.nS + spc - 1) / spc, nimg);
  k_gen_colinv<<<grid, kT, sm, st>>>(T, nsplit, A, nbins, g, tables + off_rly(g), Q, spc);  // reads slice 0
  return check_launch("k_gen_colinv");
}

int gen_launch_rowinv(const GenGeom& g, const float2* tables, const float2* Q, int nimg, int nbins, float* images,
                      cudaStream_t st) {
  if (nimg <= 0) return KL_OK;
  const int nrows = nimg * g.Ly;
  switch (g.P) {
    case 1: return launch_rowinv_t<1>(g, tables, Q, nrows, nbins, images, st);
    case 2: return launch_rowinv_t<2>(g, tables, Q, nrows, nbins, images, st);
    case 4: return launch_rowinv_t<4>(g, tables, Q, nrows, nbins, images, st);
    case 8: return launch_rowinv_t<8>(g, tables, Q, nrows, nbins, images, st);
    case 16: return launch_rowinv_t<16>(g, tables, Q, nrows, nbins, images, st);
    case 32: return launch_rowinv_t<32>(g, tables, Q, nrows, nbins, images, st);
    case 64: return launch_rowinv_t<64>(g, tables, Q, nrows, nbins, images, st);
  }
  set_error("gen_launch_rowinv: unsupported row transform length");
  return KL_ERR_UNSUPPORTED;
}

int gen_launch_bandout(const GenGeom& g, const float2* band, int nparts, int nclips, float2* out,
                       cudaStream_t st) {
  if (nclips <= 0) return KL_OK;
  k_gen_bandout<<<nclips, kT, 0, st>>>(band, nparts, g, out);
  return check_launch("k_gen_bandout");
}

}  // namespace kl
