// fp64_path.cu -- the plain FP64 GPU imaging path: a direct restatement of
// the reference's FT_r2c (K-Litho-SOCS/klitho_socs.cpp:70-121), calcSOCS
// (:196-241) with the K coherent fields materialised one g x g array each,
// FI (:158-194), and calcImage + FT_c2r (K-Litho-TCC/klitho_tcc.cpp:269-290,
// :150-183), all in FP64 on the CUDA cores with the library's own FFTs:
//   * power-of-two L x L transforms: radix-2 FFT along rows in shared memory
//     (one CTA per row, bit-reversed load, in-place butterflies) and a tiled
//     transpose between the row and column passes;
//   * the odd SOCS grid g = 4N + 1: a direct DFT along rows (g <= 255 terms).
// It is the FP64 correctness anchor of the GPU code (1e-12 of the oracle) and
// the denominator the mixed-precision fused path is measured against, so it
// does nothing clever: full-size spectra, every field written to memory.
#include <algorithm>
#include <string>
#include <vector>

#include "kl_internal.h"
#include "kl_plans.h"

namespace kl {
namespace f64 {

namespace {

constexpr int kFftThreads = 512;
constexpr int kMaxFftLog2 = 13;  // rows up to 8192 points (128 KB of shared memory)

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// w[j] = e^{+2 pi i j / n}, j < n
__global__ void k_twiddle(double2* w, int n) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * j / n, &s, &c);
    w[j] = make_double2(c, s);
  }
}

// data[r][k] <- scale * sum_j data[r][j] e^{sign 2 pi i j k / n}, n = 2^m
__global__ void __launch_bounds__(kFftThreads) k_fft_rows(double2* __restrict__ data, int n, int m,
                                                          const double2* __restrict__ w, int sign,
                                                          double scale) {
  extern __shared__ double2 a[];
  double2* row = data + (size_t)blockIdx.x * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) a[__brev(i) >> (32 - m)] = row[i];
  __syncthreads();
  for (int s = 0; s < m; ++s) {
    const int half = 1 << s, wstep = n >> (s + 1);
    for (int t = threadIdx.x; t < n / 2; t += blockDim.x) {
      const int pos = t & (half - 1), i = ((t >> s) << (s + 1)) + pos, j = i + half;
      double2 tw = w[pos * wstep];
      if (sign < 0) tw.y = -tw.y;
      const double2 u = a[i], v = cmul(a[j], tw);
      a[i] = make_double2(u.x + v.x, u.y + v.y);
      a[j] = make_double2(u.x - v.x, u.y - v.y);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) row[i] = make_double2(a[i].x * scale, a[i].y * scale);
}

// out[b][c][r] = in[b][r][c] for nb matrices of rows x cols
__global__ void k_transpose(const double2* __restrict__ in, double2* __restrict__ out, int rows, int cols) {
  __shared__ double2 tile[32][33];
  const size_t off = (size_t)blockIdx.z * rows * cols;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + k, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[k][threadIdx.x] = in[off + (size_t)r * cols + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = c0 + k, r = r0 + threadIdx.x;
    if (r < rows && c < cols) out[off + (size_t)c * rows + r] = tile[threadIdx.x][k];
  }
}

// out[r][k] = scale * sum_j in[r][j] e^{sign 2 pi i j k / n} (any n; w has n entries)
__global__ void k_dft_rows(const double2* __restrict__ in, double2* __restrict__ out, int n, int nrows,
                           const double2* __restrict__ w, int sign, double scale) {
  const size_t total = (size_t)nrows * n;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const size_t r = idx / n;
    const int k = (int)(idx - r * n);
    const double2* x = in + r * n;
    double re = 0.0, im = 0.0;
    int e = 0;  // j k mod n
    for (int j = 0; j < n; ++j) {
      double2 tw = w[e];
      if (sign < 0) tw.y = -tw.y;
      const double2 v = x[j];
      re += v.x * tw.x - v.y * tw.y;
      im += v.x * tw.y + v.y * tw.x;
      e += k;
      if (e >= n) e -= n;
    }
    out[idx] = make_double2(re * scale, im * scale);
  }
}

// myShift (klitho_socs.cpp:37-50) of the float mask by ((L+1)/2), as complex:
// d[y][x] = m[(y - yh) mod Ly][(x - xh) mod Lx]
__global__ void k_load_shifted(const float* __restrict__ m, int Lx, int Ly, double2* __restrict__ d) {
  const int xh = (Lx + 1) / 2, yh = (Ly + 1) / 2;
  const size_t n = (size_t)Lx * Ly;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / Lx), x = (int)(i - (size_t)y * Lx);
    const int ys = (y - yh + Ly) % Ly, xs = (x - xh + Lx) % Lx;
    d[i] = make_double2((double)m[(size_t)ys * Lx + xs], 0.0);
  }
}

// centred spectrum entry (kx, ky) of FT_r2c from the natural-order DFT D
__device__ __forceinline__ double2 spec(const double2* D, int Lx, int Ly, int kx, int ky, double inv) {
  const double2 v = D[(size_t)((ky + Ly) % Ly) * Lx + (kx + Lx) % Lx];
  return make_double2(v.x * inv, v.y * inv);
}

// calcSOCS input arrays (klitho_socs.cpp:218-224): X_k = 0 except the band
// X_k[difY + y + Ny][difX + x + Nx] = H_k[y][x] * M^(x, y), one g x g array per kernel
__global__ void k_socs_embed(const double2* __restrict__ D, int Lx, int Ly, const float2* __restrict__ H,
                             int nk, int Nx, int Ny, int gx, int gy, double2* __restrict__ X) {
  const int bw = 2 * Nx + 1, bh = 2 * Ny + 1, nb = bw * bh;
  const int difX = gx - bw, difY = gy - bh;
  const double inv = 1.0 / ((double)Lx * Ly);
  const size_t total = (size_t)nk * nb;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i / nb), f = (int)(i - (size_t)k * nb);
    const int yy = f / bw, xx = f - yy * bw;  // y + Ny, x + Nx
    const float2 h = H[i];
    const double2 m = spec(D, Lx, Ly, xx - Nx, yy - Ny, inv);
    const double hr = h.x, hi = h.y;
    X[(size_t)k * gx * gy + (size_t)(difY + yy) * gx + difX + xx] =
        make_double2(hr * m.x - hi * m.y, hr * m.y + hi * m.x);
  }
}

// acc[i] = sum_k lam_k |E_k[i]|^2 in kernel order (klitho_socs.cpp:227-230)
__global__ void k_socs_accumulate(const double2* __restrict__ E, const float* __restrict__ lam, int nk,
                                  size_t ng, double* __restrict__ acc) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < ng; i += (size_t)gridDim.x * blockDim.x) {
    double a = 0.0;
    for (int k = 0; k < nk; ++k) {
      const double2 e = E[(size_t)k * ng + i];
      a += (double)lam[k] * (e.x * e.x + e.y * e.y);
    }
    acc[i] = a;
  }
}

// myShift(g/2) of the accumulator (klitho_socs.cpp:233) then FI's own
// myShift((g+1)/2) (:166), as one complex array for the DFT
__global__ void k_fi_load(const double* __restrict__ acc, int gx, int gy, double2* __restrict__ out) {
  const int ax = gx / 2 + (gx + 1) / 2, ay = gy / 2 + (gy + 1) / 2;  // total shift
  const size_t n = (size_t)gx * gy;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / gx), x = (int)(i - (size_t)y * gx);
    const int ys = ((y - ay) % gy + gy) % gy, xs = ((x - ax) % gx + gx) % gx;
    out[i] = make_double2(acc[(size_t)ys * gx + xs], 0.0);
  }
}

// Full L x L spectrum Z from a half-plane spectrum h(kx >= 0, ky) given as a
// function; negative kx by Hermitian symmetry, the kx = 0 column symmetrised
// (what a complex-to-real transform of the half plane computes).
// FI (klitho_socs.cpp:174-183): h(kx, ky) = A[ky mod g][kx], |kx|, |ky| <= g/2.
__global__ void k_fi_spectrum(const double2* __restrict__ A, int gx, int gy, int Lx, int Ly,
                              double2* __restrict__ Z) {
  const int hx = gx / 2, hy = gy / 2;
  const size_t n = (size_t)(2 * hx + 1) * (2 * hy + 1);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int ky = (int)(i / (2 * hx + 1)) - hy, kx = (int)(i % (2 * hx + 1)) - hx;
    double2 v;
    if (kx > 0) {
      v = A[(size_t)((ky + gy) % gy) * gx + kx];
    } else if (kx < 0) {
      const double2 u = A[(size_t)((-ky + gy) % gy) * gx - kx];
      v = make_double2(u.x, -u.y);
    } else {
      const double2 u = A[(size_t)((ky + gy) % gy) * gx], c = A[(size_t)((-ky + gy) % gy) * gx];
      v = make_double2(0.5 * (u.x + c.x), 0.5 * (u.y - c.y));
    }
    Z[(size_t)((ky + Ly) % Ly) * Lx + (kx + Lx) % Lx] = v;
  }
}

// calcImage (klitho_tcc.cpp:269-290): half-plane Hopkins spectrum,
// h(nx2, ny2) = sum_f1 M(f1 + f2) conj(M(f1)) TCC(f1, f1 + f2), then the
// full spectrum as in k_fi_spectrum
__global__ void k_hopkins_half(const double2* __restrict__ D, int Lx, int Ly, const double2* __restrict__ tcc,
                               int N, int Nx, int Ny, double2* __restrict__ half) {
  const int bw = 2 * Nx + 1, tch = (N - 1) / 2;
  const int nxs = 2 * Nx + 1, nys = 4 * Ny + 1;
  const double inv = 1.0 / ((double)Lx * Ly);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nxs * nys; i += gridDim.x * blockDim.x) {
    const int nx2 = i % nxs, ny2 = i / nxs - 2 * Ny;
    double vr = 0.0, vi = 0.0;
    for (int ny1 = -Ny; ny1 <= Ny; ++ny1) {
      if (abs(ny2 + ny1) > Ny) continue;
      for (int nx1 = -Nx; nx1 <= Nx; ++nx1) {
        if (abs(nx2 + nx1) > Nx) continue;
        const double2 a = spec(D, Lx, Ly, nx2 + nx1, ny2 + ny1, inv);
        const double2 b = spec(D, Lx, Ly, nx1, ny1, inv);
        const double2 t = tcc[(size_t)(ny1 * bw + nx1 + tch) * N + (size_t)((ny2 + ny1) * bw + (nx2 + nx1) + tch)];
        const double pr = a.x * b.x + a.y * b.y, pi = a.y * b.x - a.x * b.y;
        vr += pr * t.x - pi * t.y;
        vi += pr * t.y + pi * t.x;
      }
    }
    half[i] = make_double2(vr, vi);
  }
}

__global__ void k_hopkins_spectrum(const double2* __restrict__ half, int Nx, int Ny, int Lx, int Ly,
                                   double2* __restrict__ Z) {
  const int nxs = 2 * Nx + 1, hy = 2 * Ny;
  const int wx = 4 * Nx + 1, wy = 4 * Ny + 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < wx * wy; i += gridDim.x * blockDim.x) {
    const int kx = i % wx - 2 * Nx, ky = i / wx - hy;
    double2 v;
    if (kx > 0) {
      v = half[(ky + hy) * nxs + kx];
    } else if (kx < 0) {
      const double2 u = half[(-ky + hy) * nxs - kx];
      v = make_double2(u.x, -u.y);
    } else {
      const double2 u = half[(ky + hy) * nxs], c = half[(-ky + hy) * nxs];
      v = make_double2(0.5 * (u.x + c.x), 0.5 * (u.y - c.y));
    }
    Z[(size_t)((ky + Ly) % Ly) * Lx + (kx + Lx) % Lx] = v;
  }
}

// image[y][x] = Re z[(y - yh) mod Ly][(x - xh) mod Lx] (FT_c2r's final myShift)
__global__ void k_store_image(const double2* __restrict__ z, int Lx, int Ly, double* __restrict__ img) {
  const int xh = (Lx + 1) / 2, yh = (Ly + 1) / 2;
  const size_t n = (size_t)Lx * Ly;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / Lx), x = (int)(i - (size_t)y * Lx);
    img[i] = z[(size_t)((y - yh + Ly) % Ly) * Lx + (x - xh + Lx) % Lx].x;
  }
}

// Adjoint of the resist loss L = sum (sigmoid(alpha (I - thr)) - t)^2:
// G = dL/dI = 2 (s - t) s (1 - s) alpha; loss summed per clip (double atomics)
__global__ void k_resist_grad(const double* __restrict__ I, const float* __restrict__ t, size_t n, double alpha,
                              double thr, double* __restrict__ G, double* __restrict__ loss) {
  double part = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double sg = 1.0 / (1.0 + exp(-alpha * (I[i] - thr)));
    const double d = sg - (double)t[i];
    part += d * d;
    G[i] = 2.0 * d * sg * (1.0 - sg) * alpha;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w];
    atomicAdd(loss, v);
  }
}

// the image-space gradient at the unshifted (pre-myShift) positions, as complex:
// g[z] = G[(z + yh) mod Ly][(x + xh) mod Lx]
__global__ void k_unshift_load(const double* __restrict__ G, int Lx, int Ly, double2* __restrict__ d) {
  const int xh = (Lx + 1) / 2, yh = (Ly + 1) / 2;
  const size_t n = (size_t)Lx * Ly;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / Lx), x = (int)(i - (size_t)y * Lx);
    d[i] = make_double2(G[(size_t)((y + yh) % Ly) * Lx + (x + xh) % Lx], 0.0);
  }
}

// Y[ky mod g][kx mod g] = ghat(kx, ky) for |kx| <= gx/2, |ky| <= gy/2 (ghat natural order, L x L)
__global__ void k_band_to_grid(const double2* __restrict__ ghat, int Lx, int Ly, int gx, int gy,
                               double2* __restrict__ Y) {
  const int hx = gx / 2, hy = gy / 2;
  const size_t n = (size_t)gx * gy;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int u = (int)(i / gx), v = (int)(i - (size_t)u * gx);
    const int ky = u <= hy ? u : u - gy, kx = v <= hx ? v : v - gx;
    Y[i] = ghat[(size_t)((ky + Ly) % Ly) * Lx + (kx + Lx) % Lx];
  }
}

// Ebar_k = 2 lam_k Re(abar) E_k  (dL/dE_k from acc = sum_k lam_k |E_k|^2)
__global__ void k_field_adjoint(const double2* __restrict__ abar, const double2* __restrict__ E,
                                const float* __restrict__ lam, int nk, size_t ng, double2* __restrict__ Eb) {
  const size_t total = (size_t)nk * ng;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(i / ng);
    const double f = 2.0 * (double)lam[k] * abar[i - (size_t)k * ng].x;
    const double2 e = E[i];
    Eb[i] = make_double2(f * e.x, f * e.y);
  }
}

// Mbar(f) = sum_k conj(H_k(f)) Xbar_k(f) on the band, into the L x L array D
// (natural order, zero elsewhere)
__global__ void k_spectrum_adjoint(const double2* __restrict__ Xb, const float2* __restrict__ H, int nk, int Nx,
                                   int Ny, int gx, int gy, int Lx, int Ly, double2* __restrict__ D) {
  const int bw = 2 * Nx + 1, bh = 2 * Ny + 1, nb = bw * bh;
  const int difX = gx - bw, difY = gy - bh;
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nb; f += gridDim.x * blockDim.x) {
    const int yy = f / bw, xx = f - yy * bw;
    const size_t gi = (size_t)(difY + yy) * gx + difX + xx;
    double re = 0.0, im = 0.0;
    for (int k = 0; k < nk; ++k) {
      const float2 h = H[(size_t)k * nb + f];
      const double2 x = Xb[(size_t)k * gx * gy + gi];
      re += (double)h.x * x.x + (double)h.y * x.y;  // conj(h) x
      im += (double)h.x * x.y - (double)h.y * x.x;
    }
    D[(size_t)((yy - Ny + Ly) % Ly) * Lx + (xx - Nx + Lx) % Lx] = make_double2(re, im);
  }
}

// dL/dmask[y][x] = Re z[(y + yh) mod Ly][(x + xh) mod Lx] / (Lx Ly)
__global__ void k_store_grad(const double2* __restrict__ z, int Lx, int Ly, double* __restrict__ grad) {
  const int xh = (Lx + 1) / 2, yh = (Ly + 1) / 2;
  const double inv = 1.0 / ((double)Lx * Ly);
  const size_t n = (size_t)Lx * Ly;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / Lx), x = (int)(i - (size_t)y * Lx);
    grad[i] = z[(size_t)((y + yh) % Ly) * Lx + (x + xh) % Lx].x * inv;
  }
}

// FT_r2c's centred, 1/(Lx Ly)-scaled layout: out[y][x] = M^(x - Lx/2, y - Ly/2)
__global__ void k_centre(const double2* __restrict__ D, int Lx, int Ly, double2* __restrict__ out) {
  const double inv = 1.0 / ((double)Lx * Ly);
  const size_t n = (size_t)Lx * Ly;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int y = (int)(i / Lx), x = (int)(i - (size_t)y * Lx);
    out[i] = spec(D, Lx, Ly, x - Lx / 2, y - Ly / 2, inv);
  }
}

int ilog2_exact(int n) {
  int m = 0;
  while ((1 << m) < n) ++m;
  return (1 << m) == n ? m : -1;
}

unsigned grid_for(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

}  // namespace

// Device scratch of the FP64 path for one clip at a time.
struct Fp64Work {
  int Lx = 0, Ly = 0, gx = 0, gy = 0, nk = 0;
  double2 *D = nullptr, *T = nullptr, *wx = nullptr, *wy = nullptr;  // L^2 data, transpose, twiddles
  double2 *X = nullptr, *E = nullptr, *wg = nullptr, *wgy = nullptr;  // K g^2 fields, grid twiddles
  double* acc = nullptr;
  double2* Y = nullptr;               // adjoint: 2 g^2 (band of dL/dI, scratch)
  double *I = nullptr, *G = nullptr;  // adjoint: image and dL/dI, L^2
  cudaStream_t st = nullptr;
  std::vector<void*> owned;
  ~Fp64Work() {
    for (void* v : owned) scratch_free(v, st);
  }
};

namespace {

int alloc(Fp64Work& w, void** p, size_t bytes, const char* what) {
  const int rc = scratch_alloc(p, bytes, w.st, what);
  if (!rc) w.owned.push_back(*p);
  return rc;
}

int fft_rows(double2* d, int nrows, int n, const double2* w, int sign, double scale, cudaStream_t st) {
  const int m = ilog2_exact(n);
  const size_t sm = sizeof(double2) * (size_t)n;
  if (sm > 48 * 1024)
    KL_CUDA_TRY(cudaFuncSetAttribute(k_fft_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_fft_rows<<<nrows, kFftThreads, sm, st>>>(d, n, m, w, sign, scale);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

int transpose(const double2* in, double2* out, int rows, int cols, int nb, cudaStream_t st) {
  k_transpose<<<dim3((cols + 31) / 32, (rows + 31) / 32, nb), dim3(32, 8), 0, st>>>(in, out, rows, cols);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

// 2D FFT of the Ly x Lx array w.D (natural order in and out), T scratch
int fft2(Fp64Work& w, int sign, cudaStream_t st) {
  int rc;
  if ((rc = fft_rows(w.D, w.Ly, w.Lx, w.wx, sign, 1.0, st))) return rc;
  if ((rc = transpose(w.D, w.T, w.Ly, w.Lx, 1, st))) return rc;
  if ((rc = fft_rows(w.T, w.Lx, w.Ly, w.wy, sign, 1.0, st))) return rc;
  return transpose(w.T, w.D, w.Lx, w.Ly, 1, st);
}

// 2D DFT of nb arrays gy x gx (natural order), in -> out, tmp scratch (tmp
// may be in; out must differ from both)
int dft2(const double2* in, double2* out, double2* tmp, int gx, int gy, int nb, const double2* wgx,
         const double2* wgy, int sign, double scale, cudaStream_t st) {
  k_dft_rows<<<grid_for((size_t)nb * gy * gx), 256, 0, st>>>(in, out, gx, nb * gy, wgx, sign, 1.0);
  KL_CUDA_TRY(cudaGetLastError());
  int rc;
  if ((rc = transpose(out, tmp, gy, gx, nb, st))) return rc;
  k_dft_rows<<<grid_for((size_t)nb * gy * gx), 256, 0, st>>>(tmp, out, gy, nb * gx, wgy, sign, scale);
  KL_CUDA_TRY(cudaGetLastError());
  if ((rc = transpose(out, tmp, gx, gy, nb, st))) return rc;
  KL_CUDA_TRY(cudaMemcpyAsync(out, tmp, sizeof(double2) * (size_t)nb * gx * gy, cudaMemcpyDeviceToDevice, st));
  return KL_OK;
}

int prepare(Fp64Work& w, int Lx, int Ly, int gx, int gy, int nk, cudaStream_t st) {
  KL_CHECK_ARG(ilog2_exact(Lx) > 0 && ilog2_exact(Ly) > 0 && ilog2_exact(Lx) <= kMaxFftLog2 &&
                   ilog2_exact(Ly) <= kMaxFftLog2,
               "FP64 path: Lx and Ly must be powers of two in [2, 8192]");
  w.st = st;
  w.Lx = Lx;
  w.Ly = Ly;
  w.gx = gx;
  w.gy = gy;
  w.nk = nk;
  const size_t nL = (size_t)Lx * Ly;
  int rc;
  if ((rc = alloc(w, (void**)&w.D, sizeof(double2) * nL, "spectrum")) ||
      (rc = alloc(w, (void**)&w.T, sizeof(double2) * nL, "transpose")) ||
      (rc = alloc(w, (void**)&w.wx, sizeof(double2) * Lx, "twiddles")) ||
      (rc = alloc(w, (void**)&w.wy, sizeof(double2) * Ly, "twiddles")))
    return rc;
  k_twiddle<<<(Lx + 255) / 256, 256, 0, st>>>(w.wx, Lx);
  k_twiddle<<<(Ly + 255) / 256, 256, 0, st>>>(w.wy, Ly);
  KL_CUDA_TRY(cudaGetLastError());
  if (gx > 0) {
    const size_t ng = (size_t)gx * gy, nb = std::max(nk, 3);  // >= 3: FI uses three slots
    if ((rc = alloc(w, (void**)&w.X, sizeof(double2) * ng * nb, "fields")) ||
        (rc = alloc(w, (void**)&w.E, sizeof(double2) * ng * nb, "fields")) ||
        (rc = alloc(w, (void**)&w.wg, sizeof(double2) * gx, "grid twiddles")) ||
        (rc = alloc(w, (void**)&w.wgy, sizeof(double2) * gy, "grid twiddles")) ||
        (rc = alloc(w, (void**)&w.acc, sizeof(double) * ng, "accumulator")))
      return rc;
    k_twiddle<<<(gx + 255) / 256, 256, 0, st>>>(w.wg, gx);
    k_twiddle<<<(gy + 255) / 256, 256, 0, st>>>(w.wgy, gy);
    KL_CUDA_TRY(cudaGetLastError());
  }
  return KL_OK;
}

// FT_r2c of one mask into w.D (natural-order unscaled DFT of the shifted mask)
int mask_dft(Fp64Work& w, const float* mask, cudaStream_t st) {
  const size_t nL = (size_t)w.Lx * w.Ly;
  k_load_shifted<<<grid_for(nL), 256, 0, st>>>(mask, w.Lx, w.Ly, w.D);
  KL_CUDA_TRY(cudaGetLastError());
  return fft2(w, -1, st);
}

// image = FT_c2r-style inverse of the full spectrum already in w.D
int image_from_spectrum(Fp64Work& w, double* img, cudaStream_t st) {
  int rc = fft2(w, +1, st);
  if (rc) return rc;
  k_store_image<<<grid_for((size_t)w.Lx * w.Ly), 256, 0, st>>>(w.D, w.Lx, w.Ly, img);
  KL_CUDA_TRY(cudaGetLastError());
  return KL_OK;
}

}  // namespace

namespace {

// image (double, L x L) of one clip; leaves the K fields in w.E and the mask
// DFT overwritten
int socs_clip(Fp64Work& w, const float* mask, int Nx, int Ny, const float2* H, const float* lam, int nk,
              double* image, cudaStream_t st) {
  const int Lx = w.Lx, Ly = w.Ly, gx = w.gx, gy = w.gy;
  const size_t ng = (size_t)gx * gy, nL = (size_t)Lx * Ly;
  const int nb = (2 * Nx + 1) * (2 * Ny + 1);
  int rc;
  if ((rc = mask_dft(w, mask, st))) return rc;
  KL_CUDA_TRY(cudaMemsetAsync(w.X, 0, sizeof(double2) * ng * nk, st));
  k_socs_embed<<<grid_for((size_t)nk * nb), 256, 0, st>>>(w.D, Lx, Ly, H, nk, Nx, Ny, gx, gy, w.X);
  KL_CUDA_TRY(cudaGetLastError());
  // K backward FFTs of the g x g grid, unnormalised (klitho_socs.cpp:226)
  if ((rc = dft2(w.X, w.E, w.X, gx, gy, nk, w.wg, w.wgy, +1, 1.0, st))) return rc;
  k_socs_accumulate<<<grid_for(ng), 256, 0, st>>>(w.E, lam, nk, ng, w.acc);
  KL_CUDA_TRY(cudaGetLastError());
  // FI: shift, r2c / g^2, band copy into the L x L spectrum, c2r, shift
  k_fi_load<<<grid_for(ng), 256, 0, st>>>(w.acc, gx, gy, w.X);
  KL_CUDA_TRY(cudaGetLastError());
  if ((rc = dft2(w.X, w.X + 2 * ng, w.X + ng, gx, gy, 1, w.wg, w.wgy, -1, 1.0 / (double)ng, st))) return rc;
  KL_CUDA_TRY(cudaMemsetAsync(w.D, 0, sizeof(double2) * nL, st));
  k_fi_spectrum<<<grid_for(ng), 256, 0, st>>>(w.X + 2 * ng, gx, gy, Lx, Ly, w.D);
  KL_CUDA_TRY(cudaGetLastError());
  return image_from_spectrum(w, image, st);
}

int check_socs_args(int Lx, int Ly, int Nx, int Ny, int nk, const char* who) {
  KL_CHECK_ARG(nk > 0 && Nx >= 0 && Ny >= 0 && 4 * Nx + 1 <= Lx && 4 * Ny + 1 <= Ly,
               std::string(who) + ": the SOCS grid (4N+1) must fit in the clip");
  return KL_OK;
}

}  // namespace

int socs_forward(const float* masks, int nclips, int Lx, int Ly, int Nx, int Ny, const float2* H,
                 const float* lam, int nk, double* images, cudaStream_t st) {
  KL_CHECK_ARG(masks && images && H && lam && nclips >= 0, "kl_fp64_socs_forward: NULL argument");
  int rc = check_socs_args(Lx, Ly, Nx, Ny, nk, "kl_fp64_socs_forward");
  if (rc) return rc;
  Fp64Work w;
  if ((rc = prepare(w, Lx, Ly, 4 * Nx + 1, 4 * Ny + 1, nk, st))) return rc;
  const size_t nL = (size_t)Lx * Ly;
  for (int c = 0; c < nclips; ++c)
    if ((rc = socs_clip(w, masks + (size_t)c * nL, Nx, Ny, H, lam, nk, images + (size_t)c * nL, st))) return rc;
  return KL_OK;
}

int socs_vjp(const float* masks, const float* targets, int nclips, int Lx, int Ly, int Nx, int Ny,
             const float2* H, const float* lam, int nk, double alpha, double thr, double* images, double* grad,
             double* loss, cudaStream_t st) {
  KL_CHECK_ARG(masks && targets && grad && loss && H && lam && nclips >= 0, "kl_fp64_socs_vjp: NULL argument");
  int rc = check_socs_args(Lx, Ly, Nx, Ny, nk, "kl_fp64_socs_vjp");
  if (rc) return rc;
  const int gx = 4 * Nx + 1, gy = 4 * Ny + 1;
  Fp64Work w;
  if ((rc = prepare(w, Lx, Ly, gx, gy, nk, st))) return rc;
  const size_t ng = (size_t)gx * gy, nL = (size_t)Lx * Ly;
  if ((rc = alloc(w, (void**)&w.Y, sizeof(double2) * 2 * ng, "adjoint grid")) ||
      (rc = alloc(w, (void**)&w.G, sizeof(double) * nL, "dL/dI")) ||
      (!images && (rc = alloc(w, (void**)&w.I, sizeof(double) * nL, "image"))))
    return rc;
  KL_CUDA_TRY(cudaMemsetAsync(loss, 0, sizeof(double) * nclips, st));
  const int nb = (2 * Nx + 1) * (2 * Ny + 1);
  for (int c = 0; c < nclips; ++c) {
    double* I = images ? images + (size_t)c * nL : w.I;
    if ((rc = socs_clip(w, masks + (size_t)c * nL, Nx, Ny, H, lam, nk, I, st))) return rc;
    k_resist_grad<<<grid_for(nL), 256, 0, st>>>(I, targets + (size_t)c * nL, nL, alpha, thr, w.G, loss + c);
    KL_CUDA_TRY(cudaGetLastError());
    // dL/dacc: band of sum_z g[z] e^{+2 pi i k z / L}, then the g-grid DFT / g^2
    k_unshift_load<<<grid_for(nL), 256, 0, st>>>(w.G, Lx, Ly, w.D);
    KL_CUDA_TRY(cudaGetLastError());
    if ((rc = fft2(w, +1, st))) return rc;
    k_band_to_grid<<<grid_for(ng), 256, 0, st>>>(w.D, Lx, Ly, gx, gy, w.Y);
    KL_CUDA_TRY(cudaGetLastError());
    if ((rc = dft2(w.Y, w.Y + ng, w.Y, gx, gy, 1, w.wg, w.wgy, -1, 1.0 / (double)ng, st))) return rc;
    // dL/dE_k, then dL/dX_k = DFT(dL/dE_k) (adjoint of the unnormalised backward FFT)
    k_field_adjoint<<<grid_for((size_t)nk * ng), 256, 0, st>>>(w.Y + ng, w.E, lam, nk, ng, w.X);
    KL_CUDA_TRY(cudaGetLastError());
    if ((rc = dft2(w.X, w.E, w.X, gx, gy, nk, w.wg, w.wgy, -1, 1.0, st))) return rc;
    // dL/dM^ on the band, then the adjoint of FT_r2c: Re IFFT / (Lx Ly), unshifted
    KL_CUDA_TRY(cudaMemsetAsync(w.D, 0, sizeof(double2) * nL, st));
    k_spectrum_adjoint<<<(nb + 127) / 128, 128, 0, st>>>(w.E, H, nk, Nx, Ny, gx, gy, Lx, Ly, w.D);
    KL_CUDA_TRY(cudaGetLastError());
    if ((rc = fft2(w, +1, st))) return rc;
    k_store_grad<<<grid_for(nL), 256, 0, st>>>(w.D, Lx, Ly, grad + (size_t)c * nL);
    KL_CUDA_TRY(cudaGetLastError());
  }
  return KL_OK;
}

int hopkins_image(const float* masks, int nclips, int Lx, int Ly, int Nx, int Ny, const double2* tcc,
                  double* images, cudaStream_t st) {
  KL_CHECK_ARG(masks && images && tcc && nclips >= 0, "kl_fp64_hopkins_image: bad argument");
  KL_CHECK_ARG(4 * Nx + 1 <= Lx && 4 * Ny + 1 <= Ly, "kl_fp64_hopkins_image: band too wide for the clip");
  Fp64Work w;
  int rc = prepare(w, Lx, Ly, 0, 0, 0, st);
  if (rc) return rc;
  const int N = (2 * Nx + 1) * (2 * Ny + 1), nh = (2 * Nx + 1) * (4 * Ny + 1);
  double2* half = nullptr;
  if ((rc = alloc(w, (void**)&half, sizeof(double2) * nh, "Hopkins spectrum"))) return rc;
  const size_t nL = (size_t)Lx * Ly;
  for (int c = 0; c < nclips && !rc; ++c) {
    if ((rc = mask_dft(w, masks + (size_t)c * nL, st))) break;
    k_hopkins_half<<<(nh + 127) / 128, 128, 0, st>>>(w.D, Lx, Ly, tcc, N, Nx, Ny, half);
    if (cudaGetLastError() != cudaSuccess) {
      rc = KL_ERR_CUDA;
      break;
    }
    if (cudaMemsetAsync(w.D, 0, sizeof(double2) * nL, st) != cudaSuccess) {
      rc = KL_ERR_CUDA;
      break;
    }
    const int nz = (4 * Nx + 1) * (4 * Ny + 1);
    k_hopkins_spectrum<<<(nz + 255) / 256, 256, 0, st>>>(half, Nx, Ny, Lx, Ly, w.D);
    if (cudaGetLastError() != cudaSuccess) {
      rc = KL_ERR_CUDA;
      break;
    }
    rc = image_from_spectrum(w, images + (size_t)c * nL, st);
  }
  if (rc == KL_ERR_CUDA) set_error("kl_fp64_hopkins_image: kernel launch failed");
  return rc;
}

int mask_spectrum(const float* mask, int Lx, int Ly, double2* out, cudaStream_t st) {
  KL_CHECK_ARG(mask && out, "kl_fp64_mask_spectrum: NULL argument");
  Fp64Work w;
  int rc = prepare(w, Lx, Ly, 0, 0, 0, st);
  if (rc) return rc;
  if ((rc = mask_dft(w, mask, st))) return rc;
  k_centre<<<grid_for((size_t)Lx * Ly), 256, 0, st>>>(w.D, Lx, Ly, out);
  KL_CUDA_TRY(cudaGetLastError());
  KL_CUDA_TRY(cudaStreamSynchronize(st));
  return KL_OK;
}

}  // namespace f64
}  // namespace kl
