// kl_device.cuh -- device building blocks shared by the SOCS kernels:
// complex helpers, compile-time twiddle tables, register-resident radix-2
// FFTs, a warp-cooperative FFT (four-step: in-register DFT over the high
// index digit, twiddle, 32-point DIF butterflies across lanes by shuffles)
// and a warp reduce-scatter.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace kl {

// ---------------------------------------------------------------------------
// complex float helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// a + b * w
__device__ __forceinline__ float2 cfma(float2 b, float2 w, float2 a) {
  return make_float2(fmaf(b.x, w.x, fmaf(-b.y, w.y, a.x)), fmaf(b.x, w.y, fmaf(b.y, w.x, a.y)));
}
__device__ __forceinline__ float cabs2(float2 a) { return fmaf(a.x, a.x, a.y * a.y); }

// exp(i*2*pi*num/den) with exact argument reduction (num taken mod den in
// integers, then sincospi in double) -- used to fill twiddle tables.
__device__ __forceinline__ float2 expi2pi_frac(long long num, long long den) {
  long long r = num % den;
  if (r < 0) r += den;
  double s, c;
  sincospi(2.0 * (double)r / (double)den, &s, &c);
  return make_float2((float)c, (float)s);
}

// ---------------------------------------------------------------------------
// compile-time twiddles: cos/sin(2*pi*k/256) evaluated by the compiler from a
// Taylor series on the octant-reduced angle, stored in constant memory.
// ---------------------------------------------------------------------------
namespace cx {
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double sin_poly(double x) {
  double x2 = x * x, term = x, sum = x;
  for (int n = 1; n < 14; ++n) {
    term *= -x2 / (double)((2 * n) * (2 * n + 1));
    sum += term;
  }
  return sum;
}
constexpr double cos_poly(double x) {
  double x2 = x * x, term = 1.0, sum = 1.0;
  for (int n = 1; n < 14; ++n) {
    term *= -x2 / (double)((2 * n - 1) * (2 * n));
    sum += term;
  }
  return sum;
}
// angle 2*pi*k/n split as quadrant q and remainder r in [-pi/4, pi/4]
constexpr double cos2pi(long k, long n) {
  long kk = ((k % n) + n) % n;
  long q = (4 * kk + n / 2) / n;  // nearest quadrant (0..4)
  double r = 2.0 * kPi * ((double)(4 * kk - q * n) / (double)(4 * n));
  switch (q & 3) {
    case 0: return cos_poly(r);
    case 1: return -sin_poly(r);
    case 2: return -cos_poly(r);
    default: return sin_poly(r);
  }
}
constexpr double sin2pi(long k, long n) {
  long kk = ((k % n) + n) % n;
  long q = (4 * kk + n / 2) / n;
  double r = 2.0 * kPi * ((double)(4 * kk - q * n) / (double)(4 * n));
  switch (q & 3) {
    case 0: return sin_poly(r);
    case 1: return cos_poly(r);
    case 2: return -sin_poly(r);
    default: return -cos_poly(r);
  }
}
}  // namespace cx

constexpr int kTwN = 256;
struct TwTable {
  float c[kTwN];
  float s[kTwN];
  constexpr TwTable() : c(), s() {
    for (int k = 0; k < kTwN; ++k) {
      c[k] = (float)cx::cos2pi(k, kTwN);
      s[k] = (float)cx::sin2pi(k, kTwN);
    }
  }
};
// e^{+2*pi*i*k/256}; other power-of-two lengths use a stride
__constant__ const TwTable c_tw = TwTable();

// the same table in global memory, for lane-dependent indices (the constant
// cache serialises divergent addresses)
__device__ const TwTable g_twd = TwTable();

// e^{+2*pi*i*num/den} for den a power of two dividing 256
__device__ __forceinline__ float2 expi2pi_pow2(int num, int den) {
  const int idx = (num & (den - 1)) * (kTwN / den);
  return make_float2(g_twd.c[idx], g_twd.s[idx]);
}

// e^{SIGN*2*pi*i*k/N}, k and N compile-time after unrolling
template <int N, int SIGN>
__device__ __forceinline__ float2 tw_const(int k) {
  static_assert(kTwN % N == 0, "twiddle table too short");
  int idx = ((k % N) + N) % N * (kTwN / N);
  return make_float2(c_tw.c[idx], SIGN > 0 ? c_tw.s[idx] : -c_tw.s[idx]);
}

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }
__host__ __device__ constexpr int brevc(int v, int bits) {
  int r = 0;
  for (int i = 0; i < bits; ++i) r |= ((v >> i) & 1) << (bits - 1 - i);
  return r;
}

// ---------------------------------------------------------------------------
// In-register radix-2 DIT FFT of length N (natural order in and out).
// X[k] = sum_n x[n] e^{SIGN 2 pi i k n / N}, unnormalised.
// ---------------------------------------------------------------------------
// one radix-2 stage of butterfly span LEN, then the next (compile-time recursion
// keeps every register index a constant expression)
template <int N, int SIGN, int LEN>
__device__ __forceinline__ void fft_stages(float2 (&a)[N]) {
  if constexpr (LEN <= N) {
#pragma unroll
    for (int i = 0; i < N; i += LEN) {
#pragma unroll
      for (int k = 0; k < LEN / 2; ++k) {
        float2 u = a[i + k];
        float2 v = a[i + k + LEN / 2];
        if (k != 0) v = cmul(v, tw_const<N, SIGN>(k * (N / LEN)));
        a[i + k] = cadd(u, v);
        a[i + k + LEN / 2] = csub(u, v);
      }
    }
    fft_stages<N, SIGN, LEN * 2>(a);
  }
}

template <int N, int SIGN>
__device__ __forceinline__ void fft_reg(float2 (&a)[N]) {
  constexpr int B = ilog2c(N);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const int j = brevc(i, B);
    if (i < j) {
      float2 t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
  fft_stages<N, SIGN, 2>(a);
}

// Real-input DFT of length P (P even, P/2 <= 64): out[k] for k in [0, P/2],
// S[k] = sum_i v[i] e^{-2 pi i k i / P}.  Packs pairs into a P/2 complex FFT.
template <int P>
__device__ __forceinline__ void rdft_reg(const float (&v)[P], float2 (&S)[P / 2 + 1]) {
  constexpr int H = P / 2;
  float2 z[H];
#pragma unroll
  for (int m = 0; m < H; ++m) z[m] = make_float2(v[2 * m], v[2 * m + 1]);
  fft_reg<H, -1>(z);
  // S[k] = (Z[k] + conj Z[H-k])/2 - i e^{-2 pi i k/P} (Z[k] - conj Z[H-k])/2
#pragma unroll
  for (int k = 0; k <= H; ++k) {
    float2 a = z[k % H];
    float2 b = cconj(z[(H - k) % H]);
    float2 ev = cscale(cadd(a, b), 0.5f);
    float2 od = cscale(csub(a, b), 0.5f);
    float2 w = tw_const<P, -1>(k);
    // -i * w * od
    float2 t = cmul(w, od);
    S[k] = make_float2(ev.x + t.y, ev.y - t.x);
  }
}

// Real part of a length-P inverse DFT of arbitrary complex input Z:
// out[i] = Re sum_k Z[k] e^{+2 pi i k i / P}, via one P/2 complex FFT.
template <int P>
__device__ __forceinline__ void re_idft_reg(const float2 (&Z)[P], float (&out)[P]) {
  constexpr int H = P / 2;
  float2 x[H];
#pragma unroll
  for (int k = 0; k < H; ++k) {
    // Hermitian part Zh[k] = (Z[k] + conj Z[-k]) / 2 at k and k + H
    float2 za = cscale(cadd(Z[k], cconj(Z[(P - k) % P])), 0.5f);
    float2 zb = cscale(cadd(Z[k + H], cconj(Z[(P - k - H) % P])), 0.5f);
    float2 ze = cadd(za, zb);
    float2 zo = cmul(csub(za, zb), tw_const<P, +1>(k));
    x[k] = make_float2(ze.x - zo.y, ze.y + zo.x);  // ze + i zo
  }
  fft_reg<H, +1>(x);
#pragma unroll
  for (int m = 0; m < H; ++m) {
    out[2 * m] = x[m].x;
    out[2 * m + 1] = x[m].y;
  }
}

// S[k] = sum_i v[i] e^{-2 pi i k i / P}, k in [0, P/2], any power-of-two P >= 1
template <int P>
__device__ __forceinline__ void rdft_any(const float (&v)[P], float2 (&S)[P / 2 + 1]) {
  if constexpr (P == 1) {
    S[0] = make_float2(v[0], 0.f);
  } else {
    rdft_reg<P>(v, S);
  }
}

// out[i] = Re sum_{k=0}^{P/2} Y[k] e^{+2 pi i k i / P}, where Y holds the
// Hermitian fold of a length-P spectrum Z: Y[0] = Z[0], Y[P/2] = Z[P/2],
// Y[k] = Z[k] + conj Z[P-k] (so out = Re IDFT_P(Z)).  One P/2-point FFT;
// accumulating Y instead of Z halves the registers of a row synthesis.
template <int P>
__device__ __forceinline__ void c2r_half(const float2 (&Y)[P / 2 + 1], float (&out)[P]) {
  if constexpr (P == 1) {
    out[0] = Y[0].x;
  } else {
    constexpr int H = P / 2;
    float2 x[H];
#pragma unroll
    for (int k = 0; k < H; ++k) {
      // F[k] and F[k+H] of the Hermitian spectrum F[k] = Y[k]/2 (0<k<H), F[P-k] = conj F[k]
      const float2 a = k == 0 ? make_float2(Y[0].x, 0.f) : cscale(Y[k], 0.5f);
      const float2 b = k == 0 ? make_float2(Y[H].x, 0.f) : cscale(cconj(Y[H - k]), 0.5f);
      const float2 fe = cadd(a, b);
      const float2 fo = cmul(csub(a, b), tw_const<P, +1>(k));
      x[k] = make_float2(fe.x - fo.y, fe.y + fo.x);
    }
    fft_reg<H, +1>(x);
#pragma unroll
    for (int m = 0; m < H; ++m) {
      out[2 * m] = x[m].x;
      out[2 * m + 1] = x[m].y;
    }
  }
}

// The columns fx = fxs + 32 t (t < kGenMaxFold, fx <= Nx) of band row r of a
// kernel (row-major (2Ny+1) x (2Nx+1), 2Nx+1 <= 128), issued as independent
// loads so that several are in flight at once.
constexpr int kGenMaxFold = 4;
__device__ __forceinline__ void gen_load_hrow(const float2* __restrict__ Hk, int r, int nbx, int Nx, int fxs,
                                              float2 (&h)[kGenMaxFold]) {
  const float2* hr = Hk + (size_t)r * nbx + Nx;
#pragma unroll
  for (int t = 0; t < kGenMaxFold; ++t) {
    const int fx = fxs + 32 * t;
    h[t] = fx <= Nx ? __ldg(hr + fx) : make_float2(0.f, 0.f);
  }
}

// Coefficients b = lane + 32 t (t < 4, b < nbins <= 128) of one row of a
// row-coefficient array, as independent loads.
__device__ __forceinline__ void gen_load_qrow(const float2* __restrict__ qr, int nbins, int lane, float2 (&q)[4]) {
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int b = lane + 32 * t;
    q[t] = b < nbins ? __ldg(qr + b) : make_float2(0.f, 0.f);
  }
}

// ---------------------------------------------------------------------------
// Warp FFT of length N = 32*R.  Input: v[j] = x[lane + 32 j].  Output:
// v[q1] = X[q1 + R * brev5(lane)].  Twiddles are per lane, made once.
// ---------------------------------------------------------------------------
template <int R, int SIGN>
struct WarpFFT {
  float2 tw4[R];   // e^{SIGN 2 pi i q1 lane / (32R)}
  float2 tws[5];   // stage twiddles e^{SIGN 2 pi i (lane mod h) / (2h)}, h = 16..1
  __device__ __forceinline__ void init(int lane) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      float2 e = expi2pi_pow2(q * lane, 32 * R);
      tw4[q] = make_float2(e.x, SIGN > 0 ? e.y : -e.y);
    }
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      int h = 16 >> s;
      float2 e = expi2pi_pow2(lane & (h - 1), 2 * h);
      tws[s] = make_float2(e.x, SIGN > 0 ? e.y : -e.y);
    }
  }
  __device__ __forceinline__ void run(float2 (&v)[R], int lane) const {
    if (R > 1) fft_reg<R, SIGN>(v);
#pragma unroll
    for (int q = 1; q < R; ++q) v[q] = cmul(v[q], tw4[q]);
#pragma unroll
    for (int s = 0; s < 5; ++s) {
      const int h = 16 >> s;
      const bool upper = (lane & h) != 0;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        float ox = __shfl_xor_sync(0xffffffffu, v[q].x, h);
        float oy = __shfl_xor_sync(0xffffffffu, v[q].y, h);
        float2 o = make_float2(ox, oy);
        // lower lane: a + b ; upper lane: (a - b) * w, a = lower value
        float2 r = upper ? cmul(csub(o, v[q]), tws[s]) : cadd(v[q], o);
        v[q] = r;
      }
    }
  }
  // The transpose of run(): input v[q1] = x[q1 + R * brev5(lane)] (the
  // layout run() produces), output v[j] = X[lane + 32 j], the same DFT.  The
  // lane stages run in reverse order as decimation-in-time butterflies
  // (x + w y, x - w y), then the diagonal twiddle, then the register DFT.
  __device__ __forceinline__ void run_rev(float2 (&v)[R], int lane) const {
#pragma unroll
    for (int s = 4; s >= 0; --s) {
      const int h = 16 >> s;
      const bool upper = (lane & h) != 0;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const float2 t = upper ? cmul(v[q], tws[s]) : v[q];
        const float2 o = make_float2(__shfl_xor_sync(0xffffffffu, t.x, h), __shfl_xor_sync(0xffffffffu, t.y, h));
        v[q] = upper ? csub(o, t) : cadd(v[q], o);
      }
    }
#pragma unroll
    for (int q = 1; q < R; ++q) v[q] = cmul(v[q], tw4[q]);
    if (R > 1) fft_reg<R, SIGN>(v);
  }
};

// ---------------------------------------------------------------------------
// Warp reduce-scatter of M floats (M a multiple of 32): on return lane l holds
// the warp sums of indices [l*M/32, (l+1)*M/32) in a[0 .. M/32).
// ---------------------------------------------------------------------------
template <int M>
__device__ __forceinline__ void warp_reduce_scatter(float (&a)[M], int lane) {
  static_assert(M % 32 == 0, "M must be a multiple of 32");
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    const int cnt = M >> (s + 1);
    const bool up = (lane & h) != 0;
#pragma unroll
    for (int i = 0; i < cnt; ++i) {
      float keep = up ? a[i + cnt] : a[i];
      float send = up ? a[i] : a[i + cnt];
      a[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
    }
  }
}

}  // namespace kl
