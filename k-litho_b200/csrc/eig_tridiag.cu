// eig_tridiag.cu -- top-K eigenpairs of a Hermitian B x B matrix (64 <= B <= 256)
// by Householder reduction to tridiagonal form, bisection and inverse
// iteration: the zhetrd + dstebz + dstein route of LAPACK, which the
// reference's zheevr (K-Litho-TCC/klitho_tcc.cpp:300-377) starts from too
// (zheevr finishes with MRRR instead of bisection + inverse iteration).
//
// Five launches per batch of matrices:
//   k_hermitian_tridiag  one thread-block cluster of 8 CTAs per matrix, the
//                        matrix's rows dealt round-robin over the CTAs'
//                        shared memory; B - 2 reflector steps, each a
//                        distributed matvec and a rank-2 update, with the
//                        reflector and the matvec exchanged as st.async
//                        stores completing on the receivers' mbarriers; the
//                        next reflector is formed by the warp that updates
//                        its row as soon as it has
//   k_tridiag_bisect     one CTA per wanted eigenvalue: 256-point multisection
//                        on division-free Sturm counts of the real tridiagonal
//                        D^H T D
//   k_tridiag_invit      one thread per eigenvector: inverse iteration with
//                        the unpivoted L D L^T factorisation of T - lambda I,
//                        Gram-Schmidt against the earlier members of a cluster
//                        of close eigenvalues (clusters run in rounds); the
//                        vectors stay in shared memory when they fit
//   k_tridiag_wy         the compact WY factor T of each block of 8 reflectors
//   k_tridiag_back       one warp per eigenvector: phases, then the reflector
//                        blocks in reverse order, 8 reflectors per round
// Everything is complex / real FP64.  The reduction's exchange waits are
// bounded (2 s): a timeout sets the job's error word instead of spinning.
#include <cooperative_groups.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "kl_internal.h"
#include "kl_tcc.h"

namespace kl {

namespace {

constexpr int kTdCl = 8;            // CTAs per matrix (a portable cluster)
constexpr int kTdThreads = 512;     // threads per CTA of the reduction
constexpr int kTdMaxJobs = 16;      // matrices per launch
constexpr int kTdBisPoints = 256;   // Sturm counts per pass of the bisection (threads per eigenvalue)
constexpr int kTdBackWarps = 8;     // eigenvectors per CTA of the back-transform (threads = kTridiagMaxB)
constexpr int kTdNB = 8;            // reflectors per block of the back-transform
constexpr size_t kTdInvSmemCap = 200 * 1024;  // inverse iteration keeps its vectors on chip up to this
constexpr int kTdInvIters = 2;      // inverse-iteration solves per eigenvector (from a shift exact to a few ulps)
constexpr int kTdChunk = 8;         // elements staged in registers per memory pass
// eigenvalues closer than this multiple of ||T|| are one cluster: their vectors
// are orthogonalised against each other (the others are orthogonal to within
// eps ||T|| / gap by inverse iteration itself)
constexpr double kTdClusterTol = 1e-7;
constexpr double kEps = 2.220446049250313e-16;  // 2^-52
constexpr double kSafeMin = 2.2250738585072014e-308;  // smallest normal double
constexpr unsigned long long kTdWaitNs = 2000000000ull;  // bound on one exchange wait of the reduction

struct TridiagJobs {
  TridiagJob j[kTdMaxJobs];
};

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__host__ __device__ inline int td_rows(int B) { return (B + kTdCl - 1) / kTdCl; }
// shared memory of k_hermitian_tridiag: the CTA's rows, two reflector and two
// matvec buffers (by step parity)
__host__ __device__ inline size_t td_smem(int B) {
  return sizeof(double2) * ((size_t)td_rows(B) * B + 4 * (size_t)B);
}

// bytes one step k of order B delivers into each CTA's reflector (and matvec) buffer
__host__ __device__ inline uint32_t td_step_bytes(int B, int k) { return (uint32_t)(B - k - 1) * 16u; }

__device__ __forceinline__ uint32_t td_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
// address of `p`'s counterpart in the shared memory of CTA `cta` of the cluster
__device__ __forceinline__ uint32_t td_cluster_addr(const void* p, uint32_t cta) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(td_smem_u32(p)), "r"(cta));
  return r;
}
// dst[0] of CTA `cta` <- v; the 16 bytes complete on that CTA's barrier `bar`
__device__ __forceinline__ void td_push(double2* dst, double2 v, uint64_t* bar, uint32_t cta) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(
                   td_cluster_addr(dst, cta)),
               "d"(v.x), "d"(v.y), "r"(td_cluster_addr(bar, cta))
               : "memory");
}// this CTA expects `bytes` on `bar` in the barrier's current phase
__device__ __forceinline__ void td_arm(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(td_smem_u32(bar)), "r"(bytes)
               : "memory");
}
// bounded wait for the phase of `bar` with `parity`; false after kTdWaitNs
__device__ __forceinline__ bool td_wait(uint64_t* bar, uint32_t parity) {
  unsigned long long t0 = 0;
  for (int n = 0;; ++n) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(td_smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (n == 0) t0 = t;
    else if (t - t0 > kTdWaitNs) return false;
  }
}

// ---------------------------------------------------------------------------
// Householder reduction H = Q T Q^H.  Row i of H lives in CTA i % 8 (local row
// i / 8), so the trailing rows stay spread evenly as the reduction proceeds.
// Step k: warp 0 of the CTA holding row k forms v (unit, supported on
// k+1..B-1) with (I - 2 v v^H) x = alpha e_{k+1} for x = column k below the
// diagonal (= conj(row k) right of it) as soon as row k is updated, and sends
// it into every CTA; each CTA, once its copy of v has landed, forms
// p_i = sum_j H[i][j] v_j for its rows i > k and sends them into every CTA;
// once all of p has landed, every CTA updates its rows:
// H -= 2 (v w^H + w v^H), w = p - (v^H p) v.
// The sends are st.async stores that complete their bytes on the receiving
// CTA's mbarrier for that buffer (no cluster barrier per step).  Buffers
// alternate by step parity; a CTA re-arms a buffer's barrier for step k + 2
// as soon as its step-k data has landed, and the data of step k + 2 can only
// be sent after every CTA has finished step k (it depends on all of step
// k + 1's matvec), so no byte reaches an unarmed phase and no buffer is
// overwritten while it is read.  Waits are bounded; a CTA that gives up
// raises the job's error word and leaves the loop, and its peers then give
// up on their next wait.
// Outputs d[k] = T[k][k], e[k] = T[k+1][k] = alpha_k, and v_k in refl row k.
// ---------------------------------------------------------------------------
// the reflector of step k, by one warp of the CTA holding row k (hk, already
// updated through step k - 1): v into vdst of every CTA of the cluster (bytes
// on vbar) and row k of refl; d[k] and e[k] = alpha
__device__ __forceinline__ void td_reflector(const TridiagJob& job, const double2* hk, double2* vdst,
                                             uint64_t* vbar, int k, int lane, bool send) {
  const int B = job.B, j0 = k + 1;
  double s2a = 0.0, s2b = 0.0;  // two partial sums: half the FP64 dependency chain
  for (int j = j0 + lane; j < B; j += 64) {
    const double2 h = hk[j];
    s2a += fma(h.x, h.x, h.y * h.y);
    if (j + 32 < B) {
      const double2 g = hk[j + 32];
      s2b += fma(g.x, g.x, g.y * g.y);
    }
  }
  const double s2 = warp_sum(s2a + s2b);
  const double2 x0 = make_double2(hk[j0].x, -hk[j0].y);
  const double ax0 = sqrt(x0.x * x0.x + x0.y * x0.y), nx = sqrt(s2);
  double2 alpha = make_double2(0.0, 0.0);
  double sc = 0.0;
  if (nx > 0.0) {
    const double2 ph = ax0 > 0.0 ? make_double2(x0.x / ax0, x0.y / ax0) : make_double2(1.0, 0.0);
    alpha = make_double2(-ph.x * nx, -ph.y * nx);
    sc = 1.0 / sqrt(2.0 * nx * (nx + ax0));  // 1 / ||x - alpha e||
  }
  for (int j = j0 + lane; j < B; j += 32) {
    double2 x = make_double2(hk[j].x, -hk[j].y);
    if (j == j0) x = make_double2(x.x - alpha.x, x.y - alpha.y);
    const double2 vj = make_double2(x.x * sc, x.y * sc);
    job.refl[(size_t)k * B + j] = vj;
    if (send)
#pragma unroll
      for (int c = 0; c < kTdCl; ++c) td_push(vdst + j, vj, vbar, (uint32_t)c);
  }
  if (lane == 0) {
    job.d[k] = hk[k].x;
    job.e[k] = alpha;
  }
}

__global__ void __cluster_dims__(kTdCl, 1, 1) __launch_bounds__(kTdThreads, 1)
    k_hermitian_tridiag(TridiagJobs jobs) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char tsm[];
  __shared__ __align__(8) uint64_t s_vbar[2], s_pbar[2];
  __shared__ int s_fail;
  const int me = (int)cl.block_rank();
  const TridiagJob job = jobs.j[blockIdx.x / kTdCl];
  const int B = job.B, R = td_rows(B), nsteps = B - 2;
  double2* rows = reinterpret_cast<double2*>(tsm);  // R x B
  double2* vbuf = rows + (size_t)R * B;             // 2 x B (by step parity)
  double2* pbuf = vbuf + 2 * (size_t)B;             // 2 x B
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = kTdThreads / 32;
  const double2 zero = make_double2(0.0, 0.0);
  for (int x = tid; x < R * B; x += kTdThreads) {
    const int l = x / B, j = x - l * B, i = kTdCl * l + me;
    rows[x] = i < B ? job.H[(size_t)i * B + j] : zero;
  }
  if (tid == 0) {
    for (int b = 0; b < 2; ++b) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(td_smem_u32(&s_vbar[b])), "r"(1) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(td_smem_u32(&s_pbar[b])), "r"(1) : "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int k = 0; k < 2 && k < nsteps; ++k) {
      td_arm(&s_vbar[k], td_step_bytes(B, k));
      td_arm(&s_pbar[k], td_step_bytes(B, k));
    }
    s_fail = 0;
  }
  cl.sync();  // every CTA's barriers are armed before the first bytes are sent
  bool fail = false;
  if (nsteps > 0 && me == 0 && warp == 0) td_reflector(job, rows, vbuf, &s_vbar[0], 0, lane, true);
  for (int k = 0; k < nsteps; ++k) {
    const int par = k & 1;
    const uint32_t ph = (uint32_t)((k >> 1) & 1);
    const double2* v = vbuf + (size_t)par * B;
    double2* pb = pbuf + (size_t)par * B;
    // v of step k has landed, and every row of this CTA is updated through step k - 1
    fail = !td_wait(&s_vbar[par], ph);
    if (__syncthreads_or(fail)) break;
    if (tid == 0 && k + 2 < nsteps) td_arm(&s_vbar[par], td_step_bytes(B, k + 2));
    const int j0 = k + 1;
    const int lfirst = k < me ? 0 : (k - me) / kTdCl + 1;  // first local row below row k
    for (int l = lfirst + warp; l < R; l += nwarp) {
      const int i = kTdCl * l + me;
      if (i >= B) break;
      const double2* hr = rows + (size_t)l * B;
      double ax = 0.0, ay = 0.0, bx = 0.0, by = 0.0;  // two partial sums per part
      for (int j = j0 + lane; j < B; j += 64) {
        const double2 h = hr[j], vj = v[j];
        ax += fma(h.x, vj.x, -h.y * vj.y);
        ay += fma(h.x, vj.y, h.y * vj.x);
        if (j + 32 < B) {
          const double2 g = hr[j + 32], wj = v[j + 32];
          bx += fma(g.x, wj.x, -g.y * wj.y);
          by += fma(g.x, wj.y, g.y * wj.x);
        }
      }
      ax = warp_sum(ax + bx);
      ay = warp_sum(ay + by);
      if (lane < kTdCl && !s_fail) td_push(pb + i, make_double2(ax, ay), &s_pbar[par], (uint32_t)lane);
    }
    // all of p has landed
    fail = !td_wait(&s_pbar[par], ph);
    if (__syncthreads_or(fail)) break;
    if (tid == 0 && k + 2 < nsteps) td_arm(&s_pbar[par], td_step_bytes(B, k + 2));
    // c = Re(v^H p), the same sum in every warp
    double ca = 0.0, cb = 0.0;
    for (int j = j0 + lane; j < B; j += 64) {
      const double2 a = v[j], b = pb[j];
      ca += fma(a.x, b.x, a.y * b.y);
      if (j + 32 < B) {
        const double2 a2 = v[j + 32], b2 = pb[j + 32];
        cb += fma(a2.x, b2.x, a2.y * b2.y);
      }
    }
    const double c = warp_sum(ca + cb);
    // row k + 1 is the first row below k of its CTA, so warp 0 there updates it
    // first and then forms and sends the next step's reflector at once
    const bool next = k + 1 < nsteps && me == (k + 1) % kTdCl;
    for (int l = lfirst + warp; l < R; l += nwarp) {
      const int i = kTdCl * l + me;
      if (i >= B) break;
      double2* hr = rows + (size_t)l * B;
      const double2 vi = v[i], pi = pb[i];
      // 2 v_i and 2 w_i
      const double2 v2 = make_double2(2.0 * vi.x, 2.0 * vi.y);
      const double2 w2 = make_double2(2.0 * (pi.x - c * vi.x), 2.0 * (pi.y - c * vi.y));
      for (int j = j0 + lane; j < B; j += 32) {
        const double2 vj = v[j], pj = pb[j];
        const double2 wj = make_double2(pj.x - c * vj.x, pj.y - c * vj.y);
        double2 h = hr[j];
        // h -= 2 v_i conj(w_j) + 2 w_i conj(v_j)
        h.x -= fma(v2.x, wj.x, fma(v2.y, wj.y, fma(w2.x, vj.x, w2.y * vj.y)));
        h.y -= fma(v2.y, wj.x, fma(-v2.x, wj.y, fma(w2.y, vj.x, -w2.x * vj.y)));
        hr[j] = h;
      }
      if (next && l == lfirst) {
        __syncwarp();
        td_reflector(job, hr, vbuf + (size_t)(par ^ 1) * B, &s_vbar[par ^ 1], k + 1, lane, !s_fail);
      }
    }
    __syncthreads();  // the rows are updated before the next step's matvec reads them
  }
  if (fail && tid == 0) {
    if (job.err) atomicExch(job.err, 41);
    for (int c = 0; c < kTdCl; ++c) *cl.map_shared_rank(&s_fail, c) = 1;  // peers stop sending
  }
  __syncthreads();
  // the trailing 2 x 2 block (or the 1 x 1 matrix)
  if (tid == 0) {
    for (int i = B >= 2 ? B - 2 : 0; i < B; ++i) {
      if (i % kTdCl != me) continue;
      const double2* hr = rows + (size_t)(i / kTdCl) * B;
      job.d[i] = hr[i].x;
      if (i + 1 < B) job.e[i] = make_double2(hr[i + 1].x, -hr[i + 1].y);  // T[i+1][i] = conj(H[i][i+1])
    }
  }
  cl.sync();  // no CTA leaves while a peer may still address its shared memory
}

// Sturm count of the real tridiagonal: the number of eigenvalues below x, as
// the sign changes along p_0 = 1, p_i = (d_{i-1} - x) p_{i-1} - e2_{i-2} p_{i-2}
// (the characteristic polynomials of the leading submatrices; Sturm's theorem).
// d and e2 = |e|^2 come scaled by powers of two so that ||T|| is near 1; the
// pair (p_{i-1}, p_i) is rescaled by a power of two every 4 steps, which keeps
// it in range (a step grows it by at most ~3) and changes no sign.  A zero
// takes the sign opposite to its predecessor.  One FMA per step on the
// dependency chain (the ratio form q_i = p_i / p_{i-1} needs a division).
__device__ __forceinline__ int sturm_count(const double* d, const double* e2, int B, double x) {
  double pm = 1.0, p = d[0] - x;
  int neg = p < 0.0 || p == 0.0;  // sign of p_1 (a zero counts as negative after p_0 = 1)
  int c = neg;
  int i = 1;
  // four steps per pass, their table entries loaded ahead of the chain
  for (; i + 3 < B; i += 4) {
    double dx[4], ee[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      dx[u] = d[i + u] - x;
      ee[u] = e2[i + u - 1];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const double pn = fma(dx[u], p, -ee[u] * pm);
      pm = p;
      p = pn;
      const int n = p < 0.0 || (p == 0.0 && !neg);
      c += n != neg;
      neg = n;
    }
    const double a = fabs(p);
    if (a > 0x1p400 || (a < 0x1p-400 && a > 0.0)) {
      const double s = scalbn(1.0, -ilogb(a));
      p *= s;
      pm *= s;
    }
  }
  for (; i < B; ++i) {
    const double pn = fma(d[i] - x, p, -e2[i - 1] * pm);
    pm = p;
    p = pn;
    const int n = p < 0.0 || (p == 0.0 && !neg);
    c += n != neg;
    neg = n;
  }
  return c;
}

// w[j] = the j-th largest eigenvalue, one CTA each: its threads count at
// kTdBisPoints points splitting the interval into kTdBisPoints + 1 parts, and
// the interval shrinks to the part holding eigenvalue B - 1 - j (ascending)
// until it is a few ulps wide (7 passes from the Gershgorin interval).
__global__ void __launch_bounds__(kTdBisPoints) k_tridiag_bisect(TridiagJobs jobs) {
  const TridiagJob job = jobs.j[blockIdx.y];
  const int B = job.B, j = blockIdx.x, tid = threadIdx.x;
  if (j >= job.K) return;  // the whole CTA
  __shared__ double s_d[kTridiagMaxB], s_e2[kTridiagMaxB];
  __shared__ double s_lo[kTdBisPoints / 32], s_hi[kTdBisPoints / 32];
  // Gershgorin interval and the norm scale
  double lo = 1e300, hi = -1e300;
  for (int i = tid; i < B; i += blockDim.x) {
    const double2 e = i + 1 < B ? job.e[i] : make_double2(0.0, 0.0);
    const double2 f = i > 0 ? job.e[i - 1] : make_double2(0.0, 0.0);
    const double r = sqrt(e.x * e.x + e.y * e.y) + sqrt(f.x * f.x + f.y * f.y), di = job.d[i];
    lo = fmin(lo, di - r);
    hi = fmax(hi, di + r);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((tid & 31) == 0) {
    s_lo[tid >> 5] = lo;
    s_hi[tid >> 5] = hi;
  }
  __syncthreads();
  for (int w = 0; w < (int)blockDim.x / 32; ++w) {
    lo = fmin(lo, s_lo[w]);
    hi = fmax(hi, s_hi[w]);
  }
  const double tn = fmax(fabs(lo), fabs(hi));
  if (!(tn > 0.0)) {  // the zero matrix
    if (tid == 0) job.w[j] = 0.0;
    return;
  }
  const double sc = scalbn(1.0, -ilogb(tn)), isc = scalbn(1.0, ilogb(tn));  // exact powers of two
  for (int i = tid; i < B; i += blockDim.x) {
    const double2 e = i + 1 < B ? job.e[i] : make_double2(0.0, 0.0);
    s_d[i] = job.d[i] * sc;
    s_e2[i] = (e.x * sc) * (e.x * sc) + (e.y * sc) * (e.y * sc);
  }
  __syncthreads();
  const double tns = tn * sc;
  lo = lo * sc - 4.0 * kEps * tns;
  hi = hi * sc + 4.0 * kEps * tns;
  const int m = B - 1 - j;
  constexpr double kStep = 1.0 / (kTdBisPoints + 1);
  for (int it = 0; it < 64; ++it) {
    const double width = hi - lo;
    if (width <= fmax(2.0 * kEps * fmax(fabs(lo), fabs(hi)), 4.0 * kEps * tns)) break;  // uniform
    const double x = lo + width * ((double)(tid + 1) * kStep);
    const int nle = __syncthreads_count(sturm_count(s_d, s_e2, B, x) <= m);  // a prefix of the points
    const double xlo = lo + width * ((double)nle * kStep), xhi = lo + width * ((double)(nle + 1) * kStep);
    if (nle > 0) lo = xlo;
    if (nle < kTdBisPoints) hi = xhi;
  }
  if (tid == 0) job.w[j] = 0.5 * (lo + hi) * isc;
}

// start vector of inverse iteration: splitmix64 of (vector, row) mapped to [-0.5, 0.5)
__device__ __forceinline__ double td_start(int j, int i) {
  unsigned long long z = 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1) +
                         0xBF58476D1CE4E5B9ull * (unsigned long long)(j + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

// Y[:, j] = eigenvector j of the real tridiagonal (d, |e|) for eigenvalue w[j]:
// solves (T - w_j I) y' = y with T - w_j I = L D L^T unpivoted (pivots below
// eps ||T|| raised to it).  Round 0 gives every vector kTdInvIters solves from
// its own start vector; round r takes the r-th member of every cluster of close
// eigenvalues through Gram-Schmidt against the cluster's finished members, one
// more solve and Gram-Schmidt again (three solve times for a cluster of two
// instead of four).  The vectors and multipliers are B x K,
// row-major ([i][j]: the threads of a warp touch consecutive words), in shared
// memory when they fit (smem != 0), else in the job's work buffers.
__global__ void __launch_bounds__(kTridiagMaxB) k_tridiag_invit(TridiagJobs jobs, int smem) {
  extern __shared__ __align__(16) double ism[];
  const TridiagJob job = jobs.j[blockIdx.x];
  const int B = job.B, K = job.K, j = threadIdx.x;
  __shared__ double s_d[kTridiagMaxB], s_e[kTridiagMaxB], s_w[kTridiagMaxB];
  __shared__ int s_first[kTridiagMaxB], s_pos[kTridiagMaxB];
  __shared__ double s_tn;
  __shared__ int s_rounds;
  for (int i = j; i < B; i += blockDim.x) {
    s_d[i] = job.d[i];
    const double2 e = i + 1 < B ? job.e[i] : make_double2(0.0, 0.0);
    s_e[i] = sqrt(e.x * e.x + e.y * e.y);
  }
  for (int i = j; i < K; i += blockDim.x) s_w[i] = job.w[i];
  __syncthreads();
  if (j == 0) {
    double tn = 0.0;
    for (int i = 0; i < B; ++i) tn = fmax(tn, fabs(s_d[i]) + s_e[i] + (i ? s_e[i - 1] : 0.0));
    s_tn = tn;
    int rounds = 1;
    s_first[0] = 0;
    s_pos[0] = 0;
    for (int m = 1; m < K; ++m) {
      const bool same = s_w[m - 1] - s_w[m] <= kTdClusterTol * tn;
      s_first[m] = same ? s_first[m - 1] : m;
      s_pos[m] = same ? s_pos[m - 1] + 1 : 0;
      rounds = max(rounds, s_pos[m] + 1);
    }
    s_rounds = rounds;
  }
  __syncthreads();
  const double floor = fmax(kEps * s_tn, kSafeMin);
  double* Y = smem ? ism : job.Y;
  double* L = smem ? ism + (size_t)B * K : job.lw;
  const double lam = j < K ? s_w[j] : 0.0;
  // one solve (T - lam I) y' = y in place; returns ||y'||^2
  auto solve = [&]() -> double {
    // forward: q_i = (d_i - lam) - e_{i-1} l_{i-1}, l_i = e_i / q_i, z_i = y_i - l_{i-1} z_{i-1};
    // Y[i] <- z_i / q_i
    double q = s_d[0] - lam;
    if (fabs(q) < floor) q = copysign(floor, q);
    double z = 0.0, lprev = 0.0;
    for (int i0 = 0; i0 < B; i0 += kTdChunk) {
      double yv[kTdChunk], zq[kTdChunk], lv[kTdChunk];
#pragma unroll
      for (int u = 0; u < kTdChunk; ++u) yv[u] = i0 + u < B ? Y[(size_t)(i0 + u) * K + j] : 0.0;
#pragma unroll
      for (int u = 0; u < kTdChunk; ++u) {
        const int i = i0 + u;
        if (i < B) {
          if (i > 0) {
            q = (s_d[i] - lam) - s_e[i - 1] * lprev;
            if (fabs(q) < floor) q = copysign(floor, q);
          }
          const double rq = 1.0 / q;
          z = yv[u] - lprev * z;
          lprev = s_e[i] * rq;
          zq[u] = z * rq;
          lv[u] = lprev;
        }
      }
#pragma unroll
      for (int u = 0; u < kTdChunk; ++u)
        if (i0 + u < B) {
          Y[(size_t)(i0 + u) * K + j] = zq[u];
          L[(size_t)(i0 + u) * K + j] = lv[u];
        }
    }
    // backward: y_i = Y[i] - l_i y_{i+1}
    double y = 0.0, nrm = 0.0;
    for (int i1 = B; i1 > 0; i1 -= kTdChunk) {
      double zv[kTdChunk], lv[kTdChunk];
#pragma unroll
      for (int u = 0; u < kTdChunk; ++u) {
        const int i = i1 - 1 - u;
        zv[u] = i >= 0 ? Y[(size_t)i * K + j] : 0.0;
        lv[u] = i >= 0 ? L[(size_t)i * K + j] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < kTdChunk; ++u) {
        const int i = i1 - 1 - u;
        if (i >= 0) {
          y = i == B - 1 ? zv[u] : zv[u] - lv[u] * y;
          zv[u] = y;
          nrm = fma(y, y, nrm);
        }
      }
#pragma unroll
      for (int u = 0; u < kTdChunk; ++u) {
        const int i = i1 - 1 - u;
        if (i >= 0) Y[(size_t)i * K + j] = zv[u];
      }
    }
    return nrm;
  };
  // modified Gram-Schmidt against the cluster's finished members; returns ||y||^2
  auto orthogonalise = [&]() -> double {
    for (int m = s_first[j]; m < j; ++m) {
      double dot = 0.0;
      for (int i = 0; i < B; ++i) dot = fma(Y[(size_t)i * K + m], Y[(size_t)i * K + j], dot);
      for (int i = 0; i < B; ++i) Y[(size_t)i * K + j] -= dot * Y[(size_t)i * K + m];
    }
    double nrm = 0.0;
    for (int i = 0; i < B; ++i) nrm = fma(Y[(size_t)i * K + j], Y[(size_t)i * K + j], nrm);
    return nrm;
  };
  auto normalise = [&](double nrm) {
    const double sc = nrm > 0.0 ? 1.0 / sqrt(nrm) : 0.0;
    for (int i = 0; i < B; ++i) Y[(size_t)i * K + j] *= sc;
  };
  // round 0: every vector takes kTdInvIters solves from its start vector; round
  // r: the r-th member of each cluster is orthogonalised against the earlier
  // ones (final by now), solved once more and orthogonalised again
  const int nr = s_rounds;
  for (int r = 0; r < nr; ++r) {
    if (j < K && r == 0) {
      for (int i = 0; i < B; ++i) Y[(size_t)i * K + j] = td_start(j, i);
      for (int it = 0; it < kTdInvIters; ++it) normalise(solve());
    } else if (j < K && s_pos[j] == r) {
      normalise(orthogonalise());
      normalise(solve());
      normalise(orthogonalise());
    }
    __syncthreads();  // this round's vectors are final before the next round reads them
  }
  if (smem)
    for (int x = j; x < B * K; x += blockDim.x) job.Y[x] = ism[x];
}

// Compact WY factors of the reflector blocks: block b holds reflectors
// k0 = kTdNB b .. k0 + nb - 1, and H_k0 ... H_{k0+nb-1} = I - V T V^H with
// V = [v_k0 .. v_{k0+nb-1}] and T = (I/2 + striu(V^H V))^{-1} for unit v
// (Joffrain, Low, Quintana-Orti, van de Geijn and Van Zee, "Accumulating
// Householder transformations, revisited", ACM TOMS 2006).  One CTA per block:
// its warps form the strictly upper part of V^H V, one thread inverts the
// nb x nb triangle; T (zero-padded to kTdNB x kTdNB) goes to wy[b].
__global__ void __launch_bounds__(256) k_tridiag_wy(TridiagJobs jobs) {
  const TridiagJob job = jobs.j[blockIdx.y];
  const int B = job.B, b = blockIdx.x, k0 = kTdNB * b, nb = min(kTdNB, B - 2 - k0);
  if (nb <= 0) return;  // the whole CTA
  __shared__ double2 s_u[kTdNB][kTdNB];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int pq = warp; pq < kTdNB * kTdNB; pq += nwarp) {
    const int r = pq / kTdNB, q = pq % kTdNB;
    double ax = 0.0, ay = 0.0;
    if (r < q && q < nb) {
      const double2* vr = job.refl + (size_t)(k0 + r) * B;
      const double2* vq = job.refl + (size_t)(k0 + q) * B;
      for (int i = k0 + q + 1 + lane; i < B; i += 32) {  // v_q is supported on k0+q+1 ..
        const double2 a = vr[i], c = vq[i];
        ax += fma(a.x, c.x, a.y * c.y);
        ay += fma(a.x, c.y, -a.y * c.x);
      }
      ax = warp_sum(ax);
      ay = warp_sum(ay);
    }
    if (lane == 0) s_u[r][q] = make_double2(ax, ay);  // conj(v_r) . v_q above the diagonal, else 0
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double2 t[kTdNB][kTdNB];
    for (int c = 0; c < kTdNB; ++c)
      for (int r = kTdNB - 1; r >= 0; --r) {
        if (r > c || c >= nb) {
          t[r][c] = make_double2(0.0, 0.0);
          continue;
        }
        // (I/2 + U) T = I: T[r][c] = 2 (delta_rc - sum_{q > r} U[r][q] T[q][c])
        double sx = r == c ? 1.0 : 0.0, sy = 0.0;
        for (int q = r + 1; q <= c; ++q) {
          const double2 u = s_u[r][q], v = t[q][c];
          sx -= u.x * v.x - u.y * v.y;
          sy -= u.x * v.y + u.y * v.x;
        }
        t[r][c] = make_double2(2.0 * sx, 2.0 * sy);
      }
    double2* out = job.wy + (size_t)b * kTdNB * kTdNB;
    for (int r = 0; r < kTdNB; ++r)
      for (int c = 0; c < kTdNB; ++c) out[r * kTdNB + c] = t[r][c];
  }
}

// Q[:, j] = H_0 H_1 ... H_{B-3} D Y[:, j], D = diag(phase) making the
// subdiagonal real (phase_0 = 1, phase_{k+1} = phase_k e_k / |e_k|, a parallel
// prefix product).  A warp holds its column x in registers (lane: rows
// lane + 32 t) and applies the reflector blocks last to first, each as
// x -= V (T (V^H x)): kTdNB dot products reduced together, then the update.
// The CTA stages each block's V and T in shared memory for its warps.
__global__ void __launch_bounds__(32 * kTdBackWarps) k_tridiag_back(TridiagJobs jobs) {
  constexpr int T = kTridiagMaxB / 32;
  extern __shared__ __align__(16) double2 bsm[];  // kTdNB x B block of V, then kTdNB x kTdNB T
  const TridiagJob job = jobs.j[blockIdx.y];
  const int B = job.B, K = job.K, tid = threadIdx.x;
  if ((int)blockIdx.x * kTdBackWarps >= K) return;  // the whole CTA
  __shared__ double2 s_ph[kTridiagMaxB];
  {
    const double2 one = make_double2(1.0, 0.0);
    double2 u = one;  // factor tid of the product: e_{tid-1} / |e_{tid-1}|
    if (tid >= 1 && tid < B) {
      const double2 e = job.e[tid - 1];
      const double a = sqrt(e.x * e.x + e.y * e.y);
      if (a > 0.0) u = make_double2(e.x / a, e.y / a);
    }
    s_ph[tid] = u;
    __syncthreads();
    for (int off = 1; off < kTridiagMaxB; off <<= 1) {  // inclusive scan (Hillis-Steele)
      const double2 o = tid >= off ? s_ph[tid - off] : one;
      __syncthreads();
      s_ph[tid] = zmul(o, s_ph[tid]);
      __syncthreads();
    }
  }
  const int lane = tid & 31, j = blockIdx.x * kTdBackWarps + (tid >> 5);
  const bool act = j < K;
  double2 vc[T];
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int i = lane + 32 * t;
    const double y = (act && i < B) ? job.Y[(size_t)i * K + j] : 0.0;
    vc[t] = i < B ? make_double2(s_ph[i].x * y, s_ph[i].y * y) : make_double2(0.0, 0.0);
  }
  double2* sv = bsm;
  double2* st = bsm + (size_t)kTdNB * B;
  const int nblk = (B - 2 + kTdNB - 1) / kTdNB;
  // this thread's share (entries tid + 256 u) of a block's V and T, loaded one
  // block ahead so that the L2 latency overlaps the current block's work
  constexpr int kPre = kTdNB * kTridiagMaxB / (32 * kTdBackWarps);
  double2 pre[kPre], pret = make_double2(0.0, 0.0);
  auto fetch = [&](int b) {
    const int k0 = kTdNB * b;
#pragma unroll
    for (int u = 0; u < kPre; ++u) {
      const int x = tid + 32 * kTdBackWarps * u, r = x / B, i = x - r * B, k = k0 + r;
      pre[u] = (x < kTdNB * B && k < B - 2 && i > k) ? job.refl[(size_t)k * B + i] : make_double2(0.0, 0.0);
    }
    if (tid < kTdNB * kTdNB) pret = job.wy[(size_t)b * kTdNB * kTdNB + tid];
  };
  fetch(nblk - 1);
  for (int b = nblk - 1; b >= 0; --b) {
    __syncthreads();  // the previous block is used up
#pragma unroll
    for (int u = 0; u < kPre; ++u) {
      const int x = tid + 32 * kTdBackWarps * u;
      if (x < kTdNB * B) sv[x] = pre[u];
    }
    if (tid < kTdNB * kTdNB) st[tid] = pret;
    __syncthreads();
    if (b > 0) fetch(b - 1);
    if (!act) continue;
    // w = V^H x
    double wx[kTdNB], wy[kTdNB];
#pragma unroll
    for (int r = 0; r < kTdNB; ++r) {
      double ax = 0.0, ay = 0.0;
#pragma unroll
      for (int t = 0; t < T; ++t) {
        const int i = lane + 32 * t;
        if (i < B) {
          const double2 v = sv[r * B + i], x = vc[t];
          ax = fma(v.x, x.x, fma(v.y, x.y, ax));
          ay = fma(v.x, x.y, fma(-v.y, x.x, ay));
        }
      }
      wx[r] = ax;
      wy[r] = ay;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int r = 0; r < kTdNB; ++r) {
        wx[r] += __shfl_xor_sync(0xffffffffu, wx[r], o);
        wy[r] += __shfl_xor_sync(0xffffffffu, wy[r], o);
      }
    // w' = T w (every lane)
    double zx[kTdNB], zy[kTdNB];
#pragma unroll
    for (int r = 0; r < kTdNB; ++r) {
      double ax = 0.0, ay = 0.0;
#pragma unroll
      for (int c = r; c < kTdNB; ++c) {
        const double2 t = st[r * kTdNB + c];
        ax += t.x * wx[c] - t.y * wy[c];
        ay += t.x * wy[c] + t.y * wx[c];
      }
      zx[r] = ax;
      zy[r] = ay;
    }
    // x -= V w'
#pragma unroll
    for (int t = 0; t < T; ++t) {
      const int i = lane + 32 * t;
      if (i < B) {
        double dx = 0.0, dy = 0.0;
#pragma unroll
        for (int r = 0; r < kTdNB; ++r) {
          const double2 v = sv[r * B + i];
          dx += v.x * zx[r] - v.y * zy[r];
          dy += v.x * zy[r] + v.y * zx[r];
        }
        vc[t].x -= dx;
        vc[t].y -= dy;
      }
    }
  }
  if (!act) return;
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const int i = lane + 32 * t;
    if (i < B) job.Q[(size_t)i * job.ldq + j] = vc[t];
  }
}

std::mutex g_td_mu;

}  // namespace

bool tridiag_eig_supported(int B) {
  if (B < kTridiagMinB || B > kTridiagMaxB) return false;
  static std::vector<int> known;  // per device: -1 unknown, 0 no, 1 yes
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  std::lock_guard<std::mutex> lock(g_td_mu);
  if ((int)known.size() <= dev) known.resize(dev + 1, -1);
  int& ok = known[dev];
  if (ok < 0) {
    ok = 0;
    const size_t sm = td_smem(kTridiagMaxB);
    if (cudaFuncSetAttribute(k_hermitian_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) ==
        cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(kTdCl);
      cfg.blockDim = dim3(kTdThreads);
      cfg.dynamicSmemBytes = sm;
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, k_hermitian_tridiag, &cfg) == cudaSuccess && n > 0) ok = 1;
    }
    (void)cudaGetLastError();
  }
  return ok == 1;
}

int tridiag_eig_batch(const std::vector<TridiagJob>& all, cudaStream_t st) {
  for (const TridiagJob& j : all)
    KL_CHECK_ARG(j.B >= kTridiagMinB && j.B <= kTridiagMaxB && j.K >= 1 && j.K <= j.B && j.ldq >= j.K,
                 "tridiag_eig: matrix order or K out of range");
  for (size_t j0 = 0; j0 < all.size(); j0 += kTdMaxJobs) {
    const int nj = (int)std::min(all.size() - j0, (size_t)kTdMaxJobs);
    TridiagJobs jobs{};
    int bmax = 1, kmax = 1;
    for (int j = 0; j < nj; ++j) {
      jobs.j[j] = all[j0 + j];
      bmax = std::max(bmax, jobs.j[j].B);
      kmax = std::max(kmax, jobs.j[j].K);
    }
    const size_t sm = td_smem(bmax);
    KL_CUDA_TRY(cudaFuncSetAttribute(k_hermitian_tridiag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_hermitian_tridiag<<<nj * kTdCl, kTdThreads, sm, st>>>(jobs);
    KL_CUDA_TRY(cudaGetLastError());
    k_tridiag_bisect<<<dim3(kmax, nj), kTdBisPoints, 0, st>>>(jobs);
    KL_CUDA_TRY(cudaGetLastError());
    const size_t ism = sizeof(double) * 2 * (size_t)bmax * kmax;
    const bool on_chip = ism <= kTdInvSmemCap;
    if (on_chip)
      KL_CUDA_TRY(cudaFuncSetAttribute(k_tridiag_invit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ism));
    k_tridiag_invit<<<nj, kTridiagMaxB, on_chip ? ism : 0, st>>>(jobs, on_chip ? 1 : 0);
    KL_CUDA_TRY(cudaGetLastError());
    k_tridiag_wy<<<dim3(tridiag_wy_blocks(bmax), nj), 256, 0, st>>>(jobs);
    KL_CUDA_TRY(cudaGetLastError());
    const size_t bsm = sizeof(double2) * kTdNB * ((size_t)bmax + kTdNB);
    k_tridiag_back<<<dim3((kmax + kTdBackWarps - 1) / kTdBackWarps, nj), 32 * kTdBackWarps, bsm, st>>>(jobs);
    KL_CUDA_TRY(cudaGetLastError());
  }
  return KL_OK;
}

}  // namespace kl
