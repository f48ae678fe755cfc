// Krylov (Lanczos) square root of the mobility and the Brownian step built
// on it.
//
// The reference draws its Brownian displacement with the conformationally
// averaged truncated-expansion approximation (updateHI,
// shear/src/main26.c:745-857).  This path computes sqrt(M) z itself:
// Lanczos on M from v_1 = z/|z| with full reorthogonalisation in FP64 (the
// three-term recurrence, then one classical Gram-Schmidt pass against the
// whole basis), T_m = V_m^T M V_m tridiagonal,
// sqrt(M) z ~= |z| V_m T_m^(1/2) e_1.  The relative change d_m of the iterate
// between successive m (the quantity of Ando, Chow and Skolnick, J. Chem.
// Phys. 137, 064106 (2012)) decays geometrically; the solve stops when the
// tail it implies, d_m rho / (1 - rho) with rho = (d_m / d_(m-6))^(1/6) the
// mean decay of the last six changes, is below the tolerance, an estimate of
// the error of the iterate itself rather than of its last change.  T_m^(1/2) e_1 comes
// from an eigen-decomposition of T_m on the host by the implicit symmetric QR
// iteration with Wilkinson shifts (Golub and Van Loan, Matrix Computations,
// section 8.3).  Vectors live on the device in component-major SoA with the
// tile padding (3 x NTp); every reduction is a fixed-order two-level sum.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bd_ctx.cuh"
#include "bd_hostpool.h"

using namespace bd;

#define CU(call) BD_CU(call)

static const int kDotBlocks = 148;  // one CTA per SM for the vector reductions

// Fixed-order sum of n partials by one warp: lane-strided sums, then a
// butterfly; every lane returns the same value.
__device__ __forceinline__ double warp_sum_parts(const double* __restrict__ part, int n,
                                                 int stride) {
  int lane = threadIdx.x & 31;
  double s = 0;
  for (int b = lane; b < n; b += 32) s += part[(size_t)b * stride];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// sc[0] = sqrt(sum of part) = |w|, sc[1] = 1/|w| (one warp per right-hand
// side blockIdx.x: partials nblk further on, scalars 2 further on)
__global__ void k_norm_fin(const double* __restrict__ part, int nblk, double* sc) {
  part += (size_t)blockIdx.x * nblk;
  sc += 2 * blockIdx.x;
  double s = warp_sum_parts(part, nblk, 1);
  if (threadIdx.x == 0) {
    sc[0] = sqrt(s);
    sc[1] = sc[0] > 0 ? 1.0 / sc[0] : 0.0;
  }
}

// v (SoA, padded) = z (bead-interleaved) / |z|; padding entries are zero.
// Right-hand side blockIdx.y: z zs, v vs entries further on, scalars 2.
__global__ void k_interleaved_to_soa(const double* __restrict__ z, size_t zs,
                                     const double* __restrict__ sc, double* v, size_t vs, int N,
                                     int NTp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NTp) return;
  z += (size_t)blockIdx.y * zs;
  sc += 2 * blockIdx.y;
  v += (size_t)blockIdx.y * vs;
  double f = sc[1];
  for (int a = 0; a < 3; a++) v[(size_t)a * NTp + i] = i < N ? z[3 * i + a] * f : 0.0;
}

// y_r = |z_r| sum_k c_r[k] V_r,k for the right-hand sides of a block
// (blockIdx.y = r): Krylov dimension m[r], coefficients c + r * cst, basis
// vector k at V + k * bs + r * n, norm sc[2 r], output y + r * n.
__global__ void k_combo_m(const double* __restrict__ V, size_t bs, const double* __restrict__ c,
                          int cst, const int* __restrict__ m, const double* __restrict__ sc,
                          double* y, int n) {
  int r = blockIdx.y, nv = m[r];
  const double* Vr = V + (size_t)r * n;
  const double* cr = c + (size_t)r * cst;
  double scale = sc[2 * r];
  double* yr = y + (size_t)r * n;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0;
    for (int k = 0; k < nv; k++) s += cr[k] * Vr[(size_t)k * bs + i];
    yr[i] = scale * s;
  }
}

// y = scale * sum_k c[k] V_k
__global__ void k_combo(const double* __restrict__ V, size_t vstride,
                        const double* __restrict__ c, int nv, double scale, double* y, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = 0;
    for (int k = 0; k < nv; k++) s += c[k] * V[(size_t)k * vstride + i];
    y[i] = scale * s;
  }
}

// Fused classical Gram-Schmidt (two passes) for Lanczos step j, split over
// kDotBlocks CTAs that each own one contiguous chunk of the 3 NTp entries.
// A dot product is the sum over chunks of chunk-local dots, so a CTA can
// update its own chunk as soon as it has the full sums; every CTA re-adds the
// per-chunk partials in the same order, which keeps results deterministic.
//   stage 0: part1[k][b] = V_k . w over chunk b                 (k <= j)
//   stage 1: h = sum_b part1; w_b -= V_b h; part2[k][b] = V_k . w_b
//   stage 2: h2 = sum_b part2; w_b -= V_b h2; part3[b] = |w_b|^2;
//            CTA 0 stores alpha_j = h_j + h2_j
//   stage 3: beta_j = sqrt(sum_b part3); v_{j+1,b} = w_b / beta_j
// Chunks are multiples of 4 entries (the vectors' lengths are multiples of
// 96), so the passes over an FP32 basis can read four rows per load.
__device__ __forceinline__ void chunk_range(int n, int& lo, int& hi) {
  int per = ((n + gridDim.x - 1) / gridDim.x + 3) & ~3;
  lo = min(n, (int)blockIdx.x * per);
  hi = min(n, lo + per);
}

// chunk_dots over an FP32 basis, four rows per load (lo, hi multiples of 4)
__device__ __forceinline__ void chunk_dots4(const float* __restrict__ V, size_t vs, int nv,
                                            const double* __restrict__ w, int lo, int hi,
                                            double* part) {
  int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double2* w2 = (const double2*)w;
  for (int k0 = 4 * wp; k0 < nv; k0 += 4 * nw) {
    const float4* v0 = (const float4*)(V + (size_t)k0 * vs);
    const float4* v1 = (const float4*)(V + (size_t)min(k0 + 1, nv - 1) * vs);
    const float4* v2 = (const float4*)(V + (size_t)min(k0 + 2, nv - 1) * vs);
    const float4* v3 = (const float4*)(V + (size_t)min(k0 + 3, nv - 1) * vs);
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int i4 = (lo >> 2) + lane; i4 < (hi >> 2); i4 += 32) {
      double2 wa = w2[2 * i4], wb = w2[2 * i4 + 1];
      float4 a = v0[i4], b = v1[i4], c = v2[i4], d = v3[i4];
      s0 += ((double)a.x * wa.x + (double)a.y * wa.y) + ((double)a.z * wb.x + (double)a.w * wb.y);
      s1 += ((double)b.x * wa.x + (double)b.y * wa.y) + ((double)b.z * wb.x + (double)b.w * wb.y);
      s2 += ((double)c.x * wa.x + (double)c.y * wa.y) + ((double)c.z * wb.x + (double)c.w * wb.y);
      s3 += ((double)d.x * wa.x + (double)d.y * wa.y) + ((double)d.z * wb.x + (double)d.w * wb.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      s3 += __shfl_xor_sync(0xffffffffu, s3, o);
    }
    if (lane == 0) {
      part[(size_t)k0 * gridDim.x + blockIdx.x] = s0;
      if (k0 + 1 < nv) part[(size_t)(k0 + 1) * gridDim.x + blockIdx.x] = s1;
      if (k0 + 2 < nv) part[(size_t)(k0 + 2) * gridDim.x + blockIdx.x] = s2;
      if (k0 + 3 < nv) part[(size_t)(k0 + 3) * gridDim.x + blockIdx.x] = s3;
    }
  }
}

// w[i..i+3] -= sum_k h[k] V_k[i..i+3] over an FP32 basis (i = 4 i4), eight
// vectors' loads in flight per step.  The sum is formed in FP32: the
// coefficients h are the Gram-Schmidt pass's corrections, at the level of
// the lost orthogonality (far below |w|), so its FP32 rounding is many
// orders below w's own; w and its update stay FP64.  Returns the four new
// entries' squares summed.
__device__ __forceinline__ double combo_rows4(const float* __restrict__ V, size_t vs,
                                              const double* h, int nv, int i4, double* w) {
  float a[2][4] = {};
  int k = 0;
  const float4* V4 = (const float4*)V + i4;
  const size_t vs4 = vs >> 2;  // vs is a multiple of 4
  for (; k + 8 <= nv; k += 8) {
    float4 v[8];
#pragma unroll
    for (int q = 0; q < 8; q++) v[q] = V4[(size_t)(k + q) * vs4];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      float hq = (float)h[k + q];
      a[q & 1][0] += hq * v[q].x;
      a[q & 1][1] += hq * v[q].y;
      a[q & 1][2] += hq * v[q].z;
      a[q & 1][3] += hq * v[q].w;
    }
  }
  for (; k < nv; k++) {
    float4 v = V4[(size_t)k * vs4];
    float hk = (float)h[k];
    a[0][0] += hk * v.x;
    a[0][1] += hk * v.y;
    a[0][2] += hk * v.z;
    a[0][3] += hk * v.w;
  }
  double2* w2 = (double2*)w;
  double2 wa = w2[2 * i4], wb = w2[2 * i4 + 1];
  double x[4] = {wa.x, wa.y, wb.x, wb.y}, sq = 0;
#pragma unroll
  for (int e = 0; e < 4; e++) {
    x[e] -= (double)a[0][e] + (double)a[1][e];
    sq += x[e] * x[e];
  }
  w2[2 * i4] = make_double2(x[0], x[1]);
  w2[2 * i4 + 1] = make_double2(x[2], x[3]);
  return sq;
}

// Dots of four vectors at a time per warp (vectors k0..k0+3, warps strided
// by groups): lanes over the chunk, so each lane keeps several independent
// loads in flight; butterfly reductions.
template <typename T>
__device__ __forceinline__ void chunk_dots(const T* __restrict__ V, size_t vs, int nv,
                                           const double* __restrict__ w, int lo, int hi,
                                           double* part) {
  int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k0 = 4 * wp; k0 < nv; k0 += 4 * nw) {
    const T* v0 = V + (size_t)k0 * vs;
    const T* v1 = V + (size_t)min(k0 + 1, nv - 1) * vs;
    const T* v2 = V + (size_t)min(k0 + 2, nv - 1) * vs;
    const T* v3 = V + (size_t)min(k0 + 3, nv - 1) * vs;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int i = lo + lane; i < hi; i += 32) {
      double x = w[i];
      s0 += (double)v0[i] * x;
      s1 += (double)v1[i] * x;
      s2 += (double)v2[i] * x;
      s3 += (double)v3[i] * x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      s3 += __shfl_xor_sync(0xffffffffu, s3, o);
    }
    if (lane == 0) {
      part[(size_t)k0 * gridDim.x + blockIdx.x] = s0;
      if (k0 + 1 < nv) part[(size_t)(k0 + 1) * gridDim.x + blockIdx.x] = s1;
      if (k0 + 2 < nv) part[(size_t)(k0 + 2) * gridDim.x + blockIdx.x] = s2;
      if (k0 + 3 < nv) part[(size_t)(k0 + 3) * gridDim.x + blockIdx.x] = s3;
    }
  }
}

// sum_k h[k] V_k[i] with eight independent partial sums (loads in flight),
// combined in a fixed order.
template <typename T>
__device__ __forceinline__ double combo_row(const T* __restrict__ V, size_t vs,
                                            const double* h, int nv, int i) {
  double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int k = 0;
  for (; k + 8 <= nv; k += 8) {
#pragma unroll
    for (int q = 0; q < 8; q++) a[q] += h[k + q] * (double)V[(size_t)(k + q) * vs + i];
  }
  double t = 0;
  for (; k < nv; k++) t += h[k] * (double)V[(size_t)k * vs + i];
  a[0] += t;
  return ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
}

// h[k] = sum_b part[k][b] into shared memory, one warp per k (every CTA,
// same order)
__device__ __forceinline__ void sum_parts(const double* __restrict__ part, int nv, double* h) {
  int wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = wp; k < nv; k += nw) {
    double s = warp_sum_parts(part + (size_t)k * gridDim.x, gridDim.x, 1);
    if ((threadIdx.x & 31) == 0) h[k] = s;
  }
  __syncthreads();
}

// Buffers of a Lanczos run over one or several right-hand sides (a block of
// steps' noise); right-hand side r = blockIdx.y.  Vectors have n entries;
// basis vector j of r is at V + j * bs + r * n, the work vector at w + r * n,
// the next product input at vcur + r * n; partial dots at part1/part2 +
// r * pst and part3 + r * gridDim.x, first-pass coefficients at hsave +
// r * hst, alpha_j and beta_j at [j * kst + r].
struct Kry {
  double* V;
  float* Vs;  // FP32 copy of the basis for the reorthogonalisation pass, or null
  size_t bs;
  double *w, *vcur;
  double *part1, *part2, *part3;
  size_t pst;
  double* hsave;
  int hst;
  double *alpha, *beta;
  int kst;
  const int* jd;
  int n;
};

// The iteration index j lives on the device (*jd) so that one iteration's
// launches are the same every iteration and can be replayed as a CUDA graph;
// k_next_j advances it at the end of the iteration.
// Lanczos step j with full reorthogonalisation: the three-term recurrence
// w -= alpha v_j + beta_{j-1} v_{j-1} (alpha = v_j . w), then one classical
// Gram-Schmidt pass against the whole basis, w -= V (V^T w), whose
// coefficient on v_j corrects alpha.  Two passes over the basis per step.
//   k_orth0: partial v_j . w per chunk
//   k_orth1: alpha; three-term update; partial V^T w per chunk
//   k_orth2: d = V^T w; w -= V d; |w|^2 partials; alpha_j = alpha + d_j
//   k_orth3: beta_j = |w|; v_{j+1} = w / beta_j
// With Vs (FP32 block products) the Gram-Schmidt pass reads an FP32 copy of
// the basis: its coefficients are at the level of the lost orthogonality,
// so their FP32 error (about 1e-10 of |w|) keeps the basis orthogonal well
// within sqrt(eps_64); the recurrence, alpha, beta and the final
// combination stay on the FP64 basis.
__global__ void __launch_bounds__(256) k_orth0(Kry q) {
  __shared__ double red[8];
  int r = blockIdx.y, j = *q.jd, lo, hi;
  const double* vj = q.V + (size_t)r * q.n + (size_t)j * q.bs;
  const double* w = q.w + (size_t)r * q.n;
  chunk_range(q.n, lo, hi);
  double s = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) s += vj[i] * w[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int p = 0; p < (int)(blockDim.x >> 5); p++) t += red[p];
    q.part1[r * q.pst + blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(256, 4) k_orth1(Kry q) {
  __shared__ double sa;
  int r = blockIdx.y, j = *q.jd, nv = j + 1, lo, hi;
  const double* V = q.V + (size_t)r * q.n;
  double* w = q.w + (size_t)r * q.n;
  chunk_range(q.n, lo, hi);
  if (threadIdx.x < 32) {
    double a = warp_sum_parts(q.part1 + r * q.pst, gridDim.x, 1);
    if (threadIdx.x == 0) {
      sa = a;
      if (blockIdx.x == 0) q.hsave[(size_t)r * q.hst + j] = a;
    }
  }
  __syncthreads();
  double alpha = sa, bprev = j > 0 ? q.beta[(size_t)(j - 1) * q.kst + r] : 0.0;
  const double* vj = V + (size_t)j * q.bs;
  const double* vp = V + (size_t)(j > 0 ? j - 1 : 0) * q.bs;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x)
    w[i] = w[i] - alpha * vj[i] - bprev * vp[i];
  __syncthreads();
  if (q.Vs)
    chunk_dots4(q.Vs + (size_t)r * q.n, q.bs, nv, w, lo, hi, q.part2 + r * q.pst);
  else
    chunk_dots(V, q.bs, nv, w, lo, hi, q.part2 + r * q.pst);
}

template <bool SHADOW>  // the pass reads the FP32 copy of the basis (q.Vs)
__global__ void __launch_bounds__(256, 4) k_orth2(Kry q) {
  __shared__ double h[kMaxKrylov + 1];
  __shared__ double red[8];
  int r = blockIdx.y, j = *q.jd, nv = j + 1, lo, hi;
  const double* V = q.V + (size_t)r * q.n;
  double* w = q.w + (size_t)r * q.n;
  chunk_range(q.n, lo, hi);
  sum_parts(q.part2 + r * q.pst, nv, h);
  double s2 = 0;
  if constexpr (SHADOW) {
    const float* Vs = q.Vs + (size_t)r * q.n;
    for (int i4 = (lo >> 2) + threadIdx.x; i4 < (hi >> 2); i4 += blockDim.x)
      s2 += combo_rows4(Vs, q.bs, h, nv, i4, w);
  } else {
    for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      double x = w[i] - combo_row(V, q.bs, h, nv, i);
      w[i] = x;
      s2 += x * x;
    }
  }
  for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int p = 0; p < (int)(blockDim.x >> 5); p++) t += red[p];
    q.part3[(size_t)r * gridDim.x + blockIdx.x] = t;
    if (blockIdx.x == 0) q.alpha[(size_t)j * q.kst + r] = q.hsave[(size_t)r * q.hst + j] + h[j];
  }
}

// beta_j = |w|; v_{j+1} = w / beta_j into the basis and into vcur (the
// fixed input of the next iteration's product)
__global__ void __launch_bounds__(256) k_orth3(Kry q) {
  __shared__ double b;
  int r = blockIdx.y, j = *q.jd;
  if (threadIdx.x < 32) {
    double s = warp_sum_parts(q.part3 + (size_t)r * gridDim.x, gridDim.x, 1);
    if (threadIdx.x == 0) {
      b = sqrt(s);
      if (blockIdx.x == 0) q.beta[(size_t)j * q.kst + r] = b;
    }
  }
  __syncthreads();
  double f = b > 0 ? 1.0 / b : 0.0;
  const double* w = q.w + (size_t)r * q.n;
  double* vnext = q.V + (size_t)(j + 1) * q.bs + (size_t)r * q.n;
  double* vcur = q.vcur + (size_t)r * q.n;
  float* vsnext = q.Vs ? q.Vs + (size_t)(j + 1) * q.bs + (size_t)r * q.n : nullptr;
  int lo, hi;
  chunk_range(q.n, lo, hi);
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double x = w[i] * f;
    vnext[i] = x;
    vcur[i] = x;
    if (vsnext) vsnext[i] = (float)x;
  }
}

__global__ void k_to_f32(const double* __restrict__ a, float* __restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = (float)a[i];
}

__global__ void k_next_j(int* jd) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *jd += 1;
}

// ---------------------------------------------------------------------------
// Convergence of the noise blocks' Krylov runs, checked on the device.
//
// T^(1/2) e_1 = (2/pi) int_0^inf T (t^2 I + T)^(-1) e_1 dt.  With t = e^u the
// component along an eigenvector of T (eigenvalue lambda) is
// (2/pi) sqrt(lambda) / (2 cosh(u - ln sqrt(lambda))), analytic in the strip
// |Im u| < pi/2, so the trapezoidal rule with step h converges like
// exp(-pi^2/h) (Trefethen and Weideman, SIAM Rev. 56, 385 (2014)): nodes on
// u in [-33, 41] with h = 74/255 form T^(1/2) e_1 to about 1e-14 for every
// eigenvalue in [1e-4, 1e8], with no estimate of the spectrum.  Each node is
// one tridiagonal solve x = (T + s)^(-1) e_1, s = t^2, by the backward (UL)
// elimination, pivots psi_(m-1) = alpha_(m-1) + s,
// psi_i = alpha_i + s - beta_i^2 / psi_(i+1), then x_0 = 1/psi_0,
// x_(i+1) = -beta_i x_i / psi_(i+1); the node adds w (T x) (not e_1 - s x,
// which cancels for large s).  One CTA per right-hand side, one node per
// thread; the pivots go through a global scratch row per node.
constexpr int kQuadNodes = 256;
constexpr double kQuadU0 = -33.0, kQuadU1 = 41.0;

struct BlkCheck {
  const double* alpha;  // alpha_j of right-hand side r at [j k + r]
  const double* beta;
  int k, L1, lmax;
  double tol;
  const int* jd;        // Krylov dimension reached
  int* done;
  int* conv;
  int* neg;
  int* last;            // dimension of the coefficients in c (-1: none)
  int* nd;              // consecutive relative changes known (up to 7)
  const int* first;     // first dimension to check
  int* mr;              // Krylov dimension used per right-hand side
  double* dh;           // 8 per right-hand side, ring indexed by dimension % 8
  double* c;            // coefficients, L1 per right-hand side
  double* psi;          // k x L1 x kQuadNodes scratch
};

// One quadrature solve of T_mm^(1/2) e_1 into cm (shared, zeroed here).
__device__ void quad_sqrt_e1(const double* a, const double* b, int mm, double* cm,
                             double* psi_row, int* bad) {
  int t = threadIdx.x, lane = t & 31;
  for (int i = t; i < mm; i += blockDim.x) cm[i] = 0.0;
  __syncthreads();
  const double h = (kQuadU1 - kQuadU0) / (kQuadNodes - 1);
  double u = kQuadU0 + h * t, et = exp(u);
  double sN = et * et, w = (2.0 / M_PI) * h * et;
  // backward pivots (their inverses), node t at psi_row[i * kQuadNodes + t]
  double p = a[mm - 1] + sN;
  int badp = !(p > 0.0);
  double ip = 1.0 / p;
  psi_row[(size_t)(mm - 1) * kQuadNodes + t] = ip;
  for (int i = mm - 2; i >= 0; i--) {
    p = a[i] + sN - b[i] * b[i] * ip;
    badp |= !(p > 0.0);
    ip = 1.0 / p;
    psi_row[(size_t)i * kQuadNodes + t] = ip;
  }
  // forward: x_i, and (T x)_i = beta_(i-1) x_(i-1) + alpha_i x_i + beta_i x_(i+1)
  double xm1 = 0.0, x = ip;  // ip = 1/psi_0
  for (int i = 0; i < mm; i++) {
    double xp1 = i + 1 < mm ? -b[i] * x * psi_row[(size_t)(i + 1) * kQuadNodes + t] : 0.0;
    double y = (i > 0 ? b[i - 1] * xm1 : 0.0) + a[i] * x + (i + 1 < mm ? b[i] * xp1 : 0.0);
    double v = badp ? 0.0 : w * y;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(&cm[i], v);
    xm1 = x;
    x = xp1;
  }
  if (badp) atomicOr(bad, 1);
  __syncthreads();
}

// After an iteration: for every open right-hand side at or past the first
// checked dimension, the coefficients c_m = T_m^(1/2) e_1, the relative
// change against c_(m-1) (the previous check's, or solved here at a first
// check, with those of m-2 .. m-7), and the host path's stopping test (tail
// d_m rho/(1-rho) <= tol, rho = (d_m/d_(m-6))^(1/6) capped at 0.99; or a
// breakdown beta_(m-1) <= 1e-300; or the Krylov cap).
__global__ void __launch_bounds__(kQuadNodes) k_block_check(BlkCheck q) {
  extern __shared__ double sh[];
  int r = blockIdx.x, t = threadIdx.x, L1 = q.L1;
  int m = *q.jd;
  if (q.done[r] || (m < *q.first && m < q.lmax)) return;  // uniform over the CTA
  double* a = sh;
  double* b = sh + L1;
  double* cm = sh + 2 * L1;
  double* red = sh + 3 * L1;
  __shared__ int bad;
  if (t == 0) bad = 0;
  for (int i = t; i < m; i += blockDim.x) {
    a[i] = q.alpha[(size_t)i * q.k + r];
    b[i] = q.beta[(size_t)i * q.k + r];
  }
  __syncthreads();
  double* crow = q.c + (size_t)r * L1;
  double* psi_row = q.psi + (size_t)r * L1 * kQuadNodes;
  int mm0 = q.last[r] == m - 1 ? m : max(1, m - 7);
  if (mm0 < m && t == 0) q.nd[r] = 0;
  for (int mm = mm0; mm <= m; mm++) {
    quad_sqrt_e1(a, b, mm, cm, psi_row, &bad);
    // relative change against the coefficients of mm - 1 in crow
    double dn = 0.0, cn = 0.0;
    bool have_prev = q.last[r] == mm - 1;
    for (int i = t; i < mm; i += blockDim.x) {
      double prev = (have_prev && i < mm - 1) ? crow[i] : 0.0;
      dn += (cm[i] - prev) * (cm[i] - prev);
      cn += cm[i] * cm[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
      dn += __shfl_xor_sync(0xffffffffu, dn, o);
      cn += __shfl_xor_sync(0xffffffffu, cn, o);
    }
    if ((t & 31) == 0) {
      red[2 * (t >> 5)] = dn;
      red[2 * (t >> 5) + 1] = cn;
    }
    __syncthreads();
    if (t == 0) {
      double D = 0.0, Cn = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
        D += red[2 * w];
        Cn += red[2 * w + 1];
      }
      if (have_prev) {
        q.dh[8 * r + (mm & 7)] = Cn > 0 ? sqrt(D / Cn) : 0.0;
        q.nd[r] = min(q.nd[r] + 1, 7);
      }
    }
    __syncthreads();  // every thread has read crow and last before they change
    for (int i = t; i < mm; i += blockDim.x) crow[i] = cm[i];
    if (t == 0) q.last[r] = mm;
    __syncthreads();
  }
  if (t == 0) {
    if (bad) q.neg[r] = 1;
    bool ok = false;
    if (q.nd[r] >= 7) {
      double d1 = q.dh[8 * r + (m & 7)], d0 = q.dh[8 * r + ((m - 6) & 7)];
      double rho = d0 > 0 ? pow(d1 / d0, 1.0 / 6.0) : 0.0;
      rho = fmin(rho, 0.99);
      ok = d1 * rho / (1.0 - rho) <= q.tol;
    }
    ok = ok || b[m - 1] <= 1e-300;
    if (ok || m >= q.lmax || bad) {
      q.done[r] = 1;
      q.conv[r] = ok && !bad;
      q.mr[r] = m;
    }
  }
}

// The while node's condition: another iteration while a right-hand side is
// open and the cap is not reached.
__global__ void k_block_cond(const int* __restrict__ done, int k, const int* __restrict__ jd,
                             int lmax, cudaGraphConditionalHandle h) {
  if (threadIdx.x != 0) return;
  int nd = 0;
  for (int r = 0; r < k; r++) nd += done[r];
  cudaGraphSetConditional(h, (nd < k && *jd < lmax) ? 1u : 0u);
}

__global__ void k_set_int(int* p, int v) {
  if (threadIdx.x == 0) *p = v;
}

// |z|^2 partials over the bead-interleaved noise (right-hand side blockIdx.y:
// z zs entries further on, partials gridDim.x further on)
__global__ void __launch_bounds__(256) k_sumsq(const double* __restrict__ z, size_t zs, int n,
                                               double* part) {
  z += (size_t)blockIdx.y * zs;
  part += (size_t)blockIdx.y * gridDim.x;
  double s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += z[i] * z[i];
  __shared__ double sh[8];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += sh[q];
    part[blockIdx.x] = t;
  }
}

// Brownian step with the Krylov displacement: dr = dt M F + sqrt(2 dt) y
// + dt u(r), u = edot (y, 0, 0) in shear, edot (x, -y, 0) in extension
// (the flow terms of updateHI, shear/src/main26.c:846-847,
// extensional/src/main14.c:885-886); also accumulates dxv for the Verlet check.
__global__ void k_krylov_update(int flow, double* rx, double* ry, double* rz, double* dxv,
                                double* dyv, double* dzv, const double* __restrict__ MF,
                                const double* __restrict__ Y, int NTp, int N, double dt,
                                double edot, double sq2dt) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double du[3];
  for (int a = 0; a < 3; a++) du[a] = dt * MF[(size_t)a * NTp + i] + sq2dt * Y[(size_t)a * NTp + i];
  if (flow == 0) {
    du[0] += dt * edot * ry[i];
  } else {
    du[0] += dt * edot * rx[i];
    du[1] -= dt * edot * ry[i];
  }
  dxv[i] += du[0];
  rx[i] += du[0];
  dyv[i] += du[1];
  ry[i] += du[1];
  dzv[i] += du[2];
  rz[i] += du[2];
}

// ---------------------------------------------------------------------------
// host: symmetric tridiagonal eigen-decomposition

// Implicit symmetric QR with Wilkinson shifts on T = tridiag(e, d, e)
// (Golub & Van Loan, Alg. 8.3.2/8.3.3).  d[n] diagonal, e[n-1] off-diagonal;
// on return d holds the eigenvalues.  The eigenvector matrix is the product
// Z = R_1 R_2 ... R_T of the Givens rotations of the sweeps (R_t acting on
// columns k, k+1 as [[cs, sn], [-sn, cs]]); they are returned in order instead
// of accumulated, so that f(T) e_1 = Z f(Lambda) Z^T e_1 costs O(T) = O(n^2)
// rather than the O(n^3) of forming Z.
struct Givens {
  int k;
  double cs, sn;
};

static void tridiag_eig(int n, std::vector<double>& d, std::vector<double> e,
                        std::vector<Givens>& rot) {
  rot.clear();
  if (n == 1) return;
  e.resize(n, 0.0);
  int hi = n - 1, guard = 0;
  while (hi > 0 && guard < 60 * n) {
    guard++;
    // deflate negligible off-diagonals
    for (int i = 0; i < hi; i++)
      if (fabs(e[i]) <= 1e-15 * (fabs(d[i]) + fabs(d[i + 1]))) e[i] = 0.0;
    while (hi > 0 && e[hi - 1] == 0.0) hi--;
    if (hi == 0) break;
    int lo = hi - 1;
    while (lo > 0 && e[lo - 1] != 0.0) lo--;
    // Wilkinson shift from the trailing 2x2 block
    double dd = 0.5 * (d[hi - 1] - d[hi]);
    double b2 = e[hi - 1] * e[hi - 1];
    double mu = d[hi] - b2 / (dd + (dd >= 0 ? 1.0 : -1.0) * sqrt(dd * dd + b2));
    double x = d[lo] - mu, z = e[lo], bulge = 0.0;
    for (int k = lo; k < hi; k++) {
      double r = hypot(x, z);
      double cs = r > 0 ? x / r : 1.0, sn = r > 0 ? -z / r : 0.0;
      if (k > lo) e[k - 1] = r;
      double a = d[k], b = e[k], c2 = d[k + 1];
      // R^T T R on rows/columns k, k+1 with R = [[cs, sn], [-sn, cs]]
      d[k] = cs * cs * a - 2 * cs * sn * b + sn * sn * c2;
      d[k + 1] = sn * sn * a + 2 * cs * sn * b + cs * cs * c2;
      e[k] = cs * sn * a + (cs * cs - sn * sn) * b - cs * sn * c2;
      if (k + 1 < hi) {
        bulge = -sn * e[k + 1];
        e[k + 1] = cs * e[k + 1];
        x = e[k];
        z = bulge;
      }
      rot.push_back({k, cs, sn});
    }
  }
}

// c = T^q e_1 for T = tridiag(beta, alpha, beta) of size m, q = +1/2 or
// -1/2; non-positive Ritz values are clamped (to zero for q > 0, to 1e-12 of
// the largest for q < 0) and counted.  y = Z^T e_1 applies R_1^T .. R_T^T to
// e_1; c = Z f(Lambda) y applies R_T .. R_1.
static int sqrt_e1(const std::vector<double>& alpha, const std::vector<double>& beta, int m,
                   std::vector<double>& c, double q = 0.5) {
  if (m <= 0) {
    c.clear();
    return 0;
  }
  std::vector<double> d(alpha.begin(), alpha.begin() + m), e(beta.begin(), beta.begin() + (m - 1));
  std::vector<Givens> rot;
  tridiag_eig(m, d, e, rot);
  std::vector<double> y(m, 0.0);
  y[0] = 1.0;
  for (const Givens& g : rot) {
    double a = y[g.k], b = y[g.k + 1];
    y[g.k] = g.cs * a - g.sn * b;
    y[g.k + 1] = g.sn * a + g.cs * b;
  }
  int neg = 0;
  double lmax = 0;
  for (int k = 0; k < m; k++) lmax = std::max(lmax, d[k]);
  for (int k = 0; k < m; k++) {
    double lam = d[k];
    if (lam <= 0) {
      neg++;
      lam = q > 0 ? 0.0 : 1e-12 * lmax;
    }
    y[k] *= q > 0 ? sqrt(lam) : 1.0 / sqrt(lam);
  }
  for (size_t t = rot.size(); t-- > 0;) {
    const Givens& g = rot[t];
    double a = y[g.k], b = y[g.k + 1];
    y[g.k] = g.cs * a + g.sn * b;
    y[g.k + 1] = -g.sn * a + g.cs * b;
  }
  c.swap(y);
  return neg;
}


// Relative change d_m = |c_m - (c_(m-1), 0)| / |c_m| of the tridiagonal
// coefficients between Krylov dimensions m - 1 and m (the basis is
// orthonormal, so this is the relative change of the iterate itself).
static double rel_change(const std::vector<double>& cm, const std::vector<double>& cprev) {
  double dn = 0, cn = 0;
  for (size_t i = 0; i < cm.size(); i++) {
    double prev = i < cprev.size() ? cprev[i] : 0.0;
    dn += (cm[i] - prev) * (cm[i] - prev);
    cn += cm[i] * cm[i];
  }
  return cn > 0 ? sqrt(dn / cn) : 0.0;
}

// Stopping test at dimension m from the changes dh[m-6 .. m] (negative where
// unknown): with the changes decaying at rate rho the error left in the
// iterate is the geometric tail d_m rho / (1 - rho).  rho is the mean decay
// over the last six changes, (d_m / d_(m-6))^(1/6) (steadier than one ratio,
// which the rounding of FP32 products makes noisy near convergence), capped
// at 0.99, so that d_m <= tol / 99 is sufficient on its own.
constexpr int kTailSpan = 6;

// The stopping tolerance of a solve: the context's for sqrt(M) z; half of it
// for the preconditioned sqrt(G M G^T) z, whose error G^-1 carries into the
// displacement amplified (by up to 1.6 measured with segment blocks), so that
// the displacement itself stays within the tolerance.
static double stop_tol(const bd_ctx* c, bool pre) { return pre ? 0.5 * c->ltol : c->ltol; }

static bool tail_converged(const std::vector<double>& dh, int m, double tol) {
  if (m <= kTailSpan + 1 || (int)dh.size() <= m) return false;
  if (dh[m] < 0 || dh[m - kTailSpan] < 0) return false;
  double rho = dh[m - kTailSpan] > 0 ? pow(dh[m] / dh[m - kTailSpan], 1.0 / kTailSpan) : 0.0;
  rho = std::min(rho, 0.99);
  return dh[m] * rho / (1.0 - rho) <= tol;
}

namespace bd {

int alloc_lanczos(bd_ctx* c) {
  if (c->LV) return BD_OK;
  c->lmax = c->p.lanczos_max > 0 ? c->p.lanczos_max : 200;
  c->ltol = c->p.lanczos_tol > 0 ? c->p.lanczos_tol : 1e-6;
  size_t n = 3 * (size_t)c->NT * 32;
  CU(cudaMalloc(&c->LV, 8 * n * (c->lmax + 1)));
  CU(cudaMalloc(&c->Lw, 8 * n));
  CU(cudaMalloc(&c->Lpart, 8 * (size_t)3 * (c->lmax + 1) * kDotBlocks));
  CU(cudaMalloc(&c->Lh, 8 * (size_t)(c->lmax + 1)));
  CU(cudaMalloc(&c->Lsc, 8 * (size_t)(c->lmax + 16)));
  CU(cudaMalloc(&c->Lc, 8 * (size_t)(c->lmax + 1)));
  CU(cudaMalloc(&c->MF, 8 * n));
  CU(cudaMalloc(&c->Yz, 8 * n));
  CU(cudaMalloc(&c->Lt1, 8 * n));
  CU(cudaMalloc(&c->Lt2, 8 * n));
  CU(cudaMalloc(&c->Lvcur, 8 * n));
  CU(cudaMalloc(&c->Ljd, 16));
  // the padding entries (beads N..NTp-1) of the work vectors stay zero: the
  // orthogonalisation runs over all 3 NTp entries and the particle-mesh
  // product and the preconditioner write only the N beads
  for (double* q : {c->Lw, c->MF, c->Yz, c->Lt1, c->Lt2, c->Lvcur})
    CU(cudaMemsetAsync(q, 0, 8 * n, c->stream));
  c->bytes += 8 * n * (c->lmax + 6) + 8 * (size_t)(c->lmax + 1) * (3 * kDotBlocks + 2) +
              8 * (size_t)(c->lmax + 16);
  return BD_OK;
}

// One Lanczos iteration's launches: w = A v with v = vcur (A = M, or
// G M G^T with the block preconditioner when pre; with force also M F into
// c->MF), reorthogonalisation against the basis, beta, v_{j+1}, j += 1.  Every argument is
// the same in every iteration (the index j is read on the device), so the
// launches can be captured once and replayed as a CUDA graph.
static int lanczos_iteration(bd_ctx* c, bool pre, bool force) {
  int s, NTp = c->NT * 32, n = 3 * NTp, blk = kDotBlocks;
  size_t vs = (size_t)n;
  cudaStream_t st = c->stream;
  double* vc = c->Lvcur;
  VecIn vin = {{vc, vc + NTp, vc + 2 * NTp}, 1};
  VecIn vf = {{c->fx, c->fy, c->fz}, 1};
  if (!pre) {
    if (force) {
      if ((s = sym_matvec(c, 2, vf, vin, c->MF, c->Lw, true)) != BD_OK) return s;
    } else {
      if ((s = sym_matvec(c, 1, vin, vin, c->Lw, c->Lw, true)) != BD_OK) return s;
    }
  } else {
    precond_apply(c, 1, vc, c->Lt1);
    VecIn vt = {{c->Lt1, c->Lt1 + NTp, c->Lt1 + 2 * NTp}, 1};
    if (force) {
      if ((s = sym_matvec(c, 2, vf, vt, c->MF, c->Lt2, true)) != BD_OK) return s;
    } else {
      if ((s = sym_matvec(c, 1, vt, vt, c->Lt2, c->Lt2, true)) != BD_OK) return s;
    }
    precond_apply(c, 0, c->Lt2, c->Lw);
  }
  Kry q;
  q.V = c->LV;
  q.Vs = nullptr;
  q.bs = vs;
  q.w = c->Lw;
  q.vcur = vc;
  q.part1 = c->Lpart;
  q.part2 = c->Lpart + (size_t)(c->lmax + 1) * blk;
  q.part3 = c->Lpart + (size_t)2 * (c->lmax + 1) * blk;
  q.pst = 0;
  q.hsave = c->Lc;
  q.hst = 0;
  q.alpha = c->Lh;
  q.beta = c->Lsc + 8;
  q.kst = 1;
  q.jd = c->Ljd;
  q.n = n;
  c->launches += 5;
  k_orth0<<<blk, 256, 0, st>>>(q);
  k_orth1<<<blk, 256, 0, st>>>(q);
  k_orth2<false><<<blk, 256, 0, st>>>(q);  // single solves keep no FP32 copy
  k_orth3<<<blk, 256, 0, st>>>(q);
  k_next_j<<<1, 32, 0, st>>>(c->Ljd);
  return launch_ok(c);
}

// Launches one iteration, from the context's captured graph when graphs are
// on (capturing it on first use).
static int lanczos_iteration_graph(bd_ctx* c, bool pre) {
  int v = pre ? 1 : 0;
  if (!c->lan_graph[v]) {
    cudaGraph_t g;
    long long l0 = c->launches;
    c->capturing = true;
    CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int s = lanczos_iteration(c, pre, false);
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->capturing = false;
    if (s != BD_OK) return s;
    if (e != cudaSuccess) return cuda_fail((int)e, cudaGetErrorString(e), __FILE__, __LINE__);
    cudaGraphExec_t ex;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail((int)e, cudaGetErrorString(e), __FILE__, __LINE__);
    c->lan_graph[v] = (void*)ex;
    c->lan_graph_launches[v] = c->launches - l0;
    c->launches = l0;
  }
  CU(cudaGraphLaunch((cudaGraphExec_t)c->lan_graph[v], c->stream));
  c->launches += c->lan_graph_launches[v];
  return launch_ok(c);
}

// Lanczos for f(A) z, f(x) = x^q (q = +-1/2), z bead-interleaved on the
// device; A = M, or A = G M G^T with the block preconditioner G when pre.
// The result |z| V_m f(T_m) e_1 goes to out (Lanczos layout).  With
// with_force the first product also forms M F into c->MF.  *conv reports
// whether the tolerance was met within the Krylov cap.
static int lanczos_run(bd_ctx* c, const double* z, bool with_force, bool pre, double q,
                       double* out, int* iters, bool* conv_out) {
  int s;
  if (!out || !c->LV) return BD_ERR_STATE;
  int N = c->N, NTp = c->NT * 32, n = 3 * NTp, blk = kDotBlocks;
  size_t vs = (size_t)n;
  cudaStream_t st = c->stream;
  // |z|, v_0 (into the basis and the product input), j = 0
  c->launches += 3;
  k_sumsq<<<blk, 256, 0, st>>>(z, 0, 3 * N, c->Lpart);
  k_norm_fin<<<1, 32, 0, st>>>(c->Lpart, blk, c->Lsc);
  k_interleaved_to_soa<<<(NTp + 255) / 256, 256, 0, st>>>(z, 0, c->Lsc, c->LV, 0, N, NTp);
  if ((s = launch_ok(c)) != BD_OK) return s;
  CU(cudaMemcpyAsync(c->Lvcur, c->LV, 8 * vs, cudaMemcpyDeviceToDevice, st));
  CU(cudaMemsetAsync(c->Ljd, 0, sizeof(int), st));
  double zn = 0;
  CU(cudaMemcpyAsync(&zn, c->Lsc, 8, cudaMemcpyDeviceToHost, st));
  std::vector<double> alpha, beta, cc;
  int m = 0, neg = 0;
  bool conv = false;
  // alpha_j, beta_j stay on the device (Lh, Lsc + 8); the host reads them
  // only at checkpoints: from two before the previous call's Krylov
  // dimension on, every second iteration.  Each check needs the changes at
  // the last seven dimensions: the coefficients of the dimensions it lacks
  // are solved for (cs: the last few, by dimension), the previous check's
  // reused.
  double* d_alpha = c->Lh;
  double* d_beta = c->Lsc + 8;
  int& last = pre ? c->pre_last : c->lan_last;
  int next_check = std::max(kTailSpan + 2, last - 2);
  std::vector<double> dh;
  std::vector<std::vector<double>> cs;
  std::vector<int> cs_m;
  auto coeffs = [&](int mm) -> std::vector<double> {
    for (size_t i = 0; i < cs_m.size(); i++)
      if (cs_m[i] == mm) return cs[i];
    cs.emplace_back();
    cs_m.push_back(mm);
    int ng = sqrt_e1(alpha, beta, mm, cs.back(), q);
    if (mm == m) neg = ng;
    return cs.back();
  };
  for (int j = 0; j < c->lmax; j++) {
    if (j == 0 && with_force)
      s = lanczos_iteration(c, pre, true);
    else if (c->use_graphs)
      s = lanczos_iteration_graph(c, pre);
    else
      s = lanczos_iteration(c, pre, false);
    if (s != BD_OK) return s;
    m = j + 1;
    if (m < next_check && m < c->lmax) continue;
    alpha.resize(m);
    beta.resize(m);
    CU(cudaMemcpyAsync(alpha.data(), d_alpha, 8 * (size_t)m, cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(beta.data(), d_beta, 8 * (size_t)m, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    // keep only the coefficients that later checks can reuse
    for (size_t i = 0; i < cs_m.size();)
      if (cs_m[i] < m - kTailSpan - 1) {
        cs.erase(cs.begin() + i);
        cs_m.erase(cs_m.begin() + i);
      } else {
        i++;
      }
    dh.resize(m + 1, -1.0);
    for (int mm = std::max(2, m - kTailSpan); mm <= m; mm++)
      if (dh[mm] < 0) dh[mm] = rel_change(coeffs(mm), coeffs(mm - 1));
    cc = coeffs(m);
    if (tail_converged(dh, m, stop_tol(c, pre)) || beta[m - 1] <= 1e-300) {
      conv = true;
      break;
    }
    next_check = m + 2;
  }
  CU(cudaMemcpyAsync(c->Lc, cc.data(), 8 * (size_t)m, cudaMemcpyHostToDevice, st));
  c->launches++;
  k_combo<<<blk * 2, 256, 0, st>>>(c->LV, vs, c->Lc, m, zn, out, n);
  last = m;
  c->lan_negative += neg;
  if (iters) *iters = m;
  *conv_out = conv;
  CU(cudaStreamSynchronize(st));  // cc is a host vector read by the copy above
  return launch_ok(c);
}

// Drops the captured Lanczos iterations (their kernels hold the mobility's
// diagonal and the preconditioner's buffers by value); called whenever those
// change.
void lanczos_graphs_reset(bd_ctx* c) {
  for (int v = 0; v < 2; v++)
    if (c->lan_graph[v]) {
      cudaGraphExecDestroy((cudaGraphExec_t)c->lan_graph[v]);
      c->lan_graph[v] = nullptr;
    }
  for (int v = 0; v < 4; v++)
    for (int h = 0; h < 2; h++)
      if (c->blk_graph[v][h]) {
        cudaGraphExecDestroy((cudaGraphExec_t)c->blk_graph[v][h]);
        c->blk_graph[v][h] = nullptr;
      }
  for (int v = 0; v < 4; v++)
    if (c->blk_while[v]) {
      cudaGraphExecDestroy((cudaGraphExec_t)c->blk_while[v]);
      c->blk_while[v] = nullptr;
    }
}

// ---------------------------------------------------------------------------
// Noise blocks: sqrt(A) z_r for the noise draws z_0..z_{k-1} of k consecutive
// steps by one Lanczos run over k right-hand sides.  Each right-hand side has
// its own basis, coefficients and stopping point; they share the launches
// (the particle-mesh product of 3 k grids, the preconditioner blocks and the
// orthogonalisation kernels with blockIdx.y = r), which turns k latency-bound iterations
// into one.  The host checks convergence for all right-hand sides at once,
// one iteration behind the device (the next iteration is already queued
// while the tridiagonal problems are solved, on several host threads).

static int alloc_blocks(bd_ctx* c) {
  if (c->BV) return BD_OK;
  int k = c->nbk, L1 = c->lmax + 1, blk = kDotBlocks;
  size_t n = 3 * (size_t)c->NT * 32;
  CU(cudaMalloc(&c->BV, 8 * n * k * L1));
  if (c->p.precision == BD_PREC_FP32) {  // FP32 copy for the reorthogonalisation pass
    CU(cudaMalloc(&c->BVs, 4 * n * k * L1));
    c->bytes += 4 * n * k * L1;
  }
  for (double** q : {&c->Bw, &c->Bvcur, &c->Bt1, &c->Bt2, &c->BY}) {
    CU(cudaMalloc(q, 8 * n * k));
    CU(cudaMemsetAsync(*q, 0, 8 * n * k, c->stream));  // padding entries stay zero
  }
  CU(cudaMalloc(&c->BR, 8 * 3 * (size_t)c->N * k));
  CU(cudaMalloc(&c->Bpart, 8 * (size_t)3 * k * L1 * blk));
  CU(cudaMalloc(&c->Bh, 8 * (size_t)k * L1));
  CU(cudaMalloc(&c->Bab, 8 * (size_t)2 * k * L1));
  CU(cudaMalloc(&c->Bsc, 8 * (size_t)2 * k));
  CU(cudaMalloc(&c->Bc, 8 * (size_t)k * L1));
  CU(cudaMalloc(&c->Bm, 4 * (size_t)k));
  CU(cudaMalloc(&c->Bjd, 16));
  CU(cudaMalloc(&c->Bctl, 4 * (size_t)(5 * k + 4)));
  CU(cudaMalloc(&c->Bdh, 8 * 8 * (size_t)k));
  CU(cudaMalloc(&c->Bpsi, 8 * (size_t)k * L1 * kQuadNodes));
  c->bytes += 4 * (size_t)(5 * k + 4) + 64 * (size_t)k + 8 * (size_t)k * L1 * kQuadNodes;
  if (!c->Bhost) return BD_ERR_STATE;  // pinned at bd_create (see there)
  CU(cudaMalloc(&c->Brng, sizeof(Ran1) * (size_t)(k + 1)));
  cudaEvent_t ev;
  CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  c->blk_ev = (void*)ev;
  c->bytes += 8 * n * k * (L1 + 5) + 24 * (size_t)c->N * k + 8 * (size_t)k * L1 * (3 * blk + 4) +
              24 * (size_t)k;
  return BD_OK;
}

void lanczos_blocks_free(bd_ctx* c) {
  for (double* q : {c->BV, c->Bw, c->Bvcur, c->Bt1, c->Bt2, c->BY, c->BR, c->Bpart, c->Bh, c->Bab,
                    c->Bsc, c->Bc})
    if (q) cudaFree(q);
  if (c->Bm) cudaFree(c->Bm);
  if (c->Bjd) cudaFree(c->Bjd);
  if (c->Bctl) cudaFree(c->Bctl);
  if (c->Bdh) cudaFree(c->Bdh);
  if (c->Bpsi) cudaFree(c->Bpsi);
  if (c->BVs) cudaFree(c->BVs);
  c->BVs = nullptr;
  c->Bctl = nullptr;
  c->Bdh = c->Bpsi = nullptr;
  if (c->Bhost) cudaFreeHost(c->Bhost);
  if (c->Brng) cudaFree(c->Brng);
  c->Brng = nullptr;
  if (c->blk_ev) cudaEventDestroy((cudaEvent_t)c->blk_ev);
  c->BV = nullptr;
  c->Bhost = nullptr;
  c->blk_ev = nullptr;
}

void noise_blocks_release(bd_ctx* c) {
  if (c->blk_n > 0 && c->blk_next < c->blk_n) {
    if (c->p.noise == BD_NOISE_PHILOX)
      c->noise_draws = c->blk_draw0 + (unsigned long long)c->blk_next;
    else
      cudaMemcpyAsync(c->rng, (const Ran1*)c->Brng + c->blk_next, sizeof(Ran1),
                      cudaMemcpyDeviceToDevice, c->stream);
  }
  c->blk_n = 0;
  c->blk_next = 0;
}

// Chunks per right-hand side of the block orthogonalisation kernels.
static int block_chunks(int k) { return std::min(kDotBlocks, std::max(8, 4 * kDotBlocks / k)); }

// Layout of a block of k right-hand sides: basis vector j of r at
// BV + (j k + r) n, alpha_j and beta_j at [j k + r].
static Kry block_kry(bd_ctx* c, int k) {
  int L1 = c->lmax + 1, blk = kDotBlocks;
  size_t n = 3 * (size_t)c->NT * 32;
  Kry q;
  q.V = c->BV;
  q.Vs = c->BVs;
  q.bs = n * k;
  q.w = c->Bw;
  q.vcur = c->Bvcur;
  q.part1 = c->Bpart;
  q.part2 = c->Bpart + (size_t)k * L1 * blk;
  q.part3 = c->Bpart + (size_t)2 * k * L1 * blk;
  q.pst = (size_t)L1 * blk;
  q.hsave = c->Bh;
  q.hst = L1;
  q.alpha = c->Bab;
  q.beta = c->Bab + (size_t)L1 * k;
  q.kst = k;
  q.jd = c->Bjd;
  q.n = (int)n;
  return q;
}

// One iteration of the block, in two parts: the product W = A V_cur for the
// k inputs (part 0), then the orthogonalisation of each against its own basis, beta, next
// vectors, j += 1 (part 1).  The same launches every iteration (j is read on
// the device), so each part can be captured as a graph; the product is timed
// on its own (BD_PROF_BLOCK) between the two.
static int block_part(bd_ctx* c, int k, bool pre, int part) {
  int s;
  size_t n = 3 * (size_t)c->NT * 32;
  cudaStream_t st = c->stream;
  if (part == 0) {
    if (!pre) {
      if ((s = pme_apply_multi(c, k, c->Bvcur, n, c->Bw, n)) != BD_OK) return s;
    } else {
      precond_apply_k(c, 1, k, c->Bvcur, n, c->Bt1, n);
      if ((s = pme_apply_multi(c, k, c->Bt1, n, c->Bt2, n)) != BD_OK) return s;
      precond_apply_k(c, 0, k, c->Bt2, n, c->Bw, n);
    }
    return launch_ok(c);
  }
  Kry q = block_kry(c, k);
  // 4 x 148 CTAs in all: each right-hand side's vectors in 592 / k chunks
  // (at most 148), so every CTA re-sums only the chunk partials of its own
  // right-hand side while enough warps stay resident
  dim3 g(block_chunks(k), k);
  c->launches += 5;
  k_orth0<<<g, 256, 0, st>>>(q);
  k_orth1<<<g, 256, 0, st>>>(q);
  if (q.Vs)
    k_orth2<true><<<g, 256, 0, st>>>(q);
  else
    k_orth2<false><<<g, 256, 0, st>>>(q);
  k_orth3<<<g, 256, 0, st>>>(q);
  k_next_j<<<1, 32, 0, st>>>(c->Bjd);
  return launch_ok(c);
}

static int block_iteration(bd_ctx* c, int k, bool pre) {
  int s;
  if (!c->use_graphs) {
    prof_begin(c, BD_PROF_BLOCK);
    if ((s = block_part(c, k, pre, 0)) != BD_OK) return s;
    prof_end(c, BD_PROF_BLOCK);
    return block_part(c, k, pre, 1);
  }
  int key = 2 * k + (pre ? 1 : 0), slot = -1;
  for (int q = 0; q < 4 && slot < 0; q++)
    if (c->blk_graph[q][0] && c->blk_graph_key[q] == key) slot = q;
  if (slot < 0) {
    for (int q = 0; q < 4 && slot < 0; q++)
      if (!c->blk_graph[q][0]) slot = q;
    if (slot < 0) {
      slot = 3;
      for (int h = 0; h < 2; h++) {
        cudaGraphExecDestroy((cudaGraphExec_t)c->blk_graph[slot][h]);
        c->blk_graph[slot][h] = nullptr;
      }
    }
    for (int h = 0; h < 2; h++) {
      cudaGraph_t g;
      long long l0 = c->launches;
      c->capturing = true;
      CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      int s2 = block_part(c, k, pre, h);
      cudaError_t e = cudaStreamEndCapture(c->stream, &g);
      c->capturing = false;
      if (s2 != BD_OK) return s2;
      if (e != cudaSuccess) return cuda_fail((int)e, cudaGetErrorString(e), __FILE__, __LINE__);
      cudaGraphExec_t ex;
      e = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return cuda_fail((int)e, cudaGetErrorString(e), __FILE__, __LINE__);
      c->blk_graph[slot][h] = (void*)ex;
      c->blk_graph_launches[slot][h] = c->launches - l0;
      c->launches = l0;
    }
    c->blk_graph_key[slot] = key;
  }
  prof_begin(c, BD_PROF_BLOCK);
  CU(cudaGraphLaunch((cudaGraphExec_t)c->blk_graph[slot][0], c->stream));
  prof_end(c, BD_PROF_BLOCK);
  CU(cudaGraphLaunch((cudaGraphExec_t)c->blk_graph[slot][1], c->stream));
  c->launches += c->blk_graph_launches[slot][0] + c->blk_graph_launches[slot][1];
  return BD_OK;
}

// f(i) for i < n on the calling thread and the process's host workers.
template <class F>
static void parallel_for(int n, F f) {
  HostPool::get().run(n, f);
}

static BlkCheck block_check_args(bd_ctx* c, int k, bool pre) {
  int L1 = c->lmax + 1;
  BlkCheck q;
  q.alpha = c->Bab;
  q.beta = c->Bab + (size_t)L1 * k;
  q.k = k;
  q.L1 = L1;
  q.lmax = c->lmax;
  q.tol = stop_tol(c, pre);
  q.jd = c->Bjd;
  q.done = c->Bctl;
  q.conv = c->Bctl + k;
  q.neg = c->Bctl + 2 * k;
  q.last = c->Bctl + 3 * k;
  q.nd = c->Bctl + 4 * k;
  q.first = c->Bctl + 5 * k;
  q.mr = c->Bm;
  q.dh = c->Bdh;
  q.c = c->Bc;
  q.psi = c->Bpsi;
  return q;
}

// The whole solve of a block of k right-hand sides (preconditioned or not) as
// one graph: a conditional while node whose body is one block iteration
// (product, orthogonalisation), the device check and the condition kernel.
// Built once per (k, pre) and kept until the captured buffers change.
static int block_while_graph(bd_ctx* c, int k, bool pre, cudaGraphExec_t* out) {
  int key = 2 * k + (pre ? 1 : 0), slot = -1;
  for (int q = 0; q < 4 && slot < 0; q++)
    if (c->blk_while[q] && c->blk_while_key[q] == key) slot = q;
  if (slot >= 0) {
    *out = (cudaGraphExec_t)c->blk_while[slot];
    return BD_OK;
  }
  for (int q = 0; q < 4 && slot < 0; q++)
    if (!c->blk_while[q]) slot = q;
  if (slot < 0) {
    slot = 3;
    cudaGraphExecDestroy((cudaGraphExec_t)c->blk_while[slot]);
    c->blk_while[slot] = nullptr;
  }
  cudaStream_t st = c->stream;
  cudaGraph_t g = nullptr;
  CU(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  cudaGraphNode_t node;
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
  int s = BD_OK;
  long long l0 = c->launches;
  if (e == cudaSuccess) {
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      c->capturing = true;
      s = block_part(c, k, pre, 0);
      if (s == BD_OK) s = block_part(c, k, pre, 1);
      if (s == BD_OK) {
        BlkCheck q = block_check_args(c, k, pre);
        size_t smem = 8 * (3 * (size_t)q.L1 + 16);
        if (smem > 48 * 1024)
          cudaFuncSetAttribute(k_block_check, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
        k_block_check<<<k, kQuadNodes, smem, st>>>(q);
        k_block_cond<<<1, 32, 0, st>>>(c->Bctl, k, c->Bjd, c->lmax, h);
        c->launches += 2;
      }
      cudaGraph_t cap = nullptr;
      cudaError_t e2 = cudaStreamEndCapture(st, &cap);
      c->capturing = false;
      if (e == cudaSuccess) e = e2;
    }
  }
  cudaGraphExec_t ex = nullptr;
  if (s == BD_OK && e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  long long per_iter = c->launches - l0;
  c->launches = l0;
  if (s != BD_OK || e != cudaSuccess) {
    // not sticky: the host-checked path takes over for this context
    cudaGetLastError();
    c->while_failed = true;
    return BD_ERR_STATE;
  }
  c->blk_while[slot] = (void*)ex;
  c->blk_while_key[slot] = key;
  c->blk_while_launches[slot] = per_iter;
  *out = ex;
  return BD_OK;
}

// lanczos_run_multi with the convergence checks and the iteration loop on the
// device: one graph launch for the whole block, one synchronisation at its end.
static int lanczos_run_multi_device(bd_ctx* c, int k, bool pre, double* out,
                                    std::vector<int>& mr, std::vector<char>& conv,
                                    int* iters_run) {
  int s, N = c->N, NTp = c->NT * 32, blk = kDotBlocks, L1 = c->lmax + 1;
  size_t n = 3 * (size_t)NTp;
  cudaStream_t st = c->stream;
  cudaGraphExec_t ex;
  if ((s = block_while_graph(c, k, pre, &ex)) != BD_OK) return s;
  long long per_iter = 0;
  for (int q = 0; q < 4; q++)
    if (c->blk_while[q] == (void*)ex) per_iter = c->blk_while_launches[q];
  c->launches += 5;
  k_sumsq<<<dim3(blk, k), 256, 0, st>>>(c->BR, 3 * (size_t)N, 3 * N, c->Bpart);
  k_norm_fin<<<k, 32, 0, st>>>(c->Bpart, blk, c->Bsc);
  k_interleaved_to_soa<<<dim3((NTp + 255) / 256, k), 256, 0, st>>>(c->BR, 3 * (size_t)N, c->Bsc,
                                                                   c->BV, n, N, NTp);
  CU(cudaMemcpyAsync(c->Bvcur, c->BV, 8 * n * k, cudaMemcpyDeviceToDevice, st));
  if (c->BVs) {
    c->launches++;
    k_to_f32<<<592, 256, 0, st>>>(c->BV, c->BVs, n * k);
  }
  CU(cudaMemsetAsync(c->Bjd, 0, sizeof(int), st));
  CU(cudaMemsetAsync(c->Bctl, 0, 4 * 3 * (size_t)k, st));             // done, conv, neg
  CU(cudaMemsetAsync(c->Bctl + 3 * k, 0xff, 4 * (size_t)k, st));      // last = -1
  CU(cudaMemsetAsync(c->Bctl + 4 * k, 0, 4 * (size_t)k, st));         // nd
  k_set_int<<<1, 32, 0, st>>>(c->Bctl + 5 * k, std::max(kTailSpan + 2, c->blk_last - 2));
  if ((s = launch_ok(c)) != BD_OK) return s;
  CU(cudaGraphLaunch(ex, st));
  k_combo_m<<<dim3(blk, k), 256, 0, st>>>(c->BV, n * k, c->Bc, L1, c->Bm, c->Bsc, out, (int)n);
  // Krylov dimensions, outcomes, negative-pivot flags and iterations run
  int* h = (int*)c->Bhost;
  CU(cudaMemcpyAsync(h, c->Bm, 4 * (size_t)k, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(h + k, c->Bctl + k, 4 * 2 * (size_t)k, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(h + 3 * k, c->Bjd, 4, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  if ((s = launch_ok(c)) != BD_OK) return s;
  int j = h[3 * k];
  mr.assign(h, h + k);
  conv.assign(k, 0);
  std::vector<int> negr;
  for (int r = 0; r < k; r++) {
    conv[r] = (char)h[k + r];
    if (h[2 * k + r]) negr.push_back(r);
  }
  c->launches += per_iter * j;
  if (!negr.empty()) {
    // a tridiagonal that is not positive definite (an indefinite operator):
    // the device stopped that right-hand side at its first non-positive
    // pivot.  Preconditioned, it is reported unconverged (the caller re-solves
    // it plainly); plain, it is re-solved by the host-checked single-vector
    // Lanczos, which clamps negative Ritz values, into its output slot
    c->host_fallbacks++;
    for (int r : negr) {
      conv[r] = 0;
      if (pre) continue;
      int m1 = 0;
      bool cv = false;
      if ((s = lanczos_run(c, c->BR + 3 * (size_t)N * r, false, false, 0.5, out + n * r, &m1,
                           &cv)) != BD_OK)
        return s;
      mr[r] = m1;
      conv[r] = cv;
    }
  }
  int mmin = c->lmax;
  for (int r = 0; r < k; r++) mmin = std::min(mmin, mr[r]);
  c->blk_last = mmin;
  c->blk_runs++;
  c->blk_products += j;
  c->blk_rhs_products += (long long)j * k;
  c->dev_solves++;
  if (iters_run) *iters_run = j;
  return launch_ok(c);
}

// Lanczos for sqrt(A) z_r, r < k, z_r = BR + 3 N r; the results
// |z_r| V_r,m f(T_r,m) e_1 go to out + r n.  mr[r] is the Krylov dimension of
// right-hand side r, conv[r] whether it met the tolerance within the cap.
// With device checks (and graphs, without per-product profiling) the loop runs
// on the device; otherwise the host checks one iteration behind.
static int lanczos_run_multi(bd_ctx* c, int k, bool pre, double* out, std::vector<int>& mr,
                             std::vector<char>& conv, int* iters_run) {
  if (c->device_krylov && c->use_graphs && !c->prof_products && !c->while_failed) {
    int s = lanczos_run_multi_device(c, k, pre, out, mr, conv, iters_run);
    if (s != BD_ERR_STATE || !c->while_failed) return s;
  }
  int s, N = c->N, NTp = c->NT * 32, blk = kDotBlocks, L1 = c->lmax + 1;
  size_t n = 3 * (size_t)NTp;
  cudaStream_t st = c->stream;
  cudaEvent_t ev = (cudaEvent_t)c->blk_ev;
  c->launches += 3;
  k_sumsq<<<dim3(blk, k), 256, 0, st>>>(c->BR, 3 * (size_t)N, 3 * N, c->Bpart);
  k_norm_fin<<<k, 32, 0, st>>>(c->Bpart, blk, c->Bsc);
  k_interleaved_to_soa<<<dim3((NTp + 255) / 256, k), 256, 0, st>>>(c->BR, 3 * (size_t)N, c->Bsc,
                                                                   c->BV, n, N, NTp);
  CU(cudaMemcpyAsync(c->Bvcur, c->BV, 8 * n * k, cudaMemcpyDeviceToDevice, st));
  if (c->BVs) {
    c->launches++;
    k_to_f32<<<592, 256, 0, st>>>(c->BV, c->BVs, n * k);
  }
  CU(cudaMemsetAsync(c->Bjd, 0, sizeof(int), st));
  std::vector<std::vector<double>> cc(k);
  std::vector<char> done(k, 0);
  std::vector<int> negs(k, 0);
  mr.assign(k, 0);
  conv.assign(k, 0);
  int ndone = 0, pending = 0, m = 0;
  int next_check = std::max(kTailSpan + 2, c->blk_last - 2);
  const double* ha = c->Bhost;
  const double* hb = c->Bhost + (size_t)L1 * k;
  // convergence of every open right-hand side at Krylov dimension mm, from the
  // alpha and beta copied after iteration mm.  Per right-hand side: the
  // changes at every checked dimension (dh), and the coefficients of the
  // previous check (clast at dimension mlast), reused as the m - 1 iterate
  // when the checks are consecutive (every iteration after the first check,
  // which solves the three dimensions below it as well)
  std::vector<std::vector<double>> clast(k), dh(k);
  std::vector<int> mlast(k, -1);
  auto evaluate = [&](int mm) -> int {
    CU(cudaEventSynchronize(ev));
    std::vector<int> open;
    for (int r = 0; r < k; r++)
      if (!done[r]) open.push_back(r);
    parallel_for((int)open.size(), [&](int q) {
      int r = open[q];
      std::vector<double> alpha(mm), beta(mm);
      for (int i = 0; i < mm; i++) {
        alpha[i] = ha[(size_t)i * k + r];
        beta[i] = hb[(size_t)i * k + r];
      }
      std::vector<double>& d = dh[r];
      d.resize(mm + 1, -1.0);
      std::vector<double> cm, cprev;
      int neg = sqrt_e1(alpha, beta, mm, cm, 0.5);
      if (mlast[r] == mm - 1) {
        cprev.swap(clast[r]);
      } else {
        // first check: the changes at mm - 1 .. mm - 6 as well
        std::vector<double> ca, cb;
        sqrt_e1(alpha, beta, mm - 1, cprev, 0.5);
        ca = cprev;
        for (int j = mm - 1; j >= std::max(2, mm - kTailSpan); j--) {
          sqrt_e1(alpha, beta, j - 1, cb, 0.5);
          d[j] = rel_change(ca, cb);
          ca.swap(cb);
        }
      }
      d[mm] = rel_change(cm, cprev);
      bool ok = tail_converged(d, mm, stop_tol(c, pre)) || beta[mm - 1] <= 1e-300;
      if (ok || mm >= c->lmax) {
        done[r] = 1;
        conv[r] = ok;
        mr[r] = mm;
        negs[r] = neg;
        cc[r].swap(cm);
      } else {
        clast[r].swap(cm);
        mlast[r] = mm;
      }
    });
    ndone = 0;
    for (int r = 0; r < k; r++) ndone += done[r];
    return BD_OK;
  };
  int j = 0;
  for (; j < c->lmax; j++) {
    s = block_iteration(c, k, pre);
    if (s != BD_OK) return s;
    m = j + 1;
    if (pending) {
      if ((s = evaluate(pending)) != BD_OK) return s;
      pending = 0;
      if (ndone == k) {
        j++;
        break;
      }
    }
    if (m >= next_check || m == c->lmax) {
      CU(cudaMemcpyAsync(c->Bhost, c->Bab, 8 * (size_t)m * k, cudaMemcpyDeviceToHost, st));
      CU(cudaMemcpyAsync(c->Bhost + (size_t)L1 * k, c->Bab + (size_t)L1 * k, 8 * (size_t)m * k,
                         cudaMemcpyDeviceToHost, st));
      CU(cudaEventRecord(ev, st));
      pending = m;
      next_check = m + 1;  // from the first check on, every iteration
    }
  }
  if (pending && (s = evaluate(pending)) != BD_OK) return s;
  std::vector<double> hc((size_t)k * L1, 0.0);
  int mmin = c->lmax;
  for (int r = 0; r < k; r++) {
    std::copy(cc[r].begin(), cc[r].end(), hc.begin() + (size_t)r * L1);
    mmin = std::min(mmin, mr[r]);
    c->lan_negative += negs[r];
  }
  CU(cudaMemcpyAsync(c->Bc, hc.data(), 8 * hc.size(), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(c->Bm, mr.data(), 4 * (size_t)k, cudaMemcpyHostToDevice, st));
  c->launches++;
  k_combo_m<<<dim3(blk, k), 256, 0, st>>>(c->BV, n * k, c->Bc, L1, c->Bm, c->Bsc, out, (int)n);
  c->blk_last = mmin;
  c->blk_runs++;
  c->blk_products += j;
  c->blk_rhs_products += (long long)j * k;
  if (iters_run) *iters_run = j;
  CU(cudaStreamSynchronize(st));  // hc and mr are read by the copies above
  return launch_ok(c);
}

// sqrt(M) z_r for the k noise draws at BR into BY (Lanczos layout, stride
// 3 NTp): the preconditioned solve G^-1 sqrt(G M G^T) z_r when a block
// preconditioner is set, with the plain single-vector solve for a right-hand
// side that misses the tolerance (a fallback, counted).
static int lanczos_sqrt_block(bd_ctx* c, int k) {
  int s;
  if (!c->hi_built) return BD_ERR_STATE;
  if ((s = alloc_lanczos(c)) != BD_OK) return s;
  if ((s = alloc_blocks(c)) != BD_OK) return s;
  if (k < 1 || k > c->nbk) return BD_ERR_ARG;
  if (k > 1 && (s = pme_multi_plan(c, k)) != BD_OK) return s;
  size_t n = 3 * (size_t)c->NT * 32;
  bool pre = c->pre_kind != BD_PRECOND_NONE && c->pre_ready;
  std::vector<int> mr;
  std::vector<char> conv;
  if ((s = lanczos_run_multi(c, k, pre, pre ? c->Bt1 : c->BY, mr, conv, nullptr)) != BD_OK)
    return s;
  if (pre) precond_apply_k(c, 2, k, c->Bt1, n, c->BY, n);
  for (int r = 0; r < k; r++) {
    c->lan_calls++;
    if (pre) {
      c->pre_calls++;
      c->pre_iters += mr[r];
      if (conv[r]) {
        c->lan_iters += mr[r];
        continue;
      }
      c->pre_fallbacks++;
      int m = 0;
      bool cv = false;
      if ((s = lanczos_run(c, c->BR + 3 * (size_t)c->N * r, false, false, 0.5, c->BY + n * r, &m,
                           &cv)) != BD_OK)
        return s;
      c->lan_iters += m;
      if (!cv) c->lan_maxed++;
    } else {
      c->lan_iters += mr[r];
      if (!conv[r]) c->lan_maxed++;
    }
  }
  return launch_ok(c);
}

// sqrt(M) z for the bead-interleaved z on the device (c->R): result in c->Yz.
// With with_force the first product also forms M F into c->MF.  With a block
// preconditioner G the result is G^(-1) sqrt(G M G^T) z; when that solve
// misses the tolerance within the Krylov cap the plain method recomputes the
// step (a fallback, counted).
int lanczos_sqrt(bd_ctx* c, const double* z, bool with_force, int* iters) {
  int s;
  if (!c->hi_built) return BD_ERR_STATE;
  if ((s = alloc_lanczos(c)) != BD_OK) return s;
  bool conv = false;
  int m = 0;
  if (c->pre_kind != BD_PRECOND_NONE && c->pre_ready) {
    if ((s = lanczos_run(c, z, with_force, true, 0.5, c->Lt1, &m, &conv)) != BD_OK) return s;
    c->pre_calls++;
    c->pre_iters += m;
    if (conv) {
      precond_apply(c, 2, c->Lt1, c->Yz);
      c->lan_calls++;
      c->lan_iters += m;
      if (iters) *iters = m;
      return launch_ok(c);
    }
    c->pre_fallbacks++;
  }
  if ((s = lanczos_run(c, z, with_force, false, 0.5, c->Yz, &m, &conv)) != BD_OK) return s;
  c->lan_calls++;
  c->lan_iters += m;
  if (!conv) c->lan_maxed++;
  if (iters) *iters = m;
  return BD_OK;
}

// A^(-1/2) z into out (Lanczos layout), A = M, or A = G M G^T when the
// segment preconditioner is active (the targets for learned blocks applied
// on top of it).
int lanczos_inv_sqrt(bd_ctx* c, const double* z, double* out, int* iters, bool* conv) {
  int s;
  if (!c->hi_built) return BD_ERR_STATE;
  if ((s = alloc_lanczos(c)) != BD_OK) return s;
  if (!out) return BD_ERR_ARG;
  bool pre = c->pre_kind == BD_PRECOND_SEGMENT && c->pre_ready;
  int keep = c->lan_last, keep_pre = c->pre_last;
  s = lanczos_run(c, z, false, pre, -0.5, out, iters, conv);
  c->lan_last = keep;
  c->pre_last = keep_pre;
  return s;
}

}  // namespace bd

extern "C" {

int bd_mobility_apply(bd_ctx* c, const double* v, double* out) {
  if (!c || !v || !out) return BD_ERR_ARG;
  if (!c->hi_built) return BD_ERR_STATE;
  int s;
  if ((s = alloc_lanczos(c)) != BD_OK) return s;
  int N = c->N, NTp = c->NT * 32;
  std::vector<double> soa(3 * (size_t)NTp, 0.0), res(3 * (size_t)NTp);
  for (int i = 0; i < N; i++)
    for (int a = 0; a < 3; a++) soa[(size_t)a * NTp + i] = v[3 * i + a];
  CU(cudaMemcpyAsync(c->Lw, soa.data(), 8 * soa.size(), cudaMemcpyHostToDevice, c->stream));
  VecIn vi = {{c->Lw, c->Lw + NTp, c->Lw + 2 * NTp}, 1};
  if ((s = sym_matvec(c, 1, vi, vi, c->Yz, c->Yz, true)) != BD_OK) return s;
  CU(cudaMemcpyAsync(res.data(), c->Yz, 8 * res.size(), cudaMemcpyDeviceToHost, c->stream));
  if ((s = check(c)) != BD_OK) return s;
  for (int i = 0; i < N; i++)
    for (int a = 0; a < 3; a++) out[3 * i + a] = res[(size_t)a * NTp + i];
  return BD_OK;
}

int bd_mobility_apply_block(bd_ctx* c, int k, const double* v, double* out) {
  if (!c || !v || !out || k < 1) return BD_ERR_ARG;
  if (!c->hi_built) return BD_ERR_STATE;
  if (!(c->p.mobility == BD_MOB_PME && k >= 2 && k <= c->nbk)) {
    for (int r = 0; r < k; r++) {
      int s = bd_mobility_apply(c, v + 3 * (size_t)r * c->N, out + 3 * (size_t)r * c->N);
      if (s != BD_OK) return s;
    }
    return BD_OK;
  }
  int s;
  if ((s = pme_multi_plan(c, k)) != BD_OK) return s;
  int N = c->N, NTp = c->NT * 32;
  size_t n = 3 * (size_t)NTp;
  std::vector<double> soa(n * k, 0.0), res(n * k);
  for (int r = 0; r < k; r++)
    for (int i = 0; i < N; i++)
      for (int a = 0; a < 3; a++) soa[r * n + (size_t)a * NTp + i] = v[(size_t)r * 3 * N + 3 * i + a];
  double *X = nullptr, *Y = nullptr;
  if (cudaMalloc(&X, 8 * n * k) != cudaSuccess || cudaMalloc(&Y, 8 * n * k) != cudaSuccess) {
    cudaGetLastError();  // not a sticky error: the next launch check must not see it
    cudaFree(X);
    return BD_ERR_OOM;
  }
  cudaError_t e = cudaMemcpyAsync(X, soa.data(), 8 * n * k, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    prof_begin(c, BD_PROF_BLOCK);  // the product alone, for timing (autotuner)
    s = pme_apply_multi(c, k, X, n, Y, n);
    prof_end(c, BD_PROF_BLOCK);
  } else {
    s = bd::cuda_fail((int)e, cudaGetErrorString(e), __FILE__, __LINE__);
  }
  if (s == BD_OK) {
    e = cudaMemcpyAsync(res.data(), Y, 8 * n * k, cudaMemcpyDeviceToHost, c->stream);
    s = e == cudaSuccess ? check(c)
                         : bd::cuda_fail((int)e, cudaGetErrorString(e), __FILE__, __LINE__);
  }
  cudaStreamSynchronize(c->stream);
  cudaFree(X);
  cudaFree(Y);
  if (s != BD_OK) return s;
  for (int r = 0; r < k; r++)
    for (int i = 0; i < N; i++)
      for (int a = 0; a < 3; a++) out[(size_t)r * 3 * N + 3 * i + a] = res[r * n + (size_t)a * NTp + i];
  return BD_OK;
}

int bd_lanczos_sqrt(bd_ctx* c, const double* z, double* out, int* iters) {
  if (!c || !z || !out) return BD_ERR_ARG;
  int s;
  CU(cudaMemcpyAsync(c->R, z, 24 * (size_t)c->N, cudaMemcpyHostToDevice, c->stream));
  if ((s = lanczos_sqrt(c, c->R, false, iters)) != BD_OK) return s;
  int N = c->N, NTp = c->NT * 32;
  std::vector<double> res(3 * (size_t)NTp);
  CU(cudaMemcpyAsync(res.data(), c->Yz, 8 * res.size(), cudaMemcpyDeviceToHost, c->stream));
  if ((s = check(c)) != BD_OK) return s;
  for (int i = 0; i < N; i++)
    for (int a = 0; a < 3; a++) out[3 * i + a] = res[(size_t)a * NTp + i];
  return BD_OK;
}

int bd_lanczos_inv_sqrt(bd_ctx* c, const double* z, double* out, int* iters) {
  if (!c || !z || !out) return BD_ERR_ARG;
  int s;
  bool conv = false;
  if (!c->hi_built) return BD_ERR_STATE;
  // the work vectors exist only after the first allocation; Lt2 is read below
  if ((s = alloc_lanczos(c)) != BD_OK) return s;
  CU(cudaMemcpyAsync(c->R, z, 24 * (size_t)c->N, cudaMemcpyHostToDevice, c->stream));
  if ((s = lanczos_inv_sqrt(c, c->R, c->Lt2, iters, &conv)) != BD_OK) return s;
  int N = c->N, NTp = c->NT * 32;
  std::vector<double> res(3 * (size_t)NTp);
  CU(cudaMemcpyAsync(res.data(), c->Lt2, 8 * res.size(), cudaMemcpyDeviceToHost, c->stream));
  if ((s = check(c)) != BD_OK) return s;
  for (int i = 0; i < N; i++)
    for (int a = 0; a < 3; a++) out[3 * i + a] = res[(size_t)a * NTp + i];
  return conv ? BD_OK : BD_ERR_LANCZOS;
}

int bd_noise_block_release(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  noise_blocks_release(c);
  return launch_ok(c);
}

int bd_noise_block_stats(bd_ctx* c, long* o) {
  if (!c || !o) return BD_ERR_ARG;
  o[0] = (long)c->blk_runs;
  o[1] = (long)c->blk_products;
  o[2] = (long)c->blk_rhs_products;
  return BD_OK;
}

int bd_lanczos_stats(bd_ctx* c, long* o) {
  if (!c || !o) return BD_ERR_ARG;
  o[0] = (long)c->lan_calls;
  o[1] = (long)c->lan_iters;
  o[2] = (long)c->lan_maxed;
  o[3] = (long)c->lan_negative;
  return BD_OK;
}

// Steps from t covered by one noise block: at most the block capacity, none
// past the next mobility rebuild, and with the reference's ran1 noise and
// sequential hop (one generator) none past the next charge-hop sweep, so that
// every draw happens in the per-step order.  A block may outlive the call that
// made it (a caller stepping one step at a time still gets blocks).
static int block_len(bd_ctx* c, unsigned long t, int with_hop) {
  unsigned long kb = (unsigned long)c->nbk;
  unsigned long sr = (unsigned long)c->srpy;
  kb = std::min(kb, (t / sr + 1) * sr - t);
  if (c->tstart > t) kb = std::min(kb, c->tstart - t);
  if (with_hop && c->nch > 0 && c->p.noise == BD_NOISE_RAN1 && c->p.hop == BD_HOP_SEQUENTIAL) {
    unsigned long ms = (unsigned long)c->p.MStep;
    unsigned long th = (t + ms - 1) / ms * ms;  // next sweep at or after t
    kb = std::min(kb, th - t + 1);
  }
  return (int)std::max(1ul, kb);
}

int bd_step_lanczos(bd_ctx* c, unsigned long t0, int nsteps, int with_hop) {
  if (!c || nsteps < 0) return BD_ERR_ARG;
  int s;
  with_hop = with_hop != 0;
  bool ext = c->p.flow == BD_FLOW_EXT;
  bool blocks = c->nbk > 1;
  size_t nl = 3 * (size_t)c->NT * 32;
  prof_begin(c, BD_PROF_STEP);
  for (int n = 0; n < nsteps; n++) {
    unsigned long t = t0 + (unsigned long)n;
    c->t = t;
    if ((s = bd_reset_force(c))) return s;
    c->strain = (double)t * c->p.dt * c->p.edot;
    host_lattice(c, t, &c->lat);
    if (ext && (s = bd_transform_coords(c))) return s;
    if ((s = bd_apply_pbc(c))) return s;
    if ((s = build_neighbors(c, false))) return s;
    prof_begin(c, BD_PROF_FORCES);
    if ((s = bd_bond_force(c))) return s;
    if ((s = bd_ev_force(c))) return s;
    if ((s = bd_coulomb_force(c))) return s;
    prof_end(c, BD_PROF_FORCES);
    const double* Y = nullptr;  // this step's sqrt(M) z (the solve allocates its buffers)
    if (!blocks) {
      noise_blocks_release(c);
      if ((s = draw_noise(c, c->R))) return s;
      if (t % (unsigned long)c->srpy == 0 || t == c->tstart || !c->hi_built)
        if ((s = calc_hi(c))) return s;
      if (ext) rotate_coords(c, 1);
      if ((s = lanczos_sqrt(c, c->R, true, nullptr))) return s;
      Y = c->Yz;
    } else {
      if (t % (unsigned long)c->srpy == 0 || t == c->tstart || !c->hi_built)
        if ((s = calc_hi(c))) return s;
      bool have = c->blk_n > 0 && c->blk_next < c->blk_n &&
                  t == c->blk_t0 + (unsigned long)c->blk_next && c->blk_hiv == c->hi_version &&
                  c->blk_hop == with_hop;
      if (!have) {
        // the draws of the block's steps, in step order, and their displacements
        noise_blocks_release(c);
        if ((s = alloc_lanczos(c)) != BD_OK || (s = alloc_blocks(c)) != BD_OK) return s;
        int kb = block_len(c, t, with_hop);
        c->blk_draw0 = c->noise_draws;
        for (int r = 0; r < kb; r++) {
          if (c->p.noise != BD_NOISE_PHILOX)
            CU(cudaMemcpyAsync((Ran1*)c->Brng + r, c->rng, sizeof(Ran1),
                               cudaMemcpyDeviceToDevice, c->stream));
          if ((s = draw_noise(c, c->BR + 3 * (size_t)c->N * r))) return s;
        }
        c->blk_t0 = t;
        c->blk_n = kb;
        c->blk_next = 0;
        c->blk_hiv = c->hi_version;
        c->blk_hop = with_hop;
        if ((s = lanczos_sqrt_block(c, kb))) {
          c->blk_n = 0;
          return s;
        }
      }
      int r = c->blk_next++;
      // this step's draw stays readable as the context's noise vector
      CU(cudaMemcpyAsync(c->R, c->BR + 3 * (size_t)c->N * r, 24 * (size_t)c->N,
                         cudaMemcpyDeviceToDevice, c->stream));
      if (ext) rotate_coords(c, 1);
      VecIn vf = {{c->fx, c->fy, c->fz}, 1};
      if ((s = sym_matvec(c, 1, vf, vf, c->MF, c->MF, true)) != BD_OK) return s;
      Y = c->BY + nl * r;
    }
    if (!Y || !c->MF) return BD_ERR_STATE;
    c->launches++;
    k_krylov_update<<<(c->N + 255) / 256, 256, 0, c->stream>>>(
        c->p.flow, c->rx, c->ry, c->rz, c->dxv, c->dyv, c->dzv, c->MF, Y, c->NT * 32, c->N,
        c->p.dt, c->p.edot, sqrt(2.0 * c->p.dt));
    if ((s = launch_ok(c)) != BD_OK) return s;
    if (with_hop && c->nch > 0 && t % (unsigned long)c->p.MStep == 0) {
      if (ext && (s = bd_transform_coords(c))) return s;
      if ((s = charge_hop(c))) return s;
      if (ext && (s = bd_inverse_coords(c))) return s;
    }
  }
  prof_end(c, BD_PROF_STEP);
  return check(c);
}

}  // extern "C"
