// Matrix-free Rotne-Prager-Yamakawa mobility by smooth particle-mesh Ewald.
//
// No counterpart in the reference, whose mobility is a dense 3N x 3N matrix
// (calcHI, shear/src/main26.c:1530-1806).  It uses the same Beenakker Ewald
// split as calcHI, M = M_real + M_self + M_recip:
//  * M_real: for pairs closer than rc (lattice minimum image, rc below half
//    the narrowest cell width) the real-space Beenakker kernel with the
//    overlap form for r <= 2 (the C1..C4 terms of shear/src/main26.c:
//    1727-1741); the 3x3 pair tensors are built once per step into a row
//    list and applied as a sparse block product;
//  * M_self: 1 - 6 alpha/sqrt(pi) + 40 alpha^3/(3 sqrt(pi)) on the diagonal;
//  * M_recip = sum over k != 0 of (phi(k)/V)(I - k k^T/k^2) cos(k.r_ij),
//    phi(k) = (1 - k^2/3)(1 + k^2/4a^2 + k^4/8a^4)(6 pi/k^2) exp(-k^2/4a^2)
//    (the coefficient of shear/src/main26.c:1622), evaluated by smooth PME
//    (Essmann et al., J. Chem. Phys. 103, 8577 (1995)) on the deforming
//    cell: fractional coordinates s = H^-1 r, cardinal B-splines of even
//    order p on a K^3 grid, three-component R2C FFT, multiplication by
//    (phi/V)(I - k k^T/k^2) |b1 b2 b3|^2 with k = 2 pi H^-T m, C2R FFT and
//    interpolation with the same weights.
// The periodic lattice is described by its Gauss-reduced basis (shortest
// vectors of the lattice spanned by L1, L2 and L e_z): the lattice sums do
// not depend on the basis, and the reduced one keeps the grid spacing and the
// minimum-image cell widths bounded over the whole deformation period
// (|a| <= 1.16 L, widths >= 0.86 L for planar extension).
// Two conventions of calcHI are kept so that the sum reproduces its tensor:
//  * for overlapping beads (r < 2) its real-space form depends on the split
//    parameter; those pairs get that dependence at calcHI's own parameter
//    M_HI / rce (shear/src/main26.c:1536-1552) rather than at the PME one;
//  * calcHI stores only the diagonal entries of the self blocks
//    (shear/src/main26.c:1663-1700); the off-diagonal entries of the k-space
//    self sum, which a sheared or stretched cell makes non-zero, are removed.
// cuFFT is used for the transforms only.  Spreading uses atomics in the grid
// precision; several right-hand sides share each launch (blockIdx.y).  The
// spline weights and pair tensors are computed once per step because the
// positions do not change during a Krylov solve.
#include <cufft.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bd_ctx.cuh"
#include "bd_cell.cuh"

using namespace bd;

#define CU(call) BD_CU(call)
#define CF(call) BD_CF(call)

// Per bead: base grid index floor(u) and the p weights in each lattice
// direction (u = K s, s wrapped into [0,1)).  Positions held in the rotated
// frame are taken to the lab frame with (cr, sr) = (cos, sin) of the lattice
// angle, x = x' cr - y' sr, y = x' sr + y' cr (inverseCoords,
// extensional/src/main14.c:1525-1535); lab-frame positions pass (1, 0).
__global__ void k_pme_weights(Cell cell, const double* __restrict__ rx,
                              const double* __restrict__ ry, const double* __restrict__ rz,
                              double cr, double sr, int N, int K, int p, int* base, double* w,
                              double4* pos, int* err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double x = rx[i] * cr - ry[i] * sr, y = rx[i] * sr + ry[i] * cr, z = rz[i];
  pos[i] = make_double4(x, y, z, 0.0);
  double s[3];
  frac_of(cell, x, y, z, s);
  for (int d = 0; d < 3; d++) {
    double sd = s[d] - floor(s[d]);
    double u = sd * K;
    if (!(u >= 0.0 && u <= (double)K)) {  // non-finite position: keep indices in range
      u = 0.0;
      atomicOr(err, ERRB_NONFINITE);
    }
    int fl = (int)floor(u);
    double f = u - fl;
    if (fl >= K) fl -= K;
    base[3 * i + d] = fl;
    bspline(f, p, w + ((size_t)3 * i + d) * kMaxOrder);
  }
}

// FP32 grids: the spread skips stencil points whose weight W_i(g) is below
// 1e-9 (for order 8, 35 % of the 512 points, carrying at most 2.7e-8 of the
// stencil's unit weight, mean 1.4e-8: below FP32 rounding, 6e-8, and two
// orders below the particle-mesh error), saving their atomics; the
// interpolation keeps every point (skipping there only added divergence), so
// the product is symmetric to ~3e-8, inside the rounding of its FP32 grids.
// (1e-8 would skip 42 % but drop up to 3e-7 of the weight, the size of the
// FP32 storage error itself.)  The FP64 path keeps every point.
constexpr double kSkipWeight = 1e-9;

// Q_r[c][g] += v_r,c(i) W_i(g) for the right-hand sides r0 .. r0 + kc - 1
// of chunk blockIdx.y (r0 = KS blockIdx.y; KS = 1 for single products): one
// warp per bead, the P^3 stencil points spread over the lanes with the
// fastest index along the contiguous grid direction, so each atomic
// instruction of a warp covers runs of P adjacent grid values; the weights
// and the bead's values are loaded once for the chunk.  Right-hand side r
// reads its vector vr entries further on and owns the grids 3 K^3 entries
// further on.

template <int P, typename R, int KS>
__global__ void __launch_bounds__(256) k_pme_spread(const int* __restrict__ base,
                                                    const double* __restrict__ w, int N, int K,
                                                    VecIn v, size_t vr, int k, R* grid) {
  int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  int r0 = KS * blockIdx.y, kc = min(KS, k - r0);
  size_t K3 = (size_t)K * K * K;
  R f[3 * KS];
#pragma unroll
  for (int r = 0; r < KS; r++) {
    size_t o = (size_t)(r0 + (r < kc ? r : 0)) * vr + (size_t)i * v.stride;
    f[3 * r] = (R)v.p[0][o];
    f[3 * r + 1] = (R)v.p[1][o];
    f[3 * r + 2] = (R)v.p[2][o];
  }
  R* g0p = grid + (size_t)r0 * 3 * K3;
  const double* w0 = w + ((size_t)3 * i + 0) * kMaxOrder;
  const double* w1 = w + ((size_t)3 * i + 1) * kMaxOrder;
  const double* w2 = w + ((size_t)3 * i + 2) * kMaxOrder;
  int b0 = base[3 * i], b1 = base[3 * i + 1], b2 = base[3 * i + 2];
  // fully unrolled: the stencil index of each lane is a compile-time
  // function of the iteration, so the weights stay in registers
#pragma unroll
  for (int it = 0; it < (P * P * P + 31) / 32; it++) {
    int q = lane + 32 * it;
    if (q >= P * P * P) break;
    int c = q % P, b = (q / P) % P, a = q / (P * P);
    int g0 = b0 - a, g1 = b1 - b, g2 = b2 - c;
    g0 += g0 < 0 ? K : 0;
    g1 += g1 < 0 ? K : 0;
    g2 += g2 < 0 ? K : 0;
    double wt = w0[a] * w1[b] * w2[c];
    if (sizeof(R) == 4 && wt < kSkipWeight) continue;  // FP32: negligible corner
    R wr = (R)wt;
    size_t g = ((size_t)g0 * K + g1) * K + g2;
#pragma unroll
    for (int r = 0; r < KS; r++) {
      if (r >= kc) break;
      R* gr = g0p + (size_t)r * 3 * K3 + g;
      if constexpr (sizeof(R) == 8) {
        atomicAdd(gr, wt * f[3 * r]);
        atomicAdd(gr + K3, wt * f[3 * r + 1]);
        atomicAdd(gr + 2 * K3, wt * f[3 * r + 2]);
      } else {
        atomicAdd(gr, wr * f[3 * r]);
        atomicAdd(gr + K3, wr * f[3 * r + 1]);
        atomicAdd(gr + 2 * K3, wr * f[3 * r + 2]);
      }
    }
  }
}

// Products of k >= 2 right-hand sides pack them in pairs: right-hand sides
// 2p and 2p + 1 are the real and imaginary parts of one complex grid per
// component (pair p, component c at (3 p + c) K^3).  The influence tensor is
// real and even in k, so one complex transform, the multiplication and the
// inverse transform give both products, with no unpacking: spreading takes
// one float2 atomic per pair and grid point, interpolation one float2 load,
// and the transforms are contiguous C2C batches.
template <typename R>
struct Pair;
template <>
struct Pair<float> {
  using T = float2;
};
template <>
struct Pair<double> {
  using T = double2;
};

// With vpk (FP32), lanes 0..7 of a bead's warp also store the pair's six
// input values (plus two zeros) at vpk[(p N + i) 8], for the real-space sums
// to read as a float4 and a float2.
template <int P, typename R>
__global__ void __launch_bounds__(256) k_pme_spread_pairs(const int* __restrict__ base,
                                                          const double* __restrict__ w, int N,
                                                          int K, VecIn v, size_t vr, int k,
                                                          typename Pair<R>::T* cgrid,
                                                          float* vpk) {
  using C2 = typename Pair<R>::T;
  int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  int pr = blockIdx.y, ra = 2 * pr, rb = 2 * pr + 1;
  size_t K3 = (size_t)K * K * K;
  size_t oa = (size_t)ra * vr + (size_t)i * v.stride;
  size_t ob = (size_t)(rb < k ? rb : ra) * vr + (size_t)i * v.stride;
  R fb_on = rb < k ? (R)1 : (R)0;
  R fa0 = (R)v.p[0][oa], fa1 = (R)v.p[1][oa], fa2 = (R)v.p[2][oa];
  R fb0 = fb_on * (R)v.p[0][ob], fb1 = fb_on * (R)v.p[1][ob], fb2 = fb_on * (R)v.p[2][ob];
  if (vpk && lane < 8) {
    R x = lane == 0 ? fa0 : lane == 1 ? fa1 : lane == 2 ? fa2
        : lane == 3 ? fb0 : lane == 4 ? fb1 : lane == 5 ? fb2 : (R)0;
    vpk[((size_t)pr * N + i) * 8 + lane] = (float)x;
  }
  C2* gp = cgrid + (size_t)pr * 3 * K3;
  const double* w0 = w + ((size_t)3 * i + 0) * kMaxOrder;
  const double* w1 = w + ((size_t)3 * i + 1) * kMaxOrder;
  const double* w2 = w + ((size_t)3 * i + 2) * kMaxOrder;
  int b0 = base[3 * i], b1 = base[3 * i + 1], b2 = base[3 * i + 2];
#pragma unroll
  for (int it = 0; it < (P * P * P + 31) / 32; it++) {
    int q = lane + 32 * it;
    if (q >= P * P * P) break;
    int c = q % P, b = (q / P) % P, a = q / (P * P);
    int g0 = b0 - a, g1 = b1 - b, g2 = b2 - c;
    g0 += g0 < 0 ? K : 0;
    g1 += g1 < 0 ? K : 0;
    g2 += g2 < 0 ? K : 0;
    double wt = w0[a] * w1[b] * w2[c];
    if (sizeof(R) == 4 && wt < kSkipWeight) continue;  // FP32: negligible corner
    size_t g = ((size_t)g0 * K + g1) * K + g2;
    if constexpr (sizeof(R) == 4) {
      float wr = (float)wt;
      atomicAdd(gp + g, make_float2(wr * fa0, wr * fb0));
      atomicAdd(gp + K3 + g, make_float2(wr * fa1, wr * fb1));
      atomicAdd(gp + 2 * K3 + g, make_float2(wr * fa2, wr * fb2));
    } else {
      atomicAdd(&gp[g].x, wt * fa0);
      atomicAdd(&gp[g].y, wt * fb0);
      atomicAdd(&gp[K3 + g].x, wt * fa1);
      atomicAdd(&gp[K3 + g].y, wt * fb1);
      atomicAdd(&gp[2 * K3 + g].x, wt * fa2);
      atomicAdd(&gp[2 * K3 + g].y, wt * fb2);
    }
  }
}

// The influence tensor on the full spectrum of the packed pairs (thread per
// point and pair): points with m2 > K/2 take the tensor of their mirror -m,
// stored in the half spectrum (the tensor is even in k; on the Nyquist planes
// of an even K the stored pairs differ in the sign of off-diagonal entries,
// where the influence is below 1e-14 of its peak).
template <typename R, typename Cx>
__global__ void k_pme_apply_influence_full(const R* __restrict__ infl, Cx* cgrid, int K,
                                           size_t np3) {
  size_t K3 = (size_t)K * K * K;
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= K3 * np3) return;
  size_t m = e % K3, pc = e / K3;  // pair index (components 3 apart)
  int Kh = K / 2 + 1;
  int m0 = (int)(m / ((size_t)K * K)), m1 = (int)((m / K) % K), m2 = (int)(m % K);
  if (m2 > K / 2) {
    m0 = (K - m0) % K;
    m1 = (K - m1) % K;
    m2 = K - m2;
  }
  const R* t = infl + 6 * (((size_t)m0 * K + m1) * Kh + m2);
  Cx* b = cgrid + pc * 3 * K3 + m;
  Cx x = b[0], y = b[K3], z = b[2 * K3];
  Cx u, v, ww;
  u.x = t[0] * x.x + t[1] * y.x + t[2] * z.x;
  u.y = t[0] * x.y + t[1] * y.y + t[2] * z.y;
  v.x = t[1] * x.x + t[3] * y.x + t[4] * z.x;
  v.y = t[1] * x.y + t[3] * y.y + t[4] * z.y;
  ww.x = t[2] * x.x + t[4] * y.x + t[5] * z.x;
  ww.y = t[2] * x.y + t[4] * y.y + t[5] * z.y;
  b[0] = u;
  b[K3] = v;
  b[2 * K3] = ww;
}

// Influence tensor on the half spectrum: (phi(k)/V)(I - k k^T/k^2) |b|^2,
// six components per point, zero at m = 0.
// Also the off-diagonal entries of sum_{k != 0} (phi/V)(I - k k^T/k^2) over
// the full spectrum (half spectrum with Hermitian multiplicity), one partial
// sum per block in soff_part[3 * block + (xy, xz, yz)].
template <typename R>
__global__ void __launch_bounds__(256) k_pme_influence(Cell cell, int K, double alpha,
                                                       const double* __restrict__ bsq, R* infl,
                                                       double* soff_part) {
  int Kh = K / 2 + 1;
  size_t n = (size_t)K * K * Kh;
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double sxy = 0, sxz = 0, syz = 0;
  __shared__ double red[3][256];
  if (e < n) {
    int m2 = (int)(e % Kh), m1 = (int)((e / Kh) % K), m0 = (int)(e / ((size_t)Kh * K));
    R* o = infl + 6 * e;
    if (m0 == 0 && m1 == 0 && m2 == 0) {
      for (int a = 0; a < 6; a++) o[a] = (R)0;
    } else {
      int s0 = m0 < (K + 1) / 2 ? m0 : m0 - K, s1 = m1 < (K + 1) / 2 ? m1 : m1 - K, s2 = m2;
      // k = 2 pi (s0 b0 + s1 b1 + s2 b2), b_d = row d of H^-1
      double k[3];
      for (int a = 0; a < 3; a++)
        k[a] = 2.0 * M_PI *
               (s0 * cell.Hi[0 * 3 + a] + s1 * cell.Hi[1 * 3 + a] + s2 * cell.Hi[2 * 3 + a]);
      double kk = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
      double a2 = alpha * alpha;
      double phi = (1.0 - kk / 3.0) * (1.0 + kk / (4.0 * a2) + kk * kk / (8.0 * a2 * a2)) * 6.0 *
                   M_PI / kk * exp(-kk / (4.0 * a2)) / cell.V;
      double f = phi * bsq[m0] * bsq[K + m1] * bsq[2 * K + m2];
      o[0] = (R)(f * (1.0 - k[0] * k[0] / kk));
      o[1] = (R)(f * (-k[0] * k[1] / kk));
      o[2] = (R)(f * (-k[0] * k[2] / kk));
      o[3] = (R)(f * (1.0 - k[1] * k[1] / kk));
      o[4] = (R)(f * (-k[1] * k[2] / kk));
      o[5] = (R)(f * (1.0 - k[2] * k[2] / kk));
      double mult = (m2 == 0 || (K % 2 == 0 && m2 == K / 2)) ? 1.0 : 2.0;
      sxy = -mult * phi * k[0] * k[1] / kk;
      sxz = -mult * phi * k[0] * k[2] / kk;
      syz = -mult * phi * k[1] * k[2] / kk;
    }
  }
  red[0][threadIdx.x] = sxy;
  red[1][threadIdx.x] = sxz;
  red[2][threadIdx.x] = syz;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int a = 0; a < 3; a++) red[a][threadIdx.x] += red[a][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 3) soff_part[3 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

// Fixed-order sum of the per-block self off-diagonal partials.
__global__ void k_pme_soff_fin(const double* __restrict__ part, int nb, double* soff) {
  __shared__ double red[3][256];
  double a0 = 0, a1 = 0, a2 = 0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    a0 += part[3 * b];
    a1 += part[3 * b + 1];
    a2 += part[3 * b + 2];
  }
  red[0][threadIdx.x] = a0;
  red[1][threadIdx.x] = a1;
  red[2][threadIdx.x] = a2;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int a = 0; a < 3; a++) red[a][threadIdx.x] += red[a][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 3) soff[threadIdx.x] = red[threadIdx.x][0];
}

// Right-hand side blockIdx.y owns the spectra 3 n entries further on.
template <typename R, typename Cx>
__global__ void k_pme_apply_influence(const R* __restrict__ infl, Cx* spec, size_t n) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  spec += (size_t)blockIdx.y * 3 * n;
  const R* t = infl + 6 * e;
  Cx x = spec[e], y = spec[n + e], z = spec[2 * n + e];
  Cx u, v, w;
  u.x = t[0] * x.x + t[1] * y.x + t[2] * z.x;
  u.y = t[0] * x.y + t[1] * y.y + t[2] * z.y;
  v.x = t[1] * x.x + t[3] * y.x + t[4] * z.x;
  v.y = t[1] * x.y + t[3] * y.y + t[4] * z.y;
  w.x = t[2] * x.x + t[4] * y.x + t[5] * z.x;
  w.y = t[2] * x.y + t[4] * y.y + t[5] * z.y;
  spec[e] = u;
  spec[n + e] = v;
  spec[2 * n + e] = w;
}

// Real-space Beenakker kernel t1 I + t2 r r^T/r^2 (shear/src/main26.c:
// 1727-1741) at split parameter alpha; with far the r > 2 form at any r.
__device__ __forceinline__ void real_kernel(double alpha, double rr, bool far, double& t1,
                                            double& t2) {
  double r = sqrt(rr), a = alpha, a2 = a * a, a3 = a2 * a, a5 = a3 * a2, a7 = a5 * a2;
  double C1, C2, C3, C4;
  if (far || r > 2.0) {
    C1 = 0.75 / r + 0.5 / (r * rr);
    C2 = 4.0 * a7 * rr * rr + 3.0 * a3 * rr - 20.0 * a5 * rr - 4.5 * a + 14.0 * a3 + a / rr;
    C3 = 0.75 / r - 1.5 / (r * rr);
    C4 = -4.0 * a7 * rr * rr - 3.0 * a3 * rr + 16.0 * a5 * rr + 1.5 * a - 2.0 * a3 - 3.0 * a / rr;
  } else {
    C1 = 1.0 - 0.28125 * r;
    C2 = 64.0 * a7 + 12.0 * a3 - 80.0 * a5 - 4.5 * a + 14.0 * a3 + 0.25 * a;
    C3 = 0.09375 * r;
    C4 = -64.0 * a7 - 12.0 * a3 + 64.0 * a5 + 1.5 * a - 2.0 * a3 - 0.75 * a;
  }
  double ec = erfc(a * r), ex = exp(-a2 * rr) / sqrt(M_PI);
  t1 = C1 * ec + C2 * ex;
  t2 = C3 * ec + C4 * ex;
}

// The overlap branch (bonded and touching beads), kept out of line.
__device__ __noinline__ void overlap_terms(double alpha, double alpha_ref, double rr,
                                           double* t) {
  double f1, f2, o1, o2, g1, g2;
  real_kernel(alpha, rr, true, f1, f2);
  real_kernel(alpha_ref, rr, false, o1, o2);
  real_kernel(alpha_ref, rr, true, g1, g2);
  t[0] = f1 + (o1 - g1);
  t[1] = f2 + (o2 - g2);
}

// t1, t2 of the real-space pair tensor at split alpha, with calcHI's overlap
// convention for r < 2 (the far form at alpha plus the overlap correction at
// its own split parameter alpha_ref).
__device__ __forceinline__ void pair_terms(double alpha, double alpha_ref, double rr, double& t1,
                                           double& t2) {
  if (rr < 4.0) {
    double t[2];
    overlap_terms(alpha, alpha_ref, rr, t);
    t1 = t[0];
    t2 = t[1];
  } else {
    real_kernel(alpha, rr, false, t1, t2);
  }
}

// out_r,c(i) = sum_g W_i(g) grid_r,c(g) + self v_r,c(i) - (S_off v_r(i))_c
//              + sum_j (T_ij v_r,j)_c (row list)
// for the right-hand sides r0 .. r0 + kc - 1 of chunk blockIdx.y (r0 =
// KG blockIdx.y; KG = 1 for single products).  One warp per bead: the lanes
// share the stencil points (weights computed once for the chunk) and the pair
// row (pair terms, positions and minimum image once for the chunk), then a
// butterfly reduction; lane e < 3 kc writes component e % 3 of right-hand
// side r0 + e / 3.
template <int P, typename R, int KG, bool PK, bool RS = false>
__global__ void __launch_bounds__(256) k_pme_gather(
    const int* __restrict__ base, const double* __restrict__ w, int N, int K,
    const R* __restrict__ grid, int k, double self, const double* __restrict__ soff, VecIn v,
    size_t vr, const int* __restrict__ rcnt, const int* __restrict__ rrows,
    const double4* __restrict__ pos, Cell cell, const R* __restrict__ tt, int rcap,
    double* o0, double* o1, double* o2, int ostride, size_t orr,
    const double* __restrict__ rsum) {
  constexpr int NA = 3 * KG;
  int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  int r0 = KG * blockIdx.y, kc = min(KG, k - r0), nj = 3 * kc;
  size_t K3 = (size_t)K * K * K;
  const R* gbase = grid + (size_t)r0 * 3 * K3;
  const double* w0 = w + ((size_t)3 * i + 0) * kMaxOrder;
  const double* w1 = w + ((size_t)3 * i + 1) * kMaxOrder;
  const double* w2 = w + ((size_t)3 * i + 2) * kMaxOrder;
  int b0 = base[3 * i], b1 = base[3 * i + 1], b2 = base[3 * i + 2];
  double u[NA];
#pragma unroll
  for (int e = 0; e < NA; e++) u[e] = 0.0;
#pragma unroll
  for (int it = 0; it < (P * P * P + 31) / 32; it++) {
    int q = lane + 32 * it;
    if (q >= P * P * P) break;
    int c = q % P, b = (q / P) % P, a = q / (P * P);
    int g0 = b0 - a, g1 = b1 - b, g2 = b2 - c;
    g0 += g0 < 0 ? K : 0;
    g1 += g1 < 0 ? K : 0;
    g2 += g2 < 0 ? K : 0;
    double wt = w0[a] * w1[b] * w2[c];
    const R* gp = gbase + ((size_t)g0 * K + g1) * K + g2;
    if constexpr (PK) {
      // packed pair blockIdx.y: right-hand sides r0, r0 + 1 as real and
      // imaginary parts (the grid argument is the pairs' complex grid)
      using C2 = typename Pair<R>::T;
      const C2* gq = (const C2*)grid + (size_t)blockIdx.y * 3 * K3 +
                     (((size_t)g0 * K + g1) * K + g2);
      C2 x0 = gq[0], x1 = gq[K3], x2 = gq[2 * K3];
      u[0] += wt * (double)x0.x;
      u[1] += wt * (double)x1.x;
      u[2] += wt * (double)x2.x;
      u[3] += wt * (double)x0.y;
      u[4] += wt * (double)x1.y;
      u[5] += wt * (double)x2.y;
    } else {
#pragma unroll
      for (int r = 0; r < KG; r++) {
        if (r >= kc) break;
        const R* gr = gp + (size_t)r * 3 * K3;
        u[3 * r] += wt * (double)gr[0];
        u[3 * r + 1] += wt * (double)gr[K3];
        u[3 * r + 2] += wt * (double)gr[2 * K3];
      }
    }
  }
  // real-space pairs: the tensor t1 I + t2 d d^T/r^2 of the minimum-image
  // displacement d; t1 and t2/r^2 are stored per pair (8 or 16 bytes), d is
  // recomputed from the frozen lab-frame positions (L2-resident)
  int n = rcnt[i];
  const int* prow = rrows + (size_t)i * rcap;
  // the cell is (b1, b2) in the xy plane and L e_z: a 2 x 2 block and L
  double4 pi = pos[i];
  const double h00 = cell.H[0], h01 = cell.H[1], h10 = cell.H[3], h11 = cell.H[4];
  const double g00 = cell.Hi[0], g01 = cell.Hi[1], g10 = cell.Hi[3], g11 = cell.Hi[4];
  const double Lz = cell.H[8], iLz = cell.Hi[8];
  if constexpr (RS) {
    // the real-space sums of this packed pair, formed for all pairs at once
    // by k_pme_real_pairs (added below)
  } else {
    for (int kk = lane; kk < n; kk += 32) {
      int j = prow[kk];
      double4 pj = pos[j];
      double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
      double s0 = g00 * dx + g01 * dy, s1 = g10 * dx + g11 * dy, s2 = iLz * dz;
      s0 -= rint(s0);
      s1 -= rint(s1);
      s2 -= rint(s2);
      dx = h00 * s0 + h01 * s1;
      dy = h10 * s0 + h11 * s1;
      dz = Lz * s2;
      const R* tk = tt + 2 * ((size_t)i * rcap + kk);
      double t1 = tk[0], t2r = tk[1];  // t1 and t2 / r^2 of the pair
#pragma unroll
      for (int r = 0; r < KG; r++) {
        if (r >= kc) break;
        size_t o = (size_t)(r0 + r) * vr + (size_t)j * v.stride;
        double x0 = v.p[0][o], x1 = v.p[1][o], x2 = v.p[2][o];
        double qq = t2r * (dx * x0 + dy * x1 + dz * x2);
        u[3 * r] += t1 * x0 + qq * dx;
        u[3 * r + 1] += t1 * x1 + qq * dy;
        u[3 * r + 2] += t1 * x2 + qq * dz;
      }
    }
  }

#pragma unroll
  for (int e = 0; e < NA; e++) {
    if (e >= nj) break;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) u[e] += __shfl_xor_sync(0xffffffffu, u[e], o);
  }
  double mine = 0.0;
#pragma unroll
  for (int e = 0; e < NA; e++)
    if (e == lane) mine = u[e];
  if constexpr (RS)
    if (lane < nj) mine += rsum[((size_t)blockIdx.y * N + i) * 6 + lane];
  if (lane < nj) {
    int r = lane / 3, c = lane % 3;
    size_t o = (size_t)(r0 + r) * vr + (size_t)i * v.stride;
    double vi0 = v.p[0][o], vi1 = v.p[1][o], vi2 = v.p[2][o];
    double sxy = soff[0], sxz = soff[1], syz = soff[2];
    double out;
    if (c == 0)
      out = mine + self * vi0 - sxy * vi1 - sxz * vi2;
    else if (c == 1)
      out = mine + self * vi1 - sxy * vi0 - syz * vi2;
    else
      out = mine + self * vi2 - sxz * vi0 - syz * vi1;
    double* dst = c == 0 ? o0 : (c == 1 ? o1 : o2);
    dst[(size_t)(r0 + r) * orr + (size_t)i * ostride] = out;
  }
}

// The real-space part of a block product (FP32 block products): for every
// packed pair p and bead i, rsum[(p N + i) 6 + 3h + c] = sum_j (T_ij v_j)_c of
// the pair's vector h (0: real part, 1: imaginary part), for NP pairs (at
// most five) in one pass over the pair rows.  One warp per bead; a lane takes
// row entries, each an index and the preparation's float4 (t1, w): T_ij =
// t1 I + s w w^T, the sign s of t2 kept in the lowest mantissa bit of t1;
// then it reads the neighbour's six inputs of every pair (the spread's
// vpk[(p N + j) 8], a float4 and a float2) and adds T_ij v into 6 NP FP32
// partial sums (a lane sums about a 32nd of the row).  The
// partials are summed over the warp by a transposing butterfly (31 exchanges
// per 32 values, lane l ends with the sum of value l), its first two stages
// in FP32 and the last three in FP64.
template <int NP>
__global__ void __launch_bounds__(256, 3) k_pme_real_pairs(
    const int* __restrict__ rcnt, const int* __restrict__ rrows, const float4* __restrict__ rw,
    int rcap, const float* __restrict__ vpk, int N, double* __restrict__ rsum) {
  constexpr int NV = 6 * NP;
  int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  float u[NV];
#pragma unroll
  for (int e = 0; e < NV; e++) u[e] = 0.f;
  int n = rcnt[i];
  const int* prow = rrows + (size_t)i * rcap;
  const float4* prw = rw + (size_t)i * rcap;
  for (int kk = lane; kk < n; kk += 32) {
    int j = __ldg(prow + kk);
    float4 q = __ldg(prw + kk);
    float s = (__float_as_uint(q.x) & 1u) ? -1.f : 1.f;
#pragma unroll
    for (int p = 0; p < NP; p++) {
      const float4* vj = (const float4*)(vpk + ((size_t)p * N + j) * 8);
      float4 a = __ldg(vj);
      float2 b = __ldg((const float2*)(vj + 1));
      float qa = s * (q.y * a.x + q.z * a.y + q.w * a.z);
      float qb = s * (q.y * a.w + q.z * b.x + q.w * b.y);
      u[6 * p] += q.x * a.x + qa * q.y;
      u[6 * p + 1] += q.x * a.y + qa * q.z;
      u[6 * p + 2] += q.x * a.z + qa * q.w;
      u[6 * p + 3] += q.x * a.w + qb * q.y;
      u[6 * p + 4] += q.x * b.x + qb * q.z;
      u[6 * p + 5] += q.x * b.y + qb * q.w;
    }
  }
  // the first two exchanges in FP32 (sums of 2 and 4 lanes), the rest in FP64
  float f[32];
#pragma unroll
  for (int e = 0; e < 32; e++) f[e] = e < NV ? u[e] : 0.f;
#pragma unroll
  for (int off = 16; off >= 8; off >>= 1) {
    bool up = lane & off;
#pragma unroll
    for (int e = 0; e < off; e++) {
      float send = up ? f[e] : f[e + off];
      float keep = up ? f[e + off] : f[e];
      f[e] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  double d[8];
#pragma unroll
  for (int e = 0; e < 8; e++) d[e] = (double)f[e];
#pragma unroll
  for (int off = 4; off >= 1; off >>= 1) {
    bool up = lane & off;
#pragma unroll
    for (int e = 0; e < off; e++) {
      double send = up ? d[e] : d[e + off];
      double keep = up ? d[e + off] : d[e];
      d[e] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  // value e = 6 p + 3 h + c
  if (lane < NV) rsum[((size_t)(lane / 6) * N + i) * 6 + lane % 6] = d[0];
}

// The real-space part of a single product (FP32 contexts that hold the
// mobility build's pair data): one warp per bead; per row entry the index
// and (t1, w) as for the block products, the neighbour's three input values
// taken to FP32, FP32 partial sums per lane, summed over the warp in FP64;
// rsum[6 i + c] for c < 3, which the interpolation adds.
__global__ void __launch_bounds__(256) k_pme_real_single(
    const int* __restrict__ rcnt, const int* __restrict__ rrows, const float4* __restrict__ rw,
    int rcap, VecIn v, int N, double* __restrict__ rsum) {
  int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f;
  int n = rcnt[i];
  const int* prow = rrows + (size_t)i * rcap;
  const float4* prw = rw + (size_t)i * rcap;
  for (int kk = lane; kk < n; kk += 32) {
    int j = __ldg(prow + kk);
    float4 q = __ldg(prw + kk);
    size_t o = (size_t)j * v.stride;
    float x0 = (float)v.p[0][o], x1 = (float)v.p[1][o], x2 = (float)v.p[2][o];
    float d = q.y * x0 + q.z * x1 + q.w * x2;
    d = (__float_as_uint(q.x) & 1u) ? -d : d;
    a0 += q.x * x0 + d * q.y;
    a1 += q.x * x1 + d * q.z;
    a2 += q.x * x2 + d * q.w;
  }
  double d0 = a0, d1 = a1, d2 = a2;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    d0 += __shfl_xor_sync(0xffffffffu, d0, o);
    d1 += __shfl_xor_sync(0xffffffffu, d1, o);
    d2 += __shfl_xor_sync(0xffffffffu, d2, o);
  }
  if (lane == 0) {
    rsum[6 * (size_t)i] = d0;
    rsum[6 * (size_t)i + 1] = d1;
    rsum[6 * (size_t)i + 2] = d2;
  }
}

// Cells of the real-space list (fractional, width >= rc).
struct RGeom {
  int n[3];
};

__device__ __forceinline__ int rcell(const Cell& cell, const RGeom& g, double x, double y, double z,
                                     int* cd) {
  double s[3];
  frac_of(cell, x, y, z, s);
  for (int d = 0; d < 3; d++) {
    double sd = s[d] - floor(s[d]);
    int c = (sd >= 0.0 && sd <= 1.0) ? (int)(sd * g.n[d]) : 0;  // 0 for non-finite input
    cd[d] = c >= g.n[d] ? g.n[d] - 1 : c;
  }
  return (cd[0] * g.n[1] + cd[1]) * g.n[2] + cd[2];
}

__global__ void k_rl_count(Cell cell, RGeom g, const double* __restrict__ rx,
                           const double* __restrict__ ry, const double* __restrict__ rz,
                           double cr, double sr, int N, int* cell_of, int* cell_count) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int cd[3];
  double x = rx[i] * cr - ry[i] * sr, y = rx[i] * sr + ry[i] * cr;
  int c = rcell(cell, g, x, y, rz[i], cd);
  cell_of[i] = c;
  atomicAdd(&cell_count[c], 1);
}

__global__ void k_rl_scan(int ncell, int* cell_count, int* cell_start, int* cursor) {
  __shared__ int part[1024];
  int t = threadIdx.x, nt = blockDim.x;
  int per = (ncell + nt - 1) / nt, lo = t * per, hi = min(ncell, lo + per), s = 0;
  for (int c = lo; c < hi; c++) s += cell_count[c];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < nt; o <<= 1) {
    int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int b = part[t] - s;
  for (int c = lo; c < hi; c++) {
    cell_start[c] = b;
    cursor[c] = 0;
    b += cell_count[c];
    cell_count[c] = 0;
  }
  if (t == nt - 1) cell_start[ncell] = part[t];
}

__global__ void k_rl_fill(const int* __restrict__ cell_of, const int* __restrict__ cell_start,
                          int* cursor, int* beads, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int c = cell_of[i];
  beads[cell_start[c] + atomicAdd(&cursor[c], 1)] = i;
}

// Pairs within rc (lattice minimum image): rows of bead indices and, per
// pair, t1 and t2 / r^2 of the real-space tensor.
template <typename R>
__global__ void k_rl_rows(Cell cell, RGeom g, const double4* __restrict__ pos, int N,
                          const int* __restrict__ cell_start, const int* __restrict__ beads,
                          double rc2, double alpha, double alpha_ref, int rcap, int* cnt,
                          int* rows, R* tt, float4* rw, int* need, int* err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double4 p = pos[i];
  int cd[3];
  rcell(cell, g, p.x, p.y, p.z, cd);
  int lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = g.n[d] >= 3 ? -1 : 0;
    hi[d] = g.n[d] >= 3 ? 1 : g.n[d] - 1;
  }
  int n = 0, nall = 0;
  bool over = false;
  for (int a = lo[0]; a <= hi[0]; a++)
    for (int b = lo[1]; b <= hi[1]; b++)
      for (int c = lo[2]; c <= hi[2]; c++) {
        int e0 = g.n[0] >= 3 ? (cd[0] + a + g.n[0]) % g.n[0] : a;
        int e1 = g.n[1] >= 3 ? (cd[1] + b + g.n[1]) % g.n[1] : b;
        int e2 = g.n[2] >= 3 ? (cd[2] + c + g.n[2]) % g.n[2] : c;
        int cc = (e0 * g.n[1] + e1) * g.n[2] + e2;
        for (int q = cell_start[cc]; q < cell_start[cc + 1]; q++) {
          int j = beads[q];
          if (j == i) continue;
          double4 pj = pos[j];
          double dx = pj.x - p.x, dy = pj.y - p.y, dz = pj.z - p.z, s[3];
          frac_of(cell, dx, dy, dz, s);
          for (int d = 0; d < 3; d++) s[d] -= rint(s[d]);
          dx = cell.H[0] * s[0] + cell.H[1] * s[1] + cell.H[2] * s[2];
          dy = cell.H[3] * s[0] + cell.H[4] * s[1] + cell.H[5] * s[2];
          dz = cell.H[6] * s[0] + cell.H[7] * s[1] + cell.H[8] * s[2];
          double rr = dx * dx + dy * dy + dz * dz;
          if (rr >= rc2) continue;
          if (n >= rcap) {
            over = true;
            nall++;
            continue;
          }
          double t1, t2;
          pair_terms(alpha, alpha_ref, rr, t1, t2);
          rows[(size_t)i * rcap + n] = j;
          tt[2 * ((size_t)i * rcap + n)] = (R)t1;
          tt[2 * ((size_t)i * rcap + n) + 1] = (R)(t2 / rr);
          if (rw) {
            double sw = sqrt(fabs(t2 / rr));
            unsigned b = (__float_as_uint((float)t1) & ~1u) | (t2 < 0.0 ? 1u : 0u);
            rw[(size_t)i * rcap + n] =
                make_float4(__uint_as_float(b), (float)(sw * dx), (float)(sw * dy), (float)(sw * dz));
          }
          n++;
          nall++;
        }
      }
  cnt[i] = n;
  if (over) {
    if (need)
      atomicMax(need, nall);  // the host grows the rows and builds them again
    else
      atomicOr(err, ERRB_NBR_OVERFLOW);
  }
}

namespace bd {

int pme_alloc(bd_ctx* c) {
  if (c->pme_grid) return BD_OK;
  int K = c->pmeK, N = c->N;
  size_t K3 = (size_t)K * K * K, Ks = (size_t)K * K * (K / 2 + 1);
  c->pme_f32 = c->p.precision == BD_PREC_FP32;
  size_t es = c->pme_f32 ? 4 : 8;  // grid, spectrum, influence and pair tensors
  // grids and spectra for the largest number of right-hand sides of a product
  size_t nr = (size_t)std::max(1, c->nbk);
  CU(cudaMalloc(&c->pme_grid, es * 3 * K3 * nr));
  // the spectra; for products of several right-hand sides the same buffer
  // holds the packed pairs' complex grids (3 ceil(k/2) K^3 complex values)
  size_t spec_bytes = std::max(2 * es * 3 * Ks * nr, nr > 1 ? 2 * es * 3 * K3 * ((nr + 1) / 2) : 0);
  CU(cudaMalloc(&c->pme_spec, spec_bytes));
  CU(cudaMalloc(&c->pme_infl, es * 6 * Ks));
  CU(cudaMalloc(&c->pme_bsq, 8 * 3 * (size_t)K));
  c->pme_nblk = (int)((Ks + 255) / 256);
  CU(cudaMalloc(&c->pme_soff, 8 * (3 * (size_t)c->pme_nblk + 3)));
  CU(cudaMalloc(&c->pme_base, 4 * 3 * (size_t)N));
  CU(cudaMalloc(&c->pme_w, 8 * 3 * (size_t)N * kMaxOrder));
  // default row cap: 2.5 times the mean number of beads within the cutoff at
  // the system's density, at least 512, a multiple of 32
  if (c->p.pme_max_pairs > 0) {
    c->rl_cap = c->p.pme_max_pairs;
  } else {
    double mean = 4.0 / 3.0 * M_PI * c->pme_rc * c->pme_rc * c->pme_rc * N / c->boxvol;
    c->rl_cap = std::max(512, ((int)ceil(2.5 * mean) + 31) / 32 * 32);
  }
  CU(cudaMalloc(&c->rl_cnt, 4 * (size_t)N));
  CU(cudaMalloc(&c->rl_need, 4));
  CU(cudaMemsetAsync(c->rl_need, 0, 4, c->stream));
  CU(cudaMalloc(&c->rl_rows, 4 * (size_t)N * c->rl_cap));
  CU(cudaMalloc(&c->rl_pos, 32 * (size_t)N));
  if (c->pme_f32 && nr > 1) {
    CU(cudaMalloc(&c->pme_vpk, 32 * (size_t)N * ((nr + 1) / 2)));
    CU(cudaMalloc(&c->pme_rsum, 48 * (size_t)N * ((nr + 1) / 2)));
    CU(cudaMalloc(&c->rl_w, 16 * (size_t)N * c->rl_cap));
    c->bytes += 80 * (size_t)N * ((nr + 1) / 2) + 16 * (size_t)N * c->rl_cap;
  }
  CU(cudaMalloc(&c->rl_tt, 2 * es * (size_t)N * c->rl_cap));
  c->rl_ncell_cap = 4096;
  CU(cudaMalloc(&c->rl_cell_of, 4 * (size_t)N));
  CU(cudaMalloc(&c->rl_beads, 4 * (size_t)N));
  CU(cudaMalloc(&c->rl_cell_count, 4 * (size_t)c->rl_ncell_cap));
  CU(cudaMalloc(&c->rl_cell_start, 4 * (size_t)(c->rl_ncell_cap + 1)));
  CU(cudaMalloc(&c->rl_cursor, 4 * (size_t)c->rl_ncell_cap));
  CU(cudaMemsetAsync(c->rl_cell_count, 0, 4 * (size_t)c->rl_ncell_cap, c->stream));
  c->bytes += es * (3 * K3 * nr + 6 * Ks) + spec_bytes + 24 * (size_t)K + 12 * (size_t)N +
              24 * (size_t)N * kMaxOrder + 4 * (size_t)N + (size_t)N * c->rl_cap * (4 + 2 * es) + 32 * (size_t)N +
              8 * (size_t)N + 12 * (size_t)c->rl_ncell_cap;
  int n[3] = {K, K, K};
  cufftHandle f, b;
  CF(cufftPlanMany(&f, 3, n, nullptr, 1, (int)K3, nullptr, 1, (int)Ks,
                   c->pme_f32 ? CUFFT_R2C : CUFFT_D2Z, 3));
  CF(cufftPlanMany(&b, 3, n, nullptr, 1, (int)Ks, nullptr, 1, (int)K3,
                   c->pme_f32 ? CUFFT_C2R : CUFFT_Z2D, 3));
  CF(cufftSetStream(f, c->stream));
  CF(cufftSetStream(b, c->stream));
  c->pme_plan_f = (int)f;
  c->pme_plan_b = (int)b;
  std::vector<double> bs(3 * (size_t)K);
  bspline_moduli(K, c->pme_p, bs.data());
  for (int d = 1; d < 3; d++)
    for (int m = 0; m < K; m++) bs[(size_t)d * K + m] = bs[m];
  CU(cudaMemcpyAsync(c->pme_bsq, bs.data(), 8 * bs.size(), cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return BD_OK;
}

// In-place complex transforms of the 3 ceil(k/2) packed-pair grids of a
// k-right-hand-side product (one plan, used forward and inverse), created
// outside any stream capture and kept for up to four values of k (replacing
// one drops the captured iterations that use it).
int pme_multi_plan(bd_ctx* c, int k) {
  int slot = -1;
  for (int q = 0; q < 4; q++)
    if (c->pme_mplan_k[q] == k) return BD_OK;
  for (int q = 0; q < 4 && slot < 0; q++)
    if (c->pme_mplan_k[q] == 0) slot = q;
  if (slot < 0) {
    slot = 3;
    lanczos_graphs_reset(c);
    cufftDestroy((cufftHandle)c->pme_mplan_f[slot]);
    c->pme_mplan_k[slot] = 0;
  }
  int K = c->pmeK;
  size_t K3 = (size_t)K * K * K;
  int n[3] = {K, K, K};
  cufftHandle f;
  CF(cufftPlanMany(&f, 3, n, nullptr, 1, (int)K3, nullptr, 1, (int)K3,
                   c->pme_f32 ? CUFFT_C2C : CUFFT_Z2Z, 3 * ((k + 1) / 2)));
  if (cufftSetStream(f, c->stream) != CUFFT_SUCCESS) {
    cufftDestroy(f);
    return BD_ERR_CUDA;
  }
  c->pme_mplan_f[slot] = (int)f;
  c->pme_mplan_k[slot] = k;
  return BD_OK;
}

void pme_free(bd_ctx* c) {
  if (c->pme_plan_f) cufftDestroy((cufftHandle)c->pme_plan_f);
  if (c->pme_plan_b) cufftDestroy((cufftHandle)c->pme_plan_b);
  for (int q = 0; q < 4; q++)
    if (c->pme_mplan_k[q]) {
      cufftDestroy((cufftHandle)c->pme_mplan_f[q]);
      c->pme_mplan_k[q] = 0;
    }
  void* ptrs[] = {c->pme_vpk, c->pme_rsum, c->rl_w, c->rl_need, c->pme_grid, c->pme_spec, c->pme_infl, c->pme_bsq, c->pme_soff, c->pme_base, c->pme_w,
                  c->rl_cnt, c->rl_rows, c->rl_pos, c->rl_tt, c->rl_cell_of, c->rl_beads, c->rl_cell_count,
                  c->rl_cell_start, c->rl_cursor};
  for (void* q : ptrs)
    if (q) cudaFree(q);
}

// Preparation for the current positions, in the frame calcHI reads them
// (extension: rotated by the lattice angle, taken to the lab frame here):
// spline weights, influence tensor of the current cell, self off-diagonal
// sums, real-space pair list and tensors.  The products that follow use this
// configuration until the next preparation, as the dense matrix does.
// Pair rows of a larger cap (the rows are rebuilt by the caller).
static int rl_grow(bd_ctx* c, int cap) {
  size_t N = c->N, es = c->pme_f32 ? 4 : 8, old = (size_t)c->rl_cap;
  CU(cudaStreamSynchronize(c->stream));
  cudaFree(c->rl_rows);
  cudaFree(c->rl_tt);
  c->rl_rows = nullptr;
  c->rl_tt = nullptr;
  CU(cudaMalloc(&c->rl_rows, 4 * N * cap));
  CU(cudaMalloc(&c->rl_tt, 2 * es * N * cap));
  c->bytes += (4 + 2 * es) * N * (cap - old);
  if (c->rl_w) {
    cudaFree(c->rl_w);
    c->rl_w = nullptr;
    CU(cudaMalloc(&c->rl_w, 16 * N * cap));
    c->bytes += 16 * N * (cap - old);
  }
  c->rl_cap = cap;
  CU(cudaMemsetAsync(c->rl_need, 0, 4, c->stream));
  return BD_OK;
}

int pme_prepare(bd_ctx* c, const Lat& l) {
  int s;
  if ((s = pme_alloc(c)) != BD_OK) return s;
  Cell cell = make_cell(l);
  double cr = 1.0, sr = 0.0;
  if (l.flow == BD_FLOW_EXT) {
    cr = l.cth;
    sr = l.sth;
  }
  double rc = c->pme_rc, alpha = c->pme_alpha;
  int K = c->pmeK, N = c->N;
  // calcHI's split parameter at this step, for its overlap convention
  double rce = l.treal <= c->tp / 2 ? l.L2yp : 2.0 * l.L2yp;
  double alpha_ref = 4.0 / rce;
  c->launches += 3;
  k_pme_weights<<<nblk(N, 256), 256, 0, c->stream>>>(cell, c->rx, c->ry, c->rz, cr, sr, N, K,
                                                     c->pme_p, c->pme_base, c->pme_w,
                                                     (double4*)c->rl_pos, c->err);
  if (c->pme_f32)
    k_pme_influence<float><<<c->pme_nblk, 256, 0, c->stream>>>(
        cell, K, alpha, c->pme_bsq, (float*)c->pme_infl, c->pme_soff + 3);
  else
    k_pme_influence<double><<<c->pme_nblk, 256, 0, c->stream>>>(
        cell, K, alpha, c->pme_bsq, (double*)c->pme_infl, c->pme_soff + 3);
  k_pme_soff_fin<<<1, 256, 0, c->stream>>>(c->pme_soff + 3, c->pme_nblk, c->pme_soff);
  if ((s = launch_ok(c)) != BD_OK) return s;
  // real-space cells: perpendicular widths V/|a_j x a_k|
  double w[3];
  {
    const double* H = cell.H;
    double a[3][3];
    for (int j = 0; j < 3; j++)
      for (int d = 0; d < 3; d++) a[j][d] = H[d * 3 + j];
    for (int j = 0; j < 3; j++) {
      const double* u = a[(j + 1) % 3];
      const double* v = a[(j + 2) % 3];
      double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2],
             cz = u[0] * v[1] - u[1] * v[0];
      w[j] = cell.V / sqrt(cx * cx + cy * cy + cz * cz);
    }
  }
  if (2 * rc > std::min(w[0], std::min(w[1], w[2]))) return BD_ERR_ARG;  // rc beyond half a width
  RGeom g;
  for (int d = 0; d < 3; d++) g.n[d] = std::max(1, (int)floor(w[d] / rc));
  while ((long)g.n[0] * g.n[1] * g.n[2] > c->rl_ncell_cap) {
    int d = g.n[0] >= g.n[1] && g.n[0] >= g.n[2] ? 0 : (g.n[1] >= g.n[2] ? 1 : 2);
    g.n[d]--;
  }
  int ncell = g.n[0] * g.n[1] * g.n[2];
  c->launches += 4;
  k_rl_count<<<nblk(N, 256), 256, 0, c->stream>>>(cell, g, c->rx, c->ry, c->rz, cr, sr, N,
                                                  c->rl_cell_of, c->rl_cell_count);
  k_rl_scan<<<1, 1024, 0, c->stream>>>(ncell, c->rl_cell_count, c->rl_cell_start, c->rl_cursor);
  k_rl_fill<<<nblk(N, 256), 256, 0, c->stream>>>(c->rl_cell_of, c->rl_cell_start, c->rl_cursor,
                                                 c->rl_beads, N);
  if ((s = launch_ok(c)) != BD_OK) return s;
  // the pair rows; with the default cap (no pme_max_pairs), rows that
  // overflow it are grown to 1.25 times the longest row and built again
  int* need = c->p.pme_max_pairs > 0 ? nullptr : c->rl_need;
  for (int pass = 0; pass < 2; pass++) {
    if (c->pme_f32)
      k_rl_rows<float><<<nblk(N, 128), 128, 0, c->stream>>>(
          cell, g, (const double4*)c->rl_pos, N, c->rl_cell_start, c->rl_beads, rc * rc, alpha,
          alpha_ref, c->rl_cap, c->rl_cnt, c->rl_rows, (float*)c->rl_tt, c->rl_w, need, c->err);
    else
      k_rl_rows<double><<<nblk(N, 128), 128, 0, c->stream>>>(
          cell, g, (const double4*)c->rl_pos, N, c->rl_cell_start, c->rl_beads, rc * rc, alpha,
          alpha_ref, c->rl_cap, c->rl_cnt, c->rl_rows, (double*)c->rl_tt, nullptr, need, c->err);
    if (!need) break;
    int longest = 0;
    CU(cudaMemcpyAsync(&longest, need, 4, cudaMemcpyDeviceToHost, c->stream));
    if ((s = check(c)) != BD_OK) return s;
    if (longest <= c->rl_cap) break;
    if ((s = rl_grow(c, ((int)ceil(1.25 * longest) + 31) / 32 * 32)) != BD_OK) return s;
  }
  // the cell and calcHI's split parameter of this configuration, for the
  // products until the next preparation
  memcpy(c->pme_cellbuf, cell.H, sizeof(cell.H));
  memcpy(c->pme_cellbuf + 9, cell.Hi, sizeof(cell.Hi));
  c->pme_cellbuf[18] = cell.V;
  c->pme_alpha_ref = alpha_ref;
  double a = alpha;
  c->pme_self = 1.0 - 6.0 / sqrt(M_PI) * a + 40.0 / (3.0 * sqrt(M_PI)) * a * a * a;
  c->Dtr[0] = c->Dtr[1] = c->Dtr[2] = c->pme_self;
  c->pme_ready = true;
  c->hi_built = true;
  return launch_ok(c);
}

// out_r = M v_r by PME for k right-hand sides given by component pointers
// (VecIn) and RHS strides vr (input) and orr (output); k = 1 is the
// single-vector product with the context's own transforms.
template <typename R, typename Cx>
static int pme_apply_t(bd_ctx* c, int k, const VecIn& v, size_t vr, double* o0, double* o1,
                       double* o2, int ostride, size_t orr) {
  int K = c->pmeK, N = c->N, p = c->pme_p;
  size_t K3 = (size_t)K * K * K, Ks = (size_t)K * K * (K / 2 + 1);
  if (k < 1 || k > std::max(1, c->nbk)) return BD_ERR_ARG;
  int nb8 = nblk(N, 8);
  Cell cell;
  memcpy(cell.H, c->pme_cellbuf, sizeof(cell.H));
  memcpy(cell.Hi, c->pme_cellbuf + 9, sizeof(cell.Hi));
  cell.V = c->pme_cellbuf[18];
  c->launches += 3;  // spread, influence, gather (the transforms are cuFFT's)
  if (k == 1) {
    // one right-hand side: three real grids, R2C / C2R
    R* grid = (R*)c->pme_grid;
    Cx* spec = (Cx*)c->pme_spec;
    CU(cudaMemsetAsync(grid, 0, sizeof(R) * 3 * K3, c->stream));
#define PME_SPREAD(P_) \
  k_pme_spread<P_, R, 1><<<nb8, 256, 0, c->stream>>>(c->pme_base, c->pme_w, N, K, v, vr, 1, grid)
    switch (p) {
      case 4: PME_SPREAD(4); break;
      case 6: PME_SPREAD(6); break;
      default: PME_SPREAD(8);
    }
#undef PME_SPREAD
    if constexpr (sizeof(R) == 4)
      CF(cufftExecR2C((cufftHandle)c->pme_plan_f, (cufftReal*)grid, (cufftComplex*)spec));
    else
      CF(cufftExecD2Z((cufftHandle)c->pme_plan_f, (cufftDoubleReal*)grid,
                      (cufftDoubleComplex*)spec));
    k_pme_apply_influence<R, Cx><<<nblk((long long)Ks, 256), 256, 0, c->stream>>>(
        (const R*)c->pme_infl, spec, Ks);
    if constexpr (sizeof(R) == 4)
      CF(cufftExecC2R((cufftHandle)c->pme_plan_b, (cufftComplex*)spec, (cufftReal*)grid));
    else
      CF(cufftExecZ2D((cufftHandle)c->pme_plan_b, (cufftDoubleComplex*)spec,
                      (cufftDoubleReal*)grid));
    // FP32 with the stored pair data: the real-space sums in their own pass
    // (as for the block products), the interpolation then only reads the grid
    bool rs = sizeof(R) == 4 && c->rl_w && c->pme_rsum;
    if (rs) {
      c->launches++;
      k_pme_real_single<<<nb8, 256, 0, c->stream>>>(c->rl_cnt, c->rl_rows, c->rl_w, c->rl_cap, v,
                                                     N, c->pme_rsum);
    }
#define PME_GATHER(P_, RS_)                                                                   \
  k_pme_gather<P_, R, 1, false, RS_><<<nb8, 256, 0, c->stream>>>(                             \
      c->pme_base, c->pme_w, N, K, grid, 1, c->pme_self, c->pme_soff, v, vr, c->rl_cnt,       \
      c->rl_rows, (const double4*)c->rl_pos, cell, (const R*)c->rl_tt, c->rl_cap, o0, o1, o2, \
      ostride, orr, RS_ ? c->pme_rsum : nullptr)
    if (rs) {
      switch (p) {
        case 4: PME_GATHER(4, true); break;
        case 6: PME_GATHER(6, true); break;
        default: PME_GATHER(8, true);
      }
    } else {
      switch (p) {
        case 4: PME_GATHER(4, false); break;
        case 6: PME_GATHER(6, false); break;
        default: PME_GATHER(8, false);
      }
    }
#undef PME_GATHER
    return BD_OK;
  }
  // k >= 2: packed pairs in the spectrum buffer, in-place complex transforms
  int q = 0;
  while (q < 4 && c->pme_mplan_k[q] != k) q++;
  if (q == 4) return BD_ERR_STATE;  // pme_multi_plan(c, k) first
  cufftHandle plan = (cufftHandle)c->pme_mplan_f[q];
  int np = (k + 1) / 2;
  using C2 = typename Pair<R>::T;
  C2* cg = (C2*)c->pme_spec;
  CU(cudaMemsetAsync(cg, 0, sizeof(C2) * 3 * K3 * np, c->stream));
  dim3 gp(nb8, np);
  float* vpk = sizeof(R) == 4 ? c->pme_vpk : nullptr;
#define PME_SPREAD(P_)                                                                       \
  k_pme_spread_pairs<P_, R><<<gp, 256, 0, c->stream>>>(c->pme_base, c->pme_w, N, K, v, vr, k, cg, \
                                                       vpk)
  switch (p) {
    case 4: PME_SPREAD(4); break;
    case 6: PME_SPREAD(6); break;
    default: PME_SPREAD(8);
  }
#undef PME_SPREAD
  if constexpr (sizeof(R) == 4)
    CF(cufftExecC2C(plan, (cufftComplex*)cg, (cufftComplex*)cg, CUFFT_FORWARD));
  else
    CF(cufftExecZ2Z(plan, (cufftDoubleComplex*)cg, (cufftDoubleComplex*)cg, CUFFT_FORWARD));
  k_pme_apply_influence_full<R, C2><<<nblk((long long)K3 * np, 256), 256, 0, c->stream>>>(
      (const R*)c->pme_infl, cg, K, (size_t)np);
  if constexpr (sizeof(R) == 4)
    CF(cufftExecC2C(plan, (cufftComplex*)cg, (cufftComplex*)cg, CUFFT_INVERSE));
  else
    CF(cufftExecZ2Z(plan, (cufftDoubleComplex*)cg, (cufftDoubleComplex*)cg, CUFFT_INVERSE));
  // FP32: the real-space sums of the packed pairs, in passes over the rows of
  // up to five pairs (30 FP32 partial sums per lane at 80 registers)
  double* rsum = nullptr;
  if constexpr (sizeof(R) == 4) {
    if (vpk && c->pme_rsum && c->rl_w) {
      rsum = c->pme_rsum;
      for (int p0 = 0; p0 < np; p0 += 5) {
        const float* vp = vpk + (size_t)p0 * N * 8;
        double* rs = rsum + (size_t)p0 * N * 6;
        c->launches++;
#define PME_REAL(NP_)                                                                        \
  k_pme_real_pairs<NP_><<<nb8, 256, 0, c->stream>>>(c->rl_cnt, c->rl_rows, c->rl_w, c->rl_cap, \
                                                    vp, N, rs)
        switch (std::min(5, np - p0)) {
          case 1: PME_REAL(1); break;
          case 2: PME_REAL(2); break;
          case 3: PME_REAL(3); break;
          case 4: PME_REAL(4); break;
          default: PME_REAL(5);
        }
#undef PME_REAL
      }
    }
  }
#define PME_GATHER(P_, RS_)                                                                   \
  k_pme_gather<P_, R, 2, true, RS_><<<gp, 256, 0, c->stream>>>(                               \
      c->pme_base, c->pme_w, N, K, (const R*)cg, k, c->pme_self, c->pme_soff, v, vr,          \
      c->rl_cnt, c->rl_rows, (const double4*)c->rl_pos, cell, (const R*)c->rl_tt, c->rl_cap,  \
      o0, o1, o2, ostride, orr, rsum)
  if (rsum) {
    switch (p) {
      case 4: PME_GATHER(4, true); break;
      case 6: PME_GATHER(6, true); break;
      default: PME_GATHER(8, true);
    }
  } else {
    switch (p) {
      case 4: PME_GATHER(4, false); break;
      case 6: PME_GATHER(6, false); break;
      default: PME_GATHER(8, false);
    }
  }
#undef PME_GATHER
  return BD_OK;
}

static int pme_apply_k(bd_ctx* c, int k, const VecIn& v, size_t vr, double* o0, double* o1,
                       double* o2, int ostride, size_t orr) {
  if (!c->pme_ready) return BD_ERR_STATE;
  prof_begin(c, BD_PROF_MATVEC);
  int s = c->pme_f32
              ? pme_apply_t<float, cufftComplex>(c, k, v, vr, o0, o1, o2, ostride, orr)
              : pme_apply_t<double, cufftDoubleComplex>(c, k, v, vr, o0, o1, o2, ostride, orr);
  prof_end(c, BD_PROF_MATVEC);
  if (s != BD_OK) return s;
  return launch_ok(c);
}

int pme_apply(bd_ctx* c, const VecIn& v, double* o0, double* o1, double* o2, int ostride) {
  return pme_apply_k(c, 1, v, 0, o0, o1, o2, ostride, 0);
}

int pme_apply_multi(bd_ctx* c, int k, const double* X, size_t xs, double* Y, size_t ys) {
  int NTp = c->NT * 32;
  VecIn v = {{X, X + NTp, X + 2 * (size_t)NTp}, 1};
  return pme_apply_k(c, k, v, xs, Y, Y + NTp, Y + 2 * (size_t)NTp, 1, ys);
}

}  // namespace bd
