// Krylov (Lanczos) square root of the mobility and the Brownian step built
// on it.
//
// The reference draws its Brownian displacement with the conformationally
// averaged truncated-expansion approximation (updateHI,
// shear/src/main26.c:745-857).  This path computes sqrt(M) z itself:
// Lanczos on M from v_1 = z/|z| with full reorthogonalisation in FP64
// (classical Gram-Schmidt, applied twice), T_m = V_m^T M V_m tridiagonal,
// sqrt(M) z ~= |z| V_m T_m^(1/2) e_1, stopped when the relative change of the
// iterate between successive m is below the tolerance (the criterion of Ando,
// Chow and Skolnick, J. Chem. Phys. 137, 064106 (2012)).  T_m^(1/2) e_1 comes
// from an eigen-decomposition of T_m on the host by the implicit symmetric QR
// iteration with Wilkinson shifts (Golub and Van Loan, Matrix Computations,
// section 8.3).  Vectors live on the device in component-major SoA with the
// tile padding (3 x NTp); every reduction is a fixed-order two-level sum.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bd_ctx.cuh"

using namespace bd;

#define CU(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return BD_ERR_CUDA;    \
  } while (0)

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

// sc[0] = sqrt(sum of part) = |w|, sc[1] = 1/|w| (one warp)
__global__ void k_norm_fin(const double* __restrict__ part, int nblk, double* sc) {
  double s = warp_sum_parts(part, nblk, 1);
  if (threadIdx.x == 0) {
    sc[0] = sqrt(s);
    sc[1] = sc[0] > 0 ? 1.0 / sc[0] : 0.0;
  }
}

// v (SoA, padded) = z (bead-interleaved) / |z|; padding entries are zero
__global__ void k_interleaved_to_soa(const double* __restrict__ z, const double* __restrict__ sc,
                                     double* v, int N, int NTp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NTp) return;
  double f = sc[1];
  for (int a = 0; a < 3; a++) v[(size_t)a * NTp + i] = i < N ? z[3 * i + a] * f : 0.0;
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
__device__ __forceinline__ void chunk_range(int n, int& lo, int& hi) {
  int per = (n + gridDim.x - 1) / gridDim.x;
  lo = blockIdx.x * per;
  hi = min(n, lo + per);
}

// Dots of four vectors at a time per warp (vectors k0..k0+3, warps strided
// by groups): lanes over the chunk, so each lane keeps several independent
// loads in flight; butterfly reductions.
__device__ __forceinline__ void chunk_dots(const double* __restrict__ V, size_t vs, int nv,
                                           const double* __restrict__ w, int lo, int hi,
                                           double* part) {
  int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k0 = 4 * wp; k0 < nv; k0 += 4 * nw) {
    const double* v0 = V + (size_t)k0 * vs;
    const double* v1 = V + (size_t)min(k0 + 1, nv - 1) * vs;
    const double* v2 = V + (size_t)min(k0 + 2, nv - 1) * vs;
    const double* v3 = V + (size_t)min(k0 + 3, nv - 1) * vs;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    for (int i = lo + lane; i < hi; i += 32) {
      double x = w[i];
      s0 += v0[i] * x;
      s1 += v1[i] * x;
      s2 += v2[i] * x;
      s3 += v3[i] * x;
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
__device__ __forceinline__ double combo_row(const double* __restrict__ V, size_t vs,
                                            const double* h, int nv, int i) {
  double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int k = 0;
  for (; k + 8 <= nv; k += 8) {
#pragma unroll
    for (int q = 0; q < 8; q++) a[q] += h[k + q] * V[(size_t)(k + q) * vs + i];
  }
  double t = 0;
  for (; k < nv; k++) t += h[k] * V[(size_t)k * vs + i];
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

// The iteration index j lives on the device (*jd) so that one iteration's
// launches are the same every iteration and can be replayed as a CUDA graph;
// k_next_j advances it at the end of the iteration.
__global__ void __launch_bounds__(256) k_orth0(const double* __restrict__ V, size_t vs,
                                               const int* __restrict__ jd,
                                               const double* __restrict__ w, int n,
                                               double* part1) {
  int nv = *jd + 1, lo, hi;
  chunk_range(n, lo, hi);
  chunk_dots(V, vs, nv, w, lo, hi, part1);
}

__global__ void __launch_bounds__(256) k_orth1(const double* __restrict__ V, size_t vs,
                                               const int* __restrict__ jd, double* w, int n,
                                               const double* __restrict__ part1,
                                               double* part2, double* hsave) {
  __shared__ double h[kMaxKrylov + 1];
  int nv = *jd + 1, lo, hi;
  chunk_range(n, lo, hi);
  sum_parts(part1, nv, h);
  if (blockIdx.x == 0)
    for (int k = threadIdx.x; k < nv; k += blockDim.x) hsave[k] = h[k];
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) w[i] -= combo_row(V, vs, h, nv, i);
  __syncthreads();
  chunk_dots(V, vs, nv, w, lo, hi, part2);
}

__global__ void __launch_bounds__(256) k_orth2(const double* __restrict__ V, size_t vs,
                                               const int* __restrict__ jd, double* w, int n,
                                               const double* __restrict__ part2,
                                               double* part3, const double* __restrict__ hsave,
                                               double* alpha) {
  __shared__ double h[kMaxKrylov + 1];
  __shared__ double red[8];
  int j = *jd, nv = j + 1, lo, hi;
  chunk_range(n, lo, hi);
  sum_parts(part2, nv, h);
  double s2 = 0;
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double x = w[i] - combo_row(V, vs, h, nv, i);
    w[i] = x;
    s2 += x * x;
  }
  for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) t += red[q];
    part3[blockIdx.x] = t;
    if (blockIdx.x == 0) alpha[j] = hsave[j] + h[j];
  }
}

// beta_j = |w|; v_{j+1} = w / beta_j into the basis and into vcur (the
// fixed input of the next iteration's product)
__global__ void __launch_bounds__(256) k_orth3(const double* __restrict__ w, int n,
                                               const double* __restrict__ part3, double* beta,
                                               const int* __restrict__ jd, double* V, size_t vs,
                                               double* vcur) {
  __shared__ double b;
  int j = *jd;
  if (threadIdx.x < 32) {
    double s = warp_sum_parts(part3, gridDim.x, 1);
    if (threadIdx.x == 0) {
      b = sqrt(s);
      if (blockIdx.x == 0) beta[j] = b;
    }
  }
  __syncthreads();
  double f = b > 0 ? 1.0 / b : 0.0;
  double* vnext = V + (size_t)(j + 1) * vs;
  int lo, hi;
  chunk_range(n, lo, hi);
  for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    double x = w[i] * f;
    vnext[i] = x;
    vcur[i] = x;
  }
}

__global__ void k_next_j(int* jd) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *jd += 1;
}

// |z|^2 partials over the bead-interleaved noise
__global__ void __launch_bounds__(256) k_sumsq(const double* __restrict__ z, int n, double* part) {
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
// on return d holds the eigenvalues and Z (n x n, Z[i*n+k] = component i of
// eigenvector k) the orthonormal eigenvectors.
static void tridiag_eig(int n, std::vector<double>& d, std::vector<double> e,
                        std::vector<double>& Z) {
  Z.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) Z[(size_t)i * n + i] = 1.0;
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
      for (int i = 0; i < n; i++) {
        double zk = Z[(size_t)i * n + k], zk1 = Z[(size_t)i * n + k + 1];
        Z[(size_t)i * n + k] = cs * zk - sn * zk1;
        Z[(size_t)i * n + k + 1] = sn * zk + cs * zk1;
      }
    }
  }
}

// c = T^q e_1 for T = tridiag(beta, alpha, beta) of size m, q = +1/2 or
// -1/2; non-positive Ritz values are clamped (to zero for q > 0, to 1e-12 of
// the largest for q < 0) and counted.
static int sqrt_e1(const std::vector<double>& alpha, const std::vector<double>& beta, int m,
                   std::vector<double>& c, double q = 0.5) {
  std::vector<double> d(alpha.begin(), alpha.begin() + m), e(beta.begin(), beta.begin() + (m - 1));
  std::vector<double> Z;
  tridiag_eig(m, d, e, Z);
  int neg = 0;
  double lmax = 0;
  for (int k = 0; k < m; k++) lmax = std::max(lmax, d[k]);
  c.assign(m, 0.0);
  for (int k = 0; k < m; k++) {
    double lam = d[k];
    if (lam <= 0) {
      neg++;
      lam = q > 0 ? 0.0 : 1e-12 * lmax;
    }
    double w = (q > 0 ? sqrt(lam) : 1.0 / sqrt(lam)) * Z[(size_t)0 * m + k];
    for (int i = 0; i < m; i++) c[i] += Z[(size_t)i * m + k] * w;
  }
  return neg;
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
// c->MF), CGS2 against the basis, beta, v_{j+1}, j += 1.  Every argument is
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
  double* part1 = c->Lpart;
  double* part2 = c->Lpart + (size_t)(c->lmax + 1) * blk;
  double* part3 = c->Lpart + (size_t)2 * (c->lmax + 1) * blk;
  c->launches += 5;
  k_orth0<<<blk, 256, 0, st>>>(c->LV, vs, c->Ljd, c->Lw, n, part1);
  k_orth1<<<blk, 256, 0, st>>>(c->LV, vs, c->Ljd, c->Lw, n, part1, part2, c->Lc);
  k_orth2<<<blk, 256, 0, st>>>(c->LV, vs, c->Ljd, c->Lw, n, part2, part3, c->Lc, c->Lh);
  k_orth3<<<blk, 256, 0, st>>>(c->Lw, n, part3, c->Lsc + 8, c->Ljd, c->LV, vs, vc);
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
    if (e != cudaSuccess) return BD_ERR_CUDA;
    cudaGraphExec_t ex;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return BD_ERR_CUDA;
    c->lan_graph[v] = (void*)ex;
    c->lan_graph_launches[v] = c->launches - l0;
    c->launches = l0;
  }
  CU(cudaGraphLaunch((cudaGraphExec_t)c->lan_graph[v], c->stream));
  c->launches += c->lan_graph_launches[v];
  return BD_OK;
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
  k_sumsq<<<blk, 256, 0, st>>>(z, 3 * N, c->Lpart);
  k_norm_fin<<<1, 32, 0, st>>>(c->Lpart, blk, c->Lsc);
  k_interleaved_to_soa<<<(NTp + 255) / 256, 256, 0, st>>>(z, c->Lsc, c->LV, N, NTp);
  CU(cudaMemcpyAsync(c->Lvcur, c->LV, 8 * vs, cudaMemcpyDeviceToDevice, st));
  CU(cudaMemsetAsync(c->Ljd, 0, sizeof(int), st));
  double zn = 0;
  CU(cudaMemcpyAsync(&zn, c->Lsc, 8, cudaMemcpyDeviceToHost, st));
  std::vector<double> alpha, beta, cc, cprev;
  int m = 0, neg = 0;
  bool conv = false;
  // alpha_j, beta_j stay on the device (Lh, Lsc + 8); the host reads them
  // only at checkpoints: from two before the previous call's Krylov
  // dimension on, every second iteration
  double* d_alpha = c->Lh;
  double* d_beta = c->Lsc + 8;
  int& last = pre ? c->pre_last : c->lan_last;
  int next_check = std::max(4, last - 2);
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
    neg = sqrt_e1(alpha, beta, m, cc, q);
    sqrt_e1(alpha, beta, m - 1, cprev, q);
    double dn = 0, cn = 0;
    for (int i = 0; i < m; i++) {
      double prev = i < m - 1 ? cprev[i] : 0.0;
      dn += (cc[i] - prev) * (cc[i] - prev);
      cn += cc[i] * cc[i];
    }
    if (sqrt(dn) <= c->ltol * sqrt(cn) || beta[m - 1] <= 1e-300) {
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

int bd_lanczos_stats(bd_ctx* c, long* o) {
  if (!c || !o) return BD_ERR_ARG;
  o[0] = (long)c->lan_calls;
  o[1] = (long)c->lan_iters;
  o[2] = (long)c->lan_maxed;
  o[3] = (long)c->lan_negative;
  return BD_OK;
}

int bd_step_lanczos(bd_ctx* c, unsigned long t0, int nsteps, int with_hop) {
  if (!c || nsteps < 0) return BD_ERR_ARG;
  int s;
  bool ext = c->p.flow == BD_FLOW_EXT;
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
    if ((s = bd_get_noise(c))) return s;
    if (t % (unsigned long)c->srpy == 0 || t == c->tstart || !c->hi_built)
      if ((s = calc_hi(c))) return s;
    if (ext) rotate_coords(c, 1);
    if ((s = lanczos_sqrt(c, c->R, true, nullptr))) return s;
    c->launches++;
    k_krylov_update<<<(c->N + 255) / 256, 256, 0, c->stream>>>(
        c->p.flow, c->rx, c->ry, c->rz, c->dxv, c->dyv, c->dzv, c->MF, c->Yz, c->NT * 32, c->N,
        c->p.dt, c->p.edot, sqrt(2.0 * c->p.dt));
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
