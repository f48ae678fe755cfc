// Ewald-summed Coulomb forces and energy between signed bead charges.
//
// No counterpart in the reference, whose electrostatics is the screened
// Debye-Hueckel pair force over all charged pairs (coulombForce,
// shear/src/main26.c:1891-1925; U = lambda_B q_i q_j exp(-kappa r)/r, in kT).
// With coulomb = BD_COULOMB_EWALD the unscreened U = lambda_B q_i q_j / r is
// summed over the periodic deforming lattice by the Ewald split
//   U = sum_pairs lambda_B q_i q_j erfc(beta r)/r                (real space)
//     + (1/2V) sum_{k != 0} (4 pi lambda_B/k^2) exp(-k^2/4beta^2) |S(k)|^2
//     - lambda_B beta/sqrt(pi) sum_i q_i^2                        (self)
//     - pi lambda_B Q^2 / (2 V beta^2)                            (background,
//       only for a net charge Q),
// the reciprocal part by smooth PME (Essmann et al., J. Chem. Phys. 103, 8577
// (1995)) on the same grid size, spline order and Gauss-reduced cell as the
// particle-mesh mobility, forces from the analytic derivative of the
// B-splines.  Real-space pairs within the cutoff come from a cell list of the
// charged beads rebuilt every call.  FP64 throughout (the energies feed
// Metropolis tests).
#include <cufft.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "bd_ctx.cuh"
#include "bd_cell.cuh"

#define CU(call) BD_CU(call)
#define CF(call) BD_CF(call)

namespace {

constexpr int kCellCap = 8192;

struct CGeom {
  int n[3];
};

__device__ __forceinline__ void lab_of(double x, double y, double cr, double sr, double& lx,
                                       double& ly) {
  lx = x * cr - y * sr;
  ly = x * sr + y * cr;
}

// Per charge: base index, B-spline weights of order p and their derivatives
// d/du M_p(u - g) = M_{p-1}(f + k) - M_{p-1}(f + k - 1) for g = floor(u) - k.
// One thread per (charge, direction d); the spline order P is a template
// parameter so the recursion stays in registers.
template <int P>
__global__ void k_cw_weights(Cell cell, const double4* __restrict__ cq, int nch, double cr,
                             double sr, int K, int* base, double* w, double* dw, int* err) {
  constexpr int p = P;
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 3 * nch) return;
  int k = e / 3, d = e % 3;
  double4 q = cq[k];
  double x, y, s[3];
  lab_of(q.x, q.y, cr, sr, x, y);
  frac_of(cell, x, y, q.z, s);
  {
    double sd = s[d] - floor(s[d]);
    double u = sd * K;
    if (!(u >= 0.0 && u <= (double)K)) {
      u = 0.0;
      atomicOr(err, ERRB_NONFINITE);
    }
    int fl = (int)floor(u);
    double f = u - fl;
    if (fl >= K) fl -= K;
    base[3 * k + d] = fl;
    double lo[P - 1], full[P];
    bspline_t<P - 1>(f, lo);  // M_{p-1}(f + k), k = 0..p-2
    bspline_t<P>(f, full);
    double* wo = w + ((size_t)3 * k + d) * kMaxOrder;
    double* dwo = dw + ((size_t)3 * k + d) * kMaxOrder;
#pragma unroll
    for (int a = 0; a < p; a++) {
      double hi = a < p - 1 ? lo[a] : 0.0, lm = a >= 1 ? lo[a - 1] : 0.0;
      wo[a] = full[a];
      dwo[a] = hi - lm;
    }
  }
}

// Q(g) += q_k W_k(g), one warp per charge, FP64 atomics.
__global__ void k_cw_spread(const double4* __restrict__ cq, const int* __restrict__ base,
                            const double* __restrict__ w, int nch, int K, int p, double* grid) {
  int k = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (k >= nch) return;
  double q = cq[k].w;
  const double* w0 = w + ((size_t)3 * k) * kMaxOrder;
  const double* w1 = w0 + kMaxOrder;
  const double* w2 = w1 + kMaxOrder;
  int b0 = base[3 * k], b1 = base[3 * k + 1], b2 = base[3 * k + 2];
  for (int e = lane; e < p * p * p; e += 32) {
    int c = e % p, b = (e / p) % p, a = e / (p * p);
    int g0 = b0 - a, g1 = b1 - b, g2 = b2 - c;
    g0 += g0 < 0 ? K : 0;
    g1 += g1 < 0 ? K : 0;
    g2 += g2 < 0 ? K : 0;
    atomicAdd(grid + ((size_t)g0 * K + g1) * K + g2, q * w0[a] * w1[b] * w2[c]);
  }
}

// Spectrum times G(m) = (4 pi lambda_B / V k^2) exp(-k^2/4 beta^2) |b(m)|^2 on
// the half spectrum; per-block partial sums of the reciprocal energy
// (1/2) sum_m G |F(Q)|^2 with Hermitian multiplicity.
__global__ void __launch_bounds__(256) k_cw_influence(Cell cell, int K, double beta,
                                                      double lambda_b,
                                                      const double* __restrict__ bsq,
                                                      cufftDoubleComplex* spec, double* epart) {
  int Kh = K / 2 + 1;
  size_t n = (size_t)K * K * Kh;
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double en = 0;
  __shared__ double red[256];
  if (e < n) {
    int m2 = (int)(e % Kh), m1 = (int)((e / Kh) % K), m0 = (int)(e / ((size_t)Kh * K));
    cufftDoubleComplex v = spec[e];
    if (m0 == 0 && m1 == 0 && m2 == 0) {
      v.x = v.y = 0.0;
    } else {
      int s0 = m0 < (K + 1) / 2 ? m0 : m0 - K, s1 = m1 < (K + 1) / 2 ? m1 : m1 - K, s2 = m2;
      double kv[3];
      for (int a = 0; a < 3; a++)
        kv[a] = 2.0 * M_PI *
                (s0 * cell.Hi[0 * 3 + a] + s1 * cell.Hi[1 * 3 + a] + s2 * cell.Hi[2 * 3 + a]);
      double kk = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
      double G = 4.0 * M_PI * lambda_b / (cell.V * kk) * exp(-kk / (4.0 * beta * beta)) *
                 bsq[m0] * bsq[K + m1] * bsq[2 * K + m2];
      double mult = (m2 == 0 || (K % 2 == 0 && m2 == K / 2)) ? 1.0 : 2.0;
      en = 0.5 * mult * G * (v.x * v.x + v.y * v.y);
      v.x *= G;
      v.y *= G;
    }
    spec[e] = v;
  }
  red[threadIdx.x] = en;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) epart[blockIdx.x] = red[0];
}

// Per-block partial sums of sum_{k != 0} A_k k_a k_b over the mesh spectrum,
// A_k = (2 pi lambda_B / V k^2) exp(-k^2/4 beta^2) (the reciprocal energy is
// sum_k A_k |S(k)|^2 over all k), six components (xx xy xz yy yz zz).
__global__ void __launch_bounds__(256) k_cw_quad(Cell cell, int K, double beta, double lambda_b,
                                                 double* part) {
  int Kh = K / 2 + 1;
  size_t n = (size_t)K * K * Kh;
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (e < n) {
    int m2 = (int)(e % Kh), m1 = (int)((e / Kh) % K), m0 = (int)(e / ((size_t)Kh * K));
    if (m0 || m1 || m2) {
      int s0 = m0 < (K + 1) / 2 ? m0 : m0 - K, s1 = m1 < (K + 1) / 2 ? m1 : m1 - K, s2 = m2;
      double kv[3];
      for (int a = 0; a < 3; a++)
        kv[a] = 2.0 * M_PI *
                (s0 * cell.Hi[0 * 3 + a] + s1 * cell.Hi[1 * 3 + a] + s2 * cell.Hi[2 * 3 + a]);
      double kk = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
      double mult = (m2 == 0 || (K % 2 == 0 && m2 == K / 2)) ? 1.0 : 2.0;
      double A = mult * 2.0 * M_PI * lambda_b / (cell.V * kk) * exp(-kk / (4.0 * beta * beta));
      acc[0] = A * kv[0] * kv[0];
      acc[1] = A * kv[0] * kv[1];
      acc[2] = A * kv[0] * kv[2];
      acc[3] = A * kv[1] * kv[1];
      acc[4] = A * kv[1] * kv[2];
      acc[5] = A * kv[2] * kv[2];
    }
  }
  __shared__ double red[8][6];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int c = 0; c < 6; c++) {
    double v = acc[c];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[w][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < 6) {
    double v = 0;
    for (int q = 0; q < 8; q++) v += red[q][threadIdx.x];
    part[(size_t)blockIdx.x * 6 + threadIdx.x] = v;
  }
}

// Q = -sum_k A_k k k^T + lambda_B (2 beta^3 / (3 sqrt(pi))) I from the block
// partials (one warp per component, fixed order).
__global__ void k_cw_quad_fin(const double* __restrict__ part, int nblk, double beta,
                              double lambda_b, double* Q) {
  int c = blockIdx.x;
  double v = 0;
  for (int b = threadIdx.x; b < nblk; b += 32) v += part[(size_t)b * 6 + c];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (threadIdx.x == 0) {
    bool diag = c == 0 || c == 3 || c == 5;
    Q[c] = -v + (diag ? lambda_b * 2.0 * beta * beta * beta / (3.0 * sqrt(M_PI)) : 0.0);
  }
}

// Cell list of the charged beads (fractional cells of the reduced cell).
__global__ void k_cc_count(Cell cell, CGeom g, const double4* __restrict__ cq, int nch,
                           double cr, double sr, int* cell_of, int* count) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nch) return;
  double4 q = cq[k];
  double x, y, s[3];
  lab_of(q.x, q.y, cr, sr, x, y);
  frac_of(cell, x, y, q.z, s);
  int cd[3];
  for (int d = 0; d < 3; d++) {
    double sd = s[d] - floor(s[d]);
    int c = (sd >= 0.0 && sd <= 1.0) ? (int)(sd * g.n[d]) : 0;
    cd[d] = c >= g.n[d] ? g.n[d] - 1 : c;
  }
  int c = (cd[0] * g.n[1] + cd[1]) * g.n[2] + cd[2];
  cell_of[k] = c;
  atomicAdd(&count[c], 1);
}

__global__ void k_cc_scan(int ncell, int* count, int* start, int* cursor) {
  __shared__ int part[1024];
  int t = threadIdx.x, nt = blockDim.x;
  int per = (ncell + nt - 1) / nt, lo = t * per, hi = min(ncell, lo + per), s = 0;
  for (int c = lo; c < hi; c++) s += count[c];
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
    start[c] = b;
    cursor[c] = 0;
    b += count[c];
    count[c] = 0;
  }
  if (t == nt - 1) start[ncell] = part[t];
}

__global__ void k_cc_fill(const int* __restrict__ cell_of, const int* __restrict__ start,
                          int* cursor, int* idx, int nch) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nch) return;
  int c = cell_of[k];
  idx[start[c] + atomicAdd(&cursor[c], 1)] = k;
}

// Forces on each charge: reciprocal part from the potential grid and the
// spline derivatives, real-space pairs within rc; adds to the bead forces and
// writes the charge's real-space energy share (half of its pair sum).
template <int P>
__global__ void __launch_bounds__(256)
    k_cw_forces(Cell cell, CGeom g, const double4* __restrict__ cq, const int* __restrict__ track,
                int nch, double cr, double sr, int K, const int* __restrict__ base,
                const double* __restrict__ w, const double* __restrict__ dw,
                const double* __restrict__ phi, const int* __restrict__ cell_of,
                const int* __restrict__ start, const int* __restrict__ idx, double rc2,
                double beta, double lambda_b, double* fx, double* fy, double* fz,
                double* ereal) {
  int k = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (k >= nch) return;
  double4 me = cq[k];
  const double* w0 = w + ((size_t)3 * k) * kMaxOrder;
  const double* w1 = w0 + kMaxOrder;
  const double* w2 = w1 + kMaxOrder;
  const double* d0 = dw + ((size_t)3 * k) * kMaxOrder;
  const double* d1 = d0 + kMaxOrder;
  const double* d2 = d1 + kMaxOrder;
  int b0 = base[3 * k], b1 = base[3 * k + 1], b2 = base[3 * k + 2];
  double gu0 = 0, gu1 = 0, gu2 = 0;  // dPhi/du_d at the charge
  constexpr int p = P;
#pragma unroll
  for (int it = 0; it < (p * p * p + 31) / 32; it++) {
    int e = lane + 32 * it;
    if (e >= p * p * p) break;
    int c = e % p, b = (e / p) % p, a = e / (p * p);
    int g0 = b0 - a, g1 = b1 - b, g2 = b2 - c;
    g0 += g0 < 0 ? K : 0;
    g1 += g1 < 0 ? K : 0;
    g2 += g2 < 0 ? K : 0;
    double ph = phi[((size_t)g0 * K + g1) * K + g2];
    gu0 += d0[a] * w1[b] * w2[c] * ph;
    gu1 += w0[a] * d1[b] * w2[c] * ph;
    gu2 += w0[a] * w1[b] * d2[c] * ph;
  }
  // real space
  double xi, yi;
  lab_of(me.x, me.y, cr, sr, xi, yi);
  double zi = me.z;
  int ci = cell_of[k];
  int cd[3] = {ci / (g.n[1] * g.n[2]), (ci / g.n[2]) % g.n[1], ci % g.n[2]};
  double f0 = 0, f1 = 0, f2 = 0, en = 0;
  const double rtpi = sqrt(M_PI);
  int lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    lo[d] = g.n[d] >= 3 ? -1 : 0;
    hi[d] = g.n[d] >= 3 ? 1 : g.n[d] - 1;
  }
  // the (at most 27) neighbour cells as one candidate list: lane l < ncell
  // takes cell l's range; a warp scan of the counts places candidate m in
  // the cell whose range holds it, so the lanes walk all cells at once (no
  // chain of dependent loads per cell)
  __shared__ int c_start[8][32], c_excl[8][32], c_incl[8][32];
  const int wl = threadIdx.x >> 5;
  int nd[3] = {hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1};
  int ncell = nd[0] * nd[1] * nd[2];
  int my_s = 0, my_n = 0;
  if (lane < ncell) {
    int a = lo[0] + lane / (nd[1] * nd[2]), b = lo[1] + (lane / nd[2]) % nd[1],
        c = lo[2] + lane % nd[2];
    int e0 = g.n[0] >= 3 ? (cd[0] + a + g.n[0]) % g.n[0] : a;
    int e1 = g.n[1] >= 3 ? (cd[1] + b + g.n[1]) % g.n[1] : b;
    int e2 = g.n[2] >= 3 ? (cd[2] + c + g.n[2]) % g.n[2] : c;
    int cc = (e0 * g.n[1] + e1) * g.n[2] + e2;
    my_s = start[cc];
    my_n = start[cc + 1] - my_s;
  }
  int incl = my_n;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  c_start[wl][lane] = my_s;
  c_excl[wl][lane] = incl - my_n;
  c_incl[wl][lane] = incl;
  __syncwarp();
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  int cl = 0;
  for (int m = lane; m < total; m += 32) {
    while (m >= c_incl[wl][cl]) cl++;  // ends at the last cell: m < total
    int j = idx[c_start[wl][cl] + (m - c_excl[wl][cl])];
    if (j == k) continue;
    double4 ot = cq[j];
    double xj, yj;
    lab_of(ot.x, ot.y, cr, sr, xj, yj);
    double dx = xi - xj, dy = yi - yj, dz = zi - ot.z, s[3];
    frac_of(cell, dx, dy, dz, s);
    for (int d = 0; d < 3; d++) s[d] -= rint(s[d]);
    dx = cell.H[0] * s[0] + cell.H[1] * s[1] + cell.H[2] * s[2];
    dy = cell.H[3] * s[0] + cell.H[4] * s[1] + cell.H[5] * s[2];
    dz = cell.H[6] * s[0] + cell.H[7] * s[1] + cell.H[8] * s[2];
    double rr = dx * dx + dy * dy + dz * dz;
    if (rr >= rc2) continue;
    double r = sqrt(rr), qq = lambda_b * me.w * ot.w;
    double ec = erfc(beta * r) / r;
    double fr = qq * (ec + 2.0 * beta / rtpi * exp(-beta * beta * rr)) / rr;
    f0 += fr * dx;
    f1 += fr * dy;
    f2 += fr * dz;
    en += 0.5 * qq * ec;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    gu0 += __shfl_xor_sync(0xffffffffu, gu0, o);
    gu1 += __shfl_xor_sync(0xffffffffu, gu1, o);
    gu2 += __shfl_xor_sync(0xffffffffu, gu2, o);
    f0 += __shfl_xor_sync(0xffffffffu, f0, o);
    f1 += __shfl_xor_sync(0xffffffffu, f1, o);
    f2 += __shfl_xor_sync(0xffffffffu, f2, o);
    en += __shfl_xor_sync(0xffffffffu, en, o);
  }
  if (lane == 0) {
    // F = -q dPhi/dr, dPhi/dr_a = sum_d dPhi/du_d K Hi[d][a]
    double gq = -me.w * K;
    double fr0 = gq * (gu0 * cell.Hi[0] + gu1 * cell.Hi[3] + gu2 * cell.Hi[6]);
    double fr1 = gq * (gu0 * cell.Hi[1] + gu1 * cell.Hi[4] + gu2 * cell.Hi[7]);
    double fr2 = gq * (gu0 * cell.Hi[2] + gu1 * cell.Hi[5] + gu2 * cell.Hi[8]);
    // forces in the lab frame, as the other force routines accumulate them
    int i = track[k];
    fx[i] += f0 + fr0;
    fy[i] += f1 + fr1;
    fz[i] += f2 + fr2;
    ereal[k] = en;
  }
}

// Fixed-order sums: out[0] += sum part[0..n) (one warp)
__global__ void k_sum_into(const double* __restrict__ part, int n, double* out) {
  double s = 0;
  for (int b = threadIdx.x; b < n; b += 32) s += part[b];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) *out = s;
}

}  // namespace

namespace bd {

static int coul_alloc(bd_ctx* c) {
  if (c->cw_grid) return BD_OK;
  // per-charge arrays sized for every bead charged (charges can be reset)
  int K = c->pmeK, n = std::max(c->N, 1);
  size_t K3 = (size_t)K * K * K, Ks = (size_t)K * K * (K / 2 + 1);
  CU(cudaMalloc(&c->cw_grid, 8 * K3));
  CU(cudaMalloc(&c->cw_spec, 16 * Ks));
  CU(cudaMalloc(&c->cw_bsq, 24 * (size_t)K));
  c->cw_nblk = (int)((Ks + 255) / 256);
  CU(cudaMalloc(&c->cw_epart, 8 * (size_t)std::max(6 * c->cw_nblk, n)));
  CU(cudaMalloc(&c->cw_energy, 8 * 4));
  CU(cudaMalloc(&c->cw_base, 12 * (size_t)n));
  CU(cudaMalloc(&c->cw_w, 2 * 8 * 3 * (size_t)n * kMaxOrder));
  CU(cudaMalloc(&c->cw_cell_of, 4 * (size_t)n));
  CU(cudaMalloc(&c->cw_idx, 4 * (size_t)n));
  CU(cudaMalloc(&c->cw_count, 4 * (size_t)kCellCap));
  CU(cudaMalloc(&c->cw_start, 4 * (size_t)(kCellCap + 1)));
  CU(cudaMalloc(&c->cw_cursor, 4 * (size_t)kCellCap));
  CU(cudaMemsetAsync(c->cw_count, 0, 4 * (size_t)kCellCap, c->stream));
  CU(cudaMemsetAsync(c->cw_energy, 0, 32, c->stream));
  c->bytes += 8 * K3 + 16 * Ks + 24 * (size_t)K + 8 * (size_t)std::max(6 * c->cw_nblk, n) + 32 +
              (size_t)n * (12 + 48 * kMaxOrder + 8) + 12 * (size_t)kCellCap;
  int dims[3] = {K, K, K};
  cufftHandle f, b;
  CF(cufftPlanMany(&f, 3, dims, nullptr, 1, (int)K3, nullptr, 1, (int)Ks, CUFFT_D2Z, 1));
  CF(cufftPlanMany(&b, 3, dims, nullptr, 1, (int)Ks, nullptr, 1, (int)K3, CUFFT_Z2D, 1));
  CF(cufftSetStream(f, c->stream));
  CF(cufftSetStream(b, c->stream));
  c->cw_plan_f = (int)f;
  c->cw_plan_b = (int)b;
  std::vector<double> bs(3 * (size_t)K);
  bspline_moduli(K, c->pme_p, bs.data());
  for (int d = 1; d < 3; d++)
    for (int m = 0; m < K; m++) bs[(size_t)d * K + m] = bs[m];
  CU(cudaMemcpyAsync(c->cw_bsq, bs.data(), 8 * bs.size(), cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return BD_OK;
}

void coulomb_free(bd_ctx* c) {
  if (c->cw_plan_f) cufftDestroy((cufftHandle)c->cw_plan_f);
  if (c->cw_plan_b) cufftDestroy((cufftHandle)c->cw_plan_b);
  void* ptrs[] = {c->cw_grid, c->cw_spec, c->cw_bsq, c->cw_epart, c->cw_energy, c->cw_base,
                  c->cw_w, c->cw_cell_of, c->cw_idx, c->cw_count, c->cw_start, c->cw_cursor};
  for (void* q : ptrs)
    if (q) cudaFree(q);
}

// Reciprocal-space potential of the charges gathered in cq on the mesh:
// c->cw_grid = phi with Phi(r) = sum_g W(r - g) phi(g) the smooth-PME
// reciprocal potential (kT per unit charge, lambda_B included) at any point r
// (the same weights, spread, transform and influence as coulomb_ewald; the
// energies it keeps are not touched).  Used by the charge-hop sweep's Ewald
// energy differences.
int coulomb_mesh_potential(bd_ctx* c, const Lat& l, const double4* cq) {
  int s;
  if ((s = coul_alloc(c)) != BD_OK) return s;
  int K = c->pmeK, p = c->pme_p, nch = c->nch;
  Cell cell = make_cell(l);
  double cr = 1.0, sr = 0.0;
  if (l.flow == BD_FLOW_EXT) {
    cr = l.cth;
    sr = l.sth;
  }
  size_t K3 = (size_t)K * K * K;
  double* w = c->cw_w;
  double* dw = c->cw_w + 3 * (size_t)nch * kMaxOrder;
  c->launches += 5;
#define CW_WEIGHTS(P_)                                                                      \
  k_cw_weights<P_><<<nblk(3 * (long long)nch, 128), 128, 0, c->stream>>>(cell, cq, nch, cr, sr, K, \
                                                                        c->cw_base, w, dw, c->err)
  switch (p) {
    case 4: CW_WEIGHTS(4); break;
    case 6: CW_WEIGHTS(6); break;
    default: CW_WEIGHTS(8);
  }
#undef CW_WEIGHTS
  CU(cudaMemsetAsync(c->cw_grid, 0, 8 * K3, c->stream));
  k_cw_spread<<<nblk(nch, 8), 256, 0, c->stream>>>(cq, c->cw_base, w, nch, K, p, c->cw_grid);
  CF(cufftExecD2Z((cufftHandle)c->cw_plan_f, c->cw_grid, (cufftDoubleComplex*)c->cw_spec));
  k_cw_influence<<<c->cw_nblk, 256, 0, c->stream>>>(cell, K, c->cw_beta, c->p.lambda_b,
                                                    c->cw_bsq, (cufftDoubleComplex*)c->cw_spec,
                                                    c->cw_epart);
  CF(cufftExecZ2D((cufftHandle)c->cw_plan_b, (cufftDoubleComplex*)c->cw_spec, c->cw_grid));
  return launch_ok(c);
}

// Quadratic form of the periodic remainder of the reciprocal pair term near
// the origin: G(r) = lambda_B erf(beta r)/r + r^T Q r + const + O(r^4), into
// Q6 (device, xx xy xz yy yz zz), for the lattice l.  For a cubic lattice
// Q = (2 pi lambda_B / 3 V) I.
int coulomb_quadform(bd_ctx* c, const Lat& l, double* Q6) {
  int s;
  if ((s = coul_alloc(c)) != BD_OK) return s;
  Cell cell = make_cell(l);
  c->launches += 2;
  k_cw_quad<<<c->cw_nblk, 256, 0, c->stream>>>(cell, c->pmeK, c->cw_beta, c->p.lambda_b,
                                              c->cw_epart);
  k_cw_quad_fin<<<6, 32, 0, c->stream>>>(c->cw_epart, c->cw_nblk, c->cw_beta, c->p.lambda_b, Q6);
  return launch_ok(c);
}

// Ewald Coulomb forces for the charges gathered in cq (positions in the frame
// the force routines receive them: stored frame, rotated to the lab frame by
// the lattice angle in extension), added to fx, fy, fz; energies into
// c->cw_energy = {real, reciprocal, self + background, total}.
int coulomb_ewald(bd_ctx* c, const Lat& l, const double4* cq) {
  int s;
  if ((s = coul_alloc(c)) != BD_OK) return s;
  int K = c->pmeK, p = c->pme_p, nch = c->nch;
  Cell cell = make_cell(l);
  double cr = 1.0, sr = 0.0;
  if (l.flow == BD_FLOW_EXT) {
    cr = l.cth;
    sr = l.sth;
  }
  // cell list: widths V / |a_j x a_k| >= rc
  double wdt[3];
  for (int j = 0; j < 3; j++) {
    double a[3][3];
    for (int q = 0; q < 3; q++)
      for (int d = 0; d < 3; d++) a[q][d] = cell.H[d * 3 + q];
    const double* u = a[(j + 1) % 3];
    const double* v = a[(j + 2) % 3];
    double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2],
           cz = u[0] * v[1] - u[1] * v[0];
    wdt[j] = cell.V / sqrt(cx * cx + cy * cy + cz * cz);
  }
  double rc = c->cw_rc;
  if (2 * rc > std::min(wdt[0], std::min(wdt[1], wdt[2]))) return BD_ERR_ARG;
  CGeom g;
  for (int d = 0; d < 3; d++) g.n[d] = std::max(1, (int)floor(wdt[d] / rc));
  while ((long)g.n[0] * g.n[1] * g.n[2] > kCellCap) {
    int d = g.n[0] >= g.n[1] && g.n[0] >= g.n[2] ? 0 : (g.n[1] >= g.n[2] ? 1 : 2);
    g.n[d]--;
  }
  int ncell = g.n[0] * g.n[1] * g.n[2];
  size_t K3 = (size_t)K * K * K;
  double* w = c->cw_w;
  double* dw = c->cw_w + 3 * (size_t)nch * kMaxOrder;
  c->launches += 9;
#define CW_WEIGHTS(P_)                                                                      \
  k_cw_weights<P_><<<nblk(3 * (long long)nch, 128), 128, 0, c->stream>>>(cell, cq, nch, cr, sr, K, \
                                                                        c->cw_base, w, dw, c->err)
  switch (p) {
    case 4: CW_WEIGHTS(4); break;
    case 6: CW_WEIGHTS(6); break;
    default: CW_WEIGHTS(8);
  }
#undef CW_WEIGHTS
  CU(cudaMemsetAsync(c->cw_grid, 0, 8 * K3, c->stream));
  k_cw_spread<<<nblk(nch, 8), 256, 0, c->stream>>>(cq, c->cw_base, w, nch, K, p, c->cw_grid);
  CF(cufftExecD2Z((cufftHandle)c->cw_plan_f, c->cw_grid, (cufftDoubleComplex*)c->cw_spec));
  k_cw_influence<<<c->cw_nblk, 256, 0, c->stream>>>(cell, K, c->cw_beta, c->p.lambda_b,
                                                    c->cw_bsq, (cufftDoubleComplex*)c->cw_spec,
                                                    c->cw_epart);
  k_sum_into<<<1, 32, 0, c->stream>>>(c->cw_epart, c->cw_nblk, c->cw_energy + 1);
  CF(cufftExecZ2D((cufftHandle)c->cw_plan_b, (cufftDoubleComplex*)c->cw_spec, c->cw_grid));
  k_cc_count<<<nblk(nch, 256), 256, 0, c->stream>>>(cell, g, cq, nch, cr, sr, c->cw_cell_of,
                                                    c->cw_count);
  k_cc_scan<<<1, 1024, 0, c->stream>>>(ncell, c->cw_count, c->cw_start, c->cw_cursor);
  k_cc_fill<<<nblk(nch, 256), 256, 0, c->stream>>>(c->cw_cell_of, c->cw_start, c->cw_cursor,
                                                   c->cw_idx, nch);
#define CW_FORCES(P_)                                                                        \
  k_cw_forces<P_><<<nblk(nch, 8), 256, 0, c->stream>>>(                                       \
      cell, g, cq, c->track, nch, cr, sr, K, c->cw_base, w, dw, c->cw_grid, c->cw_cell_of,    \
      c->cw_start, c->cw_idx, rc * rc, c->cw_beta, c->p.lambda_b, c->fx, c->fy, c->fz,        \
      c->cw_epart)
  switch (p) {
    case 4: CW_FORCES(4); break;
    case 6: CW_FORCES(6); break;
    default: CW_FORCES(8);
  }
#undef CW_FORCES
  k_sum_into<<<1, 32, 0, c->stream>>>(c->cw_epart, nch, c->cw_energy);
  c->cw_cell_V = cell.V;
  return launch_ok(c);
}

}  // namespace bd

extern "C" {

int bd_set_charge_values(bd_ctx* c, const double* qk) {
  if (!c || (c->nch > 0 && !qk)) return BD_ERR_ARG;
  std::vector<int> track(c->nch);
  if (c->nch)
    CU(cudaMemcpyAsync(track.data(), c->track, 4 * (size_t)c->nch, cudaMemcpyDeviceToHost,
                       c->stream));
  CU(cudaStreamSynchronize(c->stream));
  std::vector<double> q(c->N, 0.0);
  double q2 = 0, Q = 0;
  for (int k = 0; k < c->nch; k++) {
    q[track[k]] = qk[k];
    q2 += qk[k] * qk[k];
    Q += qk[k];
  }
  CU(cudaMemcpyAsync(c->q, q.data(), 8 * (size_t)c->N, cudaMemcpyHostToDevice, c->stream));
  c->cw_q2 = q2;
  c->cw_Q = Q;
  return check(c);
}

int bd_coulomb_energy(bd_ctx* c, double* out4) {
  if (!c || !out4) return BD_ERR_ARG;
  if (c->p.coulomb != BD_COULOMB_EWALD || !c->cw_energy) return BD_ERR_STATE;
  double e[2];
  CU(cudaMemcpyAsync(e, c->cw_energy, 16, cudaMemcpyDeviceToHost, c->stream));
  int s;
  if ((s = check(c)) != BD_OK) return s;
  double lb = c->p.lambda_b, b = c->cw_beta;
  double self = -lb * b / sqrt(M_PI) * c->cw_q2;
  double bg = c->cw_cell_V > 0 ? -M_PI * lb * c->cw_Q * c->cw_Q / (2.0 * c->cw_cell_V * b * b) : 0.0;
  out4[0] = e[0];
  out4[1] = e[1];
  out4[2] = self + bg;
  out4[3] = e[0] + e[1] + self + bg;
  return BD_OK;
}

}  // extern "C"
