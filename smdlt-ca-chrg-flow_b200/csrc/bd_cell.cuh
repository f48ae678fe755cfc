// Periodic cell of the deforming lattice and cardinal B-splines, shared by
// the particle-mesh mobility (bd_pme.cu) and the Ewald Coulomb sum
// (bd_coulomb.cu).
#pragma once

#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bd_ctx.cuh"

using namespace bd;

struct Cell {
  double H[9];     // lattice vectors as columns (lab frame), row-major 3x3
  double Hi[9];    // inverse
  double V;        // volume
};

static const int kMaxOrder = 8;

__device__ __forceinline__ void frac_of(const Cell& c, double x, double y, double z, double s[3]) {
  s[0] = c.Hi[0] * x + c.Hi[1] * y + c.Hi[2] * z;
  s[1] = c.Hi[3] * x + c.Hi[4] * y + c.Hi[5] * z;
  s[2] = c.Hi[6] * x + c.Hi[7] * y + c.Hi[8] * z;
}

// Cardinal B-spline weights: w[k] = M_p(f + k), k = 0..p-1, for the grid point
// floor(u) - k, from M_n(x) = (x M_{n-1}(x) + (n - x) M_{n-1}(x - 1))/(n - 1).
__device__ __forceinline__ void bspline(double f, int p, double* w) {
  double a[kMaxOrder], b[kMaxOrder];
  a[0] = f;
  a[1] = 1.0 - f;
  for (int n = 3; n <= p; n++) {
    for (int k = 0; k < n; k++) {
      double hi = k < n - 1 ? a[k] : 0.0, lo = k >= 1 ? a[k - 1] : 0.0;
      b[k] = ((f + k) * hi + (n - f - k) * lo) / (n - 1);
    }
    for (int k = 0; k < n; k++) a[k] = b[k];
  }
  for (int k = 0; k < p; k++) w[k] = a[k];
}

// bspline with the order known at compile time (loops unrolled, the
// recursion's arrays in registers).
template <int P>
__device__ __forceinline__ void bspline_t(double f, double* w) {
  double a[P], b[P];
  a[0] = f;
  a[1] = 1.0 - f;
#pragma unroll
  for (int n = 3; n <= P; n++) {
#pragma unroll
    for (int k = 0; k < n; k++) {
      double hi = k < n - 1 ? a[k] : 0.0, lo = k >= 1 ? a[k - 1] : 0.0;
      b[k] = ((f + k) * hi + (n - f - k) * lo) / (n - 1);
    }
#pragma unroll
    for (int k = 0; k < n; k++) a[k] = b[k];
  }
#pragma unroll
  for (int k = 0; k < P; k++) w[k] = a[k];
}

static inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

// Lab-frame cell of the current lattice: columns b1, b2, L e_z with (b1, b2)
// the Gauss-reduced basis of the lattice spanned by L1 and L2
// (|b1| <= |b2|, |b1.b2| <= |b1|^2/2).
static Cell make_cell(const Lat& l) {
  Cell c;
  double a[2] = {l.L1x, l.L1y}, b[2] = {l.L2x, l.L2y};
  for (int it = 0; it < 64; it++) {
    double aa = a[0] * a[0] + a[1] * a[1], bb = b[0] * b[0] + b[1] * b[1];
    if (aa > bb) {
      std::swap(a[0], b[0]);
      std::swap(a[1], b[1]);
      std::swap(aa, bb);
    }
    double mu = rint((a[0] * b[0] + a[1] * b[1]) / aa);
    if (mu == 0.0) break;
    b[0] -= mu * a[0];
    b[1] -= mu * a[1];
  }
  double H[9] = {a[0], b[0], 0.0, a[1], b[1], 0.0, 0.0, 0.0, l.L};
  memcpy(c.H, H, sizeof(H));
  double det = H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) +
               H[2] * (H[3] * H[7] - H[4] * H[6]);
  c.V = fabs(det);
  double* I = c.Hi;
  I[0] = (H[4] * H[8] - H[5] * H[7]) / det;
  I[1] = (H[2] * H[7] - H[1] * H[8]) / det;
  I[2] = (H[1] * H[5] - H[2] * H[4]) / det;
  I[3] = (H[5] * H[6] - H[3] * H[8]) / det;
  I[4] = (H[0] * H[8] - H[2] * H[6]) / det;
  I[5] = (H[2] * H[3] - H[0] * H[5]) / det;
  I[6] = (H[3] * H[7] - H[4] * H[6]) / det;
  I[7] = (H[1] * H[6] - H[0] * H[7]) / det;
  I[8] = (H[0] * H[4] - H[1] * H[3]) / det;
  return c;
}

// |b(m)|^2 = 1/|sum_{k=0}^{p-2} M_p(k+1) exp(2 pi i m k / K)|^2
static void bspline_moduli(int K, int p, double* out) {
  std::vector<double> Mk(p + 1, 0.0);
  // M_p at the integers 1..p-1 from the same recursion (f = 0)
  std::vector<double> a = {0.0, 1.0};
  for (int n = 3; n <= p; n++) {
    std::vector<double> b(n, 0.0);
    for (int k = 0; k < n; k++) {
      double hi = k < n - 1 ? a[k] : 0.0, lo = k >= 1 ? a[k - 1] : 0.0;
      b[k] = (k * hi + (n - k) * lo) / (n - 1);
    }
    a = b;
  }
  for (int m = 0; m < K; m++) {
    double re = 0, im = 0;
    for (int k = 0; k <= p - 2; k++) {
      double w = a[k + 1];  // M_p(k + 1)
      re += w * cos(2 * M_PI * m * k / K);
      im += w * sin(2 * M_PI * m * k / K);
    }
    double d = re * re + im * im;
    out[m] = d > 1e-300 ? 1.0 / d : 0.0;
  }
}

