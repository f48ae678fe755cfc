// Internal declarations shared by the bd_b200 CUDA translation units.
//
// Arithmetic that the reference decides by comparisons -- the minimum-image
// vector of getNID/getNIDbin, squared distances, periodic wrapping -- is
// written with explicit round-to-nearest intrinsics (__dmul_rn, __dadd_rn,
// __dsub_rn) so nvcc cannot contract it into FMAs.  With the same operation
// order as the reference this makes neighbour sets and charge-hop proposals
// bit-identical to the host code, which is compiled without FMA.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "bd_b200.h"

namespace bd {

// Records the failing CUDA or cuFFT call (code, message, source line) for
// bd_last_error_detail and returns BD_ERR_CUDA.
int cuda_fail(int code, const char* msg, const char* file, int line);
// Replaces the calling thread's bd_last_error_detail text.
void set_error_detail(const char* msg);

// Lattice of the deforming cell at one step (updateLattice,
// shear/src/main26.c:1382-1408, extensional/src/main14.c:1426-1450).  Built
// on the host with the C library's transcendental functions and passed to
// kernels by value.
struct Lat {
  int flow;   // 0 shear, 1 extension
  int treal;  // t % tp
  int tp;
  int nmax;   // Ewald image range: 1 for treal <= tp/2 else 2
  double L;
  double L1x, L1y, L2x, L2y;      // cell vectors, lab frame
  double L1xp, L1yp, L2xp, L2yp;  // cell vectors, frame rotated by theta
  double detL;
  double cth, sth;                // cos/sin of theta = atan(L1y/L1x)
  double delx;                    // edot * treal * dt (shear brick offset)
};

// Error bits recorded by kernels in the context's device error word.
enum : int {
  ERRB_OVERSTRETCH = 1 << 0,
  ERRB_NONFINITE = 1 << 1,
  ERRB_NBR_OVERFLOW = 1 << 2,
  ERRB_GRID_RANGE = 1 << 3,
  ERRB_TIMEOUT = 1 << 4,
};

__device__ __forceinline__ double mulx(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double addx(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double subx(double a, double b) { return __dsub_rn(a, b); }

__device__ __forceinline__ double rr3(double x, double y, double z) {
  return addx(addx(mulx(x, x), mulx(y, y)), mulx(z, z));
}

// getNID on a raw difference d = r_i - r_j (shear/src/main26.c:1429-1457,
// extensional/src/main14.c:1462-1480).
__device__ __forceinline__ void min_image(const Lat& l, double dx, double dy, double dz,
                                          double& ox, double& oy, double& oz) {
  dx = subx(dx, mulx(l.L2xp, round(dy / l.L2yp)));
  if (l.flow == 0) {
    if (dy > l.L2yp / 2) {
      dx = subx(dx, l.delx);
      dy = subx(dy, mulx(l.L2yp, round(dy / l.L2yp)));
    } else if (dy < -l.L2yp / 2) {
      dx = addx(dx, l.delx);
      dy = subx(dy, mulx(l.L2yp, round(dy / l.L2yp)));
    }
    dx = subx(dx, mulx(l.L1xp, round(dx / l.L1xp)));
    dz = subx(dz, mulx(l.L, round(dz / l.L)));
    ox = dx;
    oy = dy;
    oz = dz;
  } else {
    dy = subx(dy, mulx(l.L2yp, round(dy / l.L2yp)));
    dx = subx(dx, mulx(l.L1xp, round(dx / l.L1xp)));
    dz = subx(dz, mulx(l.L, round(dz / l.L)));
    ox = subx(mulx(dx, l.cth), mulx(dy, l.sth));
    oy = addx(mulx(dx, l.sth), mulx(dy, l.cth));
    oz = dz;
  }
}

__device__ __forceinline__ void nid(const Lat& l, const double* __restrict__ rx,
                                    const double* __restrict__ ry, const double* __restrict__ rz,
                                    int i, int j, double& ox, double& oy, double& oz) {
  min_image(l, subx(rx[i], rx[j]), subx(ry[i], ry[j]), subx(rz[i], rz[j]), ox, oy, oz);
}

// getNIDbin: minimum over the (nx,ny) images in the rotated frame
// (shear/src/main26.c:1458-1497, extensional/src/main14.c:1481-1513).
__device__ __forceinline__ void min_image_bin(const Lat& l, double dx, double dy, double dz,
                                              double& ox, double& oy, double& oz) {
  int nmax = l.nmax;
  dz = subx(dz, mulx(l.L, round(dz / l.L)));
  double dxmin = dx, dymin = dy;
  double rmin = sqrt(addx(mulx(dx, dx), mulx(dy, dy)));
  if (l.flow == 0) {
    if (dy > l.L2yp / 2)
      dx = subx(dx, l.delx);
    else if (dy < -l.L2yp / 2)
      dx = addx(dx, l.delx);
  }
  for (int nx = -nmax; nx < nmax + 1; nx++)
    for (int ny = -nmax; ny < nmax + 1; ny++) {
      double dxp = addx(addx(dx, mulx((double)nx, l.L1xp)), mulx((double)ny, l.L2xp));
      double dyp = addx(dy, mulx((double)ny, l.L2yp));
      double rp = sqrt(addx(mulx(dxp, dxp), mulx(dyp, dyp)));
      if (rp < rmin) {
        dxmin = dxp;
        dymin = dyp;
        rmin = rp;
      }
    }
  if (l.flow == 0) {
    ox = dxmin;
    oy = dymin;
  } else {
    ox = subx(mulx(dxmin, l.cth), mulx(dymin, l.sth));
    oy = addx(mulx(dxmin, l.sth), mulx(dymin, l.cth));
  }
  oz = dz;
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with a Weyl key
// schedule.
__device__ __forceinline__ uint4 philox4x32_10(uint4 ctr, uint2 key) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = __umulhi(M0, ctr.x), lo0 = M0 * ctr.x;
    uint32_t hi1 = __umulhi(M1, ctr.z), lo1 = M1 * ctr.z;
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += W0;
    key.y += W1;
  }
  return ctr;
}

// Device copy of the reference's ran1 state (64-bit longs).
struct Ran1 {
  long long idum, idum2, iy;
  long long iv[32];
  int iset;
  float gset;
};

// ran1 (shear/src/Initialization.c:601-634), including that idum2 is never
// advanced.
__device__ __forceinline__ float ran1_dev(Ran1& g) {
  const long long IM1 = 2147483563LL, IA1 = 40014LL, IQ1 = 53668LL, IR1 = 12211LL;
  const long long IMM1 = IM1 - 1, NDIV = 1 + IMM1 / 32;
  long long k;
  if (g.idum <= 0) {
    if (-(g.idum) < 1)
      g.idum = 1;
    else
      g.idum = -(g.idum);
    g.idum2 = g.idum;
    for (int j = 32 + 7; j >= 0; --j) {
      k = g.idum / IQ1;
      g.idum = IA1 * (g.idum - k * IQ1) - k * IR1;
      if (g.idum < 0) g.idum += IM1;
      if (j < 32) g.iv[j] = g.idum;
    }
    g.iy = g.iv[0];
  }
  k = g.idum / IQ1;
  g.idum = IA1 * (g.idum - k * IQ1) - k * IR1;
  if (g.idum < 0) g.idum += IM1;
  int j = (int)(g.iy / NDIV);
  g.iy = g.iv[j] - g.idum2;
  g.iv[j] = g.idum;
  if (g.iy < 1) g.iy += IMM1;
  float temp = (float)((1.0 / (double)IM1) * (double)g.iy);
  if ((double)temp > (1.0 - 1.2e-7)) return (float)(1.0 - 1.2e-7);
  return temp;
}

}  // namespace bd

// Checked CUDA runtime and cuFFT calls inside functions returning a status.
#define BD_CU(call)                                                                   \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return bd::cuda_fail((int)e_, cudaGetErrorString(e_), __FILE__, __LINE__);      \
  } while (0)
#define BD_CF(call)                                                                   \
  do {                                                                                \
    int r_ = (int)(call);                                                             \
    if (r_ != 0) return bd::cuda_fail(r_, "cuFFT call failed", __FILE__, __LINE__);   \
  } while (0)
