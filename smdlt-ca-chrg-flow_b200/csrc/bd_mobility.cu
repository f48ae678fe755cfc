// Dense hybrid Rotne-Prager-Yamakawa mobility (reference mode) and the TEA
// Brownian displacement.
//
// Storage.  M is symmetric with symmetric 3x3 blocks, so only the upper
// triangle of 32x32-bead tiles is stored, six unique components per block,
// component-major inside a tile: tile(I,J), I <= J, at packed index
// I*NT - I*(I-1)/2 + (J-I), element (c, il, jl) at c*1024 + il*32 + jl.
// A warp reading one (c, il) row reads 256 contiguous bytes.  The diagonal
// blocks are the reference's uniform self term Dtr (calcHI writes only their
// diagonal entries, shear/src/main26.c:1687-1692) and are kept as 3 scalars.
//
// Build (calcHI, shear/src/main26.c:1530-1806).  A far pass evaluates the
// minimum image over the (nx,ny) images for every pair (getNIDbin), copies
// the lookup tensor for pairs at 12 or more, and appends nearer pairs to a
// list with one atomic per warp.  A near pass gives each listed pair a warp
// whose lanes split the real-space image sum and the k-space cosine sum.
// The k-vectors, their coefficients and Dtr are generated on the host with
// the reference's loop bounds and arithmetic.
//
// Matvec.  One CTA per tile applies the block to both the tile's rows and its
// columns (block symmetry) for two right-hand sides at once, and writes the
// two partial sums to scratch; a two-level reduction sums them per bead in a
// fixed order, so results are deterministic without atomics.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bd_ctx.cuh"

using namespace bd;

#define CU(call) BD_CU(call)

static const int kRedSplit = 16;  // column-range splits of the matvec reduction

struct Ewald {
  double alpha, alpha2, alpha3, alpha5, alpha7, rce, rtpi;
  int nmax, nt, nk;
};

__device__ __forceinline__ long long tile_off(int I, int NT) {
  return (long long)I * NT - (long long)I * (I - 1) / 2;
}

// Real-space Beenakker RPY terms for one image at squared distance rr
// (shear/src/main26.c:1727-1741), with the overlap form for r <= 2.
__device__ __forceinline__ void rpy_real(const Ewald& e, double rr, double& t1, double& t2) {
  double r = sqrt(rr), C1, C2, C3, C4;
  double a = e.alpha, a3 = e.alpha3, a5 = e.alpha5, a7 = e.alpha7;
  if (r > 2.0) {
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
  double ec = erfc(a * r), ex = exp(-e.alpha2 * rr) / e.rtpi;
  t1 = C1 * ec + C2 * ex;
  t2 = C3 * ec + C4 * ex;
}

__global__ void __launch_bounds__(256) k_hi_far(Lat l, Ewald ew, const double* __restrict__ rx,
                                                const double* __restrict__ ry,
                                                const double* __restrict__ rz, int N, int NT,
                                                const int* __restrict__ tileI,
                                                const double* __restrict__ grid, int nbx,
                                                int nby, int nbz, int nhx, int nhy, int nhz,
                                                double bsx, double bsy, double bsz, int nbins,
                                                double* Mt, int2* near, int* near_count,
                                                long long near_cap, int* err) {
  long long tile = blockIdx.x;
  int I = tileI[tile];
  int J = I + (int)(tile - tile_off(I, NT));
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* tb = Mt + tile * 6144;
  const double* gt = grid + (size_t)ew.nt * nbins * 6;
  for (int q = 0; q < 4; q++) {
    int il = w + 8 * q;
    int i = I * 32 + il, j = J * 32 + lane;
    bool pair = (i < j) && (j < N);
    bool is_near = false;
    double m[6] = {0, 0, 0, 0, 0, 0};
    if (pair) {
      double vx, vy, vz;
      // getNIDbin(j, i) (shear/src/main26.c:1709)
      min_image_bin(l, subx(rx[j], rx[i]), subx(ry[j], ry[i]), subx(rz[j], rz[i]), vx, vy, vz);
      double d = sqrt(rr3(vx, vy, vz));
      if (d < 12.0) {
        is_near = true;
      } else {
        // binij(i, j) uses getNIDbin(j, i) as well (shear/src/main26.c:1518-1529)
        // the flattened index is used as the reference computes it: a bin
        // just off the table on one axis aliases to a neighbouring table row
        int bx = (int)(round(vx / bsx) + nhx), by = (int)(round(vy / bsy) + nhy);
        int bz = (int)(round(vz / bsz) + nhz);
        long long b = (long long)nby * nbz * bx + (long long)nbz * by + bz;
        if (b < 0 || b >= nbins) {
          atomicOr(err, ERRB_GRID_RANGE);
        } else {
          const double* g = gt + (size_t)b * 6;
          for (int a = 0; a < 6; a++) m[a] = g[a];
        }
      }
    }
    unsigned bal = __ballot_sync(0xffffffffu, is_near);
    if (bal) {
      int base = 0;
      int leader = __ffs(bal) - 1;
      if (lane == leader) base = atomicAdd(near_count, __popc(bal));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (is_near) {
        long long k = base + __popc(bal & ((1u << lane) - 1));
        if (k < near_cap)
          near[k] = make_int2(i, j);
        else
          atomicOr(err, ERRB_NBR_OVERFLOW);
      }
    }
    for (int a = 0; a < 6; a++) tb[a * 1024 + il * 32 + lane] = m[a];
  }
}

// kvec rows: rkx rky rkz m00 m01 m02 m11 m12 m22
// Lane share of the Ewald-summed RPY tensor at raw displacement (dxo,dyo,dzo):
// real-space images within rce (shear/src/main26.c:1722-1763) and the
// k-space cosine sum (shear/src/main26.c:1764-1788); lanes stride over both.
__device__ __forceinline__ void ewald6(const Lat& l, const Ewald& ew, double dxo, double dyo,
                                       double dzo, const double* __restrict__ kvec, int lane,
                                       double acc[6]) {
  for (int a = 0; a < 6; a++) acc[a] = 0.0;
  int side = 2 * ew.nmax + 1, nimg = side * side * side;
  for (int m = lane; m < nimg; m += 32) {
    int nz = m % side - ew.nmax, ny = (m / side) % side - ew.nmax, nx = m / (side * side) - ew.nmax;
    double dx = dxo + nx * l.L1x + ny * l.L2x;
    double dy = dyo + nx * l.L1y + ny * l.L2y;
    double dz = dzo + nz * l.L;
    double rr = dx * dx + dy * dy + dz * dz;
    if (sqrt(rr) < ew.rce) {
      double t1, t2;
      rpy_real(ew, rr, t1, t2);
      acc[0] += t1 + t2 * dx * dx / rr;
      acc[1] += t2 * dx * dy / rr;
      acc[2] += t2 * dx * dz / rr;
      acc[3] += t1 + t2 * dy * dy / rr;
      acc[4] += t2 * dy * dz / rr;
      acc[5] += t1 + t2 * dz * dz / rr;
    }
  }
  for (int c = lane; c < ew.nk; c += 32) {
    const double* kv = kvec + 9 * c;
    double ck = cos(kv[0] * dxo + kv[1] * dyo + kv[2] * dzo);
    acc[0] += kv[3] * ck;
    acc[1] += kv[4] * ck;
    acc[2] += kv[5] * ck;
    acc[3] += kv[6] * ck;
    acc[4] += kv[7] * ck;
    acc[5] += kv[8] * ck;
  }
}

__device__ __forceinline__ void near_pair(const Lat& l, const Ewald& ew,
                                          const double* __restrict__ rx,
                                          const double* __restrict__ ry,
                                          const double* __restrict__ rz, int NT, int2 ij,
                                          const double* __restrict__ kvec, double* Mt, int lane);

// Grid-stride over the near-pair list, one warp per pair.
__global__ void __launch_bounds__(256) k_hi_near(Lat l, Ewald ew, const double* __restrict__ rx,
                                                 const double* __restrict__ ry,
                                                 const double* __restrict__ rz, int NT,
                                                 const int2* __restrict__ near,
                                                 const int* __restrict__ near_count,
                                                 long long near_cap,
                                                 const double* __restrict__ kvec, double* Mt) {
  int lane = threadIdx.x & 31;
  long long np = min((long long)*near_count, near_cap);
  long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long p = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += nw)
    near_pair(l, ew, rx, ry, rz, NT, near[p], kvec, Mt, lane);
}

__device__ __forceinline__ void near_pair(const Lat& l, const Ewald& ew,
                                          const double* __restrict__ rx,
                                          const double* __restrict__ ry,
                                          const double* __restrict__ rz, int NT, int2 ij,
                                          const double* __restrict__ kvec, double* Mt, int lane) {
  int i = ij.x, j = ij.y;
  double rxi, ryi, rxj, ryj;
  if (l.flow == 0) {
    rxi = rx[i];
    ryi = ry[i];
    rxj = rx[j];
    ryj = ry[j];
  } else {
    // positions are held in the rotated frame; calcHI rotates them back
    // (extensional/src/main14.c:1720-1726)
    rxi = rx[i] * l.cth - ry[i] * l.sth;
    ryi = rx[i] * l.sth + ry[i] * l.cth;
    rxj = rx[j] * l.cth - ry[j] * l.sth;
    ryj = rx[j] * l.sth + ry[j] * l.cth;
  }
  double dxo = rxj - rxi, dyo = ryj - ryi, dzo = rz[j] - rz[i];
  double acc[6];
  ewald6(l, ew, dxo, dyo, dzo, kvec, lane, acc);
  for (int a = 0; a < 6; a++)
    for (int o = 16; o > 0; o >>= 1) acc[a] += __shfl_xor_sync(0xffffffffu, acc[a], o);
  if (lane == 0) {
    int I = i >> 5, J = j >> 5;
    double* tb = Mt + (tile_off(I, NT) + (J - I)) * 6144;
    int e = (i & 31) * 32 + (j & 31);
    for (int a = 0; a < 6; a++) tb[a * 1024 + e] = acc[a];
  }
}

// Ewald-summed RPY tensor for every pair (BD_MOB_EWALD): one CTA per packed
// tile, one lane per pair; the lane sums the real-space images and the k-space
// cosines serially (no cross-lane reduction), with the k-vector table staged
// in shared memory.  Positions held in the rotated frame are rotated back to
// the lab frame as calcHI does (extensional/src/main14.c:1720-1726).
template <bool kSmem>
__global__ void __launch_bounds__(256) k_hi_ewald_tiles(Lat l, Ewald ew,
                                                        const double* __restrict__ rx,
                                                        const double* __restrict__ ry,
                                                        const double* __restrict__ rz, int N,
                                                        int NT, const int* __restrict__ tileI,
                                                        const double* __restrict__ kvec_g,
                                                        double* Mt) {
  extern __shared__ double ksh[];
  long long tile = blockIdx.x;
  int I = tileI[tile];
  int J = I + (int)(tile - tile_off(I, NT));
  const double* kvec = kvec_g;
  if (kSmem) {
    for (int e = threadIdx.x; e < 9 * ew.nk; e += blockDim.x) ksh[e] = kvec_g[e];
    __syncthreads();
    kvec = ksh;
  }
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* tb = Mt + tile * 6144;
  int j = J * 32 + lane;
  double rxj = 0, ryj = 0, rzj = 0;
  if (j < N) {
    rxj = l.flow ? rx[j] * l.cth - ry[j] * l.sth : rx[j];
    ryj = l.flow ? rx[j] * l.sth + ry[j] * l.cth : ry[j];
    rzj = rz[j];
  }
  int side = 2 * ew.nmax + 1, nimg = side * side * side;
  for (int q = 0; q < 4; q++) {
    int il = w + 8 * q, i = I * 32 + il;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (i < j && j < N) {
      double rxi = l.flow ? rx[i] * l.cth - ry[i] * l.sth : rx[i];
      double ryi = l.flow ? rx[i] * l.sth + ry[i] * l.cth : ry[i];
      double dxo = rxj - rxi, dyo = ryj - ryi, dzo = rzj - rz[i];
      for (int m = 0; m < nimg; m++) {
        int nz = m % side - ew.nmax, ny = (m / side) % side - ew.nmax;
        int nx = m / (side * side) - ew.nmax;
        double dx = dxo + nx * l.L1x + ny * l.L2x;
        double dy = dyo + nx * l.L1y + ny * l.L2y;
        double dz = dzo + nz * l.L;
        double rr = dx * dx + dy * dy + dz * dz;
        if (sqrt(rr) < ew.rce) {
          double t1, t2;
          rpy_real(ew, rr, t1, t2);
          acc[0] += t1 + t2 * dx * dx / rr;
          acc[1] += t2 * dx * dy / rr;
          acc[2] += t2 * dx * dz / rr;
          acc[3] += t1 + t2 * dy * dy / rr;
          acc[4] += t2 * dy * dz / rr;
          acc[5] += t1 + t2 * dz * dz / rr;
        }
      }
      for (int c = 0; c < ew.nk; c++) {
        const double* kv = kvec + 9 * c;
        double ck = cos(kv[0] * dxo + kv[1] * dyo + kv[2] * dzo);
        acc[0] += kv[3] * ck;
        acc[1] += kv[4] * ck;
        acc[2] += kv[5] * ck;
        acc[3] += kv[6] * ck;
        acc[4] += kv[7] * ck;
        acc[5] += kv[8] * ck;
      }
    }
    for (int a = 0; a < 6; a++) tb[a * 1024 + il * 32 + lane] = acc[a];
  }
}

__global__ void k_to_fp32(const double* __restrict__ a, float* b, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t st = (size_t)gridDim.x * blockDim.x;
  for (; i < n; i += st) b[i] = (float)a[i];
}

// gridHI (shear/src/gridHI.c:145-240): one warp per bin of one lattice frame;
// the bin centre is the displacement, except the origin bin at (0.6,0.6,0.6).
__global__ void __launch_bounds__(256) k_grid_bins(Lat l, Ewald ew,
                                                   const double* __restrict__ kvec, int nbins,
                                                   int nby, int nbz, int nhx, int nhy, int nhz,
                                                   double bsx, double bsy, double bsz,
                                                   int origin, double* out) {
  int lane = threadIdx.x & 31;
  int nw = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nbins; b += nw) {
    double dx, dy, dz;
    if (b != origin) {
      int bb = b, bx = bb / (nby * nbz);
      bb -= bx * nby * nbz;
      int by = bb / nbz, bz = bb - by * nbz;
      dx = (bx - nhx) * bsx;
      dy = (by - nhy) * bsy;
      dz = (bz - nhz) * bsz;
    } else {
      dx = dy = dz = 0.6;
    }
    double acc[6];
    ewald6(l, ew, dx, dy, dz, kvec, lane, acc);
    for (int a = 0; a < 6; a++)
      for (int o = 16; o > 0; o >>= 1) acc[a] += __shfl_xor_sync(0xffffffffu, acc[a], o);
    if (lane == 0)
      for (int a = 0; a < 6; a++) out[(size_t)b * 6 + a] = acc[a];
  }
}

__device__ __forceinline__ double vin(const VecIn& v, int c, int i) {
  return v.p[c][(size_t)i * v.stride];
}

// Loads four consecutive tile entries (one row, four columns) as 16-byte
// vectors: one float4, or two double2.
__device__ __forceinline__ void load4(const float* p, double o[4]) {
  float4 v = *reinterpret_cast<const float4*>(p);
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
  o[3] = v.w;
}
__device__ __forceinline__ void load4(const double* p, double o[4]) {
  double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  o[0] = a.x;
  o[1] = a.y;
  o[2] = b.x;
  o[3] = b.y;
}

// Partial products of packed tiles with R right-hand sides (R = 1, 2).  T is
// the tile storage type (double, or float with FP64 accumulation).  A group of
// 64 threads owns one tile; thread (rg, cg) owns the 4x4 sub-block of 3x3
// blocks at rows 4rg.. and columns 4cg.., read with 16-byte loads.  Each
// block multiplies x_J into its row and, by block symmetry, x_I into its
// column; row sums are finished across the 8 threads of a row group by
// shuffles, column sums across the 8 row groups by shuffles and one shared
// exchange between the group's two warps.  Four tiles per 256-thread CTA.
// Per-tile partials go to scratch: 96 R doubles for rows, 96 R for columns.
template <typename T, int R>
__global__ void __launch_bounds__(256) k_sym_matvec(const T* __restrict__ Mt,
                                                    const int* __restrict__ tileI, int NT, int N,
                                                    long long ntiles, VecIn v0, VecIn v1,
                                                    double* rowpart, double* colpart) {
  const int g = threadIdx.x >> 6, t = threadIdx.x & 63;
  const int rg = t >> 3, cg = t & 7, lane = threadIdx.x & 31;
  long long tile = (long long)blockIdx.x * 4 + g;
  bool active = tile < ntiles;
  int I = 0, J = 0;
  if (active) {
    I = tileI[tile];
    J = I + (int)(tile - tile_off(I, NT));
  }
  __shared__ double xs[4][R][2][3][32];
  __shared__ double cx[4][R][3][4][8];  // column partials of the upper warp, per (rhs, comp, col, cg)
  for (int e = t; e < 2 * R * 96; e += 64) {
    int r = e / 192, rem = e % 192, side = rem / 96, c = (rem / 32) % 3, k = rem & 31;
    int idx = (side ? J : I) * 32 + k;
    xs[g][r][side][c][k] = (active && idx < N) ? vin(r ? v1 : v0, c, idx) : 0.0;
  }
  __syncthreads();
  double rs[R][4][3], cs[R][4][3];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int k = 0; k < 4; k++) rs[r][k][0] = rs[r][k][1] = rs[r][k][2] = cs[r][k][0] = cs[r][k][1] = cs[r][k][2] = 0.0;
  double xj[R][3][4];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int k = 0; k < 4; k++) xj[r][a][k] = xs[g][r][1][a][4 * cg + k];
  const T* tb = Mt + (active ? tile : 0) * 6144;
#pragma unroll
  for (int rr = 0; rr < 4; rr++) {
    int il = 4 * rg + rr;
    double m[6][4];
#pragma unroll
    for (int c = 0; c < 6; c++) load4(tb + c * 1024 + il * 32 + 4 * cg, m[c]);
    double xi[R][3];
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int a = 0; a < 3; a++) xi[r][a] = xs[g][r][0][a][il];
#pragma unroll
    for (int cc = 0; cc < 4; cc++) {
      int jl = 4 * cg + cc;
      bool valid = active && ((I != J) || (il < jl));
      double m0 = valid ? m[0][cc] : 0.0, m1 = valid ? m[1][cc] : 0.0, m2 = valid ? m[2][cc] : 0.0;
      double m3 = valid ? m[3][cc] : 0.0, m4 = valid ? m[4][cc] : 0.0, m5 = valid ? m[5][cc] : 0.0;
#pragma unroll
      for (int r = 0; r < R; r++) {
        double x0 = xj[r][0][cc], x1 = xj[r][1][cc], x2 = xj[r][2][cc];
        rs[r][rr][0] += m0 * x0 + m1 * x1 + m2 * x2;
        rs[r][rr][1] += m1 * x0 + m3 * x1 + m4 * x2;
        rs[r][rr][2] += m2 * x0 + m4 * x1 + m5 * x2;
        double y0 = xi[r][0], y1 = xi[r][1], y2 = xi[r][2];
        cs[r][cc][0] += m0 * y0 + m1 * y1 + m2 * y2;
        cs[r][cc][1] += m1 * y0 + m3 * y1 + m4 * y2;
        cs[r][cc][2] += m2 * y0 + m4 * y1 + m5 * y2;
      }
    }
  }
  // rows: sum over the 8 column groups (lane bits 0..2)
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int a = 0; a < 3; a++) {
        double v = rs[r][k][a];
        v += __shfl_xor_sync(0xffffffffu, v, 1);
        v += __shfl_xor_sync(0xffffffffu, v, 2);
        v += __shfl_xor_sync(0xffffffffu, v, 4);
        rs[r][k][a] = v;
      }
  // columns: sum over the 4 row groups of this warp (lane bits 3..4)
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int a = 0; a < 3; a++) {
        double v = cs[r][k][a];
        v += __shfl_xor_sync(0xffffffffu, v, 8);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        cs[r][k][a] = v;
      }
  bool upper = t >= 32;  // second warp of the group: row groups 4..7
  if (upper && lane < 8)
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int k = 0; k < 4; k++) cx[g][r][a][k][cg] = cs[r][k][a];
  __syncthreads();
  if (!active) return;
  double* rp = rowpart + tile * (96 * R);
  double* cp = colpart + tile * (96 * R);
  if (cg == 0)
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int k = 0; k < 4; k++) rp[r * 96 + a * 32 + 4 * rg + k] = rs[r][k][a];
  if (!upper && lane < 8)
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int a = 0; a < 3; a++)
#pragma unroll
        for (int k = 0; k < 4; k++)
          cp[r * 96 + a * 32 + 4 * cg + k] = cs[r][k][a] + cx[g][r][a][k][cg];
}

// First reduction level: block (K, s) sums its share of the row partials of
// tiles (K, J >= K) and the column partials of tiles (I <= K, K);
// blockDim = 96 R.
__global__ void k_matvec_reduce1(const double* __restrict__ rowpart,
                                 const double* __restrict__ colpart, int NT, double* part) {
  int K = blockIdx.x, s = blockIdx.y, e = threadIdx.x, E = blockDim.x;
  double acc = 0;
  for (int J = K + s; J < NT; J += kRedSplit) acc += rowpart[(tile_off(K, NT) + (J - K)) * E + e];
  for (int I = s; I <= K; I += kRedSplit) acc += colpart[(tile_off(I, NT) + (K - I)) * E + e];
  part[((size_t)K * kRedSplit + s) * E + e] = acc;
}

// Second level: Y_r[a*NT*32 + K*32 + k] = sum over splits, plus the diagonal
// block diag(D0,D1,D2) applied to the input when addiag is set.
__global__ void k_matvec_reduce2(const double* __restrict__ part, int NT, int N, double* Y0,
                                 double* Y1, VecIn v0, VecIn v1, int addiag, double D0,
                                 double D1, double D2) {
  int K = blockIdx.x, e = threadIdx.x, E = blockDim.x;
  double acc = 0;
  for (int s = 0; s < kRedSplit; s++) acc += part[((size_t)K * kRedSplit + s) * E + e];
  int r = e / 96, a = (e / 32) % 3, k = e & 31;
  int i = K * 32 + k;
  if (addiag && i < N) acc += (a == 0 ? D0 : a == 1 ? D1 : D2) * vin(r ? v1 : v0, a, i);
  double* Y = r ? Y1 : Y0;
  Y[(size_t)a * NT * 32 + i] = acc;
}

// TEA displacement and position update (updateHI, shear/src/main26.c:787-855;
// extensional/src/main14.c:825-893).  U = sum_{j != i} M_ij F_j and
// W = sum_{j != i} M_ij R_j; the diagonal block contributes
// Dtr_a (F_a + p C_a R_a), beta applying only off the diagonal.
__global__ void k_tea_update(int flow, double* rx, double* ry, double* rz, double* dxv,
                             double* dyv, double* dzv, const double* __restrict__ fx,
                             const double* __restrict__ fy, const double* __restrict__ fz,
                             const double* __restrict__ R, const double* __restrict__ U,
                             const double* __restrict__ W, int NTp, const double* __restrict__ Ct,
                             int Nb, int N, double dt, double edot, double p, double bt,
                             double D0, double D1, double D2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int b = i % Nb;
  double F[3] = {fx[i], fy[i], fz[i]};
  double Dg[3] = {D0, D1, D2};
  double du[3];
  for (int a = 0; a < 3; a++) {
    double C = Ct[3 * b + a];
    double Ra = R[3 * i + a];
    du[a] = dt * (U[(size_t)a * NTp + i] + p * bt * C * W[(size_t)a * NTp + i]) +
            dt * (Dg[a] * (F[a] + p * C * Ra));
  }
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

namespace bd {

int alloc_mobility(bd_ctx* c) {
  int N = c->N;
  c->NT = (N + 31) / 32;
  c->ntiles = (size_t)c->NT * (c->NT + 1) / 2;
  size_t gsz = (size_t)c->p.nt_avg * c->nbins * 6;
  CU(cudaMalloc(&c->grid, 8 * gsz));
  CU(cudaMemsetAsync(c->grid, 0, 8 * gsz, c->stream));
  CU(cudaMalloc(&c->Ctab, 8 * (size_t)(c->sbins + 1) * 3 * c->Nb));
  CU(cudaMemsetAsync(c->Ctab, 0, 8 * (size_t)(c->sbins + 1) * 3 * c->Nb, c->stream));
  c->bytes += 8 * gsz + 8 * (size_t)(c->sbins + 1) * 3 * c->Nb;
  return BD_OK;
}

// Tile storage, tile-row table, near-pair list and matvec scratch are
// allocated on the first mobility build (they are O(N^2)).
static int ensure_tiles(bd_ctx* c) {
  if (c->Mt) return BD_OK;
  size_t nt = c->ntiles;
  if (cudaMalloc(&c->Mt, 8 * nt * 6144) != cudaSuccess) return BD_ERR_OOM;
  CU(cudaMemsetAsync(c->Mt, 0, 8 * nt * 6144, c->stream));
  std::vector<int> ti(nt);
  size_t k = 0;
  for (int I = 0; I < c->NT; I++)
    for (int J = I; J < c->NT; J++) ti[k++] = I;
  CU(cudaMalloc(&c->tileI, 4 * nt));
  CU(cudaMemcpy(c->tileI, ti.data(), 4 * nt, cudaMemcpyHostToDevice));
  long long N = c->N;
  c->near_cap = c->p.mobility == BD_MOB_EWALD ? 1 : std::min<long long>(N * (N - 1) / 2 + 1, 512 * N);
  CU(cudaMalloc(&c->near_pairs, 8 * c->near_cap));
  CU(cudaMalloc(&c->near_count, 16));
  CU(cudaMalloc(&c->rowpart, 8 * nt * 192));
  CU(cudaMalloc(&c->colpart, 8 * nt * 192 + 8 * (size_t)c->NT * kRedSplit * 192));
  CU(cudaMalloc(&c->U, 8 * 3 * (size_t)c->NT * 32));
  CU(cudaMalloc(&c->W, 8 * 3 * (size_t)c->NT * 32));
  c->bytes += 8 * nt * 6144 + 4 * nt + 8 * c->near_cap + 16 + 16 * nt * 192 +
              8 * (size_t)c->NT * kRedSplit * 192 + 48 * (size_t)c->NT * 32;
  return BD_OK;
}

// Ewald parameters, k-vector list with coefficients M2, and the self term Dtr
// of calcHI (shear/src/main26.c:1536-1686; ext k-vectors of the rotated
// reciprocal lattice, extensional/src/main14.c:1582-1588), generated with
// the reference's loop structure and arithmetic.
static void hi_setup(bd_ctx* c, const Lat& l, Ewald* ew, std::vector<double>* kv, double Dtr[3],
                     double M_HI = 4.0, int tp = 0, bool exact_self = false) {
  double L = l.L, boxvol = c->boxvol;
  if (tp == 0) tp = c->tp;
  int treal = l.treal, nmax;
  double rce;
  if (treal <= tp / 2) {
    rce = 1.0 * l.L2yp;
    nmax = 1;
  } else {
    rce = 2.0 * l.L2yp;
    nmax = 2;
  }
  double tf = (double)treal / tp;
  int nt = (int)round(tf * c->p.nt_avg) % c->p.nt_avg;
  double alpha = M_HI / rce, rkcut = 2.0 * M_HI * M_HI / rce;
  double rkkcut = rkcut * rkcut, rtpi = sqrt(M_PI);
  double alpha2 = alpha * alpha, alpha3 = alpha2 * alpha, alpha4 = alpha2 * alpha2;
  double alpha5 = alpha4 * alpha, alpha7 = alpha4 * alpha2 * alpha;
  double selfconst = 1 - 6 / rtpi * alpha + 40 / (3 * rtpi) * alpha3;
  double L1[2] = {l.L1x, l.L1y}, L2[2] = {l.L2x, l.L2y};
  int kxmax = ceil(rkcut * l.detL / (M_PI * 2.0 * L * L2[1]));
  int kymax = ceil(rkcut * l.detL / (M_PI * 2.0 * L * L1[0]));
  int kzmax = ceil(rkcut * L / (M_PI * 2.0));
  int nyw = 2 * kymax + 1;
  std::vector<int> kyup(kxmax + 2, 0), kylo(kxmax + 2, 0);
  std::vector<int> kzup((size_t)(kxmax + 2) * nyw, 0), kzlo((size_t)(kxmax + 2) * nyw, 0);
  double kcoeff = (l.flow == 0) ? M_PI * 2.0 : M_PI * 2.0 / l.detL;
  auto kvec2 = [&](int kx, int ky, double& rkx, double& rky) {
    if (l.flow == 0) {
      rky = kcoeff * (kx - ky * (L2[0] / L1[0])) / L2[1];
      rkx = kcoeff * ky / L1[0];
    } else {
      rkx = kcoeff * L * (kx * L2[1] - ky * L1[1]);
      rky = kcoeff * L * (-kx * L2[0] + ky * L1[0]);
    }
  };
  for (int kx = 0; kx < kxmax + 1; kx++) {
    int ylo = 0, yup = 0;
    for (int ky = -kymax; ky < kymax + 1; ky++) {
      double rkx, rky;
      kvec2(kx, ky, rkx, rky);
      double rkxy = rkx * rkx + rky * rky;
      int zlo = 0, zup = 0;
      for (int kz = -kzmax; kz < kzmax + 1; kz++) {
        double rkz = kz * M_PI * 2.0 / L, rkk = rkxy + rkz * rkz;
        if (rkk < rkkcut && zlo == 0) {
          kzlo[nyw * kx + ky + kymax] = kz;
          zlo = 1;
        }
        if (rkk > rkkcut && zlo == 1 && zup == 0) {
          kzup[nyw * kx + ky + kymax] = kz - 1;
          zup = 1;
        }
      }
      if (rkxy < rkkcut && ylo == 0) {
        kylo[kx] = ky;
        ylo = 1;
      }
      if (rkxy > rkkcut && ylo == 1 && yup == 0) {
        kyup[kx] = ky - 1;
        yup = 1;
      }
    }
  }
  {
    // same scan as the reference; the arrays carry one spare zero row so the
    // scan and the kxmax increment below stay inside them
    int kx = 0, rows = kxmax + 2;
    while (kx < rows && kyup[kx] != -kymax &&
           kx <= (int)(rkcut * l.detL / (M_PI * 2.0 * L * l.L2yp))) {
      kxmax = kx;
      kx++;
    }
  }
  kxmax++;
  kv->clear();
  for (int kx = 0; kx < kxmax + 1 && kx < (int)kylo.size(); kx++)
    for (int ky = kylo[kx]; ky < kyup[kx] + 1; ky++) {
      double rkx, rky;
      kvec2(kx, ky, rkx, rky);
      double rkxy = rkx * rkx + rky * rky;
      for (int kz = kzlo[nyw * kx + ky + kymax]; kz < kzup[nyw * kx + ky + kymax] + 1; kz++) {
        double rkz = kz * M_PI * 2.0 / L, rkk = rkxy + rkz * rkz;
        double m2 = 2.0 * (1.0 - rkk / 3.0) * (1.0 + rkk / (4.0 * alpha2) + rkk * rkk / (8.0 * alpha4)) * 6.0 * M_PI / rkk * exp(-rkk / (4.0 * alpha2));
        double row[9] = {rkx,
                         rky,
                         rkz,
                         m2 * (1 - rkx * rkx / rkk) / boxvol,
                         m2 * (-rkx * rky / rkk) / boxvol,
                         m2 * (-rkx * rkz / rkk) / boxvol,
                         m2 * (1 - rky * rky / rkk) / boxvol,
                         m2 * (-rky * rkz / rkk) / boxvol,
                         m2 * (1 - rkz * rkz / rkk) / boxvol};
        kv->insert(kv->end(), row, row + 9);
      }
    }
  {
    int cnt = 0;
    for (int ky = kylo[0]; ky < kyup[0] + 1; ky++)
      for (int kz = kzlo[ky + kymax]; kz < kzup[ky + kymax] + 1; kz++) {
        for (int a = 3; a < 9; a++) (*kv)[9 * cnt + a] /= 2.0;
        if (ky == 0 && kz == 0)
          for (int a = 3; a < 9; a++) (*kv)[9 * cnt + a] = 0.0;
        cnt++;
      }
  }
  int nk = (int)(kv->size() / 9);
  Dtr[0] = Dtr[1] = Dtr[2] = selfconst;
  for (int k = 0; k < nk; k++) {
    Dtr[0] += (*kv)[9 * k + 3];
    Dtr[1] += (*kv)[9 * k + 6];
    Dtr[2] += (*kv)[9 * k + 8];
  }
  // self images: the reference requires all three indices non-zero and adds
  // the yy projection to the zz entry (shear/src/main26.c:1667-1686); with
  // exact_self every image but the origin counts and zz uses dz
  for (int nx = -nmax; nx < nmax + 1; nx++)
    for (int ny = -nmax; ny < nmax + 1; ny++)
      for (int nz = -nmax; nz < nmax + 1; nz++)
        if (exact_self ? (nx != 0 || ny != 0 || nz != 0) : (nx != 0 && ny != 0 && nz != 0)) {
          double dx = nx * L1[0] + ny * L2[0], dy = nx * L1[1] + ny * L2[1], dz = nz * L;
          double rr = dx * dx + dy * dy + dz * dz, r = sqrt(rr);
          double C1 = 0.75 / r + 0.5 / (r * rr);
          double C2 = 4.0 * alpha7 * rr * rr + 3.0 * alpha3 * rr - 20.0 * alpha5 * rr - 4.5 * alpha + 14.0 * alpha3 + alpha / rr;
          double C3 = 0.75 / r - 1.5 / (r * rr);
          double C4 = -4.0 * alpha7 * rr * rr - 3.0 * alpha3 * rr + 16.0 * alpha5 * rr + 1.5 * alpha - 2.0 * alpha3 - 3.0 * alpha / rr;
          double t1 = C1 * erfc(alpha * r) + C2 * exp(-alpha2 * rr) / rtpi;
          double t2 = C3 * erfc(alpha * r) + C4 * exp(-alpha2 * rr) / rtpi;
          Dtr[0] += t1 + t2 * dx * dx / rr;
          Dtr[1] += t1 + t2 * dy * dy / rr;
          Dtr[2] += t1 + t2 * (exact_self ? dz * dz : dy * dy) / rr;
        }
  ew->alpha = alpha;
  ew->alpha2 = alpha2;
  ew->alpha3 = alpha3;
  ew->alpha5 = alpha5;
  ew->alpha7 = alpha7;
  ew->rce = rce;
  ew->rtpi = rtpi;
  ew->nmax = nmax;
  ew->nt = nt;
  ew->nk = nk;
}

static Lat step_lat(bd_ctx* c) {
  Lat l = c->lat;
  int treal = (int)(c->t % (unsigned long)c->tp);
  l.treal = treal;
  l.nmax = (treal <= c->tp / 2) ? 1 : 2;
  l.delx = c->p.edot * treal * c->p.dt;
  return l;
}

int calc_hi(bd_ctx* c) {
  int s;
  lanczos_graphs_reset(c);  // captured products hold the diagonal by value
  c->hi_version++;          // noise blocks solved with the old mobility are void
  if (c->p.mobility == BD_MOB_PME) {
    prof_begin(c, BD_PROF_HI_BUILD);
    s = pme_prepare(c, step_lat(c));
    if (s == BD_OK) s = precond_build(c, step_lat(c));
    prof_end(c, BD_PROF_HI_BUILD);
    return s;
  }
  if ((s = ensure_tiles(c)) != BD_OK) return s;
  Lat l = step_lat(c);
  Ewald ew;
  std::vector<double> kv;
  bool ewald_all = c->p.mobility == BD_MOB_EWALD;
  hi_setup(c, l, &ew, &kv, c->Dtr, 4.0, 0, ewald_all);
  if ((int)kv.size() / 9 > c->kvec_cap) {
    CU(cudaStreamSynchronize(c->stream));
    if (c->kvec) cudaFree(c->kvec);
    c->kvec_cap = (int)kv.size() / 9 + 64;
    CU(cudaMalloc(&c->kvec, 8 * 9 * (size_t)c->kvec_cap));
  }
  c->nk = ew.nk;
  if (!kv.empty())
    CU(cudaMemcpyAsync(c->kvec, kv.data(), 8 * kv.size(), cudaMemcpyHostToDevice, c->stream));
  prof_begin(c, BD_PROF_HI_BUILD);
  if (ewald_all) {
    size_t smem = 8 * 9 * (size_t)ew.nk;
    c->launches++;
    if (smem <= 96 * 1024) {
      cudaFuncSetAttribute(k_hi_ewald_tiles<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           96 * 1024);
      k_hi_ewald_tiles<true><<<(unsigned)c->ntiles, 256, smem, c->stream>>>(
          l, ew, c->rx, c->ry, c->rz, c->N, c->NT, c->tileI, c->kvec, c->Mt);
    } else {
      k_hi_ewald_tiles<false><<<(unsigned)c->ntiles, 256, 0, c->stream>>>(
          l, ew, c->rx, c->ry, c->rz, c->N, c->NT, c->tileI, c->kvec, c->Mt);
    }
  } else {
    CU(cudaMemsetAsync(c->near_count, 0, 4, c->stream));
    c->launches++;
    k_hi_far<<<(unsigned)c->ntiles, 256, 0, c->stream>>>(
        l, ew, c->rx, c->ry, c->rz, c->N, c->NT, c->tileI, c->grid, c->nbx, c->nby, c->nbz,
        c->nhx, c->nhy, c->nhz, c->bsx, c->bsy, c->bsz, c->nbins, c->Mt, (int2*)c->near_pairs,
        c->near_count, (long long)c->near_cap, c->err);
    c->launches++;
    k_hi_near<<<148 * 8, 256, 0, c->stream>>>(l, ew, c->rx, c->ry, c->rz, c->NT,
                                              (const int2*)c->near_pairs, c->near_count,
                                              (long long)c->near_cap, c->kvec, c->Mt);
  }
  if (c->p.precision == BD_PREC_FP32) {
    if (!c->Mt32) {
      CU(cudaStreamSynchronize(c->stream));
      if (cudaMalloc(&c->Mt32, 4 * c->ntiles * 6144) != cudaSuccess) return BD_ERR_OOM;
      c->bytes += 4 * c->ntiles * 6144;
    }
    c->launches++;
    k_to_fp32<<<148 * 16, 256, 0, c->stream>>>(c->Mt, c->Mt32, c->ntiles * 6144);
  }
  if ((s = precond_build(c, l)) != BD_OK) return s;
  prof_end(c, BD_PROF_HI_BUILD);
  c->hi_built = true;
  return launch_ok(c);
}

// Y_r = M v_r for R = 1 or 2 right-hand sides over the packed tiles (FP64 or
// FP32 storage); with addiag the uniform diagonal blocks are included,
// otherwise only the off-diagonal blocks.
int sym_matvec(bd_ctx* c, int R, const VecIn& v0, const VecIn& v1, double* Y0, double* Y1,
               bool addiag) {
  if (c->p.mobility == BD_MOB_PME) {
    // the particle-mesh product always includes the diagonal blocks
    if (!addiag) return BD_ERR_STATE;
    int s, NTp = c->NT * 32;
    if ((s = pme_apply(c, v0, Y0, Y0 + NTp, Y0 + 2 * NTp, 1)) != BD_OK) return s;
    if (R == 2 && (s = pme_apply(c, v1, Y1, Y1 + NTp, Y1 + 2 * NTp, 1)) != BD_OK) return s;
    return BD_OK;
  }
  long long ntl = (long long)c->ntiles;
  unsigned nb = (unsigned)((ntl + 3) / 4);
  prof_begin(c, BD_PROF_MATVEC);
  c->launches++;
  if (c->Mt32) {
    if (R == 2)
      k_sym_matvec<float, 2><<<nb, 256, 0, c->stream>>>(c->Mt32, c->tileI, c->NT, c->N, ntl, v0,
                                                        v1, c->rowpart, c->colpart);
    else
      k_sym_matvec<float, 1><<<nb, 256, 0, c->stream>>>(c->Mt32, c->tileI, c->NT, c->N, ntl, v0,
                                                        v1, c->rowpart, c->colpart);
  } else {
    if (R == 2)
      k_sym_matvec<double, 2><<<nb, 256, 0, c->stream>>>(c->Mt, c->tileI, c->NT, c->N, ntl, v0,
                                                         v1, c->rowpart, c->colpart);
    else
      k_sym_matvec<double, 1><<<nb, 256, 0, c->stream>>>(c->Mt, c->tileI, c->NT, c->N, ntl, v0,
                                                         v1, c->rowpart, c->colpart);
  }
  prof_end(c, BD_PROF_MATVEC);
  double* part = c->colpart + c->ntiles * 192;
  c->launches++;
  k_matvec_reduce1<<<dim3(c->NT, kRedSplit), 96 * R, 0, c->stream>>>(c->rowpart, c->colpart,
                                                                    c->NT, part);
  c->launches++;
  k_matvec_reduce2<<<c->NT, 96 * R, 0, c->stream>>>(part, c->NT, c->N, Y0, Y1, v0, v1,
                                                    addiag ? 1 : 0, c->Dtr[0], c->Dtr[1],
                                                    c->Dtr[2]);
  return launch_ok(c);
}

int update_hi(bd_ctx* c) {
  int s;
  if (c->t % (unsigned long)c->srpy == 0 || c->t == c->tstart) {
    if ((s = calc_hi(c)) != BD_OK) return s;
    int sb = (int)floor(c->strain / c->strain_interval);
    if (sb > c->sbins) sb = c->sbins;
    if (sb < 0) sb = 0;
    c->sbin = sb;
    c->bt = c->btab[sb];
  }
  if (!c->hi_built || c->p.mobility == BD_MOB_PME) return BD_ERR_STATE;
  if (c->p.flow == BD_FLOW_EXT) rotate_coords(c, 1);
  VecIn vf = {{c->fx, c->fy, c->fz}, 1};
  VecIn vr = {{c->R, c->R + 1, c->R + 2}, 3};
  if ((s = sym_matvec(c, 2, vf, vr, c->U, c->W, false)) != BD_OK) return s;
  double p = sqrt(2.0 / c->p.dt);
  c->launches++;
  k_tea_update<<<(c->N + 255) / 256, 256, 0, c->stream>>>(
      c->p.flow, c->rx, c->ry, c->rz, c->dxv, c->dyv, c->dzv, c->fx, c->fy, c->fz, c->R, c->U,
      c->W, c->NT * 32, c->Ctab + (size_t)c->sbin * 3 * c->Nb, c->Nb, c->N, c->p.dt, c->p.edot,
      p, c->bt, c->Dtr[0], c->Dtr[1], c->Dtr[2]);
  return launch_ok(c);
}

int download_mobility(bd_ctx* c, double* M9) {
  if (!c->hi_built || !c->Mt) return BD_ERR_STATE;  // the PME mobility has no stored matrix
  int N = c->N, NT = c->NT;
  std::vector<double> h(c->ntiles * 6144);
  CU(cudaMemcpyAsync(h.data(), c->Mt, 8 * h.size(), cudaMemcpyDeviceToHost, c->stream));
  int s = check(c);
  if (s) return s;
  memset(M9, 0, sizeof(double) * 9 * (size_t)N * N);
  static const int comp[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
  size_t t = 0;
  for (int I = 0; I < NT; I++)
    for (int J = I; J < NT; J++, t++) {
      const double* tb = h.data() + t * 6144;
      for (int il = 0; il < 32; il++)
        for (int jl = 0; jl < 32; jl++) {
          int i = I * 32 + il, j = J * 32 + jl;
          if (i >= j || j >= N) continue;
          double* blk = M9 + (size_t)9 * N * i + 9 * (size_t)j;
          for (int a = 0; a < 9; a++) blk[a] = tb[comp[a] * 1024 + il * 32 + jl];
        }
    }
  for (int i = 0; i < N; i++) {
    double* blk = M9 + (size_t)9 * N * i + 9 * (size_t)i;
    blk[0] = c->Dtr[0];
    blk[4] = c->Dtr[1];
    blk[8] = c->Dtr[2];
  }
  return BD_OK;
}

}  // namespace bd

// gridHI's main (shear/src/gridHI.c:3-278) on the device: the period and bin
// geometry follow gridHI's own time step, frame nt is taken at
// t = nt*tp/nt_avg, and the Ewald split uses M_HI = 6.
extern "C" int bd_build_grid(bd_ctx* c, double grid_dt) {
  if (!c) return BD_ERR_ARG;
  if (grid_dt <= 0) grid_dt = 0.001;
  double L = c->p.L, edot = c->p.edot;
  int tp = (int)(0.9624 / edot / grid_dt);
  if (tp < 1) return BD_ERR_ARG;
  double th = (90.0 - (45.0 + (c->p.flow == 0 ? 0.0 : 31.7))) * (M_PI / 180);
  double xmax, ymax, zmax = L / 2;
  if (c->p.flow == 0) {
    ymax = L / 2;
    xmax = L / 2 * edot * tp * grid_dt;
  } else {
    ymax = -(-sqrt(2) / 2 * L * cos(th));
    xmax = (sqrt(2) / 2 * L * cos(th)) * exp(edot * tp * grid_dt);
  }
  double bs = c->p.bin_size, bsx = bs, bsy = bs, bsz = bs;
  int nbx = 2 * ceil(xmax / bsx) + 1;
  bsx = xmax / ((nbx - 1) / 2);
  int nhx = (nbx - 1) / 2;
  int nby = 2 * ceil(ymax / bsy) + 1;
  bsy = ymax / ((nby - 1) / 2);
  int nhy = (nby - 1) / 2;
  int nbz = 2 * ceil(zmax / bsz) + 1;
  bsz = zmax / ((nbz - 1) / 2);
  int nhz = (nbz - 1) / 2;
  int nbins = nbx * nby * nbz;
  if (nbins != c->nbins || nbx != c->nbx || nby != c->nby) return BD_ERR_STATE;
  int origin = nhx * nby * nbz + nhy * nbz + nhz;
  for (int nt = 0; nt < c->p.nt_avg; nt++) {
    unsigned long t = (unsigned long)(nt * tp / c->p.nt_avg);
    Lat l;
    host_lattice_at(c, t, grid_dt, tp, &l);
    Ewald ew;
    std::vector<double> kv;
    double unused[3];
    hi_setup(c, l, &ew, &kv, unused, 6.0, tp);
    if ((int)kv.size() / 9 > c->kvec_cap) {
      CU(cudaStreamSynchronize(c->stream));
      if (c->kvec) cudaFree(c->kvec);
      c->kvec_cap = (int)kv.size() / 9 + 64;
      CU(cudaMalloc(&c->kvec, 8 * 9 * (size_t)c->kvec_cap));
    }
    if (!kv.empty())
      CU(cudaMemcpyAsync(c->kvec, kv.data(), 8 * kv.size(), cudaMemcpyHostToDevice, c->stream));
    c->launches++;
    k_grid_bins<<<148 * 4, 256, 0, c->stream>>>(l, ew, c->kvec, nbins, nby, nbz, nhx, nhy, nhz, bsx,
                                                bsy, bsz, origin,
                                                c->grid + (size_t)nt * nbins * 6);
    // the host vector kv is reused next frame: wait for the copy to finish
    CU(cudaStreamSynchronize(c->stream));
  }
  return check(c);
}

extern "C" int bd_download_grid(bd_ctx* c, int nt, double* D9) {
  if (!c || !D9 || nt < 0 || nt >= c->p.nt_avg) return BD_ERR_ARG;
  std::vector<double> g((size_t)c->nbins * 6);
  CU(cudaMemcpyAsync(g.data(), c->grid + (size_t)nt * c->nbins * 6, 8 * g.size(),
                     cudaMemcpyDeviceToHost, c->stream));
  int s = check(c);
  if (s) return s;
  static const int comp[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
  for (int b = 0; b < c->nbins; b++)
    for (int a = 0; a < 9; a++) D9[(size_t)b * 9 + a] = g[(size_t)b * 6 + comp[a]];
  return BD_OK;
}

extern "C" int bd_load_grid(bd_ctx* c, int nt, const double* D9) {
  if (!c || !D9 || nt < 0 || nt >= c->p.nt_avg) return BD_ERR_ARG;
  std::vector<double> g((size_t)c->nbins * 6);
  for (int b = 0; b < c->nbins; b++) {
    const double* d = D9 + 9 * (size_t)b;
    if (d[1] != d[3] || d[2] != d[6] || d[5] != d[7]) return BD_ERR_ASYMMETRIC;
    double* o = g.data() + 6 * (size_t)b;
    o[0] = d[0];
    o[1] = d[1];
    o[2] = d[2];
    o[3] = d[4];
    o[4] = d[5];
    o[5] = d[8];
  }
  CU(cudaMemcpyAsync(c->grid + (size_t)nt * c->nbins * 6, g.data(), 8 * g.size(),
                     cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return BD_OK;
}

// ---------------------------------------------------------------------------
// CA-TEA sampling: ewaldBin + CATEA (shear/src/main26.c:975-1381,
// extensional/src/main14.c:1009-1415).
//
// ewaldBin evaluates the Ewald-summed RPY tensor of every bead pair i < j
// with its own split (M_HI = 3.5; the images, k-vector box and self sums of
// calcHI, including the self-image quirks) on the positions as they are
// (no rotation) and accumulates eps = sum_pairs 2 sum_a D_a / Dtr_(a/3) over
// the nine entries and rowsum[3i + a/3], rowsum[3j + a/3] += (D_a/Dtr)^2.
// Here one CTA per packed tile computes the tensors as k_hi_ewald_tiles does
// and writes per-tile partial sums (eps, row and column contributions), which
// a second kernel adds per bead in a fixed order.

template <bool kSmem>
__global__ void __launch_bounds__(256) k_ewald_bin_tiles(Lat l, Ewald ew,
                                                         const double* __restrict__ rx,
                                                         const double* __restrict__ ry,
                                                         const double* __restrict__ rz, int N,
                                                         int NT, const int* __restrict__ tileI,
                                                         const double* __restrict__ kvec_g,
                                                         double D0, double D1, double D2,
                                                         double* part) {
  extern __shared__ double ksh[];
  __shared__ double colacc[8][96];
  __shared__ double eacc[8];
  long long tile = blockIdx.x;
  int I = tileI[tile];
  int J = I + (int)(tile - tile_off(I, NT));
  const double* kvec = kvec_g;
  if (kSmem) {
    for (int e = threadIdx.x; e < 9 * ew.nk; e += blockDim.x) ksh[e] = kvec_g[e];
    __syncthreads();
    kvec = ksh;
  }
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int j = J * 32 + lane;
  double rxj = 0, ryj = 0, rzj = 0;
  if (j < N) {
    rxj = rx[j];
    ryj = ry[j];
    rzj = rz[j];
  }
  const double Dd[3] = {D0, D1, D2};
  const int sym[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
  int side = 2 * ew.nmax + 1, nimg = side * side * side;
  double* P = part + (size_t)tile * 193;
  double col[3] = {0, 0, 0}, epsl = 0;
  for (int q = 0; q < 4; q++) {
    int il = w + 8 * q, i = I * 32 + il;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    bool pair = i < j && j < N;
    if (pair) {
      double dxo = rxj - rx[i], dyo = ryj - ry[i], dzo = rzj - rz[i];
      for (int m = 0; m < nimg; m++) {
        int nz = m % side - ew.nmax, ny = (m / side) % side - ew.nmax;
        int nx = m / (side * side) - ew.nmax;
        double dx = dxo + nx * l.L1x + ny * l.L2x;
        double dy = dyo + nx * l.L1y + ny * l.L2y;
        double dz = dzo + nz * l.L;
        double rr = dx * dx + dy * dy + dz * dz;
        if (sqrt(rr) < ew.rce) {
          double t1, t2;
          rpy_real(ew, rr, t1, t2);
          acc[0] += t1 + t2 * dx * dx / rr;
          acc[1] += t2 * dx * dy / rr;
          acc[2] += t2 * dx * dz / rr;
          acc[3] += t1 + t2 * dy * dy / rr;
          acc[4] += t2 * dy * dz / rr;
          acc[5] += t1 + t2 * dz * dz / rr;
        }
      }
      for (int c = 0; c < ew.nk; c++) {
        const double* kv = kvec + 9 * c;
        double ck = cos(kv[0] * dxo + kv[1] * dyo + kv[2] * dzo);
        acc[0] += kv[3] * ck;
        acc[1] += kv[4] * ck;
        acc[2] += kv[5] * ck;
        acc[3] += kv[6] * ck;
        acc[4] += kv[7] * ck;
        acc[5] += kv[8] * ck;
      }
    }
    double row[3] = {0, 0, 0};
    if (pair) {
      for (int a = 0; a < 9; a++) {
        double incr = acc[sym[a]] / Dd[a / 3];
        epsl += 2.0 * incr;
        row[a / 3] += incr * incr;
        col[a / 3] += incr * incr;
      }
    }
    for (int a = 0; a < 3; a++) {
      double v = row[a];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) P[1 + a * 32 + il] = v;
    }
  }
  for (int a = 0; a < 3; a++) colacc[w][a * 32 + lane] = col[a];
  for (int o = 16; o > 0; o >>= 1) epsl += __shfl_xor_sync(0xffffffffu, epsl, o);
  if (lane == 0) eacc[w] = epsl;
  __syncthreads();
  if (threadIdx.x < 96) {
    double s = 0;
    for (int ww = 0; ww < 8; ww++) s += colacc[ww][threadIdx.x];
    P[97 + threadIdx.x] = s;
  }
  if (threadIdx.x == 0) {
    double s = 0;
    for (int ww = 0; ww < 8; ww++) s += eacc[ww];
    P[0] = s;
  }
}

// rowsum[3i + a] = sum of the row parts of tiles (K, J >= K) and the column
// parts of tiles (I <= K, K); one CTA per bead block K, fixed order.
__global__ void k_ewald_bin_reduce(const double* __restrict__ part, int NT, int N,
                                   double* rowsum) {
  int K = blockIdx.x, e = threadIdx.x;  // e = a * 32 + bead
  if (e >= 96) return;
  double s = 0;
  for (int J = K; J < NT; J++) s += part[(size_t)(tile_off(K, NT) + (J - K)) * 193 + 1 + e];
  for (int I = 0; I <= K; I++) s += part[(size_t)(tile_off(I, NT) + (K - I)) * 193 + 97 + e];
  int a = e / 32, i = K * 32 + (e & 31);
  if (i < N) rowsum[3 * i + a] = s;
}

__global__ void k_ewald_bin_eps(const double* __restrict__ part, long long ntiles, double* eps) {
  double s = 0;
  for (long long t = threadIdx.x; t < ntiles; t += 32) s += part[(size_t)t * 193];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) *eps = s;
}

namespace bd {

// eps and rowsum (3N) of ewaldBin for the current positions and lattice.
int ewald_bin(bd_ctx* c, double* eps, std::vector<double>& rowsum) {
  int N = c->N, NT = (N + 31) / 32;
  long long ntl = (long long)NT * (NT + 1) / 2;
  if (!c->cb_part) {
    CU(cudaMalloc(&c->cb_part, 8 * (size_t)ntl * 193 + 8 * (3 * (size_t)N + 1)));
    CU(cudaMalloc(&c->cb_tileI, 4 * (size_t)ntl));
    std::vector<int> ti(ntl);
    size_t k = 0;
    for (int I = 0; I < NT; I++)
      for (int J = I; J < NT; J++) ti[k++] = I;
    CU(cudaMemcpyAsync(c->cb_tileI, ti.data(), 4 * (size_t)ntl, cudaMemcpyHostToDevice,
                       c->stream));
    CU(cudaStreamSynchronize(c->stream));
    c->bytes += 8 * (size_t)ntl * 193 + 8 * (3 * (size_t)N + 1) + 4 * (size_t)ntl;
  }
  Lat l = step_lat(c);
  Ewald ew;
  std::vector<double> kv;
  double Dtr[3];
  hi_setup(c, l, &ew, &kv, Dtr, 3.5, 0, false);
  double* kdev = nullptr;
  if (!kv.empty()) {
    CU(cudaMalloc(&kdev, 8 * kv.size()));
    CU(cudaMemcpyAsync(kdev, kv.data(), 8 * kv.size(), cudaMemcpyHostToDevice, c->stream));
  }
  double* rs = c->cb_part + (size_t)ntl * 193;
  size_t smem = 8 * 9 * (size_t)ew.nk;
  c->launches += 3;
  if (smem <= 96 * 1024) {
    cudaFuncSetAttribute(k_ewald_bin_tiles<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         96 * 1024);
    k_ewald_bin_tiles<true><<<(unsigned)ntl, 256, smem, c->stream>>>(
        l, ew, c->rx, c->ry, c->rz, N, NT, c->cb_tileI, kdev, Dtr[0], Dtr[1], Dtr[2],
        c->cb_part);
  } else {
    k_ewald_bin_tiles<false><<<(unsigned)ntl, 256, 0, c->stream>>>(
        l, ew, c->rx, c->ry, c->rz, N, NT, c->cb_tileI, kdev, Dtr[0], Dtr[1], Dtr[2],
        c->cb_part);
  }
  k_ewald_bin_reduce<<<NT, 96, 0, c->stream>>>(c->cb_part, NT, N, rs);
  k_ewald_bin_eps<<<1, 32, 0, c->stream>>>(c->cb_part, ntl, rs + 3 * (size_t)N);
  rowsum.resize(3 * (size_t)N);
  CU(cudaMemcpyAsync(rowsum.data(), rs, 24 * (size_t)N, cudaMemcpyDeviceToHost, c->stream));
  CU(cudaMemcpyAsync(eps, rs + 3 * (size_t)N, 8, cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  if (kdev) cudaFree(kdev);
  return launch_ok(c);
}

}  // namespace bd
