// bd_b200 context, state transfer, lattice/PBC, pair forces, free-draining
// update, reference noise and the reference-mode step driver.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bd_ctx.cuh"

using namespace bd;

#define CU(call) BD_CU(call)

namespace bd {

int set_error_from_bits(int bits) {
  if (bits & ERRB_OVERSTRETCH) return BD_ERR_OVERSTRETCH;
  if (bits & ERRB_NONFINITE) return BD_ERR_NONFINITE;
  if (bits & ERRB_NBR_OVERFLOW) return BD_ERR_NBR_OVERFLOW;
  if (bits & ERRB_GRID_RANGE) return BD_ERR_GRID_RANGE;
  if (bits & ERRB_TIMEOUT) return BD_ERR_TIMEOUT;
  return BD_OK;
}

static thread_local char g_detail[320];

void set_error_detail(const char* msg) { snprintf(g_detail, sizeof(g_detail), "%s", msg); }

int cuda_fail(int code, const char* msg, const char* file, int line) {
  const char* base = file;
  for (const char* q = file; *q; q++)
    if (*q == '/') base = q + 1;
  snprintf(g_detail, sizeof(g_detail), "%s:%d: %s (code %d)", base, line, msg ? msg : "", code);
  return BD_ERR_CUDA;
}

// BD_DEBUG_SYNC=1 in the environment: every launch check also waits for the
// context's stream, so an asynchronous fault is reported at the launches
// that caused it (slow; for diagnosis only).
static bool debug_sync() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("BD_DEBUG_SYNC");
    on = (e && e[0] == '1') ? 1 : 0;
  }
  return on == 1;
}

int launch_ok_at(bd_ctx* c, const char* file, int line) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && c && !c->capturing && debug_sync()) e = cudaStreamSynchronize(c->stream);
  if (e == cudaSuccess) return BD_OK;
  return cuda_fail((int)e, cudaGetErrorString(e), file, line);
}

int check(bd_ctx* c) {
  int bits = 0;
  CU(cudaMemcpyAsync(&bits, c->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  if (bits) {
    CU(cudaMemsetAsync(c->err, 0, sizeof(int), c->stream));
    CU(cudaStreamSynchronize(c->stream));
  }
  return set_error_from_bits(bits);
}

static const double kEP = 0.9624;  // strain period constant (shear/src/Parameters.h:37)

static double theta0(int flow) {
  double th = 90.0 - (45.0 + (flow == 0 ? 0.0 : 31.7));
  return th * (M_PI / 180);
}

// Undeformed cell corners (initLattice, shear/src/Initialization.c:225-229).
static void corners0(int flow, double L, double p0[3][2]) {
  double th = theta0(flow);
  p0[0][0] = -sqrt(2) / 2 * L * cos(th);
  p0[0][1] = sqrt(2) / 2 * L * sin(th);
  p0[1][0] = -sqrt(2) / 2 * L * sin(th);
  p0[1][1] = -sqrt(2) / 2 * L * cos(th);
  p0[2][0] = sqrt(2) / 2 * L * cos(th);
  p0[2][1] = -sqrt(2) / 2 * L * sin(th);
}

// updateLattice (shear/src/main26.c:1382-1408, extensional/src/main14.c:
// 1426-1450), evaluated on the host with the C library so that every kernel
// sees the reference's lattice bit for bit.
void host_lattice(bd_ctx* c, unsigned long t, Lat* out) {
  host_lattice_at(c, t, c->p.dt, c->tp, out);
}

void host_lattice_at(bd_ctx* c, unsigned long t, double dt, int tp, Lat* out) {
  Lat l;
  memset(&l, 0, sizeof(l));
  double L = c->p.L, p0[3][2], pt[3][2];
  corners0(c->p.flow, L, p0);
  int treal = (int)(t % (unsigned long)tp);
  double edot = c->p.edot;
  if (c->p.flow == 0) {
    for (int a = 0; a < 3; a++) {
      pt[a][1] = p0[a][1];
      pt[a][0] = p0[a][0] + pt[a][1] * edot * treal * dt;
    }
  } else {
    for (int a = 0; a < 3; a++) {
      pt[a][0] = p0[a][0] * exp(edot * treal * dt);
      pt[a][1] = p0[a][1] * exp(-edot * treal * dt);
    }
  }
  l.flow = c->p.flow;
  l.treal = treal;
  l.tp = tp;
  l.nmax = (treal <= tp / 2) ? 1 : 2;
  l.L = L;
  l.L1x = pt[2][0] - pt[1][0];
  l.L1y = pt[2][1] - pt[1][1];
  l.L2x = pt[0][0] - pt[1][0];
  l.L2y = pt[0][1] - pt[1][1];
  if (c->p.flow == 0) {
    l.L1xp = l.L1x;
    l.L2xp = l.L2x;
    l.L1yp = l.L1y;
    l.L2yp = l.L2y;
    l.detL = l.L2yp * l.L1xp * L;
    l.cth = 1.0;
    l.sth = 0.0;
  } else {
    double th = atan(l.L1y / l.L1x);
    l.cth = cos(th);
    l.sth = sin(th);
    l.L1xp = l.L1x * cos(th) + l.L1y * sin(th);
    l.L2xp = l.L2x * cos(th) + l.L2y * sin(th);
    l.L1yp = -l.L1x * sin(th) + l.L1y * cos(th);
    l.L2yp = -l.L2x * sin(th) + l.L2y * cos(th);
    l.detL = L * (-l.L1yp * l.L2xp + l.L1xp * l.L2yp);
  }
  l.delx = edot * treal * dt;
  *out = l;
}

}  // namespace bd

// ---------------------------------------------------------------------------
// kernels

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sums three per-thread values over the block and adds them to out[0..2].
__device__ __forceinline__ void block_add3(double a, double b, double c, double* out) {
  __shared__ double sh[3][32];
  a = warp_sum(a);
  b = warp_sum(b);
  c = warp_sum(c);
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    sh[0][w] = a;
    sh[1][w] = b;
    sh[2][w] = c;
  }
  __syncthreads();
  if (w == 0) {
    int nw = (blockDim.x + 31) >> 5;
    a = lane < nw ? sh[0][lane] : 0.0;
    b = lane < nw ? sh[1][lane] : 0.0;
    c = lane < nw ? sh[2][lane] : 0.0;
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    if (lane == 0 && (a != 0.0 || b != 0.0 || c != 0.0)) {
      atomicAdd(out, a);
      atomicAdd(out + 1, b);
      atomicAdd(out + 2, c);
    }
  }
}

// applyPBC (shear/src/main26.c:1409-1428, extensional/src/main14.c:1451-1461)
__global__ void k_apply_pbc(Lat l, double* __restrict__ rx, double* __restrict__ ry,
                            double* __restrict__ rz, int N) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= N) return;
  double x = rx[a], y = ry[a], z = rz[a];
  x = subx(x, mulx(l.L2xp, round(y / l.L2yp)));
  if (l.flow == 0) {
    if (y > l.L2yp / 2) {
      x = subx(x, l.delx);
      y = subx(y, mulx(l.L2yp, round(y / l.L2yp)));
    } else if (y < -l.L2yp / 2) {
      x = addx(x, l.delx);
      y = subx(y, mulx(l.L2yp, round(y / l.L2yp)));
    }
  } else {
    y = subx(y, mulx(l.L2yp, round(y / l.L2yp)));
  }
  x = subx(x, mulx(l.L1xp, round(subx(x, mulx(y, l.L2xp) / l.L2yp) / l.L1xp)));
  z = subx(z, mulx(l.L, round(z / l.L)));
  rx[a] = x;
  ry[a] = y;
  rz[a] = z;
}

// transformCoords / inverseCoords (extensional/src/main14.c:1514-1535)
__global__ void k_rotate(Lat l, double* __restrict__ rx, double* __restrict__ ry, int N,
                         int inverse) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= N) return;
  double x = rx[a], y = ry[a];
  if (!inverse) {
    rx[a] = addx(mulx(x, l.cth), mulx(y, l.sth));
    ry[a] = addx(mulx(-x, l.sth), mulx(y, l.cth));
  } else {
    rx[a] = subx(mulx(x, l.cth), mulx(y, l.sth));
    ry[a] = addx(mulx(x, l.sth), mulx(y, l.cth));
  }
}

__global__ void k_zero3(double* a, double* b, double* c, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) {
    a[i] = 0.0;
    b[i] = 0.0;
    c[i] = 0.0;
  }
}

// Spring force of the bond (a, a-1) along v = NID(a, a-1).
__device__ __forceinline__ double spring_coeff(double rrv, int spring, double kappas,
                                               double qmax, double qmax2, int* err) {
  if (spring == BD_SPRING_FENE) {
    if (rrv > qmax2) {
      atomicOr(err, ERRB_OVERSTRETCH);
      return 0.0;
    }
    return -kappas / (1.0 - rrv / qmax2);
  }
  double r = sqrt(rrv);
  return -kappas * (r - qmax) / r;
}

struct BendTerms {
  double center[3], prev[3], next[3];
  double sxx, syy;
};

// Bending terms of the angle centred at bead m (shear/src/main26.c:581-617),
// including the reference's virial expression.
__device__ void bend_terms(const Lat& l, const double* rx, const double* ry, const double* rz,
                           int m, double kappab, BendTerms& o) {
  double n1[3], n2[3];
  nid(l, rx, ry, rz, m, m - 1, n1[0], n1[1], n1[2]);
  nid(l, rx, ry, rz, m, m + 1, n2[0], n2[1], n2[2]);
  double a1 = sqrt(n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2]);
  double a2 = sqrt(n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]);
  double var = (n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2]) / (a1 * a2);
  double thb = M_PI - acos(var);
  double co = -kappab * thb / sqrt(1 - var * var);
  for (int d = 0; d < 3; d++) {
    o.center[d] = co * ((n1[d] + n2[d]) / (a1 * a2) - var * (n1[d] / (a1 * a1) + n2[d] / (a2 * a2)));
    o.prev[d] = co * (var * n1[d] / (a1 * a1) - n2[d] / (a1 * a2));
    o.next[d] = co * (var * n2[d] / (a2 * a2) - n1[d] / (a1 * a2));
  }
  double sxx = 0, syy = 0;
  sxx += n1[0] * co * (var * n1[0] / (a1 * a1) - n2[0] / (a1 * a2));
  sxx -= n1[0] * co * ((n1[0]) / (a1 * a2) - var * (n1[0] / (a1 * a1)));
  sxx += n2[0] * co * ((n2[0]) / (a1 * a2) - var * (n2[0] / (a2 * a2)));
  sxx -= n2[0] * co * (var * n2[0] / (a2 * a2) - n1[0] / (a1 * a2));
  syy += n1[1] * co * (var * n1[1] / (a1 * a1) - n2[1] / (a1 * a2));
  syy -= n1[1] * co * ((n1[2]) / (a1 * a2) - var * (n1[2] / (a1 * a1)));
  syy += n2[1] * co * ((n2[2]) / (a1 * a2) - var * (n2[2] / (a2 * a2)));
  syy -= n2[1] * co * (var * n2[1] / (a2 * a2) - n1[1] / (a1 * a2));
  o.sxx = sxx;
  o.syy = syy;
}

// bondforce (shear/src/main26.c:541-618): one thread per bead gathers the
// spring forces of its two bonds (and the bending terms of the three angles
// it belongs to); each bond's virial is counted by its upper bead.
__global__ void k_bond(Lat l, const double* __restrict__ rx, const double* __restrict__ ry,
                       const double* __restrict__ rz, double* fx, double* fy, double* fz, int N,
                       int Nb, int spring, double kappas, double qmax, double qmax2,
                       double kappab, double* stress, int* err) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  double sxx = 0, syy = 0, sxy = 0;
  if (a < N) {
    int b = a % Nb;
    double f0 = 0, f1 = 0, f2 = 0, vx, vy, vz;
    if (b > 0) {
      nid(l, rx, ry, rz, a, a - 1, vx, vy, vz);
      double Fs = spring_coeff(rr3(vx, vy, vz), spring, kappas, qmax, qmax2, err);
      f0 += Fs * vx;
      f1 += Fs * vy;
      f2 += Fs * vz;
      sxx -= 2.0 * vx * Fs * vx;
      syy -= 2.0 * vy * Fs * vy;
      sxy -= 2.0 * vx * Fs * vy;
    }
    if (b < Nb - 1) {
      nid(l, rx, ry, rz, a + 1, a, vx, vy, vz);
      double Fs = spring_coeff(rr3(vx, vy, vz), spring, kappas, qmax, qmax2, err);
      f0 += -Fs * vx;
      f1 += -Fs * vy;
      f2 += -Fs * vz;
    }
    if (kappab > 0.0) {
      BendTerms bt;
      if (b >= 1 && b <= Nb - 2) {
        bend_terms(l, rx, ry, rz, a, kappab, bt);
        f0 += bt.center[0];
        f1 += bt.center[1];
        f2 += bt.center[2];
        sxx += bt.sxx;
        syy += bt.syy;
      }
      if (b + 1 >= 1 && b + 1 <= Nb - 2) {
        bend_terms(l, rx, ry, rz, a + 1, kappab, bt);
        f0 += bt.prev[0];
        f1 += bt.prev[1];
        f2 += bt.prev[2];
      }
      if (b - 1 >= 1 && b - 1 <= Nb - 2) {
        bend_terms(l, rx, ry, rz, a - 1, kappab, bt);
        f0 += bt.next[0];
        f1 += bt.next[1];
        f2 += bt.next[2];
      }
    }
    fx[a] += f0;
    fy[a] += f1;
    fz[a] += f2;
  }
  if (l.flow != 0) sxy = 0.0;
  block_add3(sxx, syy, sxy, stress);
}

// LJforce over the neighbour rows (shear/src/main26.c:619-681: LJ
// 12 eps (r6^2 - r6)/r^2 with rc = 5 in shear; extensional/src/main14.c:
// 625-685: WCA 48 eps (r6^2 - r6/2)/r^2 with rc^2 = 5.03968).  One thread per
// bead walks its full (sorted) row; the virial counts each pair once.
__global__ void __launch_bounds__(256) k_ev(Lat l, const double* __restrict__ rx,
                                            const double* __restrict__ ry,
                                            const double* __restrict__ rz, double* fx, double* fy,
                                            double* fz, int N, const int* __restrict__ cnt,
                                            const int* __restrict__ rows, int maxnb, double r2cut,
                                            double eps, double* stress) {
  // one warp per bead: the lanes split its neighbour row, then a butterfly
  int i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  double sxx = 0, syy = 0, sxy = 0;
  if (i < N) {
    double f0 = 0, f1 = 0, f2 = 0;
    int n = cnt[i];
    const int* row = rows + (size_t)i * maxnb;
    double xi = rx[i], yi = ry[i], zi = rz[i];
    for (int k = lane; k < n; k += 32) {
      int j = row[k];
      double vx, vy, vz;
      min_image(l, subx(xi, rx[j]), subx(yi, ry[j]), subx(zi, rz[j]), vx, vy, vz);
      double rrv = rr3(vx, vy, vz);
      if (rrv < r2cut) {
        double ratio = 4.00 / rrv;
        double r6 = ratio * ratio * ratio, co;
        if (l.flow == 0)
          co = (12 * eps / rrv) * (r6 * r6 - r6);
        else
          co = (48.0 * eps / rrv) * (r6 * r6 - 0.5 * r6);
        f0 += co * vx;
        f1 += co * vy;
        f2 += co * vz;
        if (j > i) {
          sxx -= 2.0 * vx * co * vx;
          syy -= 2.0 * vy * co * vy;
          sxy -= 2.0 * vx * co * vy;
        }
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      f0 += __shfl_xor_sync(0xffffffffu, f0, o);
      f1 += __shfl_xor_sync(0xffffffffu, f1, o);
      f2 += __shfl_xor_sync(0xffffffffu, f2, o);
    }
    if (lane == 0) {
      fx[i] += f0;
      fy[i] += f1;
      fz[i] += f2;
    }
  }
  if (l.flow != 0) sxy = 0.0;
  block_add3(sxx, syy, sxy, stress);
}

// Gathers the charged beads into compact arrays (x, y, z, q per charge).
__global__ void k_gather_charges(const double* __restrict__ rx, const double* __restrict__ ry,
                                 const double* __restrict__ rz, const double* __restrict__ q,
                                 const int* __restrict__ track, int nch, double4* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nch) {
    int i = track[k];
    out[k] = make_double4(rx[i], ry[i], rz[i], q[i]);
  }
}

// coulombForce: screened Coulomb (Debye-Hueckel) over all charged pairs
// (shear/src/main26.c:1891-1925).  One warp per charge; lanes stride over the
// other charges; no cutoff.
__global__ void k_coulomb(Lat l, const double4* __restrict__ cq, const int* __restrict__ track,
                          int nch, double* fx, double* fy, double* fz, double lambda_b,
                          double kappa_d) {
  int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (k >= nch) return;
  double4 me = cq[k];
  double f0 = 0, f1 = 0, f2 = 0;
  for (int o = lane; o < nch; o += 32) {
    if (o == k) continue;
    double4 ot = cq[o];
    double vx, vy, vz;
    min_image(l, subx(me.x, ot.x), subx(me.y, ot.y), subx(me.z, ot.z), vx, vy, vz);
    double rrv = rr3(vx, vy, vz);
    double r = sqrt(rrv);
    double Fc = lambda_b * me.w * ot.w * exp(-kappa_d * r) * (1 + r * kappa_d) / rrv;
    f0 += Fc * vx / r;
    f1 += Fc * vy / r;
    f2 += Fc * vz / r;
  }
  f0 = warp_sum(f0);
  f1 = warp_sum(f1);
  f2 = warp_sum(f2);
  if (lane == 0) {
    int i = track[k];
    fx[i] += f0;
    fy[i] += f1;
    fz[i] += f2;
  }
}

// updateFD (shear/src/main26.c:731-744, extensional/src/main14.c:735-782)
__global__ void k_update_fd(int flow, double* rx, double* ry, double* rz, double* dxv,
                            double* dyv, double* dzv, const double* __restrict__ fx,
                            const double* __restrict__ fy, const double* __restrict__ fz,
                            const double* __restrict__ R, int N, double dt, double edot,
                            double pc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double dx, dy, dz;
  if (flow == 0) {
    dx = dt * (fx[i] + edot * ry[i]) + pc * R[3 * i];
    dy = dt * fy[i] + pc * R[3 * i + 1];
  } else {
    dx = dt * (fx[i] + edot * rx[i]) + pc * R[3 * i];
    dy = dt * (fy[i] - edot * ry[i]) + pc * R[3 * i + 1];
  }
  dz = dt * fz[i] + pc * R[3 * i + 2];
  rx[i] += dx;
  ry[i] += dy;
  rz[i] += dz;
  dxv[i] += dx;
  dyv[i] += dy;
  dzv[i] += dz;
}

// gasdev (shear/src/main26.c:515-540): polar Box-Muller in float, products
// kept un-fused to match the host's float arithmetic.
__device__ float gasdev_dev(Ran1& g) {
  float fac, rsq, v1, v2;
  if (g.idum < 0) g.iset = 0;
  if (g.iset == 0) {
    do {
      v1 = (float)(2.0 * (double)ran1_dev(g) - 1.0);
      v2 = (float)(2.0 * (double)ran1_dev(g) - 1.0);
      rsq = __fadd_rn(__fmul_rn(v1, v1), __fmul_rn(v2, v2));
    } while (rsq >= 1.0f || rsq == 0.0f);
    fac = (float)sqrt(-2.0 * log((double)rsq) / (double)rsq);
    g.gset = __fmul_rn(v1, fac);
    g.iset = 1;
    return __fmul_rn(v2, fac);
  }
  g.iset = 0;
  return g.gset;
}


// Gaussian noise from Philox: counter (pair index, step, stream), key = seed;
// two 53-bit uniforms per draw, Box-Muller (u1 in (0,1]) for two deviates.
__global__ void k_noise_philox(double* R, int n, unsigned long long seed, unsigned long long step) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (2 * k >= n) return;
  uint4 c = make_uint4((uint32_t)k, (uint32_t)step, (uint32_t)(step >> 32), 0x42445f42u);
  uint4 x = philox4x32_10(c, make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  const double s53 = 1.0 / 9007199254740992.0;
  double u1 = ((double)(((unsigned long long)(x.x >> 5) << 26) | (x.y >> 6)) + 1.0) * s53;
  double u2 = (double)(((unsigned long long)(x.z >> 5) << 26) | (x.w >> 6)) * s53;
  double r = sqrt(-2.0 * log(u1)), sn, cs;
  sincospi(2.0 * u2, &sn, &cs);
  R[2 * k] = r * cs;
  if (2 * k + 1 < n) R[2 * k + 1] = r * sn;
}

// getNoise with the reference's generator (shear/src/main26.c:708-713).  The
// generator is a sequential chain, so one thread draws all 3N deviates; the
// shuffle table lives in shared memory.
__global__ void k_gasdev_seq(Ran1* gs, double* R, int n) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Ran1 g = *gs;
  for (int a = 0; a < n; a++) R[a] = (double)gasdev_dev(g);
  *gs = g;
}

// ---------------------------------------------------------------------------
// host side

static inline int nblk(int n, int b) { return (n + b - 1) / b; }

static int dalloc(bd_ctx* c, void** p, size_t bytes) {
  if (bytes == 0) bytes = 16;
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    *p = nullptr;
    return BD_ERR_OOM;
  }
  c->bytes += bytes;
  return BD_OK;
}

#define DALLOC(ptr, bytes)                                   \
  do {                                                       \
    int s_ = dalloc(c, (void**)&(ptr), (bytes));             \
    if (s_) {                                                \
      bd_destroy(c);                                         \
      return s_;                                             \
    }                                                        \
  } while (0)

extern "C" {

const char* bd_last_error_detail(void) { return g_detail; }

// Spacing proportional to the cutoff: the split parameter is 4 / rc, so
// alpha h stays at most 0.31, within 3.3e-6 of the converged Ewald sum over
// the lattice period of both flows (1.29 L points at rc = 10); cuFFT is
// markedly slower on sizes with a factor 7, hence 2^a 3^b 5^c.
// The raw generator behind every Philox draw of the library: block k is
// Philox4x32-10 of counter ctr[4k..4k+3] under key key[2k..2k+1].
__global__ void k_philox_raw(const uint32_t* __restrict__ ctr, const uint32_t* __restrict__ key,
                             uint32_t* __restrict__ out, int n) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint4 x = philox4x32_10(make_uint4(ctr[4 * k], ctr[4 * k + 1], ctr[4 * k + 2], ctr[4 * k + 3]),
                          make_uint2(key[2 * k], key[2 * k + 1]));
  out[4 * k] = x.x;
  out[4 * k + 1] = x.y;
  out[4 * k + 2] = x.z;
  out[4 * k + 3] = x.w;
}

int bd_philox4x32_10(const unsigned* ctr, const unsigned* key, unsigned* out, int n) {
  if (!ctr || !key || !out || n < 1 || n > (1 << 20)) return BD_ERR_ARG;
  uint32_t* d = nullptr;
  size_t bytes = 4 * (size_t)n * 10;
  cudaError_t e = cudaMalloc(&d, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return BD_ERR_OOM;
  }
  e = cudaMemcpy(d, ctr, 16 * (size_t)n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + 4 * (size_t)n, key, 8 * (size_t)n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_philox_raw<<<(n + 255) / 256, 256>>>(d, d + 4 * (size_t)n, d + 6 * (size_t)n, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d + 6 * (size_t)n, 16 * (size_t)n, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return bd::cuda_fail((int)e, cudaGetErrorString(e), __FILE__, __LINE__);
  return BD_OK;
}

int bd_pme_default_grid(double L, double rc, int* K_out) {
  if (!(L > 0) || !K_out) return BD_ERR_ARG;
  double rc0 = rc > 0 ? rc : std::min(10.0, 0.43 * L);
  double x = 12.9 * L / rc0;
  if (!(x <= 4096.0)) return BD_ERR_ARG;
  int K = std::max(1, (int)ceil(x - 1e-9));
  for (;; K++) {
    int r = K;
    for (int f : {2, 3, 5})
      while (r % f == 0) r /= f;
    if (r == 1) break;
  }
  if (K > 4096) return BD_ERR_ARG;
  *K_out = K;
  return BD_OK;
}

const char* bd_status_string(int s) {
  switch (s) {
    case BD_OK: return "ok";
    case BD_ERR_ARG: return "invalid argument";
    case BD_ERR_CUDA: return "CUDA runtime error";
    case BD_ERR_OOM: return "device out of memory";
    case BD_ERR_OVERSTRETCH: return "FENE overstretch";
    case BD_ERR_NONFINITE: return "non-finite value";
    case BD_ERR_NBR_OVERFLOW: return "neighbour row overflow";
    case BD_ERR_GRID_RANGE: return "displacement outside lookup table";
    case BD_ERR_STATE: return "call out of order";
    case BD_ERR_TIMEOUT: return "bounded device wait timed out";
    case BD_ERR_LANCZOS: return "Lanczos tolerance not met";
    case BD_ERR_ASYMMETRIC: return "asymmetric lookup tensor";
    case BD_ERR_CAPACITY: return "system larger than the fixed buffer allows";
  }
  return "unknown status";
}

int bd_create(const bd_params* p, bd_ctx** out) {
  if (!p || !out) return BD_ERR_ARG;
  *out = nullptr;
  if (p->Nb < 1 || p->Nc < 1 || p->L <= 0 || p->dt <= 0 || p->edot <= 0) return BD_ERR_ARG;
  if (p->flow != BD_FLOW_SHEAR && p->flow != BD_FLOW_EXT) return BD_ERR_ARG;
  if (p->spring != BD_SPRING_FENE && p->spring != BD_SPRING_HOOKEAN) return BD_ERR_ARG;
  if (p->nt_avg < 1 || p->bin_size <= 0 || p->lambda_d <= 0) return BD_ERR_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return BD_ERR_CUDA;
  bd_ctx* c = new bd_ctx();  // value-initialised: every plain member starts at zero
  c->p = *p;
  c->N = p->Nb * p->Nc;
  c->Nb = p->Nb;
  c->Nc = p->Nc;
  cudaGetDevice(&c->device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return BD_ERR_CUDA;
  }
  // initVerlet (shear/src/Initialization.c:300-316, extensional 289-305)
  double sigma = 2.0, rc;
  if (p->flow == 0) {
    rc = 2.5 * sigma;
    c->r2cut = rc * rc;
  } else {
    c->r2cut = 5.03968;
    rc = sqrt(c->r2cut);
  }
  c->rv = 3.0 * sigma;
  c->rnew = 0.5 * (c->rv - rc);
  c->qmax2 = p->qmax * p->qmax;
  c->kappa_d = 1 / p->lambda_d;
  c->boxvol = p->box_volume > 0 ? p->box_volume : p->L * p->L * p->L;
  c->kappas_eff = (p->flow == 0 && !p->shear_kappas_override) ? 200.0 : p->kappas;
  c->tp = (int)(kEP / p->edot / p->dt);
  if (c->tp < 1) {
    bd_destroy(c);
    return BD_ERR_ARG;
  }
  c->srpy = p->srpy > 0 ? p->srpy : 100;
  c->sbins = p->sbins > 0 ? p->sbins : 20;
  c->strain_ss = p->strain_ss > 0 ? p->strain_ss : 10.0;
  c->strain_interval = c->strain_ss / c->sbins;
  c->maxnb = p->max_neighbors > 0 ? p->max_neighbors : 256;
  // noise blocks need the particle-mesh product (any number of right-hand sides)
  c->nbk = (p->mobility == BD_MOB_PME && p->noise_block > 1) ? p->noise_block : 1;
  if (p->lanczos_max > kMaxKrylov || p->mobility < 0 || p->mobility > 2 || p->precision < 0 ||
      p->precision > 1 || p->noise_block < 0 || p->noise_block > BD_MAX_NOISE_BLOCK) {
    bd_destroy(c);
    return BD_ERR_ARG;
  }
  // smooth-PME discretisation
  {
    // default grid (bd_pme_default_grid): only the particle-mesh mobility
    // and Ewald Coulomb use it
    int K = p->pme_grid;
    if (K <= 0 && bd_pme_default_grid(p->L, p->pme_rc, &K) != BD_OK) {
      if (p->mobility == BD_MOB_PME || p->coulomb == BD_COULOMB_EWALD) {
        bd_destroy(c);
        return BD_ERR_ARG;
      }
      K = 0;
    }
    c->pmeK = K;
    c->pme_p = p->pme_order > 0 ? p->pme_order : 8;
    c->pme_rc = p->pme_rc > 0 ? p->pme_rc : std::min(10.0, 0.43 * p->L);
    c->pme_alpha = p->pme_alpha > 0 ? p->pme_alpha : 4.0 / c->pme_rc;
    c->hop_R = p->hop_radius > 0 ? p->hop_radius : 3.0 * p->lambda_d;
    if (p->hop < 0 || p->hop > 1) {
      bd_destroy(c);
      return BD_ERR_ARG;
    }
    c->cw_rc = p->coulomb_rc > 0 ? p->coulomb_rc : std::min(10.0, 0.43 * p->L);
    c->cw_beta = p->coulomb_beta > 0 ? p->coulomb_beta : 3.5 / c->cw_rc;
    if (p->coulomb < 0 || p->coulomb > 1 ||
        (p->coulomb == BD_COULOMB_EWALD && (K < 8 || K > 1024 || c->pme_p < 4 || c->pme_p > 8 ||
                                            (c->pme_p & 1) || c->cw_rc > 0.43 * p->L))) {
      bd_destroy(c);
      return BD_ERR_ARG;
    }
    if (p->mobility == BD_MOB_PME &&
        (K < 8 || K > 1024 || c->pme_p < 4 || c->pme_p > 8 || (c->pme_p & 1) || c->pme_p > K ||
         c->pme_rc > 0.43 * p->L)) {
      bd_destroy(c);
      return BD_ERR_ARG;
    }
  }
  // lookup-grid geometry (initLattice, shear/src/Initialization.c:244-295,
  // extensional/src/Initialization.c:252-285)
  {
    double L = p->L, p0[3][2];
    corners0(p->flow, L, p0);
    double xmax, ymax, zmax = L / 2;
    int treal = c->tp;
    if (p->flow == 0) {
      ymax = L / 2;
      xmax = L / 2 * p->edot * treal * p->dt;
    } else {
      ymax = -p0[1][1];
      xmax = p0[2][0] * exp(p->edot * treal * p->dt);
    }
    c->bsx = c->bsy = c->bsz = p->bin_size;
    c->nbx = 2 * ceil(xmax / c->bsx) + 1;
    c->bsx = xmax / ((c->nbx - 1) / 2);
    c->nhx = (c->nbx - 1) / 2;
    c->nby = 2 * ceil(ymax / c->bsy) + 1;
    c->bsy = ymax / ((c->nby - 1) / 2);
    c->nhy = (c->nby - 1) / 2;
    c->nbz = 2 * ceil(zmax / c->bsz) + 1;
    c->bsz = zmax / ((c->nbz - 1) / 2);
    c->nhz = (c->nbz - 1) / 2;
    c->nbins = c->nbx * c->nby * c->nbz;
  }
  int N = c->N;
  DALLOC(c->rx, 8 * N);
  DALLOC(c->ry, 8 * N);
  DALLOC(c->rz, 8 * N);
  DALLOC(c->fx, 8 * N);
  DALLOC(c->fy, 8 * N);
  DALLOC(c->fz, 8 * N);
  DALLOC(c->dxv, 8 * N);
  DALLOC(c->dyv, 8 * N);
  DALLOC(c->dzv, 8 * N);
  DALLOC(c->R, 24 * (size_t)N);
  DALLOC(c->stress, 8 * 4);
  DALLOC(c->err, 16);
  DALLOC(c->flag, 16);
  DALLOC(c->track, 4 * (size_t)std::max(N, 1));
  DALLOC(c->old, 4 * (size_t)std::max(N, 1));
  DALLOC(c->cflags, 4 * (size_t)N);
  DALLOC(c->hoplog, 12 * (size_t)std::max(N, 1));
  DALLOC(c->q, 8 * (size_t)N);
  DALLOC(c->dE, 64 * (size_t)std::max(N, 1));
  DALLOC(c->rng, sizeof(Ran1));
  cudaMemsetAsync(c->rx, 0, 8 * N, c->stream);
  cudaMemsetAsync(c->ry, 0, 8 * N, c->stream);
  cudaMemsetAsync(c->rz, 0, 8 * N, c->stream);
  cudaMemsetAsync(c->fx, 0, 8 * N, c->stream);
  cudaMemsetAsync(c->fy, 0, 8 * N, c->stream);
  cudaMemsetAsync(c->fz, 0, 8 * N, c->stream);
  cudaMemsetAsync(c->dxv, 0, 8 * N, c->stream);
  cudaMemsetAsync(c->dyv, 0, 8 * N, c->stream);
  cudaMemsetAsync(c->dzv, 0, 8 * N, c->stream);
  cudaMemsetAsync(c->R, 0, 24 * (size_t)N, c->stream);
  cudaMemsetAsync(c->stress, 0, 32, c->stream);
  cudaMemsetAsync(c->err, 0, 16, c->stream);
  cudaMemsetAsync(c->flag, 0, 16, c->stream);
  cudaMemsetAsync(c->cflags, 0, 4 * (size_t)N, c->stream);
  cudaMemsetAsync(c->q, 0, 8 * (size_t)N, c->stream);
  {
    Ran1 g;
    memset(&g, 0, sizeof(g));
    g.idum = p->seed;
    g.idum2 = 123456789LL;
    cudaMemcpyAsync(c->rng, &g, sizeof(g), cudaMemcpyHostToDevice, c->stream);
  }
  int s;
  if ((s = alloc_neighbors(c)) != BD_OK || (s = alloc_mobility(c)) != BD_OK) {
    bd_destroy(c);
    return s;
  }
  c->btab.assign(c->sbins + 1, 0.0);
  if (c->nbk > 1) {
    // pinned host copy of the noise blocks' alpha and beta, allocated here
    // rather than at the first block: a pinned allocation can synchronise
    // the device, which would void a stream capture running at that moment
    // in another thread (replicas of a batch capture their iterations
    // concurrently)
    int L1 = (p->lanczos_max > 0 ? p->lanczos_max : 200) + 1;
    if (cudaMallocHost(&c->Bhost, 8 * (size_t)2 * c->nbk * L1) != cudaSuccess) {
      bd_destroy(c);
      return BD_ERR_OOM;
    }
  }
  c->use_graphs = true;
  c->device_krylov = true;
  c->t = 0;
  c->tstart = 0;
  host_lattice(c, 0, &c->lat);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    bd_destroy(c);
    return BD_ERR_CUDA;
  }
  *out = c;
  return BD_OK;
}

int bd_destroy(bd_ctx* c) {
  if (!c) return BD_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  void* ptrs[] = {c->rx, c->ry, c->rz, c->fx, c->fy, c->fz, c->dxv, c->dyv, c->dzv, c->R,
                  c->stress, c->err, c->flag, c->track, c->old, c->cflags, c->hoplog, c->q,
                  c->dE, c->rng, c->nb_count, c->nb_rows, c->nb_half, c->cell_of, c->cell_count,
                  c->cell_start, c->cell_beads, c->cell_cursor, c->Mt, c->tileI, c->grid,
                  c->near_pairs, c->near_count, c->kvec, c->rowpart, c->colpart, c->U, c->W,
                  c->Ctab, c->Mt32, c->LV, c->Lw, c->Lpart, c->Lh, c->Lsc, c->Lc, c->MF, c->Yz};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  pme_free(c);
  coulomb_free(c);
  if (c->hop_cells) cudaFree(c->hop_cells);
  if (c->hop_de) cudaFree(c->hop_de);
  if (c->cb_part) cudaFree(c->cb_part);
  if (c->cb_tileI) cudaFree(c->cb_tileI);
  precond_free(c);
  mpnn_free(c);
  if (c->Lt1) cudaFree(c->Lt1);
  if (c->Lt2) cudaFree(c->Lt2);
  if (c->Lvcur) cudaFree(c->Lvcur);
  if (c->Ljd) cudaFree(c->Ljd);
  lanczos_graphs_reset(c);
  lanczos_blocks_free(c);
  prof_clear(c);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return BD_OK;
}

int bd_enable_graphs(bd_ctx* c, int on) {
  if (!c) return BD_ERR_ARG;
  CU(cudaStreamSynchronize(c->stream));
  c->use_graphs = on != 0;
  if (!c->use_graphs) lanczos_graphs_reset(c);
  return BD_OK;
}

int bd_set_device_krylov(bd_ctx* c, int on) {
  if (!c) return BD_ERR_ARG;
  CU(cudaStreamSynchronize(c->stream));
  c->device_krylov = on != 0;
  return BD_OK;
}

int bd_krylov_check_stats(bd_ctx* c, long* out2) {
  if (!c || !out2) return BD_ERR_ARG;
  out2[0] = (long)c->dev_solves;
  out2[1] = (long)c->host_fallbacks;
  return BD_OK;
}

int bd_profile_enable(bd_ctx* c, int on) {
  if (!c) return BD_ERR_ARG;
  CU(cudaStreamSynchronize(c->stream));
  prof_clear(c);
  c->prof_on = on != 0;
  c->prof_products = on == 1;
  return BD_OK;
}

int bd_profile_read(bd_ctx* c, int slot, double* total_ms, long* count) {
  if (!c || slot < 0 || slot >= BD_PROF_SLOTS || !total_ms || !count) return BD_ERR_ARG;
  CU(cudaStreamSynchronize(c->stream));
  double tot = 0;
  auto& a = c->prof_ev[slot][0];
  auto& b = c->prof_ev[slot][1];
  for (size_t k = 0; k < a.size() && k < b.size(); k++) {
    float ms = 0;
    CU(cudaEventElapsedTime(&ms, a[k], b[k]));
    tot += ms;
  }
  *total_ms = tot;
  *count = (long)std::min(a.size(), b.size());
  return BD_OK;
}

long long bd_launch_count(const bd_ctx* c) { return c ? c->launches : 0; }

int bd_sync(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  return check(c);
}

size_t bd_device_bytes(const bd_ctx* c) { return c ? c->bytes : 0; }

static int up3(bd_ctx* c, double* a, double* b, double* d, const double* x, const double* y,
               const double* z) {
  if (!c || !x || !y || !z) return BD_ERR_ARG;
  size_t n = 8 * (size_t)c->N;
  CU(cudaMemcpyAsync(a, x, n, cudaMemcpyHostToDevice, c->stream));
  CU(cudaMemcpyAsync(b, y, n, cudaMemcpyHostToDevice, c->stream));
  CU(cudaMemcpyAsync(d, z, n, cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return BD_OK;
}

static int down3(bd_ctx* c, const double* a, const double* b, const double* d, double* x,
                 double* y, double* z) {
  if (!c || !x || !y || !z) return BD_ERR_ARG;
  size_t n = 8 * (size_t)c->N;
  CU(cudaMemcpyAsync(x, a, n, cudaMemcpyDeviceToHost, c->stream));
  CU(cudaMemcpyAsync(y, b, n, cudaMemcpyDeviceToHost, c->stream));
  CU(cudaMemcpyAsync(z, d, n, cudaMemcpyDeviceToHost, c->stream));
  return check(c);
}

int bd_upload_positions(bd_ctx* c, const double* x, const double* y, const double* z) {
  return up3(c, c ? c->rx : 0, c ? c->ry : 0, c ? c->rz : 0, x, y, z);
}
int bd_download_positions(bd_ctx* c, double* x, double* y, double* z) {
  return down3(c, c ? c->rx : 0, c ? c->ry : 0, c ? c->rz : 0, x, y, z);
}
int bd_upload_displacements(bd_ctx* c, const double* x, const double* y, const double* z) {
  return up3(c, c ? c->dxv : 0, c ? c->dyv : 0, c ? c->dzv : 0, x, y, z);
}
int bd_download_displacements(bd_ctx* c, double* x, double* y, double* z) {
  return down3(c, c ? c->dxv : 0, c ? c->dyv : 0, c ? c->dzv : 0, x, y, z);
}
int bd_upload_forces(bd_ctx* c, const double* x, const double* y, const double* z) {
  return up3(c, c ? c->fx : 0, c ? c->fy : 0, c ? c->fz : 0, x, y, z);
}
int bd_download_forces(bd_ctx* c, double* x, double* y, double* z) {
  return down3(c, c ? c->fx : 0, c ? c->fy : 0, c ? c->fz : 0, x, y, z);
}

int bd_download_stress(bd_ctx* c, double* out3) {
  if (!c || !out3) return BD_ERR_ARG;
  CU(cudaMemcpyAsync(out3, c->stress, 24, cudaMemcpyDeviceToHost, c->stream));
  return check(c);
}

int bd_reset_stress(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  CU(cudaMemsetAsync(c->stress, 0, 24, c->stream));
  return BD_OK;
}

int bd_upload_noise(bd_ctx* c, const double* R) {
  if (!c || !R) return BD_ERR_ARG;
  CU(cudaMemcpyAsync(c->R, R, 24 * (size_t)c->N, cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return BD_OK;
}

int bd_download_noise(bd_ctx* c, double* R) {
  if (!c || !R) return BD_ERR_ARG;
  CU(cudaMemcpyAsync(R, c->R, 24 * (size_t)c->N, cudaMemcpyDeviceToHost, c->stream));
  return check(c);
}

int bd_set_charges(bd_ctx* c, const int* track, int nch) {
  if (!c || nch < 0 || nch > c->N || (nch > 0 && !track)) return BD_ERR_ARG;
  std::vector<int> flags(c->N, 0);
  std::vector<double> q(c->N, 0.0);
  for (int k = 0; k < nch; k++) {
    if (track[k] < 0 || track[k] >= c->N || flags[track[k]]) return BD_ERR_ARG;
    flags[track[k]] = 1;
    q[track[k]] = 1.0;
  }
  c->nch = nch;
  c->cw_q2 = nch;
  c->cw_Q = nch;
  if (nch) {
    CU(cudaMemcpyAsync(c->track, track, 4 * (size_t)nch, cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(c->old, track, 4 * (size_t)nch, cudaMemcpyHostToDevice, c->stream));
  }
  CU(cudaMemcpyAsync(c->cflags, flags.data(), 4 * (size_t)c->N, cudaMemcpyHostToDevice, c->stream));
  CU(cudaMemcpyAsync(c->q, q.data(), 8 * (size_t)c->N, cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return BD_OK;
}

int bd_download_charges(bd_ctx* c, int* track, int* old, int* flags) {
  if (!c) return BD_ERR_ARG;
  if (track && c->nch)
    CU(cudaMemcpyAsync(track, c->track, 4 * (size_t)c->nch, cudaMemcpyDeviceToHost, c->stream));
  if (old && c->nch)
    CU(cudaMemcpyAsync(old, c->old, 4 * (size_t)c->nch, cudaMemcpyDeviceToHost, c->stream));
  if (flags)
    CU(cudaMemcpyAsync(flags, c->cflags, 4 * (size_t)c->N, cudaMemcpyDeviceToHost, c->stream));
  return check(c);
}

int bd_set_rng(bd_ctx* c, const bd_ran1_state* s) {
  if (!c || !s) return BD_ERR_ARG;
  noise_blocks_release(c);
  Ran1 g;
  g.idum = s->idum;
  g.idum2 = s->idum2;
  g.iy = s->iy;
  for (int a = 0; a < 32; a++) g.iv[a] = s->iv[a];
  g.iset = s->iset;
  g.gset = s->gset;
  CU(cudaMemcpyAsync(c->rng, &g, sizeof(g), cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return BD_OK;
}

int bd_get_rng(bd_ctx* c, bd_ran1_state* s) {
  if (!c || !s) return BD_ERR_ARG;
  noise_blocks_release(c);
  Ran1 g;
  CU(cudaMemcpyAsync(&g, c->rng, sizeof(g), cudaMemcpyDeviceToHost, c->stream));
  int st = check(c);
  s->idum = (long)g.idum;
  s->idum2 = (long)g.idum2;
  s->iy = (long)g.iy;
  for (int a = 0; a < 32; a++) s->iv[a] = (long)g.iv[a];
  s->iset = g.iset;
  s->gset = g.gset;
  return st;
}

int bd_grid_shape(const bd_ctx* c, int* o) {
  if (!c || !o) return BD_ERR_ARG;
  o[0] = c->nbx;
  o[1] = c->nby;
  o[2] = c->nbz;
  o[3] = c->nhx;
  o[4] = c->nhy;
  o[5] = c->nhz;
  o[6] = c->nbins;
  return BD_OK;
}

int bd_set_tea(bd_ctx* c, int sbin, double beta, const double* c3nb) {
  if (!c || !c3nb || sbin < 0 || sbin > c->sbins) return BD_ERR_ARG;
  c->btab[sbin] = beta;
  CU(cudaMemcpyAsync(c->Ctab + (size_t)sbin * 3 * c->Nb, c3nb, 24 * (size_t)c->Nb,
                     cudaMemcpyHostToDevice, c->stream));
  CU(cudaStreamSynchronize(c->stream));
  return BD_OK;
}

int bd_set_time(bd_ctx* c, unsigned long t, unsigned long tstart) {
  if (!c) return BD_ERR_ARG;
  c->t = t;
  c->tstart = tstart;
  c->strain = (double)t * c->p.dt * c->p.edot;
  return BD_OK;
}

int bd_update_lattice(bd_ctx* c, unsigned long t) {
  if (!c) return BD_ERR_ARG;
  host_lattice(c, t, &c->lat);
  return BD_OK;
}

int bd_get_lattice(const bd_ctx* c, double* o) {
  if (!c || !o) return BD_ERR_ARG;
  o[0] = c->lat.L1x;
  o[1] = c->lat.L1y;
  o[2] = c->lat.L2x;
  o[3] = c->lat.L2y;
  o[4] = c->lat.L1xp;
  o[5] = c->lat.L1yp;
  o[6] = c->lat.L2xp;
  o[7] = c->lat.L2yp;
  o[8] = c->lat.detL;
  o[9] = (double)c->tp;
  return BD_OK;
}

// Kernels see the lattice of the step the context is at (c->t), while
// updateLattice(t') may have been called for another t' (the reference does
// this only with t' == t).  getNID reads the global t (shear/src/main26.c:
// 1432), so the PBC and pair kernels use the lattice of c->lat with the
// brick offset of step c->t.
static Lat kernel_lat(bd_ctx* c) {
  Lat l = c->lat;
  int treal = (int)(c->t % (unsigned long)c->tp);
  l.treal = treal;
  l.nmax = (treal <= c->tp / 2) ? 1 : 2;
  l.delx = c->p.edot * treal * c->p.dt;
  return l;
}

int bd_apply_pbc(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  c->launches++;
  k_apply_pbc<<<nblk(c->N, 256), 256, 0, c->stream>>>(kernel_lat(c), c->rx, c->ry, c->rz, c->N);
  return launch_ok(c);
}

int bd_transform_coords(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  if (c->p.flow != BD_FLOW_EXT) return BD_OK;
  c->launches++;
  k_rotate<<<nblk(c->N, 256), 256, 0, c->stream>>>(c->lat, c->rx, c->ry, c->N, 0);
  return launch_ok(c);
}

int bd_inverse_coords(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  if (c->p.flow != BD_FLOW_EXT) return BD_OK;
  c->launches++;
  k_rotate<<<nblk(c->N, 256), 256, 0, c->stream>>>(c->lat, c->rx, c->ry, c->N, 1);
  return launch_ok(c);
}

int bd_reset_force(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  c->launches++;
  k_zero3<<<nblk(c->N, 256), 256, 0, c->stream>>>(c->fx, c->fy, c->fz, c->N);
  CU(cudaMemsetAsync(c->stress, 0, 24, c->stream));
  return launch_ok(c);
}

int bd_bond_force(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  c->launches++;
  k_bond<<<nblk(c->N, 128), 128, 0, c->stream>>>(kernel_lat(c), c->rx, c->ry, c->rz, c->fx, c->fy,
                                                  c->fz, c->N, c->Nb, c->p.spring, c->kappas_eff,
                                                  c->p.qmax, c->qmax2, c->p.kappab, c->stress,
                                                  c->err);
  return launch_ok(c);
}

int bd_ev_force(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  c->launches++;
  k_ev<<<nblk(c->N, 8), 256, 0, c->stream>>>(kernel_lat(c), c->rx, c->ry, c->rz, c->fx, c->fy,
                                                c->fz, c->N, c->nb_count, c->nb_rows, c->maxnb,
                                                c->r2cut, c->p.epsilon, c->stress);
  return launch_ok(c);
}

int bd_coulomb_force(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  bool ewald = c->p.coulomb == BD_COULOMB_EWALD;
  if (c->nch < (ewald ? 1 : 2)) return BD_OK;
  double4* cq = (double4*)c->dE;
  c->launches++;
  k_gather_charges<<<nblk(c->nch, 256), 256, 0, c->stream>>>(c->rx, c->ry, c->rz, c->q, c->track,
                                                             c->nch, cq);
  if (ewald) return coulomb_ewald(c, kernel_lat(c), cq);
  c->launches++;
  k_coulomb<<<nblk(c->nch * 32, 256), 256, 0, c->stream>>>(kernel_lat(c), cq, c->track, c->nch,
                                                           c->fx, c->fy, c->fz, c->p.lambda_b,
                                                           c->kappa_d);
  return launch_ok(c);
}

int bd_get_noise(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  noise_blocks_release(c);
  return draw_noise(c, c->R);
}

int bd_update_fd(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  c->launches++;
  k_update_fd<<<nblk(c->N, 256), 256, 0, c->stream>>>(c->p.flow, c->rx, c->ry, c->rz, c->dxv,
                                                      c->dyv, c->dzv, c->fx, c->fy, c->fz, c->R,
                                                      c->N, c->p.dt, c->p.edot,
                                                      sqrt(2.0 * c->p.dt));
  return launch_ok(c);
}

int bd_build_neighbors(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  return build_neighbors(c, true);
}

int bd_check_verlet(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  return build_neighbors(c, false);
}

int bd_calc_hi(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  return calc_hi(c);
}

int bd_update_hi(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  return update_hi(c);
}

int bd_download_mobility(bd_ctx* c, double* M9) {
  if (!c || !M9) return BD_ERR_ARG;
  return download_mobility(c, M9);
}

int bd_charge_hop(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  noise_blocks_release(c);
  return charge_hop(c);
}

int bd_download_hop_log(bd_ctx* c, int* log3) {
  if (!c || !log3) return BD_ERR_ARG;
  if (c->nch)
    CU(cudaMemcpyAsync(log3, c->hoplog, 12 * (size_t)c->nch, cudaMemcpyDeviceToHost, c->stream));
  return check(c);
}

// One hydrodynamic step of the reference's loop body in its own order
// (shear/src/main26.c:65-151; extensional/src/main14.c:68-171), without the
// file output and diagnostics.  Mobility rebuild and charge-hop sweeps follow
// the reference's periods (t % srpy, t % MStep).
int bd_step_reference(bd_ctx* c, unsigned long t0, int nsteps, int with_hop) {
  if (!c || nsteps < 0) return BD_ERR_ARG;
  noise_blocks_release(c);
  int s;
  bool ext = c->p.flow == BD_FLOW_EXT;
  prof_begin(c, BD_PROF_STEP);
  for (int n = 0; n < nsteps; n++) {
    unsigned long t = t0 + (unsigned long)n;
    c->t = t;
    if (ext) {
      if ((s = bd_transform_coords(c))) return s;
      if ((s = bd_inverse_coords(c))) return s;
    }
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
    if ((s = update_hi(c))) return s;
    if (with_hop) {
      // chargeHop is called every step and sweeps when t % MStep == 0; the
      // ext driver rotates around every call (extensional/src/main14.c:117-121)
      if (ext && (s = bd_transform_coords(c))) return s;
      if ((s = charge_hop(c))) return s;
      if (ext && (s = bd_inverse_coords(c))) return s;
    }
  }
  prof_end(c, BD_PROF_STEP);
  return check(c);
}

}  // extern "C"

namespace bd {
// One draw of the Brownian noise into dst: Philox keyed by the draw count, or
// the reference's sequential ran1/gasdev stream.
int draw_noise(bd_ctx* c, double* dst) {
  c->launches++;
  if (c->p.noise == BD_NOISE_PHILOX) {
    int n = 3 * c->N, pairs = (n + 1) / 2;
    k_noise_philox<<<nblk(pairs, 256), 256, 0, c->stream>>>(dst, n, c->p.philox_seed,
                                                            c->noise_draws++);
  } else {
    k_gasdev_seq<<<1, 32, 0, c->stream>>>(c->rng, dst, 3 * c->N);
  }
  return launch_ok(c);
}

void rotate_coords(bd_ctx* c, int inverse) {
  c->launches++;
  k_rotate<<<nblk(c->N, 256), 256, 0, c->stream>>>(c->lat, c->rx, c->ry, c->N, inverse);
}
}  // namespace bd

namespace bd {
void prof_begin(bd_ctx* c, int slot) {
  if (!c->prof_on || c->capturing) return;
  if (slot == BD_PROF_BLOCK && !c->prof_products) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, c->stream);
  c->prof_ev[slot][0].push_back(e);
}
void prof_end(bd_ctx* c, int slot) {
  if (!c->prof_on || c->capturing) return;
  if (slot == BD_PROF_BLOCK && !c->prof_products) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, c->stream);
  c->prof_ev[slot][1].push_back(e);
}
void prof_clear(bd_ctx* c) {
  for (int s = 0; s < BD_PROF_SLOTS; s++)
    for (int k = 0; k < 2; k++) {
      for (cudaEvent_t e : c->prof_ev[s][k]) cudaEventDestroy(e);
      c->prof_ev[s][k].clear();
    }
}
}  // namespace bd
