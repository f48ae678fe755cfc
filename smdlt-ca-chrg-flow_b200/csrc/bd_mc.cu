// Charge-hopping Monte Carlo with the reference's sequential sweep semantics.
//
// chargeHop (shear/src/main26.c:1926-2390) visits the charges in order; each
// trial draws one uniform, looks for the first bead (by index, excluding the
// charge's own bead and its index neighbours) within |NID|^2 < 4.41, proposes
// a move from the draw, and accepts with a Metropolis test on
// exp(-barrier - (E_final - E_initial)/2), where E_initial is the
// Debye-Hueckel energy at the start of the sweep (never refreshed) and
// E_final the energy with the trial move.  The reference recomputes E_final
// over all bead pairs for every trial (O(N^2) each); here E_final is carried
// incrementally, E_final = E_current + sum over the other charges of
// U(target, o) - U(source, o), which is the same quantity with a different
// summation order.
//
// The sweep is inherently sequential, so it runs in one CTA of 1024 threads:
// the neighbour scan, the occupancy test and the energy difference are
// block-parallel with fixed-order reductions, and thread 0 owns the ran1
// stream (the same draws, in the same order, as the reference).
#include <math.h>

#include "bd_ctx.cuh"
#include "bd_cell.cuh"

#define CU(call) BD_CU(call)

static const int kHopThreads = 1024;

__device__ __forceinline__ double dh_pair(const Lat& l, double xa, double ya, double za,
                                          double xb, double yb, double zb, double lambda_b,
                                          double kappa_d) {
  double vx, vy, vz;
  min_image(l, subx(xa, xb), subx(ya, yb), subx(za, zb), vx, vy, vz);
  double r = sqrt(rr3(vx, vy, vz));
  return (lambda_b / r) * exp(-kappa_d * r);
}

// Per-charge partial sums of the sweep's starting energy (pairs o > k).
__global__ void k_dh_energy_rows(Lat l, const double4* __restrict__ cq, int nch, double lambda_b,
                                 double kappa_d, double* rowsum) {
  int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (k >= nch) return;
  double4 a = cq[k];
  double s = 0;
  for (int o = k + 1 + lane; o < nch; o += 32) {
    double4 b = cq[o];
    s += a.w * b.w * dh_pair(l, a.x, a.y, a.z, b.x, b.y, b.z, lambda_b, kappa_d);
  }
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) rowsum[k] = s;
}

// Fixed-order block sum (every thread receives the total).
__device__ double block_sum(double v, double* sh) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    double x = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    if (lane == 0) sh[32] = x;
  }
  __syncthreads();
  return sh[32];
}

__global__ void __launch_bounds__(1024) k_charge_hop(
    Lat l, const double* __restrict__ rx, const double* __restrict__ ry,
    const double* __restrict__ rz, int N, int Nb, int nch, int* track, int* old,
    const double* __restrict__ qk_in, const double* __restrict__ rowsum, Ran1* rng,
    double lambda_b, double kappa_d, double barrier, double barrier2, int* log, int* gidx,
    double* gq) {
  // charge sites and values in shared memory, or in global scratch (gidx,
  // gq non-null) when they do not fit
  extern __shared__ unsigned char smem[];
  int* sidx = gidx ? gidx : (int*)smem;
  double* sq = gq ? gq : (double*)(smem + (((size_t)nch * 4 + 15) & ~(size_t)15));
  __shared__ double red[33];
  __shared__ int s_first, s_c2, s_test, s_block, s_acc;
  __shared__ double s_mm;
  int t = threadIdx.x, nt = blockDim.x;
  for (int k = t; k < nch; k += nt) {
    sidx[k] = track[k];
    sq[k] = qk_in[k];
  }
  double e0 = 0;
  for (int k = t; k < nch; k += nt) e0 += rowsum[k];
  double E_init = (nch > 1) ? block_sum(e0, red) : 0.0;
  double E_cur = E_init;
  Ran1 g;
  if (t == 0) g = *rng;
  __syncthreads();
  for (int k = 0; k < nch; k++) {
    if (t == 0) {
      s_mm = (double)ran1_dev(g);
      s_first = 0x7fffffff;
    }
    __syncthreads();
    int c = sidx[k];
    double xc = rx[c], yc = ry[c], zc = rz[c];
    // first bead by index within |NID(c,j)|^2 < 4.41, excluding c-1, c, c+1
    for (int base = 0; base < N; base += nt) {
      int j = base + t;
      bool hit = false;
      if (j < N && j != c && j != c + 1 && j != c - 1) {
        double vx, vy, vz;
        min_image(l, subx(xc, rx[j]), subx(yc, ry[j]), subx(zc, rz[j]), vx, vy, vz);
        hit = rr3(vx, vy, vz) < 4.41;
      }
      if (hit) atomicMin(&s_first, j);
      __syncthreads();
      if (s_first != 0x7fffffff) break;
    }
    if (t == 0) {
      double mm = s_mm;
      int c2, test = 0, sblock;
      if (s_first != 0x7fffffff) {
        if (mm < .33) {
          c2 = c + 1;
          sblock = (c == N - 1 || c % Nb == Nb - 1 || c == Nb - 1);
          test = 1;
        } else if (mm > 0.66) {
          c2 = c - 1;
          sblock = (c2 < 0 || c == 0 || c % Nb == 0);
          test = 1;
        } else {
          c2 = s_first;
          sblock = 0;
          test = 2;
        }
      } else if (mm > .5) {
        c2 = c + 1;
        sblock = (c == N - 1 || c % Nb == Nb - 1 || c == Nb - 1);
      } else {
        c2 = c - 1;
        sblock = (c2 < 0 || c == 0 || c % Nb == 0);
      }
      s_c2 = c2;
      s_test = test;
      s_block = sblock;
    }
    __syncthreads();
    int c2 = s_c2;
    bool occ = false;
    for (int o = t; o < nch; o += nt) occ |= (sidx[o] == c2);
    int blocked = __syncthreads_or(occ ? 1 : 0) || s_block;
    if (blocked) {
      if (t == 0) {
        log[3 * k] = 0;
        log[3 * k + 1] = c2;
        log[3 * k + 2] = 0;  // a blocked trial never sets the move kind
      }
      __syncthreads();
      continue;
    }
    // energy change of moving charge k from c to c2 against all the others
    double x2 = rx[c2], y2 = ry[c2], z2 = rz[c2], de = 0;
    if (nch > 1) {
      double qk = sq[k];
      for (int o = t; o < nch; o += nt) {
        if (o == k) continue;
        int b = sidx[o];
        double xb = rx[b], yb = ry[b], zb = rz[b];
        de += qk * sq[o] *
              (dh_pair(l, x2, y2, z2, xb, yb, zb, lambda_b, kappa_d) -
               dh_pair(l, xc, yc, zc, xb, yb, zb, lambda_b, kappa_d));
      }
      de = block_sum(de, red);
    }
    double E_fin = (nch > 1) ? E_cur + de : 0.0;
    if (t == 0) {
      double bar = (s_test == 2) ? barrier2 : barrier;
      double x = exp((-bar - 0.5 * (E_fin - E_init)));
      int acc;
      if (1 <= x)
        acc = 1;
      else
        acc = ((double)ran1_dev(g) <= x);
      old[k] = c;
      if (acc) sidx[k] = c2;
      log[3 * k] = acc ? 1 : 2;
      log[3 * k + 1] = c2;
      log[3 * k + 2] = s_test;
      s_acc = acc;
    }
    __syncthreads();
    if (s_acc) E_cur = E_fin;
  }
  __syncthreads();
  for (int k = t; k < nch; k += nt) track[k] = sidx[k];
  if (t == 0) *rng = g;
}

__global__ void k_charge_values(const double* __restrict__ q, const int* __restrict__ track,
                                int nch, double* qk) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nch) qk[k] = q[track[k]];
}

__global__ void k_clear_charges(int* flags, double* q, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) {
    flags[i] = 0;
    q[i] = 0.0;
  }
}

__global__ void k_scatter_charges(const int* __restrict__ track, const double* __restrict__ qk,
                                  int nch, int* flags, double* q) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nch) {
    flags[track[k]] = 1;
    q[track[k]] = qk[k];
  }
}

__global__ void k_gather_charges_mc(const double* __restrict__ rx, const double* __restrict__ ry,
                                    const double* __restrict__ rz, const double* __restrict__ q,
                                    const int* __restrict__ track, int nch, double4* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nch) {
    int i = track[k];
    out[k] = make_double4(rx[i], ry[i], rz[i], q[i]);
  }
}

namespace bd {

int charge_hop_parallel(bd_ctx* c);

int charge_hop(bd_ctx* c) {
  if (c->nch == 0) return BD_OK;
  if (c->t % (unsigned long)c->p.MStep != 0) return BD_OK;
  if (c->p.hop == BD_HOP_PARALLEL) return charge_hop_parallel(c);
  int nch = c->nch, N = c->N;
  size_t smem = (((size_t)nch * 4 + 15) & ~(size_t)15) + 8 * (size_t)nch;
  // scratch in dE (64 N doubles): [0, 4 nch) gathered (x,y,z,q); then row
  // sums; then qk; then, for sweeps whose charges do not fit in shared
  // memory, the working copies of the charge values and sites
  double4* cq = (double4*)c->dE;
  double* rowsum = c->dE + 4 * (size_t)nch;
  double* qk = rowsum + nch;
  double* gq = nullptr;
  int* gidx = nullptr;
  if (smem > 200 * 1024) {
    gq = qk + nch;
    gidx = (int*)(gq + nch);
    smem = 0;
  }
  Lat l = c->lat;
  int treal = (int)(c->t % (unsigned long)c->tp);
  l.treal = treal;
  l.delx = c->p.edot * treal * c->p.dt;
  c->launches++;
  k_charge_values<<<(nch + 255) / 256, 256, 0, c->stream>>>(c->q, c->track, nch, qk);
  c->launches++;
  k_gather_charges_mc<<<(nch + 255) / 256, 256, 0, c->stream>>>(c->rx, c->ry, c->rz, c->q, c->track,
                                                             nch, cq);
  c->launches++;
  k_dh_energy_rows<<<(nch * 32 + 255) / 256, 256, 0, c->stream>>>(l, cq, nch, c->p.lambda_b,
                                                                   c->kappa_d, rowsum);
  cudaFuncSetAttribute(k_charge_hop, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  prof_begin(c, BD_PROF_HOP);
  c->launches++;
  k_charge_hop<<<1, kHopThreads, smem, c->stream>>>(l, c->rx, c->ry, c->rz, N, c->Nb, nch,
                                                    c->track, c->old, qk, rowsum, c->rng,
                                                    c->p.lambda_b, c->kappa_d, c->p.barrier,
                                                    c->p.barrier2, c->hoplog, gidx, gq);
  prof_end(c, BD_PROF_HOP);
  c->launches++;
  k_clear_charges<<<(N + 255) / 256, 256, 0, c->stream>>>(c->cflags, c->q, N);
  c->launches++;
  k_scatter_charges<<<(nch + 255) / 256, 256, 0, c->stream>>>(c->track, qk, nch, c->cflags, c->q);
  return launch_ok(c);
}

}  // namespace bd

// ---------------------------------------------------------------------------
// Parallel sweep on independent sets (no reference counterpart).
//
// The charges are binned into cells of the Gauss-reduced cell at least R
// wide (R = hop_radius, default 3 Debye lengths), with an even number of
// cells per direction; the parity of the three cell indices gives eight
// colours, and cells of one colour are at least R apart.  A sweep runs the
// eight colours in turn; within a colour every cell is one CTA that visits its
// charges in index order, each exactly once.  A trial follows the reference's
// proposal rules (partner search, chain ends, occupancy, the two barriers) and
// accepts with min(1, exp(-barrier - dE/2)) (the reference's factor, without
// its stale starting energy), dE the energy change of the move against every
// other charge: with Debye-Hueckel electrostatics the reference's screened
// pair energy; with Ewald electrostatics the unscreened energy the forces
// use, in FP64:
//   dE = q sum_o q_o [erfc(beta r)/r]_a^b   (real space, within the cutoff)
//      + q [Phi0(b) - Phi0(a)]               (mesh reciprocal potential of all
//                                              charges at the colour's start)
//      - q^2 [G(b - a) - G(0)]               (the moved charge's own term)
//      + q sum_j q_j [G(b-b_j) - G(b-a_j) - G(a-b_j) + G(a-a_j)]
//                                            (charges of the own cell moved
//                                              earlier in the colour, a_j -> b_j)
// with G(r) = lambda_B erf(beta r)/r + r^T Q r the reciprocal pair term near
// the origin (Q the quadratic form of its periodic remainder, from the
// lattice's k-space sum, (2 pi lambda_B / 3 V) I for a cubic cell; the rest is
// O(r^4 / L^5); G(0) = 2 beta lambda_B/sqrt(pi)).  The other
// charges are taken at their sites at the start of the colour, those of the
// own cell at their current sites; a move therefore ignores only the change
// of its interaction with charges moved in the same colour in other cells,
// which are at least R away: the second difference of the pair energy over
// both hops, |dU| <= 2 lambda_B d^2 / R^3 per pair (hop distance d <= 2.1),
// 0.005 kT at R = 15 for the bare Coulomb energy, less when screened.  The
// draws are Philox4x32-10
// counters (charge, sweep, purpose) under philox_seed, so a sweep does not
// depend on the launch order.  The partner is the first bead of the charge's
// Verlet row (sorted ascending, radius 6 > 2.1 plus twice the skin) within
// |NID|^2 < 4.41, as the reference's scan over all beads finds it.

namespace {

constexpr int kHopCellCap = 8192;

struct HGeom {
  int n[3];
};

__device__ __forceinline__ double philox_u01(int k, unsigned long long sweep, int tag,
                                             unsigned long long seed) {
  uint4 c = make_uint4((uint32_t)k, (uint32_t)sweep, (uint32_t)(sweep >> 32),
                       0x4d430000u | (uint32_t)tag);
  uint4 x = philox4x32_10(c, make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
  return (double)(((unsigned long long)(x.x >> 5) << 26) | (x.y >> 6)) *
         (1.0 / 9007199254740992.0);
}

__global__ void k_hop_cells(Cell cell, HGeom g, const double* __restrict__ rx,
                            const double* __restrict__ ry, const double* __restrict__ rz,
                            const int* __restrict__ track, int nch, double cr, double sr,
                            int* cell_of, int* count) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nch) return;
  int b = track[k];
  double x = rx[b] * cr - ry[b] * sr, y = rx[b] * sr + ry[b] * cr, s[3];
  frac_of(cell, x, y, rz[b], s);
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

__global__ void k_hop_scan(int ncell, int* count, int* start) {
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
    b += count[c];
    count[c] = 0;
  }
  if (t == nt - 1) start[ncell] = part[t];
}

// One thread per cell lists its charges in increasing index (a fixed order).
__global__ void k_hop_fill(const int* __restrict__ cell_of, const int* __restrict__ start,
                           int ncell, int nch, int* idx) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int p = start[c];
  for (int k = 0; k < nch; k++)
    if (cell_of[k] == c) idx[p++] = k;
}

// The Ewald energy terms of a trial (P > 0): the lab-frame reduced cell, the
// stored-frame rotation, the reciprocal potential on the mesh, the split.
struct HopEwald {
  Cell cell;
  double cr, sr;
  const double* phi;
  const double* Q;  // quadratic form of the reciprocal pair term's periodic remainder
  int K;
  double beta, rc2, lambda_b;
};

__device__ __forceinline__ void hop_lab(const HopEwald& ew, double x, double y, double& lx,
                                        double& ly) {
  lx = x * ew.cr - y * ew.sr;
  ly = x * ew.sr + y * ew.cr;
}

// Minimum image of d in the reduced cell.
__device__ __forceinline__ void hop_minimg(const HopEwald& ew, double& dx, double& dy,
                                           double& dz) {
  double s[3];
  frac_of(ew.cell, dx, dy, dz, s);
  for (int d = 0; d < 3; d++) s[d] -= rint(s[d]);
  const double* H = ew.cell.H;
  dx = H[0] * s[0] + H[1] * s[1] + H[2] * s[2];
  dy = H[3] * s[0] + H[4] * s[1] + H[5] * s[2];
  dz = H[6] * s[0] + H[7] * s[1] + H[8] * s[2];
}

__device__ __forceinline__ double hop_rr(const HopEwald& ew, double dx, double dy, double dz) {
  hop_minimg(ew, dx, dy, dz);
  return dx * dx + dy * dy + dz * dz;
}

// Real-space pair term lambda_B erfc(beta r)/r within the cutoff.
__device__ __forceinline__ double hop_real(const HopEwald& ew, double dx, double dy, double dz) {
  double rr = hop_rr(ew, dx, dy, dz);
  if (rr >= ew.rc2) return 0.0;
  double r = sqrt(rr);
  return ew.lambda_b * erfc(ew.beta * r) / r;
}

// Reciprocal pair term near the origin, G(r) = lambda_B erf(beta r)/r + r^T Q r
// (the Gaussian-screened part and the quadratic term of the periodic remainder;
// its constant cancels in every difference, its O(r^4 / L^5) rest is left
// out); G(0) = 2 beta lambda_B / sqrt(pi).
__device__ __forceinline__ double hop_recip(const HopEwald& ew, double dx, double dy, double dz) {
  hop_minimg(ew, dx, dy, dz);
  double rr = dx * dx + dy * dy + dz * dz, r = sqrt(rr);
  if (r <= 1e-12) return ew.lambda_b * 2.0 * ew.beta / sqrt(M_PI);
  const double* Q = ew.Q;
  double quad = Q[0] * dx * dx + Q[3] * dy * dy + Q[5] * dz * dz +
                2.0 * (Q[1] * dx * dy + Q[2] * dx * dz + Q[4] * dy * dz);
  return ew.lambda_b * erf(ew.beta * r) / r + quad;
}

// P = 0: Debye-Hueckel trial energies; P = 4, 6, 8: Ewald, B-spline order P.
template <int P>
__global__ void __launch_bounds__(1024) k_hop_colour(
    Lat l, HGeom g, int colour, const double* __restrict__ rx, const double* __restrict__ ry,
    const double* __restrict__ rz, int N, int Nb, int nch, const int* __restrict__ start,
    const int* __restrict__ idx, const int* __restrict__ cell_of,
    const int* __restrict__ site0, const double* __restrict__ qk, int* track, int* old,
    int* flags, const int* __restrict__ nb_count, const int* __restrict__ nb_rows, int maxnb,
    double lambda_b, double kappa_d, double barrier, double barrier2, unsigned long long seed,
    unsigned long long sweep, int* log, double* hop_de, HopEwald ew) {
  int cell = blockIdx.x;
  int cz = cell % g.n[2], cy = (cell / g.n[2]) % g.n[1], cx = cell / (g.n[1] * g.n[2]);
  int col = ((g.n[0] > 1 ? cx & 1 : 0) << 2) | ((g.n[1] > 1 ? cy & 1 : 0) << 1) |
            (g.n[2] > 1 ? cz & 1 : 0);
  if (col != colour) return;
  __shared__ double red[33];
  __shared__ int s_first, s_c2, s_test, s_block;
  __shared__ double s_w[2][3][P > 0 ? P : 1];  // Ewald: spline weights of both sites
  __shared__ int s_base[2][3];
  int t = threadIdx.x, nt = blockDim.x;
  for (int q = start[cell]; q < start[cell + 1]; q++) {
    int k = idx[q];
    int c = track[k];
    if (t == 0) s_first = 0x7fffffff;
    __syncthreads();
    double xc = rx[c], yc = ry[c], zc = rz[c];
    int nr = min(nb_count[c], maxnb);
    for (int e = t; e < nr; e += nt) {
      int j = nb_rows[(size_t)c * maxnb + e];
      if (j == c || j == c + 1 || j == c - 1) continue;
      double vx, vy, vz;
      min_image(l, subx(xc, rx[j]), subx(yc, ry[j]), subx(zc, rz[j]), vx, vy, vz);
      if (rr3(vx, vy, vz) < 4.41) atomicMin(&s_first, j);
    }
    __syncthreads();
    if (t == 0) {
      double mm = philox_u01(k, sweep, 0, seed);
      int c2, test = 0, sblock;
      if (s_first != 0x7fffffff) {
        if (mm < .33) {
          c2 = c + 1;
          sblock = (c == N - 1 || c % Nb == Nb - 1 || c == Nb - 1);
          test = 1;
        } else if (mm > 0.66) {
          c2 = c - 1;
          sblock = (c2 < 0 || c == 0 || c % Nb == 0);
          test = 1;
        } else {
          c2 = s_first;
          sblock = 0;
          test = 2;
        }
      } else if (mm > .5) {
        c2 = c + 1;
        sblock = (c == N - 1 || c % Nb == Nb - 1 || c == Nb - 1);
      } else {
        c2 = c - 1;
        sblock = (c2 < 0 || c == 0 || c % Nb == 0);
      }
      if (!sblock && flags[c2]) sblock = 1;  // occupied target
      s_c2 = c2;
      s_test = test;
      s_block = sblock;
    }
    __syncthreads();
    int c2 = s_c2;
    if (s_block) {
      if (t == 0) {
        log[3 * k] = 0;
        log[3 * k + 1] = c2;
        log[3 * k + 2] = 0;
        hop_de[k] = __longlong_as_double(0x7ff8000000000000LL);  // no trial energy
      }
      __syncthreads();
      continue;
    }
    double x2 = rx[c2], y2 = ry[c2], z2 = rz[c2], de = 0, qme = qk[k];
    if constexpr (P == 0) {
      for (int o = t; o < nch; o += nt) {
        if (o == k) continue;
        int b = cell_of[o] == cell ? track[o] : site0[o];
        double xb = rx[b], yb = ry[b], zb = rz[b];
        de += qme * qk[o] *
              (dh_pair(l, x2, y2, z2, xb, yb, zb, lambda_b, kappa_d) -
               dh_pair(l, xc, yc, zc, xb, yb, zb, lambda_b, kappa_d));
      }
    } else {
      double ax, ay, bx, by, az = zc, bz = z2;
      hop_lab(ew, xc, yc, ax, ay);
      hop_lab(ew, x2, y2, bx, by);
      // real space against every other charge
      for (int o = t; o < nch; o += nt) {
        if (o == k) continue;
        int b = cell_of[o] == cell ? track[o] : site0[o];
        double ox, oy, oz = rz[b];
        hop_lab(ew, rx[b], ry[b], ox, oy);
        de += qme * qk[o] *
              (hop_real(ew, bx - ox, by - oy, bz - oz) - hop_real(ew, ax - ox, ay - oy, az - oz));
      }
      // spline weights of the two sites (thread 3 pt + d: site pt, direction d)
      if (t < 6) {
        int pt = t / 3, d = t % 3;
        double sv[3];
        frac_of(ew.cell, pt ? bx : ax, pt ? by : ay, pt ? bz : az, sv);
        double u = (sv[d] - floor(sv[d])) * ew.K;
        if (!(u >= 0.0 && u <= (double)ew.K)) u = 0.0;
        int fl = (int)floor(u);
        double f = u - fl;
        if (fl >= ew.K) fl -= ew.K;
        s_base[pt][d] = fl;
        double wv[P];
        bspline_t<P>(f, wv);
#pragma unroll
        for (int a = 0; a < P; a++) s_w[pt][d][a] = wv[a];
      }
      __syncthreads();
      // q [Phi0(b) - Phi0(a)] from the mesh
      constexpr int P3 = P * P * P;
      const int K = ew.K;
      for (int e = t; e < 2 * P3; e += nt) {
        int pt = e / P3, m = e - pt * P3;
        int cc = m % P, bb = (m / P) % P, aa = m / (P * P);
        int g0 = s_base[pt][0] - aa, g1 = s_base[pt][1] - bb, g2 = s_base[pt][2] - cc;
        g0 += g0 < 0 ? K : 0;
        g1 += g1 < 0 ? K : 0;
        g2 += g2 < 0 ? K : 0;
        double v = s_w[pt][0][aa] * s_w[pt][1][bb] * s_w[pt][2][cc] *
                   ew.phi[((size_t)g0 * K + g1) * K + g2];
        de += pt ? qme * v : -qme * v;
      }
      // the moved charge's own reciprocal term
      if (t == 0)
        de -= qme * qme * (hop_recip(ew, bx - ax, by - ay, bz - az) - hop_recip(ew, 0, 0, 0));
      // charges of this cell that moved earlier in this colour (a_j -> b_j)
      for (int q2 = start[cell] + t; q2 < q; q2 += nt) {
        int j = idx[q2];
        if (log[3 * j] != 1) continue;
        int aj = old[j], bj = track[j];
        double ajx, ajy, bjx, bjy, ajz = rz[aj], bjz = rz[bj];
        hop_lab(ew, rx[aj], ry[aj], ajx, ajy);
        hop_lab(ew, rx[bj], ry[bj], bjx, bjy);
        de += qme * qk[j] *
              (hop_recip(ew, bx - bjx, by - bjy, bz - bjz) - hop_recip(ew, bx - ajx, by - ajy, bz - ajz) -
               hop_recip(ew, ax - bjx, ay - bjy, az - bjz) + hop_recip(ew, ax - ajx, ay - ajy, az - ajz));
      }
    }
    de = block_sum(de, red);
    if (t == 0) {
      hop_de[k] = de;
      double bar = (s_test == 2) ? barrier2 : barrier;
      double x = exp(-bar - 0.5 * de);
      int acc = (1 <= x) ? 1 : (philox_u01(k, sweep, 1, seed) <= x);
      old[k] = c;
      if (acc) {
        flags[c] = 0;
        flags[c2] = 1;
        track[k] = c2;
      }
      log[3 * k] = acc ? 1 : 2;
      log[3 * k + 1] = c2;
      log[3 * k + 2] = s_test;
    }
    __syncthreads();
  }
}

// (x, y, z, q) of each charge at its current site, in track order.
__global__ void k_gather_sites(const double* __restrict__ rx, const double* __restrict__ ry,
                               const double* __restrict__ rz, const int* __restrict__ track,
                               const double* __restrict__ qk, int nch, double4* cq) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nch) return;
  int b = track[k];
  cq[k] = make_double4(rx[b], ry[b], rz[b], qk[k]);
}

}  // namespace

namespace bd {

int charge_hop_parallel(bd_ctx* c) {
  int nch = c->nch, N = c->N;
  if (!c->hop_cells) {
    CU(cudaMalloc(&c->hop_cells, 4 * ((size_t)3 * N + 2 * (kHopCellCap + 1))));
    c->bytes += 4 * ((size_t)3 * N + 2 * (kHopCellCap + 1));
    CU(cudaMemsetAsync(c->hop_cells, 0, 4 * ((size_t)3 * N + 2 * (kHopCellCap + 1)), c->stream));
  }
  if (!c->hop_de) {
    CU(cudaMalloc(&c->hop_de, 8 * (size_t)N));
    c->bytes += 8 * (size_t)N;
    CU(cudaMemsetAsync(c->hop_de, 0, 8 * (size_t)N, c->stream));
  }
  int* cell_of = c->hop_cells;
  int* idx = cell_of + N;
  int* site0 = idx + N;
  int* count = site0 + N;
  int* start = count + kHopCellCap + 1;
  Lat l = c->lat;
  int treal = (int)(c->t % (unsigned long)c->tp);
  l.treal = treal;
  l.delx = c->p.edot * treal * c->p.dt;
  Cell cell = make_cell(l);
  double cr = 1.0, sr = 0.0;
  if (l.flow == BD_FLOW_EXT) {
    cr = l.cth;
    sr = l.sth;
  }
  double R = c->hop_R;
  HGeom g;
  for (int j = 0; j < 3; j++) {
    double a[3][3];
    for (int q = 0; q < 3; q++)
      for (int d = 0; d < 3; d++) a[q][d] = cell.H[d * 3 + q];
    const double* u = a[(j + 1) % 3];
    const double* v = a[(j + 2) % 3];
    double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2],
           cz = u[0] * v[1] - u[1] * v[0];
    int n = (int)floor(cell.V / sqrt(cx * cx + cy * cy + cz * cz) / R);
    g.n[j] = n >= 2 ? n - (n & 1) : 1;
  }
  while ((long)g.n[0] * g.n[1] * g.n[2] > kHopCellCap) {
    int d = g.n[0] >= g.n[1] && g.n[0] >= g.n[2] ? 0 : (g.n[1] >= g.n[2] ? 1 : 2);
    g.n[d] -= 2;
  }
  int ncell = g.n[0] * g.n[1] * g.n[2];
  double* qk = c->dE + 6 * (size_t)nch;  // charge values in track order
  c->launches += 4;
  k_charge_values<<<(nch + 255) / 256, 256, 0, c->stream>>>(c->q, c->track, nch, qk);
  k_hop_cells<<<(nch + 255) / 256, 256, 0, c->stream>>>(cell, g, c->rx, c->ry, c->rz, c->track,
                                                        nch, cr, sr, cell_of, count);
  k_hop_scan<<<1, 1024, 0, c->stream>>>(ncell, count, start);
  k_hop_fill<<<(ncell + 127) / 128, 128, 0, c->stream>>>(cell_of, start, ncell, nch, idx);
  unsigned long long sweep = c->hop_sweeps++;
  bool ewald = c->p.coulomb == BD_COULOMB_EWALD;
  HopEwald ew = {};
  int P = 0;
  if (ewald) {
    ew.cell = cell;
    ew.cr = cr;
    ew.sr = sr;
    ew.K = c->pmeK;
    ew.beta = c->cw_beta;
    ew.rc2 = c->cw_rc * c->cw_rc;
    ew.lambda_b = c->p.lambda_b;
    P = c->pme_p == 4 || c->pme_p == 6 ? c->pme_p : 8;
    // dE scratch (64 N doubles): [0, 4 nch) the gathered sites, [6 nch, 7 nch)
    // the charge values, then the six entries of Q
    double* Q6 = c->dE + 7 * (size_t)nch;
    int s;
    if ((s = coulomb_quadform(c, l, Q6)) != BD_OK) return s;
    ew.Q = Q6;
  }
  double4* cq = (double4*)c->dE;  // [0, 4 nch): charges at their sites (Ewald mesh)
  prof_begin(c, BD_PROF_HOP);
  for (int colour = 0; colour < 8; colour++) {
    CU(cudaMemcpyAsync(site0, c->track, 4 * (size_t)nch, cudaMemcpyDeviceToDevice, c->stream));
    if (ewald) {
      // the reciprocal potential of the charges at the colour's start
      c->launches++;
      k_gather_sites<<<(nch + 255) / 256, 256, 0, c->stream>>>(c->rx, c->ry, c->rz, c->track,
                                                              qk, nch, cq);
      int s;
      if ((s = coulomb_mesh_potential(c, l, cq)) != BD_OK) return s;
      ew.phi = c->cw_grid;
    }
    c->launches++;
    // only the cells of one colour work in a launch (ncell / 8 CTAs): 1024
    // threads share each trial's energy sum over the charges
#define HOP_COLOUR(P_)                                                                         \
  k_hop_colour<P_><<<ncell, 1024, 0, c->stream>>>(                                             \
      l, g, colour, c->rx, c->ry, c->rz, N, c->Nb, nch, start, idx, cell_of, site0, qk,        \
      c->track, c->old, c->cflags, c->nb_count, c->nb_rows, c->maxnb, c->p.lambda_b,           \
      c->kappa_d, c->p.barrier, c->p.barrier2, c->p.philox_seed, sweep, c->hoplog, c->hop_de, ew)
    switch (P) {
      case 0: HOP_COLOUR(0); break;
      case 4: HOP_COLOUR(4); break;
      case 6: HOP_COLOUR(6); break;
      default: HOP_COLOUR(8);
    }
#undef HOP_COLOUR
  }
  prof_end(c, BD_PROF_HOP);
  c->launches += 2;
  k_clear_charges<<<(N + 255) / 256, 256, 0, c->stream>>>(c->cflags, c->q, N);
  k_scatter_charges<<<(nch + 255) / 256, 256, 0, c->stream>>>(c->track, qk, nch, c->cflags, c->q);
  return launch_ok(c);
}

}  // namespace bd

extern "C" int bd_download_hop_energies(bd_ctx* c, double* de) {
  if (!c || (c->nch > 0 && !de)) return BD_ERR_ARG;
  if (c->nch == 0) return BD_OK;
  if (!c->hop_de) return BD_ERR_STATE;
  CU(cudaMemcpyAsync(de, c->hop_de, 8 * (size_t)c->nch, cudaMemcpyDeviceToHost, c->stream));
  return check(c);
}
