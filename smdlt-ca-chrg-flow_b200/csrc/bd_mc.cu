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

using namespace bd;

#define CU(call)                                  \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return BD_ERR_CUDA;    \
  } while (0)

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

int charge_hop(bd_ctx* c) {
  if (c->nch == 0) return BD_OK;
  if (c->t % (unsigned long)c->p.MStep != 0) return BD_OK;
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
