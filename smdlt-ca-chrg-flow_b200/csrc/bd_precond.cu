// Block-diagonal preconditioners for the Lanczos square root.
//
// No counterpart in the reference (its Brownian displacement is the CA-TEA
// approximation of updateHI, shear/src/main26.c:745-857).  With an
// invertible block-diagonal G the Krylov iteration runs on A = G M G^T,
// whose spectrum is narrower than that of M when G approximates M^(-1/2), and
// the displacement is y = G^(-1) sqrt(A) z: y has covariance
// G^(-1) A G^(-T) = M, so it is a valid Brownian sample (a different square
// root of M than sqrt(M) z; Ando, Chow and Skolnick, J. Chem. Phys. 137,
// 064106 (2012), section II.C).  Blocks cover S consecutive beads:
//  * segment blocks: S beads of one chain, G = L^(-1) with L L^T the
//    Cholesky factorisation of the free-space Rotne-Prager-Yamakawa mobility
//    of the segment (minimum-image pair vectors, overlap form for r < 2);
//  * bead blocks (S = 1): 3 x 3 blocks supplied by the caller or predicted
//    by the message-passing network of bd_mpnn.cu.
// Blocks are rebuilt with the mobility (same configuration) and stored as
// dense row-major 3S x 3S matrices G_b and G_b^(-1), FP64.
#include <math.h>

#include <algorithm>
#include <vector>

#include "bd_ctx.cuh"

using namespace bd;

#define CU(call) BD_CU(call)

// Free-space RPY block for the pair vector d (unit bead radius):
// (3/4r + 1/2r^3) I + (3/4r - 3/2r^3) d d^T/r^2 for r >= 2,
// (1 - 9r/32) I + (3r/32) d d^T/r^2 below.
__device__ __forceinline__ void rpy_free(double dx, double dy, double dz, double* o) {
  double rr = dx * dx + dy * dy + dz * dz, r = sqrt(rr);
  double t1, t2;
  if (r >= 2.0) {
    t1 = 0.75 / r + 0.5 / (r * rr);
    t2 = 0.75 / r - 1.5 / (r * rr);
  } else {
    t1 = 1.0 - 0.28125 * r;
    t2 = 0.09375 * r;
  }
  double d[3] = {dx, dy, dz};
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 3; q++) o[3 * p + q] = (p == q ? t1 : 0.0) + (rr > 0 ? t2 * d[p] * d[q] / rr : 0.0);
}

// One CTA per segment: assemble the 3S x 3S segment mobility, Cholesky in
// shared memory, invert the factor; G = L^(-1), Gi = L.  A non-positive pivot
// (not expected: the RPY tensor is positive definite) leaves the identity
// and counts the block in *bad.
__global__ void __launch_bounds__(128) k_seg_blocks(Lat l, const double* __restrict__ rx,
                                                    const double* __restrict__ ry,
                                                    const double* __restrict__ rz, int S,
                                                    double* G, double* Gi, int* bad) {
  extern __shared__ double sm[];
  int n = 3 * S, b = blockIdx.x, t = threadIdx.x;
  double* A = sm;           // n x n, factor in the lower triangle
  double* X = sm + n * n;   // n x n, inverse factor
  __shared__ int fail;
  if (t == 0) fail = 0;
  for (int e = t; e < S * S; e += blockDim.x) {
    int a = e / S, c = e % S;
    double blk[9];
    if (a == c) {
      for (int q = 0; q < 9; q++) blk[q] = (q % 4 == 0) ? 1.0 : 0.0;
    } else {
      double dx, dy, dz;
      nid(l, rx, ry, rz, b * S + a, b * S + c, dx, dy, dz);
      rpy_free(dx, dy, dz, blk);
    }
    for (int p = 0; p < 3; p++)
      for (int q = 0; q < 3; q++) A[(3 * a + p) * n + 3 * c + q] = blk[3 * p + q];
  }
  __syncthreads();
  for (int k = 0; k < n; k++) {
    if (t == 0) {
      double piv = A[k * n + k];
      if (!(piv > 0.0)) {
        fail = 1;
        piv = 1.0;
      }
      A[k * n + k] = sqrt(piv);
    }
    __syncthreads();
    double dk = A[k * n + k];
    for (int i = k + 1 + t; i < n; i += blockDim.x) A[i * n + k] /= dk;
    __syncthreads();
    int m = n - k - 1;
    for (int e = t; e < m * m; e += blockDim.x) {
      int i = k + 1 + e / m, j = k + 1 + e % m;
      if (j <= i) A[i * n + j] -= A[i * n + k] * A[j * n + k];
    }
    __syncthreads();
  }
  // X = L^(-1): column j by forward substitution (one thread per column)
  for (int j = t; j < n; j += blockDim.x) {
    for (int i = 0; i < n; i++) {
      double s = (i == j) ? 1.0 : 0.0;
      for (int k = j; k < i; k++) s -= A[i * n + k] * X[k * n + j];
      X[i * n + j] = i < j ? 0.0 : s / A[i * n + i];
    }
  }
  __syncthreads();
  double* Gb = G + (size_t)b * n * n;
  double* Gib = Gi + (size_t)b * n * n;
  for (int e = t; e < n * n; e += blockDim.x) {
    int i = e / n, j = e % n;
    if (fail) {
      Gb[e] = Gib[e] = (i == j) ? 1.0 : 0.0;
    } else {
      Gb[e] = j <= i ? X[e] : 0.0;
      Gib[e] = j <= i ? A[e] : 0.0;
    }
  }
  if (t == 0 && fail) atomicAdd(bad, 1);
}

// y_r = op(B_b) x_r for every block b and right-hand side r < k; x, y in the
// Lanczos layout (component-major, 3 x NTp, right-hand sides xs / ys apart).
// One CTA per block: B_b (stored transposed for op = B, as is for op = B^T,
// so that the threads of consecutive rows read consecutive words) and the
// block's slices of the k inputs are staged in shared memory once, so each
// block matrix is read from memory once for all right-hand sides.  Each output
// sums its row in a fixed order.
__global__ void __launch_bounds__(128) k_block_apply(const double* __restrict__ Bm, int S,
                                                     int trans, int k,
                                                     const double* __restrict__ x, size_t xs,
                                                     double* __restrict__ y, size_t ys, int NTp) {
  extern __shared__ double sm[];
  int n = 3 * S, b = blockIdx.x;
  double* Bs = sm;          // Bs[q * n + i] = op(B_b)[i][q]
  double* xv = sm + n * n;  // k x n inputs
  const double* Bb = Bm + (size_t)b * n * n;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x)
    Bs[trans ? e : (e % n) * n + e / n] = Bb[e];
  for (int e = threadIdx.x; e < k * n; e += blockDim.x) {
    int r = e / n, q = e % n;
    xv[e] = x[(size_t)r * xs + (size_t)(q % 3) * NTp + (size_t)b * S + q / 3];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < k * n; e += blockDim.x) {
    int r = e / n, i = e % n;
    const double* xr = xv + r * n;
    double s = 0;
    for (int q = 0; q < n; q++) s += Bs[q * n + i] * xr[q];
    y[(size_t)r * ys + (size_t)(i % 3) * NTp + (size_t)b * S + i / 3] = s;
  }
}

// 3 x 3 bead blocks: one thread per bead.
__global__ void k_bead_apply(const double* __restrict__ Bm, int N, int trans,
                             const double* __restrict__ x, size_t xs, double* __restrict__ y,
                             size_t ys, int NTp) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  x += (size_t)blockIdx.y * xs;  // right-hand side blockIdx.y
  y += (size_t)blockIdx.y * ys;
  const double* B = Bm + 9 * (size_t)i;
  double v0 = x[i], v1 = x[NTp + i], v2 = x[2 * (size_t)NTp + i];
  for (int p = 0; p < 3; p++) {
    double s = trans ? B[p] * v0 + B[3 + p] * v1 + B[6 + p] * v2
                     : B[3 * p] * v0 + B[3 * p + 1] * v1 + B[3 * p + 2] * v2;
    y[(size_t)p * NTp + i] = s;
  }
}

// Inverse of symmetric-or-not 3 x 3 bead blocks (adjugate / determinant);
// a block with |det| below 1e-12 |B|^3 is replaced by the identity in both.
__global__ void k_bead_invert(double* G, double* Gi, int N, int* bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double* B = G + 9 * (size_t)i;
  double* O = Gi + 9 * (size_t)i;
  double a = B[0], b = B[1], c = B[2], d = B[3], e = B[4], f = B[5], g = B[6], h = B[7],
         k = B[8];
  double A0 = e * k - f * h, A1 = c * h - b * k, A2 = b * f - c * e;
  double det = a * A0 + d * A1 + g * A2;
  double nrm = 0;
  for (int q = 0; q < 9; q++) nrm = fmax(nrm, fabs(B[q]));
  if (!(fabs(det) > 1e-12 * nrm * nrm * nrm)) {
    for (int q = 0; q < 9; q++) B[q] = O[q] = (q % 4 == 0) ? 1.0 : 0.0;
    atomicAdd(bad, 1);
    return;
  }
  double id = 1.0 / det;
  O[0] = A0 * id;
  O[1] = A1 * id;
  O[2] = A2 * id;
  O[3] = (f * g - d * k) * id;
  O[4] = (a * k - c * g) * id;
  O[5] = (c * d - a * f) * id;
  O[6] = (d * h - e * g) * id;
  O[7] = (b * g - a * h) * id;
  O[8] = (a * e - b * d) * id;
}

// Learned bead blocks on top of segment blocks: G'_b = B_b G_b and
// G'_b^-1 = G_b^-1 B_b^-1 with B_b the block diagonal of the segment's bead
// blocks (9 per bead in Bb, inverses in Bi).  One thread per matrix entry.
__global__ void k_combine_blocks(const double* __restrict__ Bb, const double* __restrict__ Bi,
                                 int S, int nblk, double* G, double* Gi) {
  int n = 3 * S;
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)nblk * n) return;
  // one thread per (block, column): the column of G'_b and the row of G'^-1_b
  int b = (int)(e / n), j = (int)(e % n);
  double* Gb = G + (size_t)b * n * n;
  double* Gib = Gi + (size_t)b * n * n;
  double col[3 * BD_PRECOND_MAX_SEGMENT], row[3 * BD_PRECOND_MAX_SEGMENT];
  for (int i = 0; i < n; i++) {
    col[i] = Gb[(size_t)i * n + j];
    row[i] = Gib[(size_t)j * n + i];
  }
  for (int a = 0; a < S; a++) {
    const double* B = Bb + 9 * ((size_t)b * S + a);
    const double* Binv = Bi + 9 * ((size_t)b * S + a);
    for (int p = 0; p < 3; p++) {
      Gb[(size_t)(3 * a + p) * n + j] =
          B[3 * p] * col[3 * a] + B[3 * p + 1] * col[3 * a + 1] + B[3 * p + 2] * col[3 * a + 2];
      Gib[(size_t)j * n + 3 * a + p] = row[3 * a] * Binv[p] + row[3 * a + 1] * Binv[3 + p] +
                                      row[3 * a + 2] * Binv[6 + p];
    }
  }
}

namespace bd {

static int pre_alloc(bd_ctx* c, int S) {
  size_t nb = (size_t)c->N / S, n = 3 * (size_t)S;
  size_t need = nb * n * n;
  if (c->pre_G && c->pre_cap >= need) return BD_OK;
  lanczos_graphs_reset(c);  // captured products hold the block pointers
  if (c->pre_G) cudaFree(c->pre_G);
  if (c->pre_Gi) cudaFree(c->pre_Gi);
  c->pre_G = c->pre_Gi = nullptr;
  CU(cudaMalloc(&c->pre_G, 8 * need));
  CU(cudaMalloc(&c->pre_Gi, 8 * need));
  if (!c->pre_bad) CU(cudaMalloc(&c->pre_bad, 16));
  CU(cudaMemsetAsync(c->pre_bad, 0, 16, c->stream));
  c->pre_cap = need;
  c->bytes += 16 * need;
  return BD_OK;
}

// Rebuild the preconditioner blocks for the configuration of the mobility
// build (positions in the stored frame, lattice l).
int precond_build(bd_ctx* c, const Lat& l) {
  if (c->pre_kind == BD_PRECOND_NONE || c->pre_kind == BD_PRECOND_BLOCKS) return BD_OK;
  int s;
  if (c->pre_kind == BD_PRECOND_SEGMENT) {
    int S = c->pre_S;
    if ((s = pre_alloc(c, S)) != BD_OK) return s;
    size_t smem = 2 * 8 * (size_t)(3 * S) * (3 * S);
    cudaFuncSetAttribute(k_seg_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    c->launches++;
    k_seg_blocks<<<c->N / S, 128, smem, c->stream>>>(l, c->rx, c->ry, c->rz, S, c->pre_G,
                                                     c->pre_Gi, c->pre_bad);
    c->pre_ready = true;
    return launch_ok(c);
  }
  if (c->pre_kind == BD_PRECOND_LEARNED && c->pre_S == 1) {
    if ((s = pre_alloc(c, 1)) != BD_OK) return s;
    if ((s = mpnn_blocks(c, l, c->pre_G)) != BD_OK) return s;
    c->launches++;
    k_bead_invert<<<(c->N + 127) / 128, 128, 0, c->stream>>>(c->pre_G, c->pre_Gi, c->N,
                                                             c->pre_bad);
    c->pre_ready = true;
    return launch_ok(c);
  }
  if (c->pre_kind == BD_PRECOND_LEARNED) {
    // segment blocks first, then the learned bead blocks applied on top
    int S = c->pre_S;
    if ((s = pre_alloc(c, S)) != BD_OK) return s;
    if (!c->pre_B) {
      CU(cudaMalloc(&c->pre_B, 72 * (size_t)c->N));
      CU(cudaMalloc(&c->pre_Bi, 72 * (size_t)c->N));
      c->bytes += 144 * (size_t)c->N;
    }
    size_t smem = 2 * 8 * (size_t)(3 * S) * (3 * S);
    cudaFuncSetAttribute(k_seg_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    c->launches += 3;
    k_seg_blocks<<<c->N / S, 128, smem, c->stream>>>(l, c->rx, c->ry, c->rz, S, c->pre_G,
                                                     c->pre_Gi, c->pre_bad);
    if ((s = mpnn_blocks(c, l, c->pre_B)) != BD_OK) return s;
    k_bead_invert<<<(c->N + 127) / 128, 128, 0, c->stream>>>(c->pre_B, c->pre_Bi, c->N,
                                                             c->pre_bad);
    int nb = c->N / S;
    k_combine_blocks<<<(nb * 3 * S + 127) / 128, 128, 0, c->stream>>>(c->pre_B, c->pre_Bi, S,
                                                                       nb, c->pre_G, c->pre_Gi);
    c->pre_ready = true;
    return launch_ok(c);
  }
  return BD_ERR_STATE;
}

// y = op(G) x (which = 0: G, 1: G^T, 2: G^(-1)) in the Lanczos layout.
// y_r = B x_r for k right-hand sides (RHS strides xs, ys); B = G (which 0),
// G^T (1) or G^-1 (2).
int precond_apply_k(bd_ctx* c, int which, int k, const double* x, size_t xs, double* y,
                    size_t ys) {
  int S = c->pre_S, NTp = c->NT * 32;
  const double* Bm = which == 2 ? c->pre_Gi : c->pre_G;
  int trans = which == 1;
  c->launches++;
  if (S == 1) {
    k_bead_apply<<<dim3((c->N + 127) / 128, k), 128, 0, c->stream>>>(Bm, c->N, trans, x, xs, y,
                                                                       ys, NTp);
  } else {
    size_t smem = 8 * (size_t)(3 * S) * (3 * S + k);
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_block_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_block_apply<<<c->N / S, 128, smem, c->stream>>>(Bm, S, trans, k, x, xs, y, ys, NTp);
  }
  return BD_OK;
}

int precond_apply(bd_ctx* c, int which, const double* x, double* y) {
  return precond_apply_k(c, which, 1, x, 0, y, 0);
}

void precond_free(bd_ctx* c) {
  if (c->pre_B) cudaFree(c->pre_B);
  if (c->pre_Bi) cudaFree(c->pre_Bi);
  if (c->pre_G) cudaFree(c->pre_G);
  if (c->pre_Gi) cudaFree(c->pre_Gi);
  if (c->pre_bad) cudaFree(c->pre_bad);
  c->pre_G = c->pre_Gi = nullptr;
  c->pre_bad = nullptr;
}

}  // namespace bd

extern "C" {

int bd_set_preconditioner(bd_ctx* c, int kind, int segment) {
  if (!c) return BD_ERR_ARG;
  if (kind < BD_PRECOND_NONE || kind > BD_PRECOND_BLOCKS) return BD_ERR_ARG;
  int S = 1;
  if (kind == BD_PRECOND_SEGMENT || (kind == BD_PRECOND_LEARNED && segment > 1)) {
    if (segment <= 0) {
      // 10 beads, or the largest of 5, 4, 2, 1 that divides the chain length
      const int cand[] = {10, 5, 4, 2, 1};
      for (int q : cand)
        if (c->Nb % q == 0) {
          S = q;
          break;
        }
    } else {
      S = segment;
    }
    if (S > kMaxSegment || c->Nb % S != 0) return BD_ERR_ARG;
  }
  if (kind == BD_PRECOND_LEARNED && !c->mpnn_ready) return BD_ERR_STATE;
  CU(cudaStreamSynchronize(c->stream));
  lanczos_graphs_reset(c);
  c->hi_version++;
  c->pre_kind = kind;
  c->pre_S = S;
  c->pre_ready = false;
  if (kind == BD_PRECOND_NONE) return BD_OK;
  if (kind == BD_PRECOND_BLOCKS) return BD_OK;  // blocks come from bd_set_precond_blocks
  // built with the next mobility rebuild; build now if a mobility exists
  if (c->hi_built) {
    Lat l = c->lat;
    int treal = (int)(c->t % (unsigned long)c->tp);
    l.treal = treal;
    l.nmax = (treal <= c->tp / 2) ? 1 : 2;
    l.delx = c->p.edot * treal * c->p.dt;
    return precond_build(c, l);
  }
  return BD_OK;
}

int bd_set_precond_blocks(bd_ctx* c, const double* G9) {
  if (!c || !G9) return BD_ERR_ARG;
  int s;
  if ((s = pre_alloc(c, 1)) != BD_OK) return s;
  CU(cudaMemcpyAsync(c->pre_G, G9, 72 * (size_t)c->N, cudaMemcpyHostToDevice, c->stream));
  c->launches++;
  k_bead_invert<<<(c->N + 127) / 128, 128, 0, c->stream>>>(c->pre_G, c->pre_Gi, c->N,
                                                           c->pre_bad);
  lanczos_graphs_reset(c);
  c->hi_version++;
  c->pre_kind = BD_PRECOND_BLOCKS;
  c->pre_S = 1;
  c->pre_ready = true;
  return launch_ok(c);
}

int bd_download_precond_blocks(bd_ctx* c, double* G, double* Ginv, int* block_beads) {
  if (!c || !c->pre_ready || !c->pre_G) return BD_ERR_STATE;
  int S = c->pre_S;
  size_t n = (size_t)(c->N / S) * 9 * S * S;
  if (G) CU(cudaMemcpyAsync(G, c->pre_G, 8 * n, cudaMemcpyDeviceToHost, c->stream));
  if (Ginv) CU(cudaMemcpyAsync(Ginv, c->pre_Gi, 8 * n, cudaMemcpyDeviceToHost, c->stream));
  if (block_beads) *block_beads = S;
  return check(c);
}

int bd_precond_stats(bd_ctx* c, long* o) {
  if (!c || !o) return BD_ERR_ARG;
  int bad = 0;
  if (c->pre_bad) {
    CU(cudaMemcpyAsync(&bad, c->pre_bad, 4, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
  }
  o[0] = (long)c->pre_calls;
  o[1] = (long)c->pre_iters;
  o[2] = (long)c->pre_fallbacks;
  o[3] = (long)bad;
  return BD_OK;
}

}  // extern "C"
