// Learned preconditioner: a per-bead message-passing network that predicts
// 3 x 3 blocks G_i approximating the diagonal blocks of M^(-1/2).
//
// No counterpart in the reference.  Per bead i the BD_MPNN_NEIGHBORS nearest
// beads j within BD_MPNN_CUTOFF (minimum image, taken from the Verlet rows)
// give unit pair vectors n_ij and radial features f_ij (Gaussians of |r_ij|
// centred on 2..6).  Three layers of width 64:
//   e_ij = silu(W1 f_ij + b1)                               (edges)
//   h_i  = silu(W2 mean_j e_ij + b2)                        (nodes)
//   u_i  = silu([W3 W4] [mean_j h_j ; h_i] + b3)            (messages)
// and two heads: a_i = exp(clamp(wa.u_i + ca, -4, 4)),
// c_ij = tanh(wb.(u_i * e_ij) + cb) / (2 K), K = BD_MPNN_NEIGHBORS, so that
// G_i = a_i (I + sum_j c_ij n_ij n_ij^T) is symmetric with eigenvalues
// >= a_i / 2.  The loss for a pair (z, t = M^(-1/2) z) is
// (1/N) sum_i |G_i z_i - t_i|^2, minimised by G_i = (M^(-1/2))_ii.
// The dense layers run on the tensor cores as warp-level
// mma.sync.m16n8k16 BF16 x BF16 -> FP32 (operands rounded to BF16 when staged
// in shared memory); the weight gradients are the same MMA with the row
// dimension as the reduction, summed over CTAs in a fixed order; the
// element-wise parts are FP32.  Adam (Kingma and Ba, ICLR 2015) updates FP32
// master parameters.
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "bd_ctx.cuh"

using namespace bd;

#define CU(call) BD_CU(call)

namespace {

constexpr int KN = BD_MPNN_NEIGHBORS, WD = BD_MPNN_WIDTH, NR = BD_MPNN_RBF;
constexpr float kCut = (float)BD_MPNN_CUTOFF;
// parameter layout (FP32): W1 (64 x 16), b1, W2 (64 x 64), b2,
// W34 = [W3 W4] (64 x 128), b3, wa, ca, wb, cb
constexpr int oW1 = 0, ob1 = oW1 + WD * NR, oW2 = ob1 + WD, ob2 = oW2 + WD * WD;
constexpr int oW34 = ob2 + WD, ob3 = oW34 + WD * 2 * WD, owa = ob3 + WD, oca = owa + WD;
constexpr int owb = oca + 1, ocb = owb + WD, kParams = ocb + 1;
constexpr int kGemmRows = 64;  // rows per CTA of the forward-type products
constexpr int kWgradCtas = 296;

typedef __nv_bfloat16 bf16;

struct Mpnn {
  int cap;
  float *w, *g, *m1, *m2;
  bf16 *W1b, *W2b, *W34b, *W2t, *W34t;  // W (out x in) and W^T (in x out), BF16
  int* nbr;                             // N x K neighbour (or -1)
  float *nvec, *rbf;                    // N x K x 3 unit vectors, N x K x 16 features
  float *g1, *e, *mv, *o2, *h, *X3, *p3, *u;
  float *sa, *a, *te, *ce;
  float *zt;     // z (3N) then t (3N)
  float *dG, *du, *de, *dp3, *dX3, *dh, *do2, *dm, *dg1, *hg, *lossv;
  float* part;   // kWgradCtas x 64 x 128 partial weight gradients
  double* G9;    // predicted blocks
  bool feat;
};

__device__ __forceinline__ float silu(float x) { return x / (1.0f + expf(-x)); }
__device__ __forceinline__ float silu_grad(float x) {
  float s = 1.0f / (1.0f + expf(-x));
  return s * (1.0f + x * (1.0f - s));
}

__device__ __forceinline__ uint32_t pack2(bf16 lo, bf16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma16816(float* c, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// pre = A B^T + bias (A: M x K FP32 row-major, B: NOUT x K BF16 row-major),
// post = silu(pre) when post is non-null.  64 rows per CTA, 16 per warp.
template <int K, int NOUT>
__global__ void __launch_bounds__(128) k_gemm(const float* __restrict__ A, int M,
                                              const bf16* __restrict__ B,
                                              const float* __restrict__ bias, float* pre,
                                              float* post) {
  constexpr int LD = K + 8;
  __shared__ __align__(16) bf16 As[kGemmRows * LD];
  __shared__ __align__(16) bf16 Bs[NOUT * LD];
  int r0 = blockIdx.x * kGemmRows;
  for (int e = threadIdx.x; e < kGemmRows * K; e += blockDim.x) {
    int r = e / K, k = e % K;
    float v = (r0 + r < M) ? A[(size_t)(r0 + r) * K + k] : 0.0f;
    As[r * LD + k] = __float2bfloat16_rn(v);
  }
  for (int e = threadIdx.x; e < NOUT * K; e += blockDim.x) Bs[(e / K) * LD + e % K] = B[e];
  __syncthreads();
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  float acc[NOUT / 8][4];
#pragma unroll
  for (int nt = 0; nt < NOUT / 8; nt++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[nt][q] = 0.0f;
  const bf16* Aw = As + warp * 16 * LD;
#pragma unroll
  for (int kk = 0; kk < K; kk += 16) {
    uint32_t a[4];
    a[0] = *(const uint32_t*)(Aw + g * LD + kk + 2 * t);
    a[1] = *(const uint32_t*)(Aw + (g + 8) * LD + kk + 2 * t);
    a[2] = *(const uint32_t*)(Aw + g * LD + kk + 2 * t + 8);
    a[3] = *(const uint32_t*)(Aw + (g + 8) * LD + kk + 2 * t + 8);
#pragma unroll
    for (int nt = 0; nt < NOUT / 8; nt++) {
      const bf16* Bn = Bs + (nt * 8 + g) * LD + kk + 2 * t;
      uint32_t b[2] = {*(const uint32_t*)Bn, *(const uint32_t*)(Bn + 8)};
      mma16816(acc[nt], a, b);
    }
  }
#pragma unroll
  for (int nt = 0; nt < NOUT / 8; nt++)
#pragma unroll
    for (int hh = 0; hh < 2; hh++) {
      int row = r0 + warp * 16 + g + 8 * hh;
      if (row >= M) continue;
#pragma unroll
      for (int q = 0; q < 2; q++) {
        int col = nt * 8 + 2 * t + q;
        float v = acc[nt][2 * hh + q] + (bias ? bias[col] : 0.0f);
        pre[(size_t)row * NOUT + col] = v;
        if (post) post[(size_t)row * NOUT + col] = silu(v);
      }
    }
}

// part[cta] = dY^T X over this CTA's rows (dY: M x 64, X: M x K; result
// 64 x K), BF16 operands, FP32 accumulation; the row dimension is the MMA's
// reduction dimension.
template <int K>
__global__ void __launch_bounds__(128) k_wgrad(const float* __restrict__ dY,
                                               const float* __restrict__ X, int M, int rpc,
                                               float* part) {
  __shared__ __align__(16) bf16 Ys[16][WD + 8];
  __shared__ __align__(16) bf16 Xs[16][K + 8];
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  int o0 = warp * 16;
  float acc[K / 8][4];
#pragma unroll
  for (int nt = 0; nt < K / 8; nt++)
#pragma unroll
    for (int q = 0; q < 4; q++) acc[nt][q] = 0.0f;
  int rb = blockIdx.x * rpc, re = min(M, rb + rpc);
  for (int r0 = rb; r0 < re; r0 += 16) {
    __syncthreads();
    for (int e = threadIdx.x; e < 16 * WD; e += blockDim.x) {
      int r = e / WD, o = e % WD;
      Ys[r][o] = __float2bfloat16_rn(r0 + r < re ? dY[(size_t)(r0 + r) * WD + o] : 0.0f);
    }
    for (int e = threadIdx.x; e < 16 * K; e += blockDim.x) {
      int r = e / K, k = e % K;
      Xs[r][k] = __float2bfloat16_rn(r0 + r < re ? X[(size_t)(r0 + r) * K + k] : 0.0f);
    }
    __syncthreads();
    uint32_t a[4];
    a[0] = pack2(Ys[2 * t][o0 + g], Ys[2 * t + 1][o0 + g]);
    a[1] = pack2(Ys[2 * t][o0 + g + 8], Ys[2 * t + 1][o0 + g + 8]);
    a[2] = pack2(Ys[2 * t + 8][o0 + g], Ys[2 * t + 9][o0 + g]);
    a[3] = pack2(Ys[2 * t + 8][o0 + g + 8], Ys[2 * t + 9][o0 + g + 8]);
#pragma unroll
    for (int nt = 0; nt < K / 8; nt++) {
      int n = nt * 8 + g;
      uint32_t b[2] = {pack2(Xs[2 * t][n], Xs[2 * t + 1][n]),
                       pack2(Xs[2 * t + 8][n], Xs[2 * t + 9][n])};
      mma16816(acc[nt], a, b);
    }
  }
  float* P = part + (size_t)blockIdx.x * WD * K;
#pragma unroll
  for (int nt = 0; nt < K / 8; nt++)
#pragma unroll
    for (int hh = 0; hh < 2; hh++)
#pragma unroll
      for (int q = 0; q < 2; q++)
        P[(size_t)(o0 + g + 8 * hh) * K + nt * 8 + 2 * t + q] = acc[nt][2 * hh + q];
}

// out[e] = sum over CTAs of part[cta][e] (fixed order)
__global__ void k_part_sum(const float* __restrict__ part, int nparts, int n, float* out) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float s = 0;
  for (int b = 0; b < nparts; b++) s += part[(size_t)b * n + e];
  out[e] = s;
}

// part[cta][c] = column sums of Y (M x C) over this CTA's rows
__global__ void k_colsum(const float* __restrict__ Y, int M, int C, int rpc, float* part) {
  int rb = blockIdx.x * rpc, re = min(M, rb + rpc);
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    float s = 0;
    for (int r = rb; r < re; r++) s += Y[(size_t)r * C + c];
    part[(size_t)blockIdx.x * C + c] = s;
  }
}

__global__ void k_to_bf16(const float* __restrict__ w, int rows, int cols, bf16* W, bf16* Wt) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= rows * cols) return;
  int r = e / cols, c = e % cols;
  bf16 v = __float2bfloat16_rn(w[e]);
  W[e] = v;
  if (Wt) Wt[(size_t)c * rows + r] = v;
}

// Neighbour features: the K nearest Verlet neighbours within the cutoff
// (ties by index), unit vectors and Gaussian radial features.
__global__ void k_mpnn_features(Lat l, const double* __restrict__ rx,
                                const double* __restrict__ ry, const double* __restrict__ rz,
                                int N, const int* __restrict__ nb_count,
                                const int* __restrict__ nb_rows, int maxnb, int* nbr,
                                float* nvec, float* rbf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float bd[KN];
  int bj[KN];
  for (int k = 0; k < KN; k++) {
    bd[k] = 1e30f;
    bj[k] = -1;
  }
  int n = min(nb_count[i], maxnb);
  for (int q = 0; q < n; q++) {
    int j = nb_rows[(size_t)i * maxnb + q];
    double dx, dy, dz;
    nid(l, rx, ry, rz, i, j, dx, dy, dz);
    float d = (float)sqrt(dx * dx + dy * dy + dz * dz);
    if (!(d < kCut)) continue;
    if (d > bd[KN - 1] || (d == bd[KN - 1] && j > bj[KN - 1])) continue;
    int p = KN - 1;
    while (p > 0 && (bd[p - 1] > d || (bd[p - 1] == d && bj[p - 1] > j))) {
      bd[p] = bd[p - 1];
      bj[p] = bj[p - 1];
      p--;
    }
    bd[p] = d;
    bj[p] = j;
  }
  for (int k = 0; k < KN; k++) {
    size_t ek = (size_t)i * KN + k;
    int j = bj[k];
    nbr[ek] = j;
    float v[3] = {0, 0, 0};
    if (j >= 0) {
      double dx, dy, dz;
      nid(l, rx, ry, rz, i, j, dx, dy, dz);
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      v[0] = (float)(dx / r);
      v[1] = (float)(dy / r);
      v[2] = (float)(dz / r);
    }
    for (int a = 0; a < 3; a++) nvec[ek * 3 + a] = v[a];
    for (int m = 0; m < NR; m++) {
      float mu = 2.0f + 4.0f * m / (NR - 1), x = (bd[k] - mu) / 0.35f;
      rbf[ek * NR + m] = j >= 0 ? expf(-0.5f * x * x) : 0.0f;
    }
  }
}

// mv_i = mean over neighbour slots of e_ij (missing slots count as zero)
__global__ void k_edge_mean(const float* __restrict__ e, const int* __restrict__ nbr, int N,
                            float* mv) {
  int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  for (int o = lane; o < WD; o += 32) {
    float s = 0;
    for (int k = 0; k < KN; k++)
      if (nbr[(size_t)i * KN + k] >= 0) s += e[((size_t)i * KN + k) * WD + o];
    mv[(size_t)i * WD + o] = s * (1.0f / KN);
  }
}

// X3_i = [mean_j h_j ; h_i]
__global__ void k_node_mean(const float* __restrict__ h, const int* __restrict__ nbr, int N,
                            float* X3) {
  int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  for (int o = lane; o < WD; o += 32) {
    float s = 0;
    for (int k = 0; k < KN; k++) {
      int j = nbr[(size_t)i * KN + k];
      if (j >= 0) s += h[(size_t)j * WD + o];
    }
    X3[(size_t)i * 2 * WD + o] = s * (1.0f / KN);
    X3[(size_t)i * 2 * WD + WD + o] = h[(size_t)i * WD + o];
  }
}

__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Heads and blocks, one warp per bead.
__global__ void k_heads(const float* __restrict__ w, const float* __restrict__ u,
                        const float* __restrict__ e, const int* __restrict__ nbr,
                        const float* __restrict__ nvec, int N, float* sa, float* a, float* te,
                        float* ce, double* G9) {
  int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  const float* ui = u + (size_t)i * WD;
  float s = warp_sum(w[owa + lane] * ui[lane] + w[owa + lane + 32] * ui[lane + 32]) + w[oca];
  float ai = expf(fminf(fmaxf(s, -4.0f), 4.0f));
  float G[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int k = 0; k < KN; k++) {
    size_t ek = (size_t)i * KN + k;
    const float* ek_ = e + ek * WD;
    float t = warp_sum(w[owb + lane] * ui[lane] * ek_[lane] +
                       w[owb + lane + 32] * ui[lane + 32] * ek_[lane + 32]) +
              w[ocb];
    float c = nbr[ek] >= 0 ? tanhf(t) * (0.5f / KN) : 0.0f;
    if (lane == 0) {
      te[ek] = t;
      ce[ek] = c;
    }
    const float* n = nvec + ek * 3;
    for (int p = 0; p < 3; p++)
      for (int q = 0; q < 3; q++) G[3 * p + q] += c * n[p] * n[q];
  }
  if (lane == 0) {
    sa[i] = s;
    a[i] = ai;
    for (int q = 0; q < 9; q++) G9[(size_t)9 * i + q] = (double)(ai * G[q]);
  }
}

// Loss and the head part of the backward pass, one warp per bead:
// r = G z - t, dG = (2/N) r z^T; writes du_i, the head part of de_ij, the
// per-bead head-parameter gradient rows hg_i = [ds u_i (64), ds, sum_j dt
// (u_i * e_ij) (64), sum_j dt] and the per-bead loss.
__global__ void k_loss_heads(const float* __restrict__ w, const float* __restrict__ u,
                             const float* __restrict__ e, const int* __restrict__ nbr,
                             const float* __restrict__ nvec, const float* __restrict__ sa,
                             const float* __restrict__ a, const float* __restrict__ te,
                             const float* __restrict__ ce, const double* __restrict__ G9,
                             const float* __restrict__ zt, int N, float* du, float* de,
                             float* hg, float* lossv) {
  int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  const float* z = zt + 3 * (size_t)i;
  const float* tg = zt + 3 * (size_t)N + 3 * (size_t)i;
  float G[9], r[3], dG[9];
  for (int q = 0; q < 9; q++) G[q] = (float)G9[(size_t)9 * i + q];
  for (int p = 0; p < 3; p++) r[p] = G[3 * p] * z[0] + G[3 * p + 1] * z[1] + G[3 * p + 2] * z[2] - tg[p];
  float sc = 2.0f / N;
  for (int p = 0; p < 3; p++)
    for (int q = 0; q < 3; q++) dG[3 * p + q] = sc * r[p] * z[q];
  float ai = a[i];
  // G = a (I + sum c n n^T): da = tr(dG) + sum c n^T dG n, dc = a n^T dG n
  float da = dG[0] + dG[4] + dG[8];
  const float* ui = u + (size_t)i * WD;
  float du0 = 0, du1 = 0, hb0 = 0, hb1 = 0, dtsum = 0;
  for (int k = 0; k < KN; k++) {
    size_t ek = (size_t)i * KN + k;
    float dt = 0;
    if (nbr[ek] >= 0) {
      const float* n = nvec + ek * 3;
      float ndn = 0;
      for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) ndn += n[p] * dG[3 * p + q] * n[q];
      da += ce[ek] * ndn;
      float th = tanhf(te[ek]);
      dt = ai * ndn * (0.5f / KN) * (1.0f - th * th);
    }
    const float* ek_ = e + ek * WD;
    float* dek = de + ek * WD;
    float wb0 = w[owb + lane], wb1 = w[owb + lane + 32];
    du0 += dt * wb0 * ek_[lane];
    du1 += dt * wb1 * ek_[lane + 32];
    dek[lane] = dt * wb0 * ui[lane];
    dek[lane + 32] = dt * wb1 * ui[lane + 32];
    hb0 += dt * ui[lane] * ek_[lane];
    hb1 += dt * ui[lane + 32] * ek_[lane + 32];
    dtsum += dt;
  }
  float s = sa[i];
  float ds = (s > -4.0f && s < 4.0f) ? da * ai : 0.0f;
  du[(size_t)i * WD + lane] = du0 + ds * w[owa + lane];
  du[(size_t)i * WD + lane + 32] = du1 + ds * w[owa + lane + 32];
  float* h = hg + (size_t)i * (2 * WD + 2);
  h[lane] = ds * ui[lane];
  h[lane + 32] = ds * ui[lane + 32];
  h[WD + 1 + lane] = hb0;
  h[WD + 1 + lane + 32] = hb1;
  if (lane == 0) {
    h[WD] = ds;
    h[2 * WD + 1] = dtsum;
    lossv[i] = (r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) / N;
  }
}

// dx = dy * silu'(pre)
__global__ void k_silu_back(const float* __restrict__ dy, const float* __restrict__ pre,
                            size_t n, float* dx) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < n) dx[e] = dy[e] * silu_grad(pre[e]);
}

// dh = dX3[:, 64:] + sum over beads i that list j of dX3_i[:, :64] / K
__global__ void k_dh(const float* __restrict__ dX3, const int* __restrict__ nbr, int N,
                     float* dh) {
  int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (i >= N) return;
  for (int o = lane; o < WD; o += 32) {
    float q = dX3[(size_t)i * 2 * WD + o] * (1.0f / KN);
    atomicAdd(&dh[(size_t)i * WD + o], dX3[(size_t)i * 2 * WD + WD + o]);
    for (int k = 0; k < KN; k++) {
      int j = nbr[(size_t)i * KN + k];
      if (j >= 0) atomicAdd(&dh[(size_t)j * WD + o], q);
    }
  }
}

// de_ij += dm_i / K for present neighbour slots
__global__ void k_de_add(const float* __restrict__ dm, const int* __restrict__ nbr, int N,
                         float* de) {
  size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)N * KN * WD) return;
  size_t ek = e / WD;
  int o = (int)(e % WD), i = (int)(ek / KN);
  if (nbr[ek] >= 0) de[e] += dm[(size_t)i * WD + o] * (1.0f / KN);
}

__global__ void k_adam(float* w, const float* __restrict__ g, float* m1, float* m2, int n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float gi = g[e];
  float m = b1 * m1[e] + (1.0f - b1) * gi, v = b2 * m2[e] + (1.0f - b2) * gi * gi;
  m1[e] = m;
  m2[e] = v;
  w[e] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
}

inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

Mpnn* get(bd_ctx* c) { return (Mpnn*)c->mpnn; }

int ensure(bd_ctx* c) {
  Mpnn* m = get(c);
  if (!m) {
    m = new Mpnn();
    c->mpnn = m;
    CU(cudaMalloc(&m->w, 4 * kParams));
    CU(cudaMalloc(&m->g, 4 * kParams));
    CU(cudaMalloc(&m->m1, 4 * kParams));
    CU(cudaMalloc(&m->m2, 4 * kParams));
    CU(cudaMemsetAsync(m->m1, 0, 4 * kParams, c->stream));
    CU(cudaMemsetAsync(m->m2, 0, 4 * kParams, c->stream));
    CU(cudaMalloc(&m->W1b, 2 * WD * NR));
    CU(cudaMalloc(&m->W2b, 2 * WD * WD));
    CU(cudaMalloc(&m->W2t, 2 * WD * WD));
    CU(cudaMalloc(&m->W34b, 2 * WD * 2 * WD));
    CU(cudaMalloc(&m->W34t, 2 * WD * 2 * WD));
    CU(cudaMalloc(&m->part, 4 * (size_t)kWgradCtas * WD * 2 * WD));
    c->bytes += 16 * kParams + 2 * (WD * NR + 2 * WD * WD + 4 * WD * WD) +
                4 * (size_t)kWgradCtas * WD * 2 * WD;
  }
  int N = c->N;
  if (m->cap < N) {
    void* old[] = {m->nbr, m->nvec, m->rbf, m->g1, m->e, m->mv, m->o2, m->h, m->X3, m->p3,
                   m->u, m->sa, m->a, m->te, m->ce, m->zt, m->dG, m->du, m->de, m->dp3,
                   m->dX3, m->dh, m->do2, m->dm, m->dg1, m->hg, m->lossv, m->G9};
    for (void* q : old)
      if (q) cudaFree(q);
    size_t E = (size_t)N * KN;
    CU(cudaMalloc(&m->nbr, 4 * E));
    CU(cudaMalloc(&m->nvec, 12 * E));
    CU(cudaMalloc(&m->rbf, 4 * E * NR));
    CU(cudaMalloc(&m->g1, 4 * E * WD));
    CU(cudaMalloc(&m->e, 4 * E * WD));
    CU(cudaMalloc(&m->de, 4 * E * WD));
    CU(cudaMalloc(&m->dg1, 4 * E * WD));
    CU(cudaMalloc(&m->te, 4 * E));
    CU(cudaMalloc(&m->ce, 4 * E));
    float** nodes[] = {&m->mv, &m->o2, &m->h, &m->p3, &m->u, &m->du, &m->dp3, &m->dh, &m->do2,
                       &m->dm};
    for (float** q : nodes) CU(cudaMalloc(q, 4 * (size_t)N * WD));
    CU(cudaMalloc(&m->X3, 8 * (size_t)N * WD));
    CU(cudaMalloc(&m->dX3, 8 * (size_t)N * WD));
    CU(cudaMalloc(&m->sa, 4 * (size_t)N));
    CU(cudaMalloc(&m->a, 4 * (size_t)N));
    CU(cudaMalloc(&m->lossv, 4 * (size_t)N));
    CU(cudaMalloc(&m->zt, 24 * (size_t)N));
    CU(cudaMalloc(&m->dG, 36 * (size_t)N));
    CU(cudaMalloc(&m->hg, 4 * (size_t)N * (2 * WD + 2)));
    CU(cudaMalloc(&m->G9, 72 * (size_t)N));
    m->cap = N;
    c->bytes += E * (4 + 12 + 4 * NR + 16 * WD + 8) + (size_t)N * (40 * WD + 16 * WD + 12 + 24 +
                36 + 4 * (2 * WD + 2) + 72);
  }
  return BD_OK;
}

int make_bf16(bd_ctx* c) {
  Mpnn* m = get(c);
  c->launches += 3;
  k_to_bf16<<<nblk(WD * NR, 256), 256, 0, c->stream>>>(m->w + oW1, WD, NR, m->W1b, nullptr);
  k_to_bf16<<<nblk(WD * WD, 256), 256, 0, c->stream>>>(m->w + oW2, WD, WD, m->W2b, m->W2t);
  k_to_bf16<<<nblk(2 * WD * WD, 256), 256, 0, c->stream>>>(m->w + oW34, WD, 2 * WD, m->W34b,
                                                           m->W34t);
  return BD_OK;
}

int features(bd_ctx* c, const Lat& l) {
  Mpnn* m = get(c);
  c->launches++;
  k_mpnn_features<<<nblk(c->N, 128), 128, 0, c->stream>>>(l, c->rx, c->ry, c->rz, c->N,
                                                          c->nb_count, c->nb_rows, c->maxnb,
                                                          m->nbr, m->nvec, m->rbf);
  m->feat = true;
  return BD_OK;
}

int forward(bd_ctx* c) {
  Mpnn* m = get(c);
  int N = c->N, E = N * KN;
  c->launches += 6;
  k_gemm<NR, WD><<<nblk(E, kGemmRows), 128, 0, c->stream>>>(m->rbf, E, m->W1b, m->w + ob1,
                                                            m->g1, m->e);
  k_edge_mean<<<nblk(N, 4), 128, 0, c->stream>>>(m->e, m->nbr, N, m->mv);
  k_gemm<WD, WD><<<nblk(N, kGemmRows), 128, 0, c->stream>>>(m->mv, N, m->W2b, m->w + ob2,
                                                            m->o2, m->h);
  k_node_mean<<<nblk(N, 4), 128, 0, c->stream>>>(m->h, m->nbr, N, m->X3);
  k_gemm<2 * WD, WD><<<nblk(N, kGemmRows), 128, 0, c->stream>>>(m->X3, N, m->W34b, m->w + ob3,
                                                                m->p3, m->u);
  k_heads<<<nblk(N, 4), 128, 0, c->stream>>>(m->w, m->u, m->e, m->nbr, m->nvec, N, m->sa, m->a,
                                             m->te, m->ce, m->G9);
  return BD_OK;
}

// weight gradient dY^T X (64 x K) into g + off, bias gradient colsum(dY)
template <int K>
void wgrad(bd_ctx* c, const float* dY, const float* X, int M, int off_w, int off_b) {
  Mpnn* m = get(c);
  int rpc = ((M + kWgradCtas - 1) / kWgradCtas + 15) / 16 * 16;
  int nct = nblk(M, rpc);
  c->launches += 2;
  k_wgrad<K><<<nct, 128, 0, c->stream>>>(dY, X, M, rpc, m->part);
  k_part_sum<<<nblk(WD * K, 256), 256, 0, c->stream>>>(m->part, nct, WD * K, m->g + off_w);
  if (off_b >= 0) {
    c->launches += 2;
    k_colsum<<<nct, 64, 0, c->stream>>>(dY, M, WD, rpc, m->part);
    k_part_sum<<<1, 64, 0, c->stream>>>(m->part, nct, WD, m->g + off_b);
  }
}

int backward(bd_ctx* c, double* loss_out) {
  Mpnn* m = get(c);
  int N = c->N, E = N * KN;
  size_t nN = (size_t)N * WD, nE = (size_t)E * WD;
  c->launches += 2;
  k_loss_heads<<<nblk(N, 4), 128, 0, c->stream>>>(m->w, m->u, m->e, m->nbr, m->nvec, m->sa,
                                                  m->a, m->te, m->ce, m->G9, m->zt, N, m->du,
                                                  m->de, m->hg, m->lossv);
  // head parameter gradients: column sums of hg = [dwa (64), dca, dwb (64), dcb]
  int rpc = (N + kWgradCtas - 1) / kWgradCtas;
  int nct = nblk(N, rpc);
  k_colsum<<<nct, 160, 0, c->stream>>>(m->hg, N, 2 * WD + 2, rpc, m->part);
  c->launches += 1;
  k_part_sum<<<1, 160, 0, c->stream>>>(m->part, nct, 2 * WD + 2, m->g + owa);
  // layer 3
  c->launches += 1;
  k_silu_back<<<nblk((long long)nN, 256), 256, 0, c->stream>>>(m->du, m->p3, nN, m->dp3);
  wgrad<2 * WD>(c, m->dp3, m->X3, N, oW34, ob3);
  c->launches += 3;
  k_gemm<WD, 2 * WD><<<nblk(N, kGemmRows), 128, 0, c->stream>>>(m->dp3, N, m->W34t, nullptr,
                                                                m->dX3, nullptr);
  CU(cudaMemsetAsync(m->dh, 0, 4 * nN, c->stream));
  k_dh<<<nblk(N, 4), 128, 0, c->stream>>>(m->dX3, m->nbr, N, m->dh);
  // layer 2
  k_silu_back<<<nblk((long long)nN, 256), 256, 0, c->stream>>>(m->dh, m->o2, nN, m->do2);
  wgrad<WD>(c, m->do2, m->mv, N, oW2, ob2);
  c->launches += 3;
  k_gemm<WD, WD><<<nblk(N, kGemmRows), 128, 0, c->stream>>>(m->do2, N, m->W2t, nullptr, m->dm,
                                                            nullptr);
  // layer 1
  k_de_add<<<nblk((long long)nE, 256), 256, 0, c->stream>>>(m->dm, m->nbr, N, m->de);
  k_silu_back<<<nblk((long long)nE, 256), 256, 0, c->stream>>>(m->de, m->g1, nE, m->dg1);
  wgrad<NR>(c, m->dg1, m->rbf, E, oW1, ob1);
  if (loss_out) {
    std::vector<float> lv(N);
    CU(cudaMemcpyAsync(lv.data(), m->lossv, 4 * (size_t)N, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    double s = 0;
    for (int i = 0; i < N; i++) s += lv[i];
    *loss_out = s;
  }
  return launch_ok(c);
}

}  // namespace

namespace bd {

// Predicted blocks for the configuration of the mobility build into G9
// (device, 9 N doubles).
int mpnn_blocks(bd_ctx* c, const Lat& l, double* G9) {
  if (!c->mpnn_ready) return BD_ERR_STATE;
  int s;
  if ((s = ensure(c)) != BD_OK) return s;
  features(c, l);
  forward(c);
  CU(cudaMemcpyAsync(G9, get(c)->G9, 72 * (size_t)c->N, cudaMemcpyDeviceToDevice, c->stream));
  return launch_ok(c);
}

void mpnn_free(bd_ctx* c) {
  Mpnn* m = get(c);
  if (!m) return;
  void* ptrs[] = {m->w, m->g, m->m1, m->m2, m->W1b, m->W2b, m->W34b, m->W2t, m->W34t,
                  m->part, m->nbr, m->nvec, m->rbf, m->g1, m->e, m->mv, m->o2, m->h, m->X3,
                  m->p3, m->u, m->sa, m->a, m->te, m->ce, m->zt, m->dG, m->du, m->de, m->dp3,
                  m->dX3, m->dh, m->do2, m->dm, m->dg1, m->hg, m->lossv, m->G9};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete m;
  c->mpnn = nullptr;
}

}  // namespace bd

static Lat current_lat(bd_ctx* c) {
  Lat l = c->lat;
  int treal = (int)(c->t % (unsigned long)c->tp);
  l.treal = treal;
  l.nmax = (treal <= c->tp / 2) ? 1 : 2;
  l.delx = c->p.edot * treal * c->p.dt;
  return l;
}

extern "C" {

size_t bd_mpnn_param_count(void) { return (size_t)kParams; }

int bd_mpnn_set_params(bd_ctx* c, const float* w) {
  if (!c || !w) return BD_ERR_ARG;
  int s;
  if ((s = ensure(c)) != BD_OK) return s;
  CU(cudaMemcpyAsync(get(c)->w, w, 4 * kParams, cudaMemcpyHostToDevice, c->stream));
  make_bf16(c);
  c->mpnn_ready = true;
  return launch_ok(c);
}

int bd_mpnn_get_params(bd_ctx* c, float* w) {
  if (!c || !w) return BD_ERR_ARG;
  if (!c->mpnn_ready) return BD_ERR_STATE;
  CU(cudaMemcpyAsync(w, get(c)->w, 4 * kParams, cudaMemcpyDeviceToHost, c->stream));
  return check(c);
}

int bd_mpnn_features(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  if (!c->mpnn_ready) return BD_ERR_STATE;
  int s;
  if ((s = ensure(c)) != BD_OK) return s;
  features(c, current_lat(c));
  return launch_ok(c);
}

int bd_mpnn_predict(bd_ctx* c, double* G9) {
  if (!c || !G9) return BD_ERR_ARG;
  if (!c->mpnn_ready || !get(c)->feat) return BD_ERR_STATE;
  forward(c);
  CU(cudaMemcpyAsync(G9, get(c)->G9, 72 * (size_t)c->N, cudaMemcpyDeviceToHost, c->stream));
  return check(c);
}

int bd_mpnn_loss_grad(bd_ctx* c, const double* z, const double* t, double* loss, float* grad) {
  if (!c || !z || !t) return BD_ERR_ARG;
  if (!c->mpnn_ready || !get(c)->feat) return BD_ERR_STATE;
  Mpnn* m = get(c);
  int N = c->N;
  std::vector<float> zt(6 * (size_t)N);
  for (size_t k = 0; k < 3 * (size_t)N; k++) {
    zt[k] = (float)z[k];
    zt[3 * (size_t)N + k] = (float)t[k];
  }
  CU(cudaMemcpyAsync(m->zt, zt.data(), 4 * zt.size(), cudaMemcpyHostToDevice, c->stream));
  forward(c);
  int s;
  if ((s = backward(c, loss)) != BD_OK) return s;
  if (grad) CU(cudaMemcpyAsync(grad, m->g, 4 * kParams, cudaMemcpyDeviceToHost, c->stream));
  return check(c);
}

int bd_mpnn_adam(bd_ctx* c, float lr, float beta1, float beta2, float eps, int step) {
  if (!c || step < 1) return BD_ERR_ARG;
  if (!c->mpnn_ready) return BD_ERR_STATE;
  Mpnn* m = get(c);
  float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  c->launches++;
  k_adam<<<nblk(kParams, 256), 256, 0, c->stream>>>(m->w, m->g, m->m1, m->m2, kParams, lr,
                                                    beta1, beta2, eps, c1, c2);
  make_bf16(c);
  return launch_ok(c);
}

}  // extern "C"
