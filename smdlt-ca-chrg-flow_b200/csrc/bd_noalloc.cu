// Mobility product that allocates nothing.
//
// bd_mobility_apply_noalloc computes out = M v with the mobility of the last
// bd_calc_hi, like bd_mobility_apply, but it is meant for callers that must
// not allocate device memory at the point of the call: a step loop that runs
// while another framework's memory pool owns the device, a real-time loop
// with a fixed memory budget, or code that must not trigger the implicit
// device-wide synchronisation that cudaMalloc/cudaFree can cause.  Its
// partial sums live in g_noalloc_scratch below, a file-scope device array of
// fixed size that every GPU loading this library holds until the process
// exits; it calls no cudaMalloc, cudaFree or allocating library routine.
//
// Limits and sharing:
//  - N <= BD_NOALLOC_MAX_BEADS (4096 beads, 14.3 MB of scratch); larger
//    systems get BD_ERR_CAPACITY;
//  - every call on a device shares the one array and it keeps the last
//    call's contents; the kernels overwrite every entry they read before
//    reading it, so nothing needs clearing, but calls that overlap on the
//    GPU (two streams at once, or two contexts on one device) race on it;
//  - the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (a host name for a __device__ array is not a
//    device address); make that first call before any stream capture;
//  - the address is kept per device ordinal for the life of the process: a
//    cudaDeviceReset destroys the array with the device's context (and every
//    bd_ctx made before it), and calls after a reset are not supported;
//  - it applies to the dense-tile mobilities (BD_MOB_EWALD, BD_MOB_HYBRID);
//    a particle-mesh context has no tiles and gets BD_ERR_STATE.
#include <math.h>

#include <mutex>

#include "bd_ctx.cuh"

using namespace bd;

namespace {

constexpr int kMaxNT = BD_NOALLOC_MAX_BEADS / 32;               // tile rows
constexpr long long kMaxTiles = (long long)kMaxNT * (kMaxNT + 1) / 2;
constexpr int kSplit = 16;                                        // reduction splits
constexpr long long kRowPart = kMaxTiles * 96;                   // per-tile row partials
constexpr long long kScratch = 2 * kRowPart + (long long)kMaxNT * kSplit * 96;

__device__ __forceinline__ long long na_tile_off(int I, int NT) {
  return (long long)I * NT - (long long)I * (I - 1) / 2;
}

}  // namespace

// 2 x kRowPart partial sums + the first reduction level: 14.3 MB.
static __device__ __align__(256) double g_noalloc_scratch[kScratch];

// One CTA per packed tile; tile row from the packed index by the inverse of
// tile_off; input bead-interleaved v[3 i + a].
template <typename T>
__global__ void __launch_bounds__(256) k_na_matvec(const T* __restrict__ Mt, int NT, int N,
                                                   const double* __restrict__ v,
                                                   double* __restrict__ scratch) {
  long long tile = blockIdx.x;
  // largest I with tile_off(I) <= tile
  double b = 2.0 * NT + 1.0;
  int I = (int)floor((b - sqrt(b * b - 8.0 * (double)tile)) * 0.5);
  if (I < 0) I = 0;
  while (I > 0 && na_tile_off(I, NT) > tile) I--;
  while (I + 1 < NT && na_tile_off(I + 1, NT) <= tile) I++;
  int J = I + (int)(tile - na_tile_off(I, NT));
  double* rowpart = scratch;
  double* colpart = scratch + kRowPart;
  __shared__ double xI[3][32], xJ[3][32], racc[3][32], cacc[8][3][32];
  int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid < 96) {
    int a = tid / 32, k = tid & 31, i = I * 32 + k, j = J * 32 + k;
    xI[a][k] = i < N ? v[3 * i + a] : 0.0;
    xJ[a][k] = j < N ? v[3 * j + a] : 0.0;
  }
  const T* tb = Mt + tile * 6144;
  double m[4][6];
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int a = 0; a < 6; a++) m[q][a] = (double)tb[a * 1024 + (w + 8 * q) * 32 + lane];
  __syncthreads();
  double c0 = 0, c1 = 0, c2 = 0;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    int il = w + 8 * q;
    bool valid = (I != J) || (il < lane);
    double m0 = valid ? m[q][0] : 0.0, m1 = valid ? m[q][1] : 0.0, m2 = valid ? m[q][2] : 0.0;
    double m3 = valid ? m[q][3] : 0.0, m4 = valid ? m[q][4] : 0.0, m5 = valid ? m[q][5] : 0.0;
    double x0 = xJ[0][lane], x1 = xJ[1][lane], x2 = xJ[2][lane];
    double ra = m0 * x0 + m1 * x1 + m2 * x2;
    double rb = m1 * x0 + m3 * x1 + m4 * x2;
    double rc = m2 * x0 + m4 * x1 + m5 * x2;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ra += __shfl_xor_sync(0xffffffffu, ra, o);
      rb += __shfl_xor_sync(0xffffffffu, rb, o);
      rc += __shfl_xor_sync(0xffffffffu, rc, o);
    }
    if (lane == 0) {
      racc[0][il] = ra;
      racc[1][il] = rb;
      racc[2][il] = rc;
    }
    double y0 = xI[0][il], y1 = xI[1][il], y2 = xI[2][il];
    c0 += m0 * y0 + m1 * y1 + m2 * y2;
    c1 += m1 * y0 + m3 * y1 + m4 * y2;
    c2 += m2 * y0 + m4 * y1 + m5 * y2;
  }
  cacc[w][0][lane] = c0;
  cacc[w][1][lane] = c1;
  cacc[w][2][lane] = c2;
  __syncthreads();
  if (tid < 96) {
    int a = tid / 32, k = tid & 31;
    double s = 0;
    for (int ww = 0; ww < 8; ww++) s += cacc[ww][a][k];
    colpart[tile * 96 + tid] = s;
    rowpart[tile * 96 + tid] = racc[a][k];
  }
}

__global__ void k_na_reduce1(int NT, double* __restrict__ scratch) {
  const double* rowpart = scratch;
  const double* colpart = scratch + kRowPart;
  double* part = scratch + 2 * kRowPart;
  int K = blockIdx.x, s = blockIdx.y, e = threadIdx.x;
  double acc = 0;
  for (int J = K + s; J < NT; J += kSplit) acc += rowpart[(na_tile_off(K, NT) + (J - K)) * 96 + e];
  for (int I = s; I <= K; I += kSplit) acc += colpart[(na_tile_off(I, NT) + (K - I)) * 96 + e];
  part[((size_t)K * kSplit + s) * 96 + e] = acc;
}

// out[3 i + a] = sum of the splits + Dtr_a v[3 i + a] (uniform self blocks)
__global__ void k_na_reduce2(int N, const double* __restrict__ scratch,
                             const double* __restrict__ v, double d0, double d1, double d2,
                             double* __restrict__ out) {
  const double* part = scratch + 2 * kRowPart;
  int K = blockIdx.x, e = threadIdx.x;
  double acc = 0;
  for (int s = 0; s < kSplit; s++) acc += part[((size_t)K * kSplit + s) * 96 + e];
  int a = e / 32, i = K * 32 + (e & 31);
  if (i < N) out[3 * i + a] = acc + (a == 0 ? d0 : a == 1 ? d1 : d2) * v[3 * i + a];
}

// Device address of g_noalloc_scratch per device ordinal, looked up once.
static double* scratch_address(int dev, int* status) {
  static std::mutex mu;
  static double* addr[256] = {nullptr};
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 0 || dev >= 256) {
    *status = BD_ERR_ARG;
    return nullptr;
  }
  if (!addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      // not a sticky error: clear it so that the next launch check of another
      // entry point does not report it as its own
      cudaGetLastError();
      *status = bd::cuda_fail((int)(e != cudaSuccess ? e : cudaErrorInvalidSymbol),
                              "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
      return nullptr;
    }
    addr[dev] = (double*)p;
  }
  *status = BD_OK;
  return addr[dev];
}

extern "C" int bd_mobility_apply_noalloc(bd_ctx* c, const double* v, double* out) {
  if (!c || !v || !out) return BD_ERR_ARG;
  if (c->N > BD_NOALLOC_MAX_BEADS) return BD_ERR_CAPACITY;
  if (!c->hi_built || !c->Mt) return BD_ERR_STATE;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return BD_ERR_CUDA;
  if (dev != c->device) return BD_ERR_STATE;  // the context's device must be current
  int st;
  double* scratch = scratch_address(dev, &st);
  if (!scratch) return st;
  int NT = c->NT;
  if (c->Mt32)
    k_na_matvec<float><<<(unsigned)c->ntiles, 256, 0, c->stream>>>(c->Mt32, NT, c->N, v, scratch);
  else
    k_na_matvec<double><<<(unsigned)c->ntiles, 256, 0, c->stream>>>(c->Mt, NT, c->N, v, scratch);
  k_na_reduce1<<<dim3(NT, kSplit), 96, 0, c->stream>>>(NT, scratch);
  k_na_reduce2<<<NT, 96, 0, c->stream>>>(c->N, scratch, v, c->Dtr[0], c->Dtr[1], c->Dtr[2], out);
  c->launches += 3;
  return launch_ok(c);
}
