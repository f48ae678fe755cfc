// Charge mean-squared displacement: calcMSD (shear/src/main26.c:2494-2637)
// on the GPU.
//
// Input: the charge-displacement log as the reference reads it from its CH
// file, nsamp = Ncharges (Tmax + 1) records (x, y, z) in file order (record
// i Ncharges + j is charge j's displacement over print interval i).  The
// reference rearranges the records into a flat array v with charge 0 at
// offset 0 and charge j > 0 at offset j (Tmax + 1) (entries i = 1..Tmax), but
// reads charge q's window from offset q Tmax; this keeps that layout and
// that indexing, so the averages are the reference's.  For every lag i and
// each of the first nq = min(Ncharges, 25) charges it averages
// |sum_{k<i} v[j + k + q Tmax]|^2 over the starts j = MSDstart .. wmax-i-1;
// the window sums are differences of one prefix sum of v (FP64) instead of
// the reference's O(i) loops, which makes the whole analysis O(nq Tmax^2)
// rather than O(nq Tmax^3).  One CTA per lag, fixed-order block reductions.
#include <math.h>

#include <vector>

#include "bd_ctx.cuh"

#define CU(call) BD_CU(call)

__global__ void __launch_bounds__(256) k_msd_lag(const double* __restrict__ P, int Tmax, int wmax,
                                                 int nq, int MSDstart, double* out) {
  int i = blockIdx.x + 1;  // lag
  int n = wmax - i - MSDstart;
  __shared__ double red[4][256];
  double s[4] = {0, 0, 0, 0};
  if (n > 0) {
    for (long long e = threadIdx.x; e < (long long)nq * n; e += blockDim.x) {
      int q = (int)(e / n), j = MSDstart + (int)(e % n);
      size_t a = (size_t)q * Tmax + j, b = a + i;
      double dx = P[3 * b] - P[3 * a], dy = P[3 * b + 1] - P[3 * a + 1],
             dz = P[3 * b + 2] - P[3 * a + 2];
      s[1] += dx * dx;
      s[2] += dy * dy;
      s[3] += dz * dz;
      s[0] += dx * dx + dy * dy + dz * dz;
    }
  }
  for (int c = 0; c < 4; c++) red[c][threadIdx.x] = s[c];
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o)
      for (int c = 0; c < 4; c++) red[c][threadIdx.x] += red[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[4 * (size_t)blockIdx.x + threadIdx.x] = n > 0 ? red[threadIdx.x][0] / n : 0.0;
}

extern "C" {

int bd_msd(const double* w, int ncharges, int Tmax, int MSDstart, double* avg) {
  if (!w || !avg || ncharges <= 0 || Tmax <= 0 || MSDstart < 0) return BD_ERR_ARG;
  int wmax = Tmax + 1;
  size_t nsamp = (size_t)ncharges * wmax;
  int nq = ncharges >= 25 ? 25 : ncharges;
  int nlag = wmax - MSDstart - 1;
  if (nlag <= 0) return BD_ERR_ARG;
  // the reference's rearrangement into v, then one prefix sum (host, FP64)
  std::vector<double> v(3 * nsamp, 0.0), P(3 * (nsamp + 1), 0.0);
  for (int j = 0; j < ncharges; j++)
    for (int i = 1; i < Tmax + 1; i++) {
      size_t ind1 = j == 0 ? (size_t)i : (size_t)j * (Tmax + 1) + i;
      size_t ind2 = (size_t)i * ncharges + j;
      for (int a = 0; a < 3; a++) v[3 * ind1 + a] = w[3 * ind2 + a];
    }
  for (size_t m = 0; m < nsamp; m++)
    for (int a = 0; a < 3; a++) P[3 * (m + 1) + a] = P[3 * m + a] + v[3 * m + a];
  double *dP = nullptr, *dout = nullptr;
  CU(cudaMalloc(&dP, 8 * P.size()));
  CU(cudaMalloc(&dout, 32 * (size_t)nlag));
  CU(cudaMemcpy(dP, P.data(), 8 * P.size(), cudaMemcpyHostToDevice));
  k_msd_lag<<<nlag, 256>>>(dP, Tmax, wmax, nq, MSDstart, dout);
  std::vector<double> o(4 * (size_t)nlag);
  cudaError_t e = cudaMemcpy(o.data(), dout, 32 * (size_t)nlag, cudaMemcpyDeviceToHost);
  cudaFree(dP);
  cudaFree(dout);
  if (e != cudaSuccess) return BD_ERR_CUDA;
  // avg[i-1] = {MSD, x, y, z} / nq for lag i, as the reference's output rows
  for (int i = 0; i < nlag; i++)
    for (int c = 0; c < 4; c++) avg[4 * (size_t)i + c] = o[4 * (size_t)i + c] / nq;
  return BD_OK;
}

}  // extern "C"
