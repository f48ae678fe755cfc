// Trajectory, restart and property files in the reference's formats, and
// the per-chain unwrapped-coordinate properties they need.
//
// printTrajectory, printRestart, printExt, printVisc
// (shear/src/main26.c:870-925, 963-974, 1866-1880; the extensional tree's
// printVisc, extensional/src/main14.c:1886-1899, writes tauxx and tauyy
// instead of tauxy) write text files that the
// reference's analysis notebooks read; these calls write the same lines from
// the device-resident state (the formats are the reference's printf formats).
// The unwrapped chain coordinates follow the reference's loop in its main
// (shear/src/main26.c:75-85): p_0 = 0 and p_{j+1} = p_j + getNID(j, j+1),
// so each chain is unwrapped mirrored (getNID(i, j) = r_i - r_j); the
// extension max(px) - min(px) (calcExt, shear/src/main26.c:926-942) does not
// depend on that sign.  Centres of mass and gyration tensors are computed
// with initialised accumulators (the reference's calcCOM and calcRg start
// from uninitialised ones, so theirs are not reproducible).
#include <math.h>
#include <stdio.h>

#include <vector>

#include "bd_ctx.cuh"

using namespace bd;

#define CU(call) BD_CU(call)

// One thread per chain: unwrapped coordinates, x extension, centre of mass
// and gyration tensor (xx xy xz yy yz zz) of the unwrapped chain.
__global__ void k_chain_props(Lat l, const double* __restrict__ rx, const double* __restrict__ ry,
                              const double* __restrict__ rz, int Nb, int Nc, double* px,
                              double* py, double* pz, double* ext, double* com, double* rg) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= Nc) return;
  int b0 = c * Nb;
  px[b0] = 0.0;
  py[b0] = 0.0;
  pz[b0] = 0.0;
  for (int j = 0; j < Nb - 1; j++) {
    double dx, dy, dz;
    nid(l, rx, ry, rz, b0 + j, b0 + j + 1, dx, dy, dz);
    px[b0 + j + 1] = addx(px[b0 + j], dx);
    py[b0 + j + 1] = addx(py[b0 + j], dy);
    pz[b0 + j + 1] = addx(pz[b0 + j], dz);
  }
  double mx = px[b0], mn = px[b0], sx = 0, sy = 0, sz = 0;
  for (int j = 0; j < Nb; j++) {
    mx = fmax(mx, px[b0 + j]);
    mn = fmin(mn, px[b0 + j]);
    sx += px[b0 + j];
    sy += py[b0 + j];
    sz += pz[b0 + j];
  }
  ext[c] = mx - mn;
  double cx = sx / Nb, cy = sy / Nb, cz = sz / Nb;
  com[3 * c] = cx;
  com[3 * c + 1] = cy;
  com[3 * c + 2] = cz;
  double g[6] = {0, 0, 0, 0, 0, 0};
  for (int j = 0; j < Nb; j++) {
    double a = px[b0 + j] - cx, b = py[b0 + j] - cy, d = pz[b0 + j] - cz;
    g[0] += a * a;
    g[1] += a * b;
    g[2] += a * d;
    g[3] += b * b;
    g[4] += b * d;
    g[5] += d * d;
  }
  for (int k = 0; k < 6; k++) rg[6 * c + k] = g[k] / Nb;
}

static Lat out_lat(bd_ctx* c) {
  Lat l = c->lat;
  int treal = (int)(c->t % (unsigned long)c->tp);
  l.treal = treal;
  l.delx = c->p.edot * treal * c->p.dt;
  return l;
}

extern "C" {

int bd_chain_props(bd_ctx* c, double* px, double* ext, double* com, double* rg) {
  if (!c) return BD_ERR_ARG;
  int N = c->N, Nc = c->p.Nc, Nb = c->Nb;
  double* d = nullptr;
  size_t n = 3 * (size_t)N + 10 * (size_t)Nc;
  CU(cudaMalloc(&d, 8 * n));
  c->launches++;
  k_chain_props<<<(Nc + 127) / 128, 128, 0, c->stream>>>(out_lat(c), c->rx, c->ry, c->rz, Nb, Nc, d,
                                                         d + N, d + 2 * (size_t)N, d + 3 * (size_t)N,
                                                         d + 3 * (size_t)N + Nc,
                                                         d + 3 * (size_t)N + 4 * (size_t)Nc);
  std::vector<double> h(n);
  cudaError_t e = cudaMemcpyAsync(h.data(), d, 8 * n, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d);
  if (e != cudaSuccess) return BD_ERR_CUDA;
  if (px) std::copy(h.begin(), h.begin() + 3 * (size_t)N, px);
  if (ext) std::copy(h.begin() + 3 * (size_t)N, h.begin() + 3 * (size_t)N + Nc, ext);
  if (com)
    std::copy(h.begin() + 3 * (size_t)N + Nc, h.begin() + 3 * (size_t)N + 4 * (size_t)Nc, com);
  if (rg) std::copy(h.begin() + 3 * (size_t)N + 4 * (size_t)Nc, h.end(), rg);
  return check(c);
}

int bd_write_trajectory(bd_ctx* c, const char* path, unsigned long t) {
  if (!c || !path) return BD_ERR_ARG;
  int N = c->N;
  std::vector<double> x(N), y(N), z(N);
  std::vector<int> fl(N);
  int s;
  if ((s = bd_download_positions(c, x.data(), y.data(), z.data())) != BD_OK) return s;
  if ((s = bd_download_charges(c, nullptr, nullptr, fl.data())) != BD_OK) return s;
  const Lat& l = c->lat;
  double L = c->p.L;
  FILE* f = fopen(path, "a");
  if (!f) return BD_ERR_ARG;
  fprintf(f, "%d\n", N);
  fprintf(f,
          "Lattice=\"%lf %lf %lf %lf %lf %lf %lf %lf %lf\" Origin=\"%lf %lf %lf\" "
          "Properties=\"\" Time=%lu\n",
          l.L1x, l.L1y, 0.0, l.L2x, l.L2y, 0.0, 0.0, 0.0, L, -(l.L1x + l.L2x) / 2,
          -(l.L1y + l.L2y) / 2, -L / 2, t);
  for (int i = 0; i < N; i++) {
    if (fl[i] == 0)
      fprintf(f, "A %lf %lf %lf\n", x[i], y[i], z[i]);
    else if (fl[i] == 1)
      fprintf(f, "B %lf %lf %lf\n", x[i], y[i], z[i]);
  }
  return fclose(f) == 0 ? BD_OK : BD_ERR_ARG;
}

int bd_write_restart(bd_ctx* c, const char* path, unsigned long t) {
  if (!c || !path) return BD_ERR_ARG;
  int N = c->N;
  std::vector<double> x(N), y(N), z(N);
  int s;
  if ((s = bd_download_positions(c, x.data(), y.data(), z.data())) != BD_OK) return s;
  FILE* f = fopen(path, "w");
  if (!f) return BD_ERR_ARG;
  fprintf(f, "%d\n%lu\n", N, t);
  for (int i = 0; i < N; i++) fprintf(f, "A %lf %lf %lf\n", x[i], y[i], z[i]);
  return fclose(f) == 0 ? BD_OK : BD_ERR_ARG;
}

int bd_write_ext(bd_ctx* c, const char* path, unsigned long t, double strain) {
  if (!c || !path) return BD_ERR_ARG;
  std::vector<double> ext(c->p.Nc);
  int s;
  if ((s = bd_chain_props(c, nullptr, ext.data(), nullptr, nullptr)) != BD_OK) return s;
  FILE* f = fopen(path, "a");
  if (!f) return BD_ERR_ARG;
  for (int i = 0; i < c->p.Nc; i++) {
    double e = ext[i] / (c->Nb * c->p.qmax);
    fprintf(f, "%lu %lf %lf %lf\n", t, strain, e, pow(e, 2));
  }
  return fclose(f) == 0 ? BD_OK : BD_ERR_ARG;
}

int bd_write_visc(bd_ctx* c, const char* path, unsigned long t, int printperiod) {
  if (!c || !path || printperiod <= 0) return BD_ERR_ARG;
  double st[3];
  int s;
  if ((s = bd_download_stress(c, st)) != BD_OK) return s;
  FILE* f = fopen(path, "a");
  if (!f) return BD_ERR_ARG;
  if (c->p.flow == BD_FLOW_EXT) {
    // extensional tree: tauxx and tauyy, which it then clears
    // (extensional/src/main14.c:1886-1899)
    fprintf(f, "%lu %lf %lf\n", t, st[0] / ((double)printperiod), st[1] / ((double)printperiod));
    if (fclose(f) != 0) return BD_ERR_ARG;
    CU(cudaMemsetAsync(c->stress, 0, 16, c->stream));
    return check(c);
  }
  fprintf(f, "%lu %lf\n", t, st[2] / ((double)printperiod));
  if (fclose(f) != 0) return BD_ERR_ARG;
  return bd_reset_stress(c);
}

}  // extern "C"
