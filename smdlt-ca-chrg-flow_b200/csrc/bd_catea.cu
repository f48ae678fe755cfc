// CA-TEA parameter sampling: ewaldBin + CATEA + printTEA
// (shear/src/main26.c:975-1381, 1807-1826; extensional/src/main14.c:1009-1415).
//
// bd_ewald_bin returns what the reference's ewaldBin accumulates (eps and
// rowsum) for the current positions, computed by the tile kernels in
// bd_mobility.cu.  bd_catea adds one sample as CATEA does: the beta of the
// truncated expansion from the normalised eps, the per-bead C_i from rowsum,
// summed into running totals of the current strain bin; bd_catea_averages
// and bd_write_decomp give those averages the way printTEA writes them
// (beta = brun / gwcount, C = Crun / (Nc gwcount)), and bd_catea_apply loads
// them as the TEA parameters of the step (resetAverage,
// shear/src/main26.c:1827-1840, then the running sums restart).
// The normalisation 9 N^2 - 3 N is evaluated in 64-bit arithmetic (the
// reference's int expression overflows above 15 449 beads).
#include <math.h>
#include <stdio.h>

#include <vector>

#include "bd_ctx.cuh"

using namespace bd;

static void catea_ensure(bd_ctx* c) {
  size_t nb = (size_t)c->sbins + 1;
  if (c->cat_brun.size() != nb) {
    c->cat_brun.assign(nb, 0.0);
    c->cat_gw.assign(nb, 0);
    c->cat_crun.assign(nb * 3 * (size_t)c->Nb, 0.0);
  }
}

extern "C" {

int bd_ewald_bin(bd_ctx* c, double* eps, double* rowsum) {
  if (!c || !eps || !rowsum) return BD_ERR_ARG;
  std::vector<double> rs;
  int s;
  if ((s = ewald_bin(c, eps, rs)) != BD_OK) return s;
  for (size_t i = 0; i < rs.size(); i++) rowsum[i] = rs[i];
  return check(c);
}

int bd_catea(bd_ctx* c, double strain, double* beta_out) {
  if (!c) return BD_ERR_ARG;
  catea_ensure(c);
  double eps;
  std::vector<double> rs;
  int s;
  if ((s = ewald_bin(c, &eps, rs)) != BD_OK) return s;
  if ((s = check(c)) != BD_OK) return s;
  long long N = c->N;
  int bin = (int)floor(strain / c->strain_interval);
  if (bin > c->sbins) bin = c->sbins;
  if (bin < 0) return BD_ERR_ARG;
  eps /= (double)(9 * N * N - 3 * N);
  double eps2 = eps * eps, row = 3.0 * N;
  double b = (1.0 - sqrt(1.0 - (row * eps2 - row * eps))) / (row * eps2 - row * eps);
  c->cat_brun[bin] += b;
  size_t m = 3 * (size_t)c->Nb;
  for (size_t i = 0; i < 3 * (size_t)N; i++)
    c->cat_crun[(size_t)bin * m + i % m] += sqrt(1.0 / (1.0 + rs[i] * b * b));
  c->cat_gw[bin]++;
  if (beta_out) *beta_out = b;
  return BD_OK;
}

int bd_catea_averages(bd_ctx* c, int* counts, double* beta, double* C) {
  if (!c) return BD_ERR_ARG;
  catea_ensure(c);
  size_t m = 3 * (size_t)c->Nb;
  for (int i = 0; i <= c->sbins; i++) {
    int g = c->cat_gw[i];
    if (counts) counts[i] = g;
    if (beta) beta[i] = g > 0 ? c->cat_brun[i] / g : 0.0;
    if (C)
      for (size_t j = 0; j < m; j++)
        C[(size_t)i * m + j] = g > 0 ? c->cat_crun[(size_t)i * m + j] / ((double)c->p.Nc * g) : 0.0;
  }
  return BD_OK;
}

int bd_write_decomp(bd_ctx* c, const char* path, unsigned long t) {
  if (!c || !path) return BD_ERR_ARG;
  catea_ensure(c);
  FILE* f = fopen(path, "w");
  if (!f) return BD_ERR_ARG;
  size_t m = 3 * (size_t)c->Nb;
  fprintf(f, "%lu\n", t);
  for (int i = 0; i <= c->sbins; i++) {
    int g = c->cat_gw[i];
    if (g > 0) {
      fprintf(f, "%d %d %.12e\n", i, g, c->cat_brun[i] / g);
      for (int j = 0; j < c->Nb; j++) {
        double d = (double)c->p.Nc * g;
        fprintf(f, "%d %.12e %.12e %.12e\n", j, c->cat_crun[(size_t)i * m + 3 * j] / d,
                c->cat_crun[(size_t)i * m + 3 * j + 1] / d, c->cat_crun[(size_t)i * m + 3 * j + 2] / d);
      }
    } else {
      fprintf(f, "%d %d %.12e\n", i, 0, 0.0);
      for (int j = 0; j < c->Nb; j++) fprintf(f, "%d %.12e %.12e %.12e\n", j, 0.0, 0.0, 0.0);
    }
  }
  return fclose(f) == 0 ? BD_OK : BD_ERR_ARG;
}

int bd_catea_apply(bd_ctx* c) {
  if (!c) return BD_ERR_ARG;
  catea_ensure(c);
  size_t m = 3 * (size_t)c->Nb;
  std::vector<double> Cb(m);
  for (int i = 0; i <= c->sbins; i++) {
    int g = c->cat_gw[i];
    double b = c->cat_brun[i] / g;  // the reference divides without a guard
    for (size_t j = 0; j < m; j++) Cb[j] = c->cat_crun[(size_t)i * m + j] / ((double)c->p.Nc * g);
    int s;
    if ((s = bd_set_tea(c, i, b, Cb.data())) != BD_OK) return s;
    c->cat_brun[i] = 0.0;
    c->cat_gw[i] = 0;
    for (size_t j = 0; j < m; j++) c->cat_crun[(size_t)i * m + j] = 0.0;
  }
  return BD_OK;
}

}  // extern "C"
