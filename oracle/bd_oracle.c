/* FP64 CPU restatement of the reference's per-step Brownian-dynamics path.
 *
 * TEST INFRASTRUCTURE ONLY (see bd_oracle.h).  Each routine follows the
 * arithmetic of the cited reference routine operation by operation, so that
 * results that the reference decides by comparisons (neighbour sets,
 * charge-hop acceptances) come out bit-identical, and floating-point results
 * agree to rounding.  Compiled without FMA contraction (plain x86-64 gcc
 * -O2 emits no FMA), like the reference.
 */
#include "bd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define EPK 0.9624 /* strain period constant, shear/src/Parameters.h:37 */

/* ---- configuration and lattice ------------------------------------------ */

/* initLattice: shear/src/Initialization.c:217-298,
 * extensional/src/Initialization.c:236-287 (period, initial cell corners and
 * the far-field lookup-grid bins). */
void bdo_init(bdo_sys *s, int flow, int Nb, int Nc, double L, double edot,
              double dt, int nt_avg, double bin_size, int spring,
              double kappas, double qmax, double kappab, double epsilon,
              double lambda_b, double lambda_d, double barrier,
              double barrier2, int MStep) {
  memset(s, 0, sizeof(*s));
  s->flow = flow;
  s->Nb = Nb;
  s->Nc = Nc;
  s->N = Nb * Nc;
  s->L = L;
  s->edot = edot;
  s->dt = dt;
  s->spring = spring;
  s->kappas = kappas;
  s->qmax = qmax;
  s->qmax2 = qmax * qmax;
  s->kappab = kappab;
  s->epsilon = epsilon;
  s->lambda_b = lambda_b;
  s->lambda_d = lambda_d;
  s->kappa_d = 1 / lambda_d;
  s->barrier = barrier;
  s->barrier2 = barrier2;
  s->MStep = MStep;
  s->nt_avg = nt_avg;
  /* initVerlet: sigma=2, rv=3 sigma; shear LJ cut 2.5 sigma, ext WCA
   * r2cut=5.03968 (shear/src/Initialization.c:300-316,
   * extensional/src/Initialization.c:289-305). */
  {
    double sigma = 2.0, rc;
    if (flow == 0) {
      rc = 2.5 * sigma;
      s->r2cut = rc * rc;
    } else {
      s->r2cut = 5.03968;
      rc = sqrt(s->r2cut);
    }
    s->rv = 3.0 * sigma;
    s->rnew = 0.5 * (s->rv - rc);
  }
  s->tp = (int)(EPK / edot / dt);
  double th = 90.0 - (45.0 + (flow == 0 ? 0.0 : 31.7));
  th *= M_PI / 180;
  double p0[3][2];
  p0[0][0] = -sqrt(2) / 2 * L * cos(th);
  p0[0][1] = sqrt(2) / 2 * L * sin(th);
  p0[1][0] = -sqrt(2) / 2 * L * sin(th);
  p0[1][1] = -sqrt(2) / 2 * L * cos(th);
  p0[2][0] = sqrt(2) / 2 * L * cos(th);
  p0[2][1] = -sqrt(2) / 2 * L * sin(th);
  double xmax, ymax, zmax;
  int treal = s->tp;
  if (flow == 0) {
    ymax = L / 2;
    xmax = L / 2 * edot * treal * dt;
  } else {
    ymax = -p0[1][1];
    xmax = p0[2][0] * exp(edot * treal * dt);
  }
  zmax = L / 2;
  s->bin_size = bin_size;
  s->bsx = bin_size;
  s->bsy = bin_size;
  s->bsz = bin_size;
  s->nbx = 2 * ceil(xmax / s->bsx) + 1;
  s->bsx = xmax / ((s->nbx - 1) / 2);
  s->nhx = (s->nbx - 1) / 2;
  s->nby = 2 * ceil(ymax / s->bsy) + 1;
  s->bsy = ymax / ((s->nby - 1) / 2);
  s->nhy = (s->nby - 1) / 2;
  s->nbz = 2 * ceil(zmax / s->bsz) + 1;
  s->bsz = zmax / ((s->nbz - 1) / 2);
  s->nhz = (s->nbz - 1) / 2;
  s->nbins = s->nbx * s->nby * s->nbz;
  bdo_lattice(s, 0);
}

/* updateLattice: shear/src/main26.c:1382-1408 (affine shear of the cell
 * corners), extensional/src/main14.c:1426-1450 (exponential stretch, then the
 * cell expressed in the frame rotated by theta = atan(L1y/L1x)). */
void bdo_lattice(bdo_sys *s, unsigned long t) {
  double th0 = 90.0 - (45.0 + (s->flow == 0 ? 0.0 : 31.7));
  th0 *= M_PI / 180;
  double L = s->L;
  double p0[3][2], p[3][2];
  p0[0][0] = -sqrt(2) / 2 * L * cos(th0);
  p0[0][1] = sqrt(2) / 2 * L * sin(th0);
  p0[1][0] = -sqrt(2) / 2 * L * sin(th0);
  p0[1][1] = -sqrt(2) / 2 * L * cos(th0);
  p0[2][0] = sqrt(2) / 2 * L * cos(th0);
  p0[2][1] = -sqrt(2) / 2 * L * sin(th0);
  int treal = (int)(t % (unsigned long)s->tp);
  s->t = t;
  if (s->flow == 0) {
    for (int a = 0; a < 3; a++) {
      p[a][1] = p0[a][1];
      p[a][0] = p0[a][0] + p[a][1] * s->edot * treal * s->dt;
    }
  } else {
    for (int a = 0; a < 3; a++) {
      p[a][0] = p0[a][0] * exp(s->edot * treal * s->dt);
      p[a][1] = p0[a][1] * exp(-s->edot * treal * s->dt);
    }
  }
  for (int a = 0; a < 2; a++) {
    s->L1[a] = p[2][a] - p[1][a];
    s->L2[a] = p[0][a] - p[1][a];
  }
  if (s->flow == 0) {
    s->L1xp = s->L1[0];
    s->L2xp = s->L2[0];
    s->L1yp = s->L1[1];
    s->L2yp = s->L2[1];
    s->detL = s->L2yp * s->L1xp * L;
    s->theta = 0.0;
    s->cth = 1.0;
    s->sth = 0.0;
  } else {
    double th = atan(s->L1[1] / s->L1[0]);
    s->theta = th;
    s->cth = cos(th);
    s->sth = sin(th);
    s->L1xp = s->L1[0] * cos(th) + s->L1[1] * sin(th);
    s->L2xp = s->L2[0] * cos(th) + s->L2[1] * sin(th);
    s->L1yp = -s->L1[0] * sin(th) + s->L1[1] * cos(th);
    s->L2yp = -s->L2[0] * sin(th) + s->L2[1] * cos(th);
    s->detL = L * (-s->L1yp * s->L2xp + s->L1xp * s->L2yp);
  }
  s->delx = s->edot * treal * s->dt;
}

/* applyPBC: shear/src/main26.c:1409-1428, extensional/src/main14.c:1451-1461 */
void bdo_apply_pbc(const bdo_sys *s, double *rx, double *ry, double *rz) {
  for (int a = 0; a < s->N; a++) {
    rx[a] -= s->L2xp * round(ry[a] / s->L2yp);
    if (s->flow == 0) {
      if (ry[a] > s->L2yp / 2) {
        rx[a] -= s->delx;
        ry[a] -= s->L2yp * round(ry[a] / s->L2yp);
      } else if (ry[a] < -s->L2yp / 2) {
        rx[a] += s->delx;
        ry[a] -= s->L2yp * round(ry[a] / s->L2yp);
      }
    } else {
      ry[a] -= s->L2yp * round(ry[a] / s->L2yp);
    }
    rx[a] -= s->L1xp * round((rx[a] - ry[a] * s->L2xp / s->L2yp) / s->L1xp);
    rz[a] -= s->L * round(rz[a] / s->L);
  }
}

/* transformCoords (inverse=0) / inverseCoords (inverse=1):
 * extensional/src/main14.c:1514-1535 */
void bdo_rotate(const bdo_sys *s, double *rx, double *ry, int inverse) {
  double c = s->cth, sn = s->sth;
  for (int a = 0; a < s->N; a++) {
    double x = rx[a], y = ry[a];
    if (!inverse) {
      rx[a] = x * c + y * sn;
      ry[a] = -x * sn + y * c;
    } else {
      rx[a] = x * c - y * sn;
      ry[a] = x * sn + y * c;
    }
  }
}

/* getNID: shear/src/main26.c:1429-1457, extensional/src/main14.c:1462-1480 */
static inline void nid(const bdo_sys *s, const double *rx, const double *ry,
                       const double *rz, int i, int j, double *o) {
  double dx = rx[i] - rx[j], dy = ry[i] - ry[j], dz = rz[i] - rz[j];
  dx -= s->L2xp * round(dy / s->L2yp);
  if (s->flow == 0) {
    if (dy > s->L2yp / 2) {
      dx -= s->delx;
      dy -= s->L2yp * round(dy / s->L2yp);
    } else if (dy < -s->L2yp / 2) {
      dx += s->delx;
      dy -= s->L2yp * round(dy / s->L2yp);
    }
    dx -= s->L1xp * round(dx / s->L1xp);
    dz -= s->L * round(dz / s->L);
    o[0] = dx;
    o[1] = dy;
    o[2] = dz;
  } else {
    dy -= s->L2yp * round(dy / s->L2yp);
    dx -= s->L1xp * round(dx / s->L1xp);
    dz -= s->L * round(dz / s->L);
    o[0] = dx * s->cth - dy * s->sth;
    o[1] = dx * s->sth + dy * s->cth;
    o[2] = dz;
  }
}

void bdo_nid(const bdo_sys *s, const double *rx, const double *ry,
             const double *rz, int i, int j, double *out) {
  nid(s, rx, ry, rz, i, j, out);
}

/* getNIDbin: shear/src/main26.c:1458-1497, extensional/src/main14.c:1481-1513 */
void bdo_nidbin(const bdo_sys *s, const double *rx, const double *ry,
                const double *rz, int i, int j, double *o) {
  double dx = rx[i] - rx[j], dy = ry[i] - ry[j], dz = rz[i] - rz[j];
  int treal = (int)(s->t % (unsigned long)s->tp);
  int nmax = (treal <= s->tp / 2) ? 1 : 2;
  dz -= s->L * round(dz / s->L);
  double dxmin = dx, dymin = dy, rmin = sqrt(dx * dx + dy * dy);
  if (s->flow == 0) {
    if (dy > s->L2yp / 2)
      dx -= s->delx;
    else if (dy < -s->L2yp / 2)
      dx += s->delx;
  }
  for (int nx = -nmax; nx < nmax + 1; nx++)
    for (int ny = -nmax; ny < nmax + 1; ny++) {
      double dxp = dx + nx * s->L1xp + ny * s->L2xp;
      double dyp = dy + ny * s->L2yp;
      double rp = sqrt(dxp * dxp + dyp * dyp);
      if (rp < rmin) {
        dxmin = dxp;
        dymin = dyp;
        rmin = rp;
      }
    }
  if (s->flow == 0) {
    o[0] = dxmin;
    o[1] = dymin;
  } else {
    o[0] = dxmin * s->cth - dymin * s->sth;
    o[1] = dxmin * s->sth + dymin * s->cth;
  }
  o[2] = dz;
}

/* binij: shear/src/main26.c:1518-1529.  The reference range-checks neither
 * the per-axis bins nor the flattened index, so a displacement just outside
 * the table on one axis aliases to a neighbouring row of the table; that
 * flattened index is reproduced.  Returns -1 (instead of reading outside the
 * table) only when the flattened index itself is out of range. */
int bdo_binij(const bdo_sys *s, const double *rx, const double *ry,
              const double *rz, int i, int j) {
  double v[3];
  bdo_nidbin(s, rx, ry, rz, j, i, v);
  int bx = round(v[0] / s->bsx) + s->nhx;
  int by = round(v[1] / s->bsy) + s->nhy;
  int bz = round(v[2] / s->bsz) + s->nhz;
  long b = (long)s->nby * s->nbz * bx + (long)s->nbz * by + bz;
  if (b < 0 || b >= s->nbins) return -1;
  return (int)b;
}

/* ---- forces ------------------------------------------------------------- */

/* bondforce: shear/src/main26.c:541-618, extensional/src/main14.c:549-624.
 * The shear tree sets kappas = 200 on entry (shear/src/main26.c:544).
 * stress[] accumulates tauxx, tauyy and (shear only) tauxy.
 * Returns 1 on FENE overstretch (where the reference prints and exits). */
int bdo_bond(const bdo_sys *s, const double *rx, const double *ry,
             const double *rz, double *fx, double *fy, double *fz,
             double *stress) {
  double kappas = (s->flow == 0) ? 200 : s->kappas;
  int Nb = s->Nb;
  for (int c = 0; c < s->Nc; c++)
    for (int b = 1; b < Nb; b++) {
      double v[3];
      nid(s, rx, ry, rz, Nb * c + b, Nb * c + b - 1, v);
      double rr = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      double r = sqrt(rr), Fs;
      if (s->spring == 1) {
        if (rr > s->qmax2) return 1;
        Fs = -kappas / (1.0 - rr / s->qmax2);
      } else {
        Fs = -kappas * (r - s->qmax) / r;
      }
      fx[Nb * c + b] += Fs * v[0];
      fy[Nb * c + b] += Fs * v[1];
      fz[Nb * c + b] += Fs * v[2];
      fx[Nb * c + b - 1] += -Fs * v[0];
      fy[Nb * c + b - 1] += -Fs * v[1];
      fz[Nb * c + b - 1] += -Fs * v[2];
      stress[0] -= 2.0 * v[0] * Fs * v[0];
      stress[1] -= 2.0 * v[1] * Fs * v[1];
      if (s->flow == 0) stress[2] -= 2.0 * v[0] * Fs * v[1];
    }
  if (s->kappab > 0.0) {
    for (int c = 0; c < s->Nc; c++)
      for (int b = 1; b < Nb - 1; b++) {
        double n1[3], n2[3];
        int a = Nb * c + b;
        nid(s, rx, ry, rz, a, a - 1, n1);
        nid(s, rx, ry, rz, a, a + 1, n2);
        double a1 = sqrt(n1[0] * n1[0] + n1[1] * n1[1] + n1[2] * n1[2]);
        double a2 = sqrt(n2[0] * n2[0] + n2[1] * n2[1] + n2[2] * n2[2]);
        double var = (n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2]) / (a1 * a2);
        double thb = M_PI - acos(var);
        double co = -s->kappab * thb / sqrt(1 - var * var);
        double *f[3] = {fx, fy, fz};
        for (int d = 0; d < 3; d++) {
          f[d][a] += co * ((n1[d] + n2[d]) / (a1 * a2) - var * (n1[d] / (a1 * a1) + n2[d] / (a2 * a2)));
          f[d][a - 1] += co * (var * n1[d] / (a1 * a1) - n2[d] / (a1 * a2));
          f[d][a + 1] += co * (var * n2[d] / (a2 * a2) - n1[d] / (a1 * a2));
        }
        /* the reference's bending virial, including its use of z components
         * in the yy sum (shear/src/main26.c:606-613) */
        stress[0] += n1[0] * co * (var * n1[0] / (a1 * a1) - n2[0] / (a1 * a2));
        stress[0] -= n1[0] * co * ((n1[0]) / (a1 * a2) - var * (n1[0] / (a1 * a1)));
        stress[0] += n2[0] * co * ((n2[0]) / (a1 * a2) - var * (n2[0] / (a2 * a2)));
        stress[0] -= n2[0] * co * (var * n2[0] / (a2 * a2) - n1[0] / (a1 * a2));
        stress[1] += n1[1] * co * (var * n1[1] / (a1 * a1) - n2[1] / (a1 * a2));
        stress[1] -= n1[1] * co * ((n1[2]) / (a1 * a2) - var * (n1[2] / (a1 * a1)));
        stress[1] += n2[1] * co * ((n2[2]) / (a1 * a2) - var * (n2[2] / (a2 * a2)));
        stress[1] -= n2[1] * co * (var * n2[1] / (a2 * a2) - n1[1] / (a1 * a2));
      }
  }
  return 0;
}

/* LJforce: shear LJ 12 eps (r6^2 - r6)/r^2 (shear/src/main26.c:619-681);
 * ext WCA 48 eps (r6^2 - r6/2)/r^2 (extensional/src/main14.c:625-685);
 * both with sigma^2 = 4 and the cutoff test on the Verlet half list. */
void bdo_ev(const bdo_sys *s, const double *rx, const double *ry,
            const double *rz, const int *counts, const int *rows, int maxnb,
            double *fx, double *fy, double *fz, double *stress) {
  for (int i = 0; i < s->N; i++)
    for (int k = 0; k < counts[i]; k++) {
      int j = rows[(size_t)i * maxnb + k];
      double v[3];
      nid(s, rx, ry, rz, i, j, v);
      double rr = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      if (rr < s->r2cut) {
        double ratio = 4.00 / rr;
        double r6 = ratio * ratio * ratio, co;
        if (s->flow == 0)
          co = (12 * s->epsilon / rr) * (r6 * r6 - r6);
        else
          co = (48.0 * s->epsilon / rr) * (r6 * r6 - 0.5 * r6);
        fx[i] += co * v[0];
        fy[i] += co * v[1];
        fz[i] += co * v[2];
        fx[j] -= co * v[0];
        fy[j] -= co * v[1];
        fz[j] -= co * v[2];
        stress[0] -= 2.0 * v[0] * co * v[0];
        stress[1] -= 2.0 * v[1] * co * v[1];
        if (s->flow == 0) stress[2] -= 2.0 * v[0] * co * v[1];
      }
    }
}

/* coulombForce: Debye-Hueckel over all charged pairs, no cutoff
 * (shear/src/main26.c:1891-1925).  q[] holds the bead charges (the reference
 * uses 0/1 flags). */
void bdo_coulomb(const bdo_sys *s, const double *rx, const double *ry,
                 const double *rz, const double *q, double *fx, double *fy,
                 double *fz) {
  for (int i = 0; i < s->N; i++)
    for (int j = i + 1; j < s->N; j++) {
      if (q[i] != 0 && q[j] != 0) {
        double v[3];
        nid(s, rx, ry, rz, i, j, v);
        double rr = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        double r = sqrt(rr);
        double Fc = s->lambda_b * q[i] * q[j] * exp(-s->kappa_d * r) * (1 + r * s->kappa_d) / rr;
        fx[i] += Fc * v[0] / r;
        fy[i] += Fc * v[1] / r;
        fz[i] += Fc * v[2] / r;
        fx[j] -= Fc * v[0] / r;
        fy[j] -= Fc * v[1] / r;
        fz[j] -= Fc * v[2] / r;
      }
    }
}

/* verletlist: half list j > i with |NID| < rv (shear/src/main26.c:682-707).
 * Returns -1 if a row would exceed maxnb. */
int bdo_verlet(const bdo_sys *s, const double *rx, const double *ry,
               const double *rz, int *counts, int *rows, int maxnb) {
  for (int i = 0; i < s->N; i++) counts[i] = 0;
  for (int i = 0; i < s->N - 1; i++)
    for (int j = i + 1; j < s->N; j++) {
      double v[3];
      nid(s, rx, ry, rz, i, j, v);
      double r = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      if (r < s->rv) {
        if (counts[i] >= maxnb) return -1;
        rows[(size_t)i * maxnb + counts[i]] = j;
        counts[i]++;
      }
    }
  return 0;
}

/* checkVerlet: rebuild when any accumulated displacement exceeds rnew
 * (shear/src/main26.c:858-869).  Returns 1 when a rebuild is due. */
int bdo_check_verlet(const bdo_sys *s, const double *dxv, const double *dyv,
                     const double *dzv) {
  for (int i = 0; i < s->N; i++) {
    double d = sqrt(dxv[i] * dxv[i] + dyv[i] * dyv[i] + dzv[i] * dzv[i]);
    if (d > s->rnew) return 1;
  }
  return 0;
}

/* ---- hydrodynamic mobility ---------------------------------------------- */

/* Wave vectors of the k-space mobility sum and their 3x3 coefficients
 * (shear/src/main26.c:1557-1652; ext reciprocal of the rotated lattice,
 * extensional/src/main14.c:1575-1670; identical loops in gridHI.c:38-144),
 * including the reference's bound scans, the halving of the kx = 0 plane and
 * the zeroed k = 0 term.  Returns nk and malloc'd M2[9 nk], kv[3 nk]. */
static void kvectors(const bdo_sys *s, double boxvol, double rkkcut, double rkcut,
                     double alpha2, double alpha4, int *nk_out, double **M2_out,
                     double **kv_out) {
  double L = s->L;
  const double *L1 = s->L1, *L2 = s->L2;
  int kxmax = ceil(rkcut * s->detL / (M_PI * 2.0 * L * L2[1]));
  int kymax = ceil(rkcut * s->detL / (M_PI * 2.0 * L * L1[0]));
  int kzmax = ceil(rkcut * L / (M_PI * 2.0));
  int nyw = 2 * kymax + 1;
  /* one spare row so the reference's kxmax increment never reads past */
  int *kyup = calloc(kxmax + 2, sizeof(int)), *kylo = calloc(kxmax + 2, sizeof(int));
  int *kzup = calloc((size_t)(kxmax + 2) * nyw, sizeof(int));
  int *kzlo = calloc((size_t)(kxmax + 2) * nyw, sizeof(int));
  double kcoeff = (s->flow == 0) ? M_PI * 2.0 : M_PI * 2.0 / s->detL;
#define KVEC(kx, ky, rkx, rky)                                   \
  do {                                                           \
    if (s->flow == 0) {                                          \
      rky = kcoeff * (kx - ky * (L2[0] / L1[0])) / L2[1];         \
      rkx = kcoeff * ky / L1[0];                                 \
    } else {                                                     \
      rkx = kcoeff * L * (kx * L2[1] - ky * L1[1]);              \
      rky = kcoeff * L * (-kx * L2[0] + ky * L1[0]);             \
    }                                                            \
  } while (0)
  for (int kx = 0; kx < kxmax + 1; kx++) {
    int ylo = 0, yup = 0;
    for (int ky = -kymax; ky < kymax + 1; ky++) {
      double rkx, rky;
      KVEC(kx, ky, rkx, rky);
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
    int kx = 0;
    while (kyup[kx] != -kymax && kx <= (int)(rkcut * s->detL / (M_PI * 2.0 * L * s->L2yp))) {
      kxmax = kx;
      kx++;
    }
  }
  kxmax++;
  int nk = 0;
  for (int kx = 0; kx < kxmax + 1; kx++)
    for (int ky = kylo[kx]; ky < kyup[kx] + 1; ky++)
      for (int kz = kzlo[nyw * kx + ky + kymax]; kz < kzup[nyw * kx + ky + kymax] + 1; kz++) nk++;
  double *M2 = calloc((size_t)9 * (nk + 1), sizeof(double));
  double *kv = calloc((size_t)3 * (nk + 1), sizeof(double));
  nk = 0;
  for (int kx = 0; kx < kxmax + 1; kx++)
    for (int ky = kylo[kx]; ky < kyup[kx] + 1; ky++) {
      double rkx, rky;
      KVEC(kx, ky, rkx, rky);
      double rkxy = rkx * rkx + rky * rky;
      for (int kz = kzlo[nyw * kx + ky + kymax]; kz < kzup[nyw * kx + ky + kymax] + 1; kz++) {
        double rkz = kz * M_PI * 2.0 / L, rkk = rkxy + rkz * rkz;
        double m2 = 2.0 * (1.0 - rkk / 3.0) * (1.0 + rkk / (4.0 * alpha2) + rkk * rkk / (8.0 * alpha4)) * 6.0 * M_PI / rkk * exp(-rkk / (4.0 * alpha2));
        double *m = M2 + 9 * nk;
        m[0] = m2 * (1 - rkx * rkx / rkk) / boxvol;
        m[1] = m2 * (-rkx * rky / rkk) / boxvol;
        m[2] = m2 * (-rkx * rkz / rkk) / boxvol;
        m[3] = m2 * (-rky * rkx / rkk) / boxvol;
        m[4] = m2 * (1 - rky * rky / rkk) / boxvol;
        m[5] = m2 * (-rky * rkz / rkk) / boxvol;
        m[6] = m2 * (-rkz * rkx / rkk) / boxvol;
        m[7] = m2 * (-rkz * rky / rkk) / boxvol;
        m[8] = m2 * (1 - rkz * rkz / rkk) / boxvol;
        kv[3 * nk] = rkx;
        kv[3 * nk + 1] = rky;
        kv[3 * nk + 2] = rkz;
        nk++;
      }
    }
#undef KVEC
  {
    int c = 0;
    for (int ky = kylo[0]; ky < kyup[0] + 1; ky++)
      for (int kz = kzlo[ky + kymax]; kz < kzup[ky + kymax] + 1; kz++) {
        for (int a = 0; a < 9; a++) M2[9 * c + a] /= 2.0;
        if (ky == 0 && kz == 0)
          for (int a = 0; a < 9; a++) M2[9 * c + a] = 0.0;
        c++;
      }
  }
  free(kyup);
  free(kylo);
  free(kzup);
  free(kzlo);
  *nk_out = nk;
  *M2_out = M2;
  *kv_out = kv;
}

/* calcHI: dense 3N x 3N Rotne-Prager-Yamakawa mobility with Beenakker's Ewald
 * split (shear/src/main26.c:1530-1806, extensional/src/main14.c:1548-1824).
 * Pairs whose minimum image is closer than 12 get the explicit real-space
 * image sum plus the explicit k-space cosine sum; other pairs copy the
 * lookup-table tensor of their displacement bin.  grid holds nt_avg frames of
 * nbins 3x3 tensors.  M is row-major 9 N^2 (block (i,j) at 9N i + 9 j);
 * only the upper blocks and the diagonal entries of the diagonal blocks are
 * written, as in the reference. */
static void calc_hi_impl(const bdo_sys *s, const double *rx, const double *ry,
                         const double *rz, const double *grid, double *M, int all_pairs);

void bdo_calc_hi(const bdo_sys *s, const double *rx, const double *ry,
                 const double *rz, const double *grid, double *M) {
  calc_hi_impl(s, rx, ry, rz, grid, M, 0);
}

/* The Ewald-summed RPY tensor for every pair (no lookup table) with the self
 * term summed over every image but the origin and its zz entry from dz --
 * the project's exact-mobility mode, which has no counterpart in the
 * reference; it shares calcHI's Ewald split and sums. */
void bdo_calc_hi_ewald(const bdo_sys *s, const double *rx, const double *ry,
                       const double *rz, double *M) {
  calc_hi_impl(s, rx, ry, rz, NULL, M, 1);
}

static void calc_hi_impl(const bdo_sys *s, const double *rx, const double *ry,
                         const double *rz, const double *grid, double *M, int all_pairs) {
  int N = s->N;
  double L = s->L, boxvol = L * L * L;
  int treal = (int)(s->t % (unsigned long)s->tp);
  double rce, M_HI = 4.0;
  int nmax;
  if (treal <= s->tp / 2) {
    rce = 1.0 * s->L2yp;
    nmax = 1;
  } else {
    rce = 2.0 * s->L2yp;
    nmax = 2;
  }
  double tf = (double)treal / s->tp;
  int nt = (int)round(tf * s->nt_avg) % s->nt_avg;
  double alpha = M_HI / rce, rkcut = 2.0 * M_HI * M_HI / rce;
  double rkkcut = rkcut * rkcut, rtpi = sqrt(M_PI);
  double alpha2 = alpha * alpha, alpha3 = alpha2 * alpha, alpha4 = alpha2 * alpha2;
  double alpha5 = alpha4 * alpha, alpha7 = alpha4 * alpha2 * alpha;
  double selfconst = 1 - 6 / rtpi * alpha + 40 / (3 * rtpi) * alpha3;
  const double *L1 = s->L1, *L2 = s->L2;
  int nk;
  double *M2, *kv;
  kvectors(s, boxvol, rkkcut, rkcut, alpha2, alpha4, &nk, &M2, &kv);
  double Dtr[3] = {selfconst, selfconst, selfconst};
  for (int c = 0; c < nk; c++) {
    Dtr[0] += M2[9 * c];
    Dtr[1] += M2[9 * c + 4];
    Dtr[2] += M2[9 * c + 8];
  }
  /* self images; the reference requires all three image indices non-zero and
   * adds the yy projection to the zz entry (shear/src/main26.c:1667-1686) */
  for (int nx = -nmax; nx < nmax + 1; nx++)
    for (int ny = -nmax; ny < nmax + 1; ny++)
      for (int nz = -nmax; nz < nmax + 1; nz++)
        if (all_pairs ? (nx != 0 || ny != 0 || nz != 0) : (nx != 0 && ny != 0 && nz != 0)) {
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
          Dtr[2] += t1 + t2 * (all_pairs ? dz * dz : dy * dy) / rr;
        }
  for (int i = 0; i < N; i++) {
    size_t st = (size_t)9 * N * i + 9 * i;
    M[st] = Dtr[0];
    M[st + 4] = Dtr[1];
    M[st + 8] = Dtr[2];
  }
  for (int i = 0; i < N; i++) {
    double rxi, ryi;
    if (s->flow == 0) {
      rxi = rx[i];
      ryi = ry[i];
    } else {
      rxi = rx[i] * s->cth - ry[i] * s->sth;
      ryi = rx[i] * s->sth + ry[i] * s->cth;
    }
    for (int j = i + 1; j < N; j++) {
      size_t st = (size_t)9 * N * i + 9 * j;
      double rxj, ryj;
      if (s->flow == 0) {
        rxj = rx[j];
        ryj = ry[j];
      } else {
        rxj = rx[j] * s->cth - ry[j] * s->sth;
        ryj = rx[j] * s->sth + ry[j] * s->cth;
      }
      double bm[3];
      bdo_nidbin(s, rx, ry, rz, j, i, bm);
      double dmin = sqrt(bm[0] * bm[0] + bm[1] * bm[1] + bm[2] * bm[2]);
      if (all_pairs || dmin < 12.0) {
        double Dt[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double dxo = rxj - rxi, dyo = ryj - ryi, dzo = rz[j] - rz[i];
        for (int nx = -nmax; nx < nmax + 1; nx++)
          for (int ny = -nmax; ny < nmax + 1; ny++)
            for (int nz = -nmax; nz < nmax + 1; nz++) {
              double dx = dxo + nx * L1[0] + ny * L2[0], dy = dyo + nx * L1[1] + ny * L2[1];
              double dz = dzo + nz * L;
              double rr = dx * dx + dy * dy + dz * dz, r = sqrt(rr);
              if (r < rce) {
                double C1, C2, C3, C4;
                if (r > 2.0) {
                  C1 = 0.75 / r + 0.5 / (r * rr);
                  C2 = 4.0 * alpha7 * rr * rr + 3.0 * alpha3 * rr - 20.0 * alpha5 * rr - 4.5 * alpha + 14.0 * alpha3 + alpha / rr;
                  C3 = 0.75 / r - 1.5 / (r * rr);
                  C4 = -4.0 * alpha7 * rr * rr - 3.0 * alpha3 * rr + 16.0 * alpha5 * rr + 1.5 * alpha - 2.0 * alpha3 - 3.0 * alpha / rr;
                } else {
                  C1 = 1.0 - 0.28125 * r;
                  C2 = 64.0 * alpha7 + 12.0 * alpha3 - 80.0 * alpha5 - 4.5 * alpha + 14.0 * alpha3 + 0.25 * alpha;
                  C3 = 0.09375 * r;
                  C4 = -64.0 * alpha7 - 12.0 * alpha3 + 64.0 * alpha5 + 1.5 * alpha - 2.0 * alpha3 - 0.75 * alpha;
                }
                double t1 = C1 * erfc(alpha * r) + C2 * exp(-alpha2 * rr) / rtpi;
                double t2 = C3 * erfc(alpha * r) + C4 * exp(-alpha2 * rr) / rtpi;
                double m1[9];
                m1[0] = t1 + t2 * dx * dx / rr;
                m1[1] = t2 * dx * dy / rr;
                m1[2] = t2 * dx * dz / rr;
                m1[3] = m1[1];
                m1[4] = t1 + t2 * dy * dy / rr;
                m1[5] = t2 * dy * dz / rr;
                m1[6] = m1[2];
                m1[7] = m1[5];
                m1[8] = t1 + t2 * dz * dz / rr;
                for (int a = 0; a < 9; a++) Dt[a] += m1[a];
              }
            }
        for (int c = 0; c < nk; c++) {
          double ck = cos(kv[3 * c] * dxo + kv[3 * c + 1] * dyo + kv[3 * c + 2] * dzo);
          for (int a = 0; a < 9; a++) Dt[a] += M2[9 * c + a] * ck;
        }
        memcpy(&M[st], Dt, 9 * sizeof(double));
      } else {
        int b = bdo_binij(s, rx, ry, rz, i, j);
        if (b < 0) b = 0; /* out-of-table bins are an error on the GPU path */
        memcpy(&M[st], &grid[(size_t)nt * 9 * s->nbins + 9 * (size_t)b], 9 * sizeof(double));
      }
    }
  }
  free(M2);
  free(kv);
}

/* gridHI: the far-field lookup table, nt_avg lattice frames of the full
 * Ewald-summed RPY tensor at every bin centre (shear/src/gridHI.c:13-246,
 * extensional/src/gridHI.c:13-239).  gridHI runs with its own time step
 * (dt = 0.001, shear/src/gridHI.c:288) for the period and the bin geometry,
 * takes frame nt at t = nt*tp/nt_avg, uses M_HI = 6, no self term, and
 * evaluates the origin bin at (0.6, 0.6, 0.6).  D receives nt_avg x nbins
 * row-major 3x3 tensors on gridHI's bin geometry, which is returned in
 * geom[]: nbx nby nbz nhx nhy nhz nbins origin. */
/* gridHI's period and bin geometry from its own time step
 * (shear/src/gridHI.c:367-432): geom = nbx nby nbz nhx nhy nhz nbins origin. */
static void grid_geom(bdo_sys *s, double grid_dt, int *geom) {
  double L = s->L, edot = s->edot;
  s->dt = grid_dt;
  s->tp = (int)(EPK / edot / grid_dt);
  double th = 90.0 - (45.0 + (s->flow == 0 ? 0.0 : 31.7));
  th *= M_PI / 180;
  double p0x2 = sqrt(2) / 2 * L * cos(th), p0y1 = -sqrt(2) / 2 * L * cos(th);
  double xmax, ymax, zmax = L / 2;
  int treal = s->tp;
  if (s->flow == 0) {
    ymax = L / 2;
    xmax = L / 2 * edot * treal * grid_dt;
  } else {
    ymax = -p0y1;
    xmax = p0x2 * exp(edot * treal * grid_dt);
  }
  s->bsx = s->bsy = s->bsz = s->bin_size;
  s->nbx = 2 * ceil(xmax / s->bsx) + 1;
  s->bsx = xmax / ((s->nbx - 1) / 2);
  s->nhx = (s->nbx - 1) / 2;
  s->nby = 2 * ceil(ymax / s->bsy) + 1;
  s->bsy = ymax / ((s->nby - 1) / 2);
  s->nhy = (s->nby - 1) / 2;
  s->nbz = 2 * ceil(zmax / s->bsz) + 1;
  s->bsz = zmax / ((s->nbz - 1) / 2);
  s->nhz = (s->nbz - 1) / 2;
  s->nbins = s->nbx * s->nby * s->nbz;
  geom[0] = s->nbx;
  geom[1] = s->nby;
  geom[2] = s->nbz;
  geom[3] = s->nhx;
  geom[4] = s->nhy;
  geom[5] = s->nhz;
  geom[6] = s->nbins;
  geom[7] = s->nhx * s->nby * s->nbz + s->nhy * s->nbz + s->nhz;
}

void bdo_grid_geom(const bdo_sys *s0, double grid_dt, int *geom) {
  bdo_sys s = *s0;
  grid_geom(&s, grid_dt, geom);
}

void bdo_grid(const bdo_sys *s0, double grid_dt, double boxvol, double *D, int *geom) {
  bdo_sys s = *s0;
  double L = s.L;
  grid_geom(&s, grid_dt, geom);
  int origin = geom[7];
  double rtpi = sqrt(M_PI);
  for (int nt = 0; nt < s.nt_avg; nt++) {
    unsigned long t = (unsigned long)(nt * s.tp / s.nt_avg);
    bdo_lattice(&s, t);
    int treal = (int)(t % (unsigned long)s.tp), nmax;
    double rce;
    if (treal <= s.tp / 2) {
      rce = s.L2yp;
      nmax = 1;
    } else {
      rce = 2.0 * s.L2yp;
      nmax = 2;
    }
    double M_HI = 6.0;
    double alpha = M_HI / rce, rkcut = 2.0 * M_HI * M_HI / rce, rkkcut = rkcut * rkcut;
    double alpha2 = alpha * alpha, alpha3 = alpha2 * alpha, alpha4 = alpha2 * alpha2;
    double alpha5 = alpha4 * alpha, alpha7 = alpha4 * alpha2 * alpha;
    int nk;
    double *M2, *kv;
    kvectors(&s, boxvol, rkkcut, rkcut, alpha2, alpha4, &nk, &M2, &kv);
    /* bins are independent: spread them over the host threads */
#pragma omp parallel for schedule(dynamic, 64)
    for (int b = 0; b < s.nbins; b++) {
      double dr[3];
      if (b != origin) {
        int bb = b;
        int bx = bb / (s.nby * s.nbz);
        bb -= bx * s.nby * s.nbz;
        bx -= s.nhx;
        int by = bb / s.nbz;
        bb -= by * s.nbz;
        by -= s.nhy;
        int bz = bb - s.nhz;
        dr[0] = bx * s.bsx;
        dr[1] = by * s.bsy;
        dr[2] = bz * s.bsz;
      } else {
        dr[0] = dr[1] = dr[2] = 0.6;
      }
      double Dt[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (int nx = -nmax; nx < nmax + 1; nx++)
        for (int ny = -nmax; ny < nmax + 1; ny++)
          for (int nz = -nmax; nz < nmax + 1; nz++) {
            double dx = dr[0] + nx * s.L1[0] + ny * s.L2[0];
            double dy = dr[1] + nx * s.L1[1] + ny * s.L2[1];
            double dz = dr[2] + nz * L;
            double rr = dx * dx + dy * dy + dz * dz, r = sqrt(rr);
            if (r < rce) {
              double C1, C2, C3, C4;
              if (r > 2.0) {
                C1 = 0.75 / r + 0.5 / (r * rr);
                C2 = 4.0 * alpha7 * rr * rr + 3.0 * alpha3 * rr - 20.0 * alpha5 * rr - 4.5 * alpha + 14.0 * alpha3 + alpha / rr;
                C3 = 0.75 / r - 1.5 / (r * rr);
                C4 = -4.0 * alpha7 * rr * rr - 3.0 * alpha3 * rr + 16.0 * alpha5 * rr + 1.5 * alpha - 2.0 * alpha3 - 3.0 * alpha / rr;
              } else {
                C1 = 1.0 - 0.28125 * r;
                C2 = 64.0 * alpha7 + 12.0 * alpha3 - 80.0 * alpha5 - 4.5 * alpha + 14.0 * alpha3 + 0.25 * alpha;
                C3 = 0.09375 * r;
                C4 = -64.0 * alpha7 - 12.0 * alpha3 + 64.0 * alpha5 + 1.5 * alpha - 2.0 * alpha3 - 0.75 * alpha;
              }
              double t1 = C1 * erfc(alpha * r) + C2 * exp(-alpha2 * rr) / rtpi;
              double t2 = C3 * erfc(alpha * r) + C4 * exp(-alpha2 * rr) / rtpi;
              Dt[0] += t1 + t2 * dx * dx / rr;
              Dt[1] += t2 * dx * dy / rr;
              Dt[2] += t2 * dx * dz / rr;
              Dt[3] += t2 * dx * dy / rr;
              Dt[4] += t1 + t2 * dy * dy / rr;
              Dt[5] += t2 * dy * dz / rr;
              Dt[6] += t2 * dx * dz / rr;
              Dt[7] += t2 * dy * dz / rr;
              Dt[8] += t1 + t2 * dz * dz / rr;
            }
          }
      for (int c = 0; c < nk; c++) {
        double ck = cos(kv[3 * c] * dr[0] + kv[3 * c + 1] * dr[1] + kv[3 * c + 2] * dr[2]);
        for (int a = 0; a < 9; a++) Dt[a] += M2[9 * c + a] * ck;
      }
      memcpy(D + ((size_t)nt * s.nbins + b) * 9, Dt, 9 * sizeof(double));
    }
    free(M2);
    free(kv);
  }
}

/* updateHI: TEA Brownian displacement dt M (F + sqrt(2/dt) beta C R) plus the
 * affine flow (shear/src/main26.c:745-857; ext rotates positions back to the
 * lab frame first and uses u = edot (x, -y, 0), extensional/src/main14.c:
 * 783-895).  On the diagonal block beta multiplies only the off-diagonal
 * components (shear/src/main26.c:800-803). */
void bdo_update_hi(const bdo_sys *s, double *rx, double *ry, double *rz,
                   double *dxv, double *dyv, double *dzv, const double *fx,
                   const double *fy, const double *fz, const double *R,
                   const double *M, double bt, const double *Ct) {
  int N = s->N;
  double dt = s->dt, p = sqrt(2.0 / dt);
  double *du = calloc((size_t)3 * N, sizeof(double));
  double *dxu = du, *dyu = du + N, *dzu = du + 2 * N;
  if (s->flow == 1) bdo_rotate(s, rx, ry, 1);
  for (int i = 0; i < N; i++) {
    int m = 3 * i;
    for (int j = i + 1; j < N; j++) {
      int n = 3 * j;
      const double *Mb = M + (size_t)9 * N * i + 9 * j;
      dxu[i] += dt * (Mb[0] * (fx[j] + p * bt * Ct[m] * R[n]) + Mb[1] * (fy[j] + p * bt * Ct[m] * R[n + 1]) + Mb[2] * (fz[j] + p * bt * Ct[m] * R[n + 2]));
      dyu[i] += dt * (Mb[3] * (fx[j] + p * bt * Ct[m + 1] * R[n]) + Mb[4] * (fy[j] + p * bt * Ct[m + 1] * R[n + 1]) + Mb[5] * (fz[j] + p * bt * Ct[m + 1] * R[n + 2]));
      dzu[i] += dt * (Mb[6] * (fx[j] + p * bt * Ct[m + 2] * R[n]) + Mb[7] * (fy[j] + p * bt * Ct[m + 2] * R[n + 1]) + Mb[8] * (fz[j] + p * bt * Ct[m + 2] * R[n + 2]));
      dxu[j] += dt * (Mb[0] * (fx[i] + p * bt * Ct[n] * R[m]) + Mb[1] * (fy[i] + p * bt * Ct[n] * R[m + 1]) + Mb[2] * (fz[i] + p * bt * Ct[n] * R[m + 2]));
      dyu[j] += dt * (Mb[3] * (fx[i] + p * bt * Ct[n + 1] * R[m]) + Mb[4] * (fy[i] + p * bt * Ct[n + 1] * R[m + 1]) + Mb[5] * (fz[i] + p * bt * Ct[n + 1] * R[m + 2]));
      dzu[j] += dt * (Mb[6] * (fx[i] + p * bt * Ct[n + 2] * R[m]) + Mb[7] * (fy[i] + p * bt * Ct[n + 2] * R[m + 1]) + Mb[8] * (fz[i] + p * bt * Ct[n + 2] * R[m + 2]));
    }
    const double *Mb = M + (size_t)9 * N * i + 9 * i;
    dxu[i] += dt * (Mb[0] * (fx[i] + p * Ct[m] * R[m]) + Mb[1] * (fy[i] + p * Ct[m] * bt * R[m + 1]) + Mb[2] * (fz[i] + p * Ct[m] * bt * R[m + 2]));
    dyu[i] += dt * (Mb[3] * (fx[i] + p * Ct[m + 1] * bt * R[m]) + Mb[4] * (fy[i] + p * Ct[m + 1] * R[m + 1]) + Mb[5] * (fz[i] + p * Ct[m + 1] * bt * R[m + 2]));
    dzu[i] += dt * (Mb[6] * (fx[i] + p * Ct[m + 2] * bt * R[m]) + Mb[7] * (fy[i] + p * Ct[m + 2] * bt * R[m + 1]) + Mb[8] * (fz[i] + p * Ct[m + 2] * R[m + 2]));
  }
  for (int i = 0; i < N; i++) {
    if (s->flow == 0) {
      dxu[i] += dt * s->edot * ry[i];
    } else {
      dxu[i] += dt * s->edot * rx[i];
      dyu[i] -= dt * s->edot * ry[i];
    }
    dxv[i] += dxu[i];
    rx[i] += dxu[i];
    dyv[i] += dyu[i];
    ry[i] += dyu[i];
    dzv[i] += dzu[i];
    rz[i] += dzu[i];
  }
  free(du);
}

/* updateFD: free-draining Euler-Maruyama step with the affine flow
 * (shear/src/main26.c:731-744, extensional/src/main14.c:735-782).  For ext
 * the caller has already rotated positions to the lab frame. */
void bdo_update_fd(const bdo_sys *s, double *rx, double *ry, double *rz,
                   double *dxv, double *dyv, double *dzv, const double *fx,
                   const double *fy, const double *fz, const double *R) {
  double dt = s->dt, pc = sqrt(2.0 * dt);
  for (int i = 0; i < s->N; i++) {
    double dx, dy, dz;
    if (s->flow == 0) {
      dx = dt * (fx[i] + s->edot * ry[i]) + pc * R[3 * i];
      dy = dt * fy[i] + pc * R[3 * i + 1];
    } else {
      dx = dt * (fx[i] + s->edot * rx[i]) + pc * R[3 * i];
      dy = dt * (fy[i] - s->edot * ry[i]) + pc * R[3 * i + 1];
    }
    dz = dt * fz[i] + pc * R[3 * i + 2];
    rx[i] += dx;
    ry[i] += dy;
    rz[i] += dz;
    dxv[i] += dx;
    dyv[i] += dy;
    dzv[i] += dz;
  }
}

/* ---- random numbers ----------------------------------------------------- */

#define R_IM1 2147483563L
#define R_IM2 2147483399L
#define R_AM (1.0 / R_IM1)
#define R_IMM1 (R_IM1 - 1)
#define R_IA1 40014L
#define R_IQ1 53668L
#define R_IR1 12211L
#define R_IQ2 52774L
#define R_NTAB 32
#define R_NDIV (1 + R_IMM1 / R_NTAB)
#define R_RNMX (1.0 - 1.2e-7)

/* State of ran1/gasdev in a process that has not drawn yet: the reference
 * seeds with a positive idum (shear/src/Initialization.c:438), so the shuffle
 * table starts zeroed and idum2 at its initialiser. */
void bdo_rng_fresh(bdo_rng *g, long seed) {
  memset(g, 0, sizeof(*g));
  g->idum = seed;
  g->idum2 = 123456789L;
}

/* ran1: shear/src/Initialization.c:601-634, including that idum2 is never
 * advanced (its update is guarded by a test on the already non-negative idum). */
float bdo_ran1(bdo_rng *g) {
  long k;
  int j;
  float temp;
  if (g->idum <= 0) {
    if (-(g->idum) < 1)
      g->idum = 1;
    else
      g->idum = -(g->idum);
    g->idum2 = g->idum;
    for (j = R_NTAB + 7; j >= 0; --j) {
      k = g->idum / R_IQ1;
      g->idum = R_IA1 * (g->idum - k * R_IQ1) - k * R_IR1;
      if (g->idum < 0) g->idum += R_IM1;
      if (j < R_NTAB) g->iv[j] = g->idum;
    }
    g->iy = g->iv[0];
  }
  k = g->idum / R_IQ1;
  g->idum = R_IA1 * (g->idum - k * R_IQ1) - k * R_IR1;
  if (g->idum < 0) g->idum += R_IM1;
  j = (int)(g->iy / R_NDIV);
  g->iy = g->iv[j] - g->idum2;
  g->iv[j] = g->idum;
  if (g->iy < 1) g->iy += R_IMM1;
  if ((temp = R_AM * g->iy) > R_RNMX) return R_RNMX;
  return temp;
}

/* gasdev: polar Box-Muller in float with a cached second deviate
 * (shear/src/main26.c:515-540). */
float bdo_gasdev(bdo_rng *g) {
  float fac, rsq, v1, v2;
  if (g->idum < 0) g->iset = 0;
  if (g->iset == 0) {
    do {
      v1 = 2.0 * bdo_ran1(g) - 1.0;
      v2 = 2.0 * bdo_ran1(g) - 1.0;
      rsq = v1 * v1 + v2 * v2;
    } while (rsq >= 1.0 || rsq == 0.0);
    fac = sqrt(-2.0 * log(rsq) / rsq);
    g->gset = v1 * fac;
    g->iset = 1;
    return v2 * fac;
  }
  g->iset = 0;
  return g->gset;
}

/* getNoise: shear/src/main26.c:708-713 */
void bdo_noise(bdo_rng *g, double *R, int n) {
  for (int a = 0; a < n; a++) R[a] = bdo_gasdev(g);
}

/* ---- charge hopping ----------------------------------------------------- */

/* Debye-Hueckel energy of the charged beads, summed over bead index pairs in
 * ascending order like the reference's E_initial/E_final scans
 * (shear/src/main26.c:1955-1970, 2183-2198). */
static double dh_energy_flags(const bdo_sys *s, const double *rx,
                              const double *ry, const double *rz,
                              const int *flag) {
  double E = 0;
  for (int i = 0; i < s->N; i++)
    for (int j = i + 1; j < s->N; j++)
      if (flag[i] != 0 && flag[j] != 0) {
        double v[3];
        nid(s, rx, ry, rz, i, j, v);
        double rr = v[0] * v[0] + v[1] * v[1] + v[2] * v[2], r = sqrt(rr);
        E += (s->lambda_b * flag[i] * flag[j] / r) * exp(-s->kappa_d * r);
      }
  return E;
}

double bdo_dh_energy(const bdo_sys *s, const double *rx, const double *ry,
                     const double *rz, const int *beads, int nch) {
  int *flag = calloc(s->N, sizeof(int));
  for (int k = 0; k < nch; k++) flag[beads[k]] = 1;
  double E = dh_energy_flags(s, rx, ry, rz, flag);
  free(flag);
  return E;
}

static int in_list(const int *idx, int nch, int b) {
  for (int a = 0; a < nch; a++)
    if (idx[a] == b) return 1;
  return 0;
}

/* chargeHop with chargehop_type 1: one sequential Metropolis sweep over the
 * charges (shear/src/main26.c:1926-2390).  Restated rules:
 *  - E_initial is computed once at the start of the sweep and not refreshed
 *    after accepted hops;
 *  - a bead j (not the charge's own bead nor its chain neighbours by index)
 *    with |NID|^2 < 4.41 found first in index order makes the move "near":
 *    mm < .33 right neighbour, mm > .66 left neighbour, else a jump to j
 *    (barrier2); a blocked near move blocks the whole trial, because the
 *    reference's blocked flag is never cleared for the rest of the trial;
 *  - with no near bead: mm > .5 right, else left;
 *  - acceptance: 1 <= exp(-barrier - dE/2) accepts without a draw, else a
 *    second uniform is drawn and compared with <=.
 * log, when given, receives per trial: outcome (0 skipped, 1 accepted,
 * 2 rejected), the target bead, the move kind (0/1 neighbour, 2 jump).
 * Returns the number of accepted hops.  The sweep runs only when
 * t % MStep == 0. */
int bdo_charge_hop(const bdo_sys *s, const double *rx, const double *ry,
                   const double *rz, int *track, int *idx, int *old, int nch,
                   bdo_rng *g, int *log, int logcap) {
  int N = s->N, Nb = s->Nb, nacc = 0;
  if (s->t % (unsigned long)s->MStep != 0) return 0;
  int *flag = calloc(N, sizeof(int));
  for (int a = 0; a < nch; a++) idx[a] = track[a];
  for (int a = 0; a < nch; a++) flag[track[a]] = 1;
  double E_init = 0;
  if (nch > 1) E_init = dh_energy_flags(s, rx, ry, rz, flag);
  for (int k = 0; k < nch; k++) {
    double mm = bdo_ran1(g);
    int c = idx[k], c2 = -1, test = 0, blocked = 0;
    for (int j = 0; j < N; j++) {
      if (j == c || j == c + 1 || j == c - 1) continue;
      double v[3];
      nid(s, rx, ry, rz, c, j, v);
      double rr = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      if (rr < 4.41) {
        if (mm < .33) {
          c2 = c + 1;
          blocked = (c == N - 1 || c % Nb == Nb - 1 || c == Nb - 1 || in_list(idx, nch, c2));
          if (!blocked) test = 1;
        } else if (mm > 0.66) {
          c2 = c - 1;
          blocked = (c2 < 0 || c == 0 || c % Nb == 0 || in_list(idx, nch, c2));
          if (!blocked) test = 1;
        } else {
          c2 = j;
          blocked = in_list(idx, nch, c2);
          if (!blocked) test = 2;
        }
        break;
      }
    }
    if (!blocked && test == 0) {
      if (mm > .5) {
        c2 = c + 1;
        blocked = (c == N - 1 || c % Nb == Nb - 1 || c == Nb - 1 || in_list(idx, nch, c2));
      } else {
        c2 = c - 1;
        blocked = (c2 < 0 || c == 0 || c % Nb == 0 || in_list(idx, nch, c2));
      }
    }
    if (blocked) {
      if (log && k < logcap) {
        log[3 * k] = 0;
        log[3 * k + 1] = c2;
        log[3 * k + 2] = test;
      }
      continue;
    }
    for (int a = 0; a < nch; a++)
      if (idx[a] == c) idx[a] = c2;
    for (int a = 0; a < N; a++) flag[a] = 0;
    for (int a = 0; a < nch; a++) flag[idx[a]] = 1;
    double E_fin = 0;
    if (nch > 1) E_fin = dh_energy_flags(s, rx, ry, rz, flag);
    double bar = (test == 2) ? s->barrier2 : s->barrier;
    double x = exp((-bar - 0.5 * (E_fin - E_init)));
    int acc;
    if (1 <= x)
      acc = 1;
    else
      acc = (bdo_ran1(g) <= x);
    if (acc) {
      for (int a = 0; a < nch; a++)
        if (track[a] == c) {
          old[a] = c;
          idx[a] = c2;
          track[a] = c2;
          break;
        }
      nacc++;
    } else {
      for (int a = 0; a < nch; a++)
        if (idx[a] == c2) {
          idx[a] = c;
          old[a] = c;
          break;
        }
    }
    if (log && k < logcap) {
      log[3 * k] = acc ? 1 : 2;
      log[3 * k + 1] = c2;
      log[3 * k + 2] = test;
    }
  }
  free(flag);
  return nacc;
}
