/* FP64 CPU restatement of the reference's per-step Brownian-dynamics path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA path is checked
 * against; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg may load it.  It is pinned against the reference itself (compiled from
 * its own sources into oracle/_ref/) by tests/test_oracle_pin.py and the
 * golden fixtures under tests/golden/.
 *
 * Every routine takes its state explicitly instead of through file-scope
 * globals, and follows the arithmetic of the reference routine it cites
 * (shear = shear/src/main26.c, ext = extensional/src/main14.c).
 */
#ifndef BD_ORACLE_H
#define BD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  /* configuration */
  int flow; /* 0 shear (deforming brick), 1 planar extension (KRBC) */
  int N, Nb, Nc;
  double L, edot, dt;
  int tp;
  int spring; /* 0 Hookean, 1 FENE */
  double kappas, qmax, qmax2, kappab, epsilon;
  double rv, r2cut, rnew;
  double lambda_b, lambda_d, kappa_d;
  double barrier, barrier2;
  int MStep;
  /* lattice at step t */
  unsigned long t;
  double L1[2], L2[2], L1xp, L1yp, L2xp, L2yp, detL, theta, cth, sth, delx;
  /* far-field lookup grid */
  int nt_avg, nbx, nby, nbz, nhx, nhy, nhz, nbins;
  double bsx, bsy, bsz;
  double bin_size;
} bdo_sys;

typedef struct {
  long idum, idum2, iy;
  long iv[32];
  int iset;
  float gset;
} bdo_rng;

void bdo_init(bdo_sys *s, int flow, int Nb, int Nc, double L, double edot,
              double dt, int nt_avg, double bin_size, int spring,
              double kappas, double qmax, double kappab, double epsilon,
              double lambda_b, double lambda_d, double barrier,
              double barrier2, int MStep);
void bdo_lattice(bdo_sys *s, unsigned long t);
void bdo_apply_pbc(const bdo_sys *s, double *rx, double *ry, double *rz);
void bdo_rotate(const bdo_sys *s, double *rx, double *ry, int inverse);
void bdo_nid(const bdo_sys *s, const double *rx, const double *ry,
             const double *rz, int i, int j, double *out);
void bdo_nidbin(const bdo_sys *s, const double *rx, const double *ry,
                const double *rz, int i, int j, double *out);
int bdo_binij(const bdo_sys *s, const double *rx, const double *ry,
              const double *rz, int i, int j);
int bdo_bond(const bdo_sys *s, const double *rx, const double *ry,
             const double *rz, double *fx, double *fy, double *fz,
             double *stress);
void bdo_ev(const bdo_sys *s, const double *rx, const double *ry,
            const double *rz, const int *counts, const int *rows, int maxnb,
            double *fx, double *fy, double *fz, double *stress);
void bdo_coulomb(const bdo_sys *s, const double *rx, const double *ry,
                 const double *rz, const double *q, double *fx, double *fy,
                 double *fz);
int bdo_verlet(const bdo_sys *s, const double *rx, const double *ry,
               const double *rz, int *counts, int *rows, int maxnb);
int bdo_check_verlet(const bdo_sys *s, const double *dxv, const double *dyv,
                     const double *dzv);
void bdo_calc_hi(const bdo_sys *s, const double *rx, const double *ry,
                 const double *rz, const double *grid, double *M);
void bdo_calc_hi_ewald(const bdo_sys *s, const double *rx, const double *ry,
                       const double *rz, double *M);
void bdo_grid_geom(const bdo_sys *s, double grid_dt, int *geom);
void bdo_grid(const bdo_sys *s, double grid_dt, double boxvol, double *D, int *geom);
void bdo_update_hi(const bdo_sys *s, double *rx, double *ry, double *rz,
                   double *dxv, double *dyv, double *dzv, const double *fx,
                   const double *fy, const double *fz, const double *R,
                   const double *M, double beta, const double *Ct);
void bdo_update_fd(const bdo_sys *s, double *rx, double *ry, double *rz,
                   double *dxv, double *dyv, double *dzv, const double *fx,
                   const double *fy, const double *fz, const double *R);
void bdo_rng_fresh(bdo_rng *g, long seed);
float bdo_ran1(bdo_rng *g);
float bdo_gasdev(bdo_rng *g);
void bdo_noise(bdo_rng *g, double *R, int n);
int bdo_charge_hop(const bdo_sys *s, const double *rx, const double *ry,
                   const double *rz, int *track, int *idx, int *old, int nch,
                   bdo_rng *g, int *log, int logcap);
double bdo_dh_energy(const bdo_sys *s, const double *rx, const double *ry,
                     const double *rz, const int *beads, int nch);

#ifdef __cplusplus
}
#endif
#endif
