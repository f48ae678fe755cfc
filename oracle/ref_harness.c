/* Test-only harness around the unmodified reference simulator.
 *
 * This file is test infrastructure: it is compiled only into oracle/_ref/
 * (never into the product library) by oracle/Makefile, directly from the
 * reference sources where they lie (shear/src/main26.c or
 * extensional/src/main14.c).  The reference is a single translation unit
 * whose state lives in file-scope globals (shear/src/Parameters.h:40-201), so
 * the harness renames its main() and exposes setters, getters and thin call
 * wrappers for the step-loop routines.  Everything it returns is what the
 * reference itself computed.
 *
 * REF_FLOW is 0 for the shear tree and 1 for the extensional tree; REF_MAIN
 * names the file to include.  ran1/gasdev keep function-local static state
 * (shear/src/Initialization.c:601-634, shear/src/main26.c:515-540), so every
 * scenario that depends on the random stream must run in a fresh process.
 */
#define main ref_main
#include REF_MAIN
#undef main

#include <stdint.h>

int h_flow(void) { return REF_FLOW; }

/* Sets the globals that Initialization() would derive from the command line
 * and Input.txt (shear/src/Initialization.c:25-174), with the box edge L given
 * directly instead of through c/c*, then runs the reference's own
 * initLattice/initVerlet/allocate. */
void h_setup(int Nb_, int Nc_, double L_, double edot, double dt_, int nt_avg_,
             double bin_size_, const char *spring_, double epsilon_,
             double kappab_, double kappas_, double qmax_, double lambda_b_,
             double lambda_d_, int Ncharges_, double barrier_,
             double barrier2_, int MStep_, long seed, int threads) {
  Nb = Nb_;
  Nc = Nc_;
  N = Nb * Nc;
  L = L_;
  box_side = L / 2;
  box_volume = L * L * L;
  flowrate = edot;
  dt = dt_;
  dt_eq = 0.001;
  nt_avg = nt_avg_;
  bin_size = bin_size_;
  strncpy(spring, spring_, 99);
  epsilon = epsilon_;
  kappab = kappab_;
  kappas = kappas_;
  qmax = qmax_;
  lambda_b = lambda_b_;
  lambda_d = lambda_d_;
  kappa_d = 1.0 / lambda_d;
  Ncharges = Ncharges_;
  barrier = barrier_;
  barrier2 = barrier2_;
  MStep = MStep_;
  total_strain = 10.0;
  fixSeed = 1;
  restart = 0;
  iterstart = 1;
  itermax = 2;
  itercount = 1;
  trace = 0;
  flowtype = 1;
  initLattice();
  initVerlet();
  allocate();
  *idum = seed;
  tstart = 0;
  t = 0;
  tcount = 0;
  strain = 0.0;
  omp_set_num_threads(threads);
}

int h_N(void) { return N; }
unsigned long h_tp(void) { return (unsigned long)tp; }

void h_set_pos(const double *x, const double *y, const double *z) {
  memcpy(rx, x, sizeof(double) * N);
  memcpy(ry, y, sizeof(double) * N);
  memcpy(rz, z, sizeof(double) * N);
}
void h_get_pos(double *x, double *y, double *z) {
  memcpy(x, rx, sizeof(double) * N);
  memcpy(y, ry, sizeof(double) * N);
  memcpy(z, rz, sizeof(double) * N);
}
void h_set_dv(const double *x, const double *y, const double *z) {
  memcpy(dxv, x, sizeof(double) * N);
  memcpy(dyv, y, sizeof(double) * N);
  memcpy(dzv, z, sizeof(double) * N);
}
void h_get_dv(double *x, double *y, double *z) {
  memcpy(x, dxv, sizeof(double) * N);
  memcpy(y, dyv, sizeof(double) * N);
  memcpy(z, dzv, sizeof(double) * N);
}
void h_set_force(const double *x, const double *y, const double *z) {
  memcpy(fx, x, sizeof(double) * N);
  memcpy(fy, y, sizeof(double) * N);
  memcpy(fz, z, sizeof(double) * N);
}
void h_get_force(double *x, double *y, double *z) {
  memcpy(x, fx, sizeof(double) * N);
  memcpy(y, fy, sizeof(double) * N);
  memcpy(z, fz, sizeof(double) * N);
}
void h_set_t(unsigned long tt) { t = tt; }
void h_set_tstart(unsigned long tt) { tstart = tt; }
void h_set_strain(double s) { strain = s; }

void h_update_lattice(unsigned long tt) { updateLattice(tt); }
/* L1x L1y L2x L2y L1xp L1yp L2xp L2yp detL tp */
void h_get_lattice(double *out) {
  out[0] = L1[0];
  out[1] = L1[1];
  out[2] = L2[0];
  out[3] = L2[1];
  out[4] = L1xp;
  out[5] = L1yp;
  out[6] = L2xp;
  out[7] = L2yp;
  out[8] = detL;
  out[9] = (double)tp;
}
void h_apply_pbc(void) { applyPBC(); }
#if REF_FLOW == 1
void h_transform(void) { transformCoords(); }
void h_inverse(void) { inverseCoords(); }
#endif
void h_nid(int i, int j, double *out) {
  Vector3D_t v = getNID(i, j);
  out[0] = v.x;
  out[1] = v.y;
  out[2] = v.z;
}
void h_nidbin(int i, int j, double *out) {
  Vector3D_t v = getNIDbin(i, j);
  out[0] = v.x;
  out[1] = v.y;
  out[2] = v.z;
}
int h_binij(int i, int j) { return binij(i, j); }

void h_reset_force(void) {
  resetForce();
  tauxx = 0.0;
  tauyy = 0.0;
#if REF_FLOW == 0
  tauxy = 0.0;
#endif
}
void h_get_stress(double *out) {
  out[0] = tauxx;
  out[1] = tauyy;
#if REF_FLOW == 0
  out[2] = tauxy;
#else
  out[2] = 0.0;
#endif
}
void h_bondforce(void) { bondforce(); }
void h_ljforce(void) { LJforce(); }
void h_coulomb(void) { coulombForce(); }
void h_verlet(void) { verletlist(); }
void h_check_verlet(void) { checkVerlet(); }
/* Copies the half neighbour list; returns -1 if a row exceeds maxnb. */
int h_get_verlet(int *counts, int *rows, int maxnb) {
  for (int a = 0; a < N; a++) {
    counts[a] = nlist[a];
    if (nlist[a] > maxnb) return -1;
    for (int k = 0; k < nlist[a]; k++) rows[(size_t)a * maxnb + k] = list[(size_t)a * N + k];
  }
  return 0;
}

/* Re-sizes the charge arrays allocate() sized for Ncharges
 * (shear/src/Initialization.c:351-361), with one spare printprops window
 * for the reference's dxt index that runs one past each charge's window. */
static void h_charge_arrays(int nch) {
  free(Charge_track);
  free(Charge_old);
  free(Charge_indices);
  free(check_ch);
  free(dxt);
  free(dyt);
  free(dzt);
  free(rbic);
  Charge_track = calloc(nch + 1, sizeof(int));
  Charge_old = calloc(nch + 1, sizeof(int));
  Charge_indices = calloc(nch + 1, sizeof(int));
  check_ch = calloc(3 * nch + 3, sizeof(int));
  dxt = calloc((size_t)(nch + 1) * printprops + 1, sizeof(long double));
  dyt = calloc((size_t)(nch + 1) * printprops + 1, sizeof(long double));
  dzt = calloc((size_t)(nch + 1) * printprops + 1, sizeof(long double));
  rbic = calloc(3 * nch + 3, sizeof(double));
}

void h_set_charges(const int *track, int nch) {
  h_charge_arrays(nch);
  Ncharges = nch;
  for (int a = 0; a < N; a++) Charge[a] = 0;
  for (int k = 0; k < nch; k++) {
    Charge_track[k] = track[k];
    Charge_indices[k] = track[k];
    Charge_old[k] = track[k];
    Charge[track[k]] = 1;
  }
}
void h_get_charges(int *track, int *old, int *flags) {
  for (int k = 0; k < Ncharges; k++) {
    track[k] = Charge_track[k];
    old[k] = Charge_old[k];
  }
  for (int a = 0; a < N; a++) flags[a] = Charge[a];
}
void h_set_noise(const double *r) { memcpy(R, r, sizeof(double) * 3 * N); }
void h_get_noise(double *r) { memcpy(r, R, sizeof(double) * 3 * N); }
void h_gen_noise(void) { getNoise(); }
long h_get_idum(void) { return *idum; }
void h_set_idum(long v) { *idum = v; }
float h_ran1(void) { return ran1(idum); }
float h_gasdev(void) { return gasdev(idum); }

/* num_bins_x num_bins_y num_bins_z nhx nhy nhz num_bins */
void h_bins(int *out) {
  out[0] = num_bins_x;
  out[1] = num_bins_y;
  out[2] = num_bins_z;
  out[3] = nhx;
  out[4] = nhy;
  out[5] = nhz;
  out[6] = num_bins;
}
void h_bin_sizes(double *out) {
  out[0] = bin_size_x;
  out[1] = bin_size_y;
  out[2] = bin_size_z;
}
void h_set_grid(int nt, const double *d9) {
  memcpy(D[nt], d9, sizeof(double) * 9 * num_bins);
}
void h_set_tea(int sbin, double beta, const double *c3nb) {
  bp[sbin] = beta;
  memcpy(C[sbin], c3nb, sizeof(double) * 3 * Nb);
}
void h_calc_hi(void) { calcHI(); }
void h_get_M(double *out) { memcpy(out, M, sizeof(double) * 9 * (size_t)N * N); }
void h_set_M(const double *in) { memcpy(M, in, sizeof(double) * 9 * (size_t)N * N); }
void h_update_hi(void) {
  tcount = 0;
  updateHI();
}
void h_update_fd(void) { updateFD(); }
void h_charge_hop(void) {
  tcount = 0;
  chargeHop();
}
/* The stale-energy accumulators and hop counters chargeHop increments. */
void h_hop_counters(int *out) {
  out[0] = counter1;
  out[1] = counter2;
  out[2] = counter3;
  out[3] = counter4;
  out[4] = counter5;
  out[5] = counter6;
}

/* Unwrapped chain coordinates, as computed inside the step loop
 * (shear/src/main26.c:75-83, extensional/src/main14.c:84-92). */
static void h_unwrap(void) {
  for (int c = 0; c < Nc; c++) {
    px[c * Nb] = 0.0;
    py[c * Nb] = 0.0;
    pz[c * Nb] = 0.0;
    for (int b = 0; b < Nb - 1; b++) {
      Vector3D_t v = getNID(c * Nb + b, c * Nb + b + 1);
      px[c * Nb + b + 1] = px[c * Nb + b] + v.x;
      py[c * Nb + b + 1] = py[c * Nb + b] + v.y;
      pz[c * Nb + b + 1] = pz[c * Nb + b] + v.z;
    }
  }
}

/* One hydrodynamic (itercount>=1, flowtype!=0) step of the reference's step
 * loop, in the reference's own call order (shear/src/main26.c:65-151,
 * extensional/src/main14.c:68-171), without its text-file output
 * (printExt/calcRg/calcCH/printTrajectory/printRestart/printVisc) and without
 * the iteration-0 CA-TEA sampling.  with_hop selects chargehop_type 1. */
void h_step_hi(unsigned long tt, int with_hop) {
  t = tt;
#if REF_FLOW == 1
  transformCoords();
  initPos();
  inverseCoords();
#endif
  resetForce();
  strain = (t - equil_start) * dt * flowrate;
  updateLattice(t);
#if REF_FLOW == 1
  transformCoords();
#endif
  applyPBC();
  h_unwrap();
#if REF_FLOW == 0
  calcCOM();
#endif
  if (t % printprops == 0) calcExt();
  checkVerlet();
  bondforce();
  LJforce();
  coulombForce();
  getNoise();
#if REF_FLOW == 1
  calcCOM();
#endif
  tcount = 0;
  updateHI();
  if (with_hop) {
#if REF_FLOW == 1
    transformCoords();
    chargeHop();
    inverseCoords();
#else
    chargeHop();
#endif
  }
}

/* Sequence used before the first step of an iteration
 * (shear/src/main26.c:45-48, extensional/src/main14.c:46-50). */
void h_begin_iteration(void) {
  updateLattice(tstart);
#if REF_FLOW == 1
  transformCoords();
#endif
  applyPBC();
  verletlist();
#if REF_FLOW == 1
  inverseCoords();
#endif
}

/* Wall-clock seconds, for timing the reference on the host cores. */
double h_wtime(void) { return omp_get_wtime(); }
int h_max_threads(void) { return omp_get_max_threads(); }

/* ewaldBin (shear/src/main26.c:975-1291): eps and rowsum (3N) for the current
 * positions, with the accumulators cleared first and after. */
void h_ewald_bin(double *eps_out, double *rowsum_out) {
  eps = 0.0;
  for (int i = 0; i < 3 * N; i++) rowsum[i] = 0.0;
  ewaldBin();
  *eps_out = eps;
  memcpy(rowsum_out, rowsum, sizeof(double) * 3 * N);
  eps = 0.0;
  for (int i = 0; i < 3 * N; i++) rowsum[i] = 0.0;
}

/* ewaldBin + CATEA (shear/src/main26.c:1340-1381) at the given strain; CATEA
 * appends its beta line to beta_path.  Returns the running sums brun
 * (sbins+1), Crun ((sbins+1) x 3Nb) and gwcount (sbins+1). */
void h_catea(double strain_, const char *beta_path, double *brun_out, double *crun_out,
             int *gw_out) {
  strain = strain_;
  beta = (char *)beta_path;
  ewaldBin();
  CATEA();
  for (int i = 0; i < sbins + 1; i++) {
    brun_out[i] = brun[i];
    gw_out[i] = gwcount[i];
    for (int j = 0; j < 3 * Nb; j++) crun_out[(size_t)i * 3 * Nb + j] = Crun[i][j];
  }
}

/* calcMSD (shear/src/main26.c:2494-2637) on the CH file at ch_path, writing
 * its MSD rows to out_path. */
void h_msd(const char *ch_path, const char *out_path, int ncharges, unsigned long tmax_,
           int printprops_, int msdstart, double dt_) {
  str2 = (char *)ch_path;
  outp1 = (char *)out_path;
  Ncharges = ncharges;
  tmax = tmax_;
  printprops = printprops_;
  MSDstart = msdstart;
  dt = dt_;
  calcMSD();
}

/* Output routines of the reference (shear/src/main26.c:870-974, 1866-1880)
 * writing to the given paths. */
#include <unistd.h>
void h_print_traj(const char *path) {
  xyz = (char *)path;
  printTrajectory();
}
void h_print_ext(const char *path) {
  /* the unwrapping loop of the reference's main (shear/src/main26.c:75-85) */
  for (int i = 0; i < Nc; i++) {
    px[i * Nb] = 0.0;
    py[i * Nb] = 0.0;
    pz[i * Nb] = 0.0;
    for (int j = 0; j < Nb - 1; j++) {
      Vector3D_t d = getNID(i * Nb + j, i * Nb + j + 1);
      px[i * Nb + j + 1] = px[i * Nb + j] + d.x;
      py[i * Nb + j + 1] = py[i * Nb + j] + d.y;
      pz[i * Nb + j + 1] = pz[i * Nb + j] + d.z;
    }
  }
  ext = (char *)path;
  calcExt();
  printExt();
}
void h_get_unwrapped(double *x, double *y, double *z) {
  memcpy(x, px, sizeof(double) * N);
  memcpy(y, py, sizeof(double) * N);
  memcpy(z, pz, sizeof(double) * N);
}
void h_print_visc(const char *path, int period) {
  visc = (char *)path;
  printperiod = period;
  printVisc();
}
/* printRestart names its file itself (res/R...xyz relative to the working
 * directory): run it inside dir. */
int h_print_restart(const char *dir) {
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd)) || chdir(dir) != 0) return 1;
  xyz = malloc(400);
  xyzstart = 0;
  printRestart();
  return chdir(cwd);
}
