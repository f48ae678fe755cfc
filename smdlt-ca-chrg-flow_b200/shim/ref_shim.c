/* Drop-in adapter: the reference simulator's hot step-loop routines on the
 * GPU through the bd_b200 C ABI.
 *
 * A maintainer compiles this file next to the reference's own sources
 * (shear/src: main26.c, Parameters.h; or extensional/src: main14.c, whose
 * routines of the same names it replaces alike, the flow chosen by the tree's
 * THETA0; compile it with -DREF_EXTENSIONAL there), against the tree's
 * Parameters.h
 * so that every global below is the reference's own, and links it with
 * libbd_b200.so.  The routines defined here replace the reference's bodies of
 * the same names (its object is linked with those symbols weakened, see
 * oracle/Makefile's drop-in target), while its main(), Initialization, random
 * streams (ran1/gasdev: getNoise, chargeHop, initChains), diagnostics and
 * file output stay as they are.  Each routine moves the globals it reads to
 * the device context, runs the device routine, and moves back what the
 * reference routine writes (updateHI also loads the lookup table D and the
 * CA-TEA parameters at an iteration's first step: the reference reads D in
 * resetAverage at the end of iteration 0, main26.c:1840-1860):
 *
 *   applyPBC     shear/src/main26.c:1409   rx, ry, rz
 *   verletlist   shear/src/main26.c:682    list on the device; dxv reset
 *   checkVerlet  shear/src/main26.c:858    dxv (reset when the list is rebuilt)
 *   bondforce    shear/src/main26.c:541    fx, fy, fz; tauxx, tauyy, tauxy
 *   LJforce      shear/src/main26.c:619    fx, fy, fz; tauxx, tauyy, tauxy
 *   coulombForce shear/src/main26.c:1891   fx, fy, fz (charges from Charge_track); kappa_d
 *   updateFD     shear/src/main26.c:731    rx, ry, rz, dxv
 *   updateHI     shear/src/main26.c:745    rx, ry, rz, dxv; dxt/dyt/dzt and tcount
 *                                          (the charges' displacement log)
 *
 * The neighbour list and the mobility stay on the device (the reference's
 * list/nlist and M are read only by the replaced routines).  A failing
 * device call prints the library's status and exits, as the reference does
 * on its own errors (printf + exit(1), e.g. main26.c:553-558).
 */
#include "Parameters.h"

#include "bd_b200.h"

static bd_ctx *g_bd;
static double *g_old;  /* rx, ry, rz before a displacement update (3 N) */

static void bd_fail(int s, const char *where) {
  if (s == BD_ERR_OVERSTRETCH)
    printf("FENE overstretch at t = %lu\n", t);
  else
    printf("bd_b200 %s: %s %s\n", where, bd_status_string(s), bd_last_error_detail());
  exit(1);
}
#define BD(call)                      \
  do {                                \
    int s_ = (call);                  \
    if (s_) bd_fail(s_, #call);       \
  } while (0)

/* The context, created at the first replaced call (after Initialization()
 * has read the command line and Input.txt). */
static bd_ctx *ctx(void) {
  if (g_bd) return g_bd;
  bd_params q;
  memset(&q, 0, sizeof q);
  q.flow = THETA0 == 0 ? BD_FLOW_SHEAR : BD_FLOW_EXT;
  q.Nb = Nb;
  q.Nc = Nc;
  q.L = L;
  q.box_volume = box_volume;
  q.edot = flowrate;
  q.dt = dt;
  q.spring = strcmp(spring, "FENE") == 0 ? BD_SPRING_FENE : BD_SPRING_HOOKEAN;
  q.kappas = kappas;
  q.qmax = qmax;
  q.kappab = kappab;
  q.epsilon = epsilon;
  q.lambda_b = lambda_b;
  q.lambda_d = lambda_d;
  q.Ncharges = Ncharges;
  q.barrier = barrier;
  q.barrier2 = barrier2;
  q.MStep = MStep;
  q.nt_avg = nt_avg;
  q.bin_size = bin_size;
  q.srpy = srpy;
  q.sbins = sbins;
  q.strain_ss = strain_ss;
  q.seed = *idum;
  q.noise = BD_NOISE_RAN1;
  q.mobility = BD_MOB_HYBRID;
  q.precision = BD_PREC_FP64;
  BD(bd_create(&q, &g_bd));
  g_old = malloc(sizeof(double) * 3 * (size_t)N);
  return g_bd;
}

/* The device lattice is the one the reference computed last: its main calls
 * updateLattice(t) in the step loop but updateLattice(tstart) before an
 * iteration's first applyPBC, while the global t still holds the end of the
 * previous iteration (applyPBC then takes delx from that t and the cell from
 * tstart, main26.c:44-47, 1409-1428).  The device lattice of the candidate
 * steps is compared with the reference's lattice globals (the same formula,
 * so equal to the bit); the step the kernels see is t itself. */
static unsigned long g_lat_t = 0;

static void put_state(void) {
  bd_ctx *c = ctx();
  unsigned long cand[4] = {g_lat_t, t, tstart, t > 0 ? t - 1 : 0};
  int found = 0;
  for (int k = 0; k < 4 && !found; k++) {
    double lat[10];
    BD(bd_update_lattice(c, cand[k]));
    BD(bd_get_lattice(c, lat));
    if (lat[4] == L1xp && lat[5] == L1yp && lat[6] == L2xp && lat[7] == L2yp) {
      g_lat_t = cand[k];
      found = 1;
    }
  }
  if (!found) {
    printf("bd_b200 adapter: the reference's lattice at step %lu is none of steps %lu, %lu\n", t,
           t, tstart);
    exit(1);
  }
  BD(bd_set_time(c, t, tstart));
  BD(bd_upload_positions(c, rx, ry, rz));
}

void applyPBC(void) {
  put_state();
  BD(bd_apply_pbc(g_bd));
  BD(bd_download_positions(g_bd, rx, ry, rz));
}

void verletlist(void) {
  put_state();
  BD(bd_build_neighbors(g_bd));
  for (int i = 0; i < N; i++) dxv[i] = dyv[i] = dzv[i] = 0.0;
}

void checkVerlet(void) {
  put_state();
  BD(bd_upload_displacements(g_bd, dxv, dyv, dzv));
  BD(bd_check_verlet(g_bd));
  BD(bd_download_displacements(g_bd, dxv, dyv, dzv));
}

/* forces: the host's accumulated forces in and out; the virial of this call
 * added to the reference's accumulators */
static void force_call(int (*f)(bd_ctx *)) {
  double tau[3];
  put_state();
  BD(bd_upload_forces(g_bd, fx, fy, fz));
  BD(bd_reset_stress(g_bd));
  BD(f(g_bd));
  BD(bd_download_forces(g_bd, fx, fy, fz));
  BD(bd_download_stress(g_bd, tau));
  tauxx += tau[0];
  tauyy += tau[1];
#ifndef REF_EXTENSIONAL
  tauxy += tau[2];  /* the extensional tree keeps only tauxx, tauyy */
#endif
}

void bondforce(void) { force_call(bd_bond_force); }
void LJforce(void) { force_call(bd_ev_force); }

void coulombForce(void) {
  /* the reference's coulombForce also sets the screening global that its
   * chargeHop reads for the Metropolis energies (main26.c:1899, 1966, 2194) */
  kappa_d = 1 / lambda_d;
  put_state();
  BD(bd_set_charges(g_bd, Charge_track, Ncharges));
  BD(bd_upload_forces(g_bd, fx, fy, fz));
  BD(bd_coulomb_force(g_bd));
  BD(bd_download_forces(g_bd, fx, fy, fz));
}

void updateFD(void) {
  put_state();
  BD(bd_upload_forces(g_bd, fx, fy, fz));
  BD(bd_upload_noise(g_bd, R));
  BD(bd_upload_displacements(g_bd, dxv, dyv, dzv));
  BD(bd_update_fd(g_bd));
  BD(bd_download_positions(g_bd, rx, ry, rz));
  BD(bd_download_displacements(g_bd, dxv, dyv, dzv));
}

void updateHI(void) {
  put_state();
  if (t == tstart) {  /* the lookup table and the last iteration's CA-TEA parameters */
    for (int nt = 0; nt < nt_avg; nt++) BD(bd_load_grid(g_bd, nt, D[nt]));
    for (int b = 0; b <= sbins; b++) BD(bd_set_tea(g_bd, b, bp[b], C[b]));
  }
  BD(bd_upload_forces(g_bd, fx, fy, fz));
  BD(bd_upload_noise(g_bd, R));
  BD(bd_upload_displacements(g_bd, dxv, dyv, dzv));
  memcpy(g_old, rx, sizeof(double) * N);
  memcpy(g_old + N, ry, sizeof(double) * N);
  memcpy(g_old + 2 * N, rz, sizeof(double) * N);
  BD(bd_update_hi(g_bd));
  BD(bd_download_positions(g_bd, rx, ry, rz));
  BD(bd_download_displacements(g_bd, dxv, dyv, dzv));
  /* the charges' displacement log, as the reference's updateHI writes it:
   * the hydrodynamic displacement (the step without its flow term: shear
   * dt flowrate (y, 0, 0), main26.c:845; planar extension
   * dt flowrate (x, -y, 0), extensional/src/main14.c:883-884) plus the flow
   * relative to the chain's centre of mass */
  tcount++;
  for (int i = 0; i < Ncharges; i++) {
    int j = Charge_track[i];
    int chain = (int)floor(j / Nb);
    double x0 = g_old[j], y0 = g_old[N + j];
    double dxh, dyh;
    if (THETA0 == 0) {
      dxh = (rx[j] - x0) - dt * flowrate * y0;
      dyh = ry[j] - y0;
      dxt[i * printprops + tcount] = dxh + dt * flowrate * (comy[chain] - py[j]);
      dyt[i * printprops + tcount] = dyh;
    } else {
      dxh = (rx[j] - x0) - dt * flowrate * x0;
      dyh = (ry[j] - y0) + dt * flowrate * y0;
      dxt[i * printprops + tcount] = dxh + dt * flowrate * (comx[chain] - px[j]);
      dyt[i * printprops + tcount] = dyh - dt * flowrate * (comy[chain] - py[j]);
    }
    dzt[i * printprops + tcount] = rz[j] - g_old[2 * N + j];
  }
}
