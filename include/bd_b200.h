/* bd_b200 -- B200-native Brownian-dynamics step path for charged bead-spring
 * chains in deforming-brick shear and Kraynik-Reinelt planar extension.
 *
 * C ABI of the drop-in boundary.  The reference simulator's step loop is a
 * set of `void f(void)` routines that exchange data through file-scope
 * globals (shear/src/main.h:7-65, shear/src/Parameters.h:44-201).  Each
 * routine below replaces one of them, operating on device-resident state
 * owned by a bd_ctx instead of on globals; the upload/download calls move
 * the reference's global arrays in and out, with the reference's layouts
 * (three double arrays rx/ry/rz of N beads, forces fx/fy/fz, noise R[3N]
 * interleaved x,y,z per bead, dense mobility M[9 N^2] row-major by 3x3
 * block).
 *
 * Conventions
 *  - every call returns a bd_status; 0 is success;
 *  - calls are asynchronous on the context's CUDA stream unless they return
 *    data to the host (downloads, bd_sync), which synchronise and report any
 *    error a kernel recorded since the last check;
 *  - where the reference prints a message and calls exit(1) (FENE
 *    overstretch, shear/src/main26.c:553-558), the library records a status
 *    and returns it instead; nothing in the library exits the process;
 *  - no call falls back to the CPU: without a usable CUDA device bd_create
 *    fails with BD_ERR_CUDA.
 */
#ifndef BD_B200_H
#define BD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  BD_OK = 0,
  BD_ERR_ARG = 1,          /* bad argument or size */
  BD_ERR_CUDA = 2,         /* CUDA runtime failure / no device */
  BD_ERR_OOM = 3,          /* device allocation failed */
  BD_ERR_OVERSTRETCH = 4,  /* FENE bond longer than qmax */
  BD_ERR_NONFINITE = 5,    /* NaN/Inf in a force or displacement */
  BD_ERR_NBR_OVERFLOW = 6, /* neighbour row longer than the configured cap */
  BD_ERR_GRID_RANGE = 7,   /* far-field displacement outside the lookup table */
  BD_ERR_STATE = 8,        /* call out of order (e.g. no mobility built) */
  BD_ERR_TIMEOUT = 9,      /* a bounded device wait gave up */
  BD_ERR_LANCZOS = 10,     /* Krylov square root missed its tolerance */
  BD_ERR_ASYMMETRIC = 11,  /* lookup tensor not symmetric */
  BD_ERR_CAPACITY = 12     /* system larger than a fixed-size buffer allows */
} bd_status;

typedef enum { BD_FLOW_SHEAR = 0, BD_FLOW_EXT = 1 } bd_flow;
/* Brownian noise source for bd_get_noise: the reference's sequential
 * ran1/gasdev stream (bit-identical, one device thread) or counter-based
 * Philox4x32-10 Gaussians (parallel; the production source). */
typedef enum { BD_NOISE_RAN1 = 0, BD_NOISE_PHILOX = 1 } bd_noise;
/* Pair mobility: the reference's hybrid (Ewald sum below a minimum-image
 * distance of 12, lookup table beyond, shear/src/main26.c:1714-1794), the
 * Ewald sum for every pair as a dense packed matrix, or the same Ewald sum
 * applied matrix-free by smooth particle-mesh Ewald (no reference
 * counterpart; O(N + K^3 log K) per product, for systems whose dense
 * matrix does not fit). */
typedef enum { BD_MOB_HYBRID = 0, BD_MOB_EWALD = 1, BD_MOB_PME = 2 } bd_mobility_kind;
/* Preconditioner of the Lanczos square root (no reference counterpart):
 * none; segment blocks (G = L^-1 from the Cholesky factor of the free-space
 * RPY mobility of S consecutive beads of a chain); per-bead 3x3 blocks
 * predicted by the learned message-passing network; or per-bead blocks set
 * by the caller.  The displacement is G^-1 sqrt(G M G^T) z. */
typedef enum {
  BD_PRECOND_NONE = 0,
  BD_PRECOND_SEGMENT = 1,
  BD_PRECOND_LEARNED = 2,
  BD_PRECOND_BLOCKS = 3
} bd_precond_kind;
#define BD_PRECOND_MAX_SEGMENT 25
/* Largest noise block of bd_step_lanczos (bd_params.noise_block). */
#define BD_MAX_NOISE_BLOCK 64
/* Storage of the packed mobility tiles used by the products: FP64, or FP32
 * with FP64 accumulation. */
typedef enum { BD_PREC_FP64 = 0, BD_PREC_FP32 = 1 } bd_precision;
typedef enum { BD_SPRING_HOOKEAN = 0, BD_SPRING_FENE = 1 } bd_spring;
/* Electrostatics: the reference's Debye-Hueckel pair force over all charged
 * pairs (coulombForce, shear/src/main26.c:1891-1925), or the unscreened
 * Coulomb interaction Ewald-summed over the periodic lattice (no reference
 * counterpart; real-space pairs within coulomb_rc plus a particle-mesh
 * reciprocal sum on the pme_grid / pme_order grid). */
typedef enum { BD_COULOMB_DH = 0, BD_COULOMB_EWALD = 1 } bd_coulomb_kind;
/* Charge-hop sweep: the reference's sequential sweep (chargeHop,
 * shear/src/main26.c:1926-2390, ran1 draws, bit-exact), or a parallel sweep
 * on independent sets of cells at least hop_radius apart with Philox draws
 * (no reference counterpart; bd_charge_hop documents its approximation). */
typedef enum { BD_HOP_SEQUENTIAL = 0, BD_HOP_PARALLEL = 1 } bd_hop_kind;

/* System parameters.  The names follow the reference's globals
 * (shear/src/Parameters.h:57-199) and Input.txt keys
 * (shear/src/Initialization.c:157-174). */
typedef struct {
  int flow;           /* bd_flow */
  int Nb, Nc;         /* beads per chain, chains */
  double L;           /* cubic box edge */
  double box_volume;  /* 0 -> L^3 (used by the k-space mobility sum) */
  double edot;        /* strain rate (flowrate) */
  double dt;          /* time step */
  int spring;         /* bd_spring */
  double kappas, qmax, kappab, epsilon;
  /* Reference-compatible force-law switches (0 = reference behaviour):
   * shear_kappas_override: 0 -> kappas forced to 200 in the shear tree
   * (shear/src/main26.c:544) as the reference does; 1 -> use kappas. */
  int shear_kappas_override;
  double lambda_b, lambda_d; /* Bjerrum and Debye lengths */
  int Ncharges;
  double barrier, barrier2;  /* adjacent / non-adjacent hop barriers */
  int MStep;                 /* charge-hop sweep period */
  int nt_avg;                /* lookup-table lattice frames */
  double bin_size;           /* lookup-table bin edge */
  int srpy;                  /* mobility rebuild period; 0 -> 100 */
  int sbins;                 /* CA-TEA strain bins; 0 -> 20 */
  double strain_ss;          /* CA-TEA steady-state strain; 0 -> 10 */
  int max_neighbors;         /* neighbour-row cap; 0 -> 256 */
  long seed;                 /* ran1 seed (fixSeed=1: 830062920 shear, 981272199 ext) */
  int noise;                 /* bd_noise */
  unsigned long long philox_seed;
  int mobility;              /* bd_mobility_kind */
  int precision;             /* bd_precision */
  double lanczos_tol;        /* bound on the estimated relative error of sqrt(M) z (the
                                geometric tail of the successive changes); 0 -> 1e-6 */
  int lanczos_max;           /* Krylov dimension cap, at most 400; 0 -> 200 */
  /* BD_MOB_PME discretisation (no reference counterpart): grid points per
   * reduced lattice direction (0 -> smallest 2^a 3^b 5^c >= 12.9 L / rc,
   * i.e. 1.29 L at the default cutoff 10: spacing proportional to the cutoff,
   * split parameter times spacing at most 0.31),
   * B-spline order (even, 4..8; 0 -> 8), real-space cutoff (0 -> the smaller
   * of 10 and 0.43 L; at most 0.43 L), split parameter (0 -> 4 / cutoff) and the cap on
   * real-space pairs per bead (0 -> 2.5 times the mean number of beads within
   * the cutoff, at least 512, and rows that overflow it are grown to 1.25
   * times the longest row at the mobility build; an explicit cap that
   * overflows is BD_ERR_NBR_OVERFLOW). */
  int pme_grid;
  int pme_order;
  double pme_rc;
  double pme_alpha;
  int pme_max_pairs;
  int coulomb;               /* bd_coulomb_kind */
  double coulomb_beta;       /* Ewald split; 0 -> 3.5 / coulomb_rc (erfc(3.5) = 7e-7) */
  double coulomb_rc;         /* real-space cutoff; 0 -> the smaller of 10 and 0.43 L */
  int hop;                   /* bd_hop_kind */
  double hop_radius;         /* parallel sweep: minimum distance between cells that
                                move at once; 0 -> 3 lambda_d */
  /* bd_step_lanczos with BD_MOB_PME: number of steps whose Brownian
   * displacements sqrt(M) z_t are solved together by one multi-vector Lanczos
   * run (0 or 1 -> one per step, at most BD_MAX_NOISE_BLOCK).  The mobility
   * is frozen between rebuilds and z_t does not depend on the state, so the
   * block gives every step the displacement the per-step solve gives (to the
   * Lanczos tolerance), with the same draws in the same order. */
  int noise_block;
} bd_params;

typedef struct bd_ctx bd_ctx;

/* State of the reference's ran1/gasdev generator
 * (shear/src/Initialization.c:601-634, shear/src/main26.c:515-540). */
typedef struct {
  long idum, idum2, iy;
  long iv[32];
  int iset;
  float gset;
} bd_ran1_state;

/* ---- context ------------------------------------------------------------
 * replaces Initialization()/allocate() (shear/src/Initialization.c:3-23,
 * 318-457): allocates device state for N = Nb*Nc beads. */
int bd_create(const bd_params *p, bd_ctx **out);
int bd_destroy(bd_ctx *ctx);
const char *bd_status_string(int status);
/* Source line, message and code of the last CUDA or cuFFT failure reported
 * as BD_ERR_CUDA on the calling thread ("" if none). */
const char *bd_last_error_detail(void);
int bd_sync(bd_ctx *ctx);
/* Device bytes currently held by the context. */
size_t bd_device_bytes(const bd_ctx *ctx);

/* ---- state transfer (the reference's global arrays) --------------------- */
int bd_upload_positions(bd_ctx *ctx, const double *rx, const double *ry, const double *rz);
int bd_download_positions(bd_ctx *ctx, double *rx, double *ry, double *rz);
int bd_upload_displacements(bd_ctx *ctx, const double *dxv, const double *dyv, const double *dzv);
int bd_download_displacements(bd_ctx *ctx, double *dxv, double *dyv, double *dzv);
int bd_upload_forces(bd_ctx *ctx, const double *fx, const double *fy, const double *fz);
int bd_download_forces(bd_ctx *ctx, double *fx, double *fy, double *fz);
/* tauxx, tauyy, tauxy virial accumulators (shear/src/Parameters.h:98,138) */
int bd_download_stress(bd_ctx *ctx, double *out3);
int bd_reset_stress(bd_ctx *ctx);
int bd_upload_noise(bd_ctx *ctx, const double *R);
int bd_download_noise(bd_ctx *ctx, double *R);
/* Charge_track (bead of each charge); sets Charge[] flags to 1 there
 * (shear/src/main26.c:490-506). */
int bd_set_charges(bd_ctx *ctx, const int *track, int ncharges);
int bd_download_charges(bd_ctx *ctx, int *track, int *old, int *flags);
int bd_set_rng(bd_ctx *ctx, const bd_ran1_state *s);
int bd_get_rng(bd_ctx *ctx, bd_ran1_state *s);
/* One lattice frame (nt < nt_avg) of the far-field lookup table read from
 * mm/G*.txt by initEwald (shear/src/Initialization.c:497-520): num_bins
 * row-major 3x3 tensors.  The tensors must be symmetric. */
int bd_load_grid(bd_ctx *ctx, int nt, const double *D9);
/* Builds all nt_avg frames of the lookup table on the device, as the
 * reference's separate gridHI program does (shear/src/gridHI.c:3-278),
 * instead of reading mm/G*.txt.  grid_dt is gridHI's own time step (it
 * hard-codes 0.001, shear/src/gridHI.c:288; 0 selects that).  Fails with
 * BD_ERR_STATE if gridHI's bin geometry differs from the simulation's. */
int bd_build_grid(bd_ctx *ctx, double grid_dt);
int bd_download_grid(bd_ctx *ctx, int nt, double *D9);
/* Lookup-grid geometry as initLattice derives it
 * (shear/src/Initialization.c:281-295): nbx nby nbz nhx nhy nhz num_bins. */
int bd_grid_shape(const bd_ctx *ctx, int *out7);
/* CA-TEA parameters of one strain bin (bp[sbin], C[sbin][3 Nb]) read from
 * decomp/DC*.txt (shear/src/Initialization.c:528-536). */
int bd_set_tea(bd_ctx *ctx, int sbin, double beta, const double *c3nb);

/* ---- step-loop routines (reference name in brackets) -------------------- */
int bd_set_time(bd_ctx *ctx, unsigned long t, unsigned long tstart);
int bd_update_lattice(bd_ctx *ctx, unsigned long t);   /* [updateLattice] main26.c:1382 */
/* L1x L1y L2x L2y L1xp L1yp L2xp L2yp detL tp */
int bd_get_lattice(const bd_ctx *ctx, double *out10);
int bd_apply_pbc(bd_ctx *ctx);                         /* [applyPBC] main26.c:1409 */
int bd_transform_coords(bd_ctx *ctx);                  /* [transformCoords] main14.c:1514 */
int bd_inverse_coords(bd_ctx *ctx);                    /* [inverseCoords] main14.c:1525 */
int bd_reset_force(bd_ctx *ctx);                       /* [resetForce] main26.c:509 */
int bd_build_neighbors(bd_ctx *ctx);                   /* [verletlist] main26.c:682 */
int bd_check_verlet(bd_ctx *ctx);                      /* [checkVerlet] main26.c:858 */
/* Half list as verletlist stores it: counts[N], rows[N*maxnb] ascending. */
int bd_download_neighbors(bd_ctx *ctx, int *counts, int *rows, int maxnb);
int bd_bond_force(bd_ctx *ctx);                        /* [bondforce] main26.c:541 */
int bd_ev_force(bd_ctx *ctx);                          /* [LJforce] main26.c:619 */
int bd_coulomb_force(bd_ctx *ctx);                     /* [coulombForce] main26.c:1891 */
int bd_get_noise(bd_ctx *ctx);                         /* [getNoise] main26.c:708 */
int bd_calc_hi(bd_ctx *ctx);                           /* [calcHI] main26.c:1530 */
/* Dense reference layout 9 N^2 (upper blocks and diagonal entries of the
 * diagonal blocks filled, as calcHI leaves them). */
int bd_download_mobility(bd_ctx *ctx, double *M9);
int bd_update_hi(bd_ctx *ctx);                         /* [updateHI] main26.c:745 */
int bd_update_fd(bd_ctx *ctx);                         /* [updateFD] main26.c:731 */
/* [chargeHop] main26.c:1926.  With hop = BD_HOP_PARALLEL the sweep runs on
 * independent sets: cells at least hop_radius wide in eight parity colours,
 * each cell's charges in index order, a trial seeing the charges of other
 * cells at their sites at the colour's start.  Its acceptance test uses the
 * energy the forces use: the Debye-Hueckel pair energy with
 * coulomb = BD_COULOMB_DH, the Ewald-summed unscreened energy in FP64 with
 * BD_COULOMB_EWALD (real-space pairs, the mesh reciprocal potential of the
 * colour's start, the moved charge's own reciprocal term and those of the
 * cell's earlier moves).  The coupling of simultaneous moves in different
 * cells is left out: at most 2 lambda_B d^2 / R^3 per pair (hop distance
 * d <= 2.1, cells R apart). */
int bd_charge_hop(bd_ctx *ctx);
/* Per-charge outcome of the last sweep: (0 skipped,1 accepted,2 rejected),
 * target bead, move kind; 3 ints per charge. */
int bd_download_hop_log(bd_ctx *ctx, int *log3);
/* Energy change (kT) each charge's trial of the last parallel sweep saw, in
 * track order (NaN where the move was blocked).  No reference counterpart:
 * the parallel sweep's check against its CPU model. */
int bd_download_hop_energies(bd_ctx *ctx, double *dE);

/* ---- measurement -----------------------------------------------------
 * Device time of selected kernels, measured with CUDA events recorded on
 * the context's stream around each launch while profiling is enabled. */
enum {
  BD_PROF_MATVEC = 0,   /* packed symmetric mobility product (2 right-hand sides) */
  BD_PROF_HI_BUILD = 1, /* mobility build (far + near passes) */
  BD_PROF_HOP = 2,      /* charge-hop sweep kernel */
  BD_PROF_FORCES = 3,   /* bond + excluded-volume + electrostatic kernels */
  BD_PROF_STEP = 4,     /* one whole bd_step_reference call */
  BD_PROF_BLOCK = 5,    /* particle-mesh product of a noise block or of
                           bd_mobility_apply_block (all its right-hand sides) */
  BD_PROF_SLOTS = 8
};
/* Replay each Lanczos iteration (product and orthogonalisation) as a CUDA
 * graph captured on first use (default on; off launches the kernels one by
 * one).  Captured products do not record BD_PROF_MATVEC events. */
int bd_enable_graphs(bd_ctx *ctx, int on);
/* Convergence of the noise blocks' Krylov runs checked on the device (default
 * on; no reference counterpart).  After every iteration one CTA per
 * right-hand side forms T^(1/2) e_1 of its tridiagonal T in FP64 by a
 * trapezoidal quadrature of (2/pi) int T (t^2 + T)^-1 e_1 dt (one tridiagonal
 * solve per node, no eigen-decomposition) and applies the stopping test; with
 * graphs on, the whole solve of a block is one CUDA graph whose conditional
 * while node repeats the iteration until every right-hand side has stopped,
 * with no host round trip.  Off (or with profiling on, which times each
 * product): the host checks one iteration behind with the implicit QR.  A
 * tridiagonal that is not positive definite (never expected of a mobility)
 * is re-solved on the host, which clamps its negative Ritz values. */
int bd_set_device_krylov(bd_ctx *ctx, int on);
/* Noise-block solves controlled on the device, and blocks re-solved on the
 * host (non-positive tridiagonal), since creation. */
int bd_krylov_check_stats(bd_ctx *ctx, long *out2);
/* on = 1: every slot; on = 2: every slot but BD_PROF_BLOCK, whose per-product
 * events need the host-checked Krylov loop (so 2 times the device-checked
 * one); 0: off.  Clears the accumulated events. */
int bd_profile_enable(bd_ctx *ctx, int on);
int bd_profile_read(bd_ctx *ctx, int slot, double *total_ms, long *count);
/* Number of kernels the library has launched on this context. */
long long bd_launch_count(const bd_ctx *ctx);

/* ---- Krylov Brownian displacement (no reference counterpart: the
 * reference's noise is the conformationally averaged TEA approximation of
 * updateHI, shear/src/main26.c:745-857) ----------------------------------- */
/* out = M v for a host vector v[3N] (bead-interleaved), using the mobility of
 * the last bd_calc_hi (diagonal blocks included). */
int bd_mobility_apply(bd_ctx *ctx, const double *v, double *out);
/* out_r = M v_r for k host vectors (v[r 3N + 3 i + a], out likewise), the
 * product the noise blocks use: with BD_MOB_PME and 2 <= k <= noise_block the
 * right-hand sides go through the particle-mesh transforms together, packed
 * in complex pairs; otherwise one product each. */
int bd_mobility_apply_block(bd_ctx *ctx, int k, const double *v, double *out);
/* out = sqrt(M) z by Lanczos with full FP64 reorthogonalisation, stopped when
 * the geometric tail of the successive relative changes d_m, d_m rho / (1 -
 * rho) with rho = (d_m / d_(m-6))^(1/6) capped at 0.99 (an estimate of the
 * iterate's own error), is below lanczos_tol (half of it with a
 * preconditioner, whose inverse factor amplifies the error); *iters receives
 * the Krylov dimension used. */
int bd_lanczos_sqrt(bd_ctx *ctx, const double *z, double *out, int *iters);
/* calls, total Krylov iterations, calls that hit lanczos_max, negative Ritz
 * values clamped (a hybrid mobility need not be positive definite) */
int bd_lanczos_stats(bd_ctx *ctx, long *out4);
/* Noise blocks of bd_step_lanczos: block solves run, block iterations
 * launched (one iteration = one product of every right-hand side) and the
 * sum over those iterations of their right-hand sides. */
int bd_noise_block_stats(bd_ctx *ctx, long *out3);
/* Drops the noise block solved ahead (if any): the generator is wound back to
 * the draws the per-step order has made, and the next bd_step_lanczos solves
 * a new block from its own step on. */
int bd_noise_block_release(bd_ctx *ctx);
/* No counterpart in the reference.  out = M v like bd_mobility_apply, for
 * callers that must not allocate device memory where they call it (a loop
 * running while another framework's pool owns the device, a fixed memory
 * budget, or code that must avoid the device-wide synchronisation
 * cudaMalloc/cudaFree can cause).  v and out are device pointers,
 * bead-interleaved (v[3 i + a]); the call is asynchronous on the context's
 * stream and allocates nothing: its scratch is a fixed device array of the
 * library (14.3 MB, held on every GPU that loads the library until exit), so
 * N may not exceed BD_NOALLOC_MAX_BEADS (else BD_ERR_CAPACITY).  All calls on
 * a device share that array: calls that overlap on the GPU race.  The first
 * call on a device looks up the array's device address; make it before any
 * stream capture.  The context's device must be current.  Dense-tile
 * mobilities only (BD_MOB_EWALD, BD_MOB_HYBRID): a particle-mesh context gets
 * BD_ERR_STATE.  The address is kept for the process's life: calls after a
 * cudaDeviceReset are not supported. */
#define BD_NOALLOC_MAX_BEADS 4096
int bd_mobility_apply_noalloc(bd_ctx *ctx, const double *v, double *out);

/* One Brownian-dynamics step with the Krylov displacement
 * dr = dt M F + sqrt(2 dt) M^(1/2) z + dt u(r): the reference's step order
 * (lattice, PBC, neighbour check, forces, mobility rebuild every srpy steps,
 * charge hop every MStep steps) with z from bd_get_noise; repeated nsteps
 * times.  With noise_block B > 1 (particle-mesh mobility) the displacements
 * M^(1/2) z_t of up to B consecutive steps are solved by one multi-vector
 * Lanczos run when the first of them starts; a block never spans a mobility
 * rebuild, the end of the call, or (ran1 noise with the sequential hop, which
 * draw from one generator) a charge-hop sweep. */
int bd_step_lanczos(bd_ctx *ctx, unsigned long t0, int nsteps, int with_hop);

/* One reference-mode hydrodynamic step (the body of the step loop,
 * shear/src/main26.c:65-151, extensional/src/main14.c:68-171, without file
 * output), repeated nsteps times from step t0. */
/* ---- CA-TEA sampling ---------------------------------------------------
 * [ewaldBin] main26.c:975: eps and rowsum (3 N) for the positions as they
 * are (the caller chooses the frame, as the reference does). */
int bd_ewald_bin(bd_ctx *ctx, double *eps, double *rowsum);
/* [ewaldBin + CATEA] main26.c:975, 1340: adds one sample at the given strain
 * to the running sums of its strain bin; returns the sample's beta. */
int bd_catea(bd_ctx *ctx, double strain, double *beta);
/* running averages per strain bin (sbins + 1): counts, beta = brun/count,
 * C = Crun/(Nc count) (3 Nb per bin); zeros for empty bins */
int bd_catea_averages(bd_ctx *ctx, int *counts, double *beta, double *C);
/* [printTEA] main26.c:1807: the decomp/DC file of the averages */
int bd_write_decomp(bd_ctx *ctx, const char *path, unsigned long t);
/* [resetAverage] main26.c:1827: load the averages as the TEA parameters of
 * every bin (bd_set_tea) and restart the running sums */
int bd_catea_apply(bd_ctx *ctx);

/* [calcMSD] main26.c:2494: mean-squared displacement of the charges from
 * the displacement log w (Ncharges (Tmax + 1) records x, y, z in the order of
 * the reference's CH file), with the reference's data layout; avg gets, for
 * lags 1 .. Tmax - MSDstart, the rows {MSD, MSD_x, MSD_y, MSD_z} that
 * calcMSD writes (the caller adds the lag time lag dt printprops). */
int bd_msd(const double *w, int ncharges, int Tmax, int MSDstart, double *avg);

/* ---- output files in the reference's formats --------------------------
 * Unwrapped coordinates (3 N: px, py, pz as the reference's main builds
 * them, shear/src/main26.c:75-85), per-chain x extension (Nc), centre of
 * mass (3 Nc) and gyration tensor (6 Nc: xx xy xz yy yz zz); any pointer
 * may be null. */
int bd_chain_props(bd_ctx *ctx, double *p3N, double *ext, double *com, double *rg);
int bd_write_trajectory(bd_ctx *ctx, const char *path, unsigned long t); /* [printTrajectory] main26.c:870 */
int bd_write_restart(bd_ctx *ctx, const char *path, unsigned long t);    /* [printRestart] main26.c:902 */
int bd_write_ext(bd_ctx *ctx, const char *path, unsigned long t, double strain); /* [calcExt+printExt] main26.c:926, 963 */
int bd_write_visc(bd_ctx *ctx, const char *path, unsigned long t, int printperiod); /* [printVisc] main26.c:1866 */

/* ---- signed charges and the Ewald Coulomb energy (no reference counterpart)
 * bd_set_charges gives every charge the value +1, as the reference's charge
 * flags do; bd_set_charge_values sets signed values per charge (in the order
 * of the track passed to bd_set_charges; the values move with the charges
 * when they hop).  bd_coulomb_energy returns, for the last bd_coulomb_force
 * with coulomb = BD_COULOMB_EWALD: real-space, reciprocal, self plus
 * neutralising-background, and total energy (kT). */
int bd_set_charge_values(bd_ctx *ctx, const double *qk);
int bd_coulomb_energy(bd_ctx *ctx, double *out4);

/* ---- Lanczos preconditioner (no reference counterpart) ------------------
 * kind: bd_precond_kind; segment: beads per block for BD_PRECOND_SEGMENT
 * (must divide Nb, at most BD_PRECOND_MAX_SEGMENT; 0 -> 10 or the largest of
 * 5, 4, 2, 1 dividing Nb).  For BD_PRECOND_LEARNED, segment > 1 applies the
 * learned bead blocks B on top of segment blocks (G = B L^-1, the network
 * then being trained on targets of the segment-preconditioned operator);
 * segment <= 1 uses the bead blocks alone.  Blocks are rebuilt with every
 * mobility build.  A preconditioned solve that misses lanczos_tol within
 * lanczos_max is redone without the preconditioner (counted as a fallback). */
int bd_set_preconditioner(bd_ctx *ctx, int kind, int segment);
/* per-bead blocks G (9 N, row-major 3x3) for BD_PRECOND_BLOCKS */
int bd_set_precond_blocks(bd_ctx *ctx, const double *G9);
/* current blocks: N/S blocks of (3S)^2 row-major values each */
int bd_download_precond_blocks(bd_ctx *ctx, double *G, double *Ginv, int *block_beads);
/* preconditioned calls, their Krylov iterations, fallbacks, identity blocks */
int bd_precond_stats(bd_ctx *ctx, long *out4);
/* A^-1/2 z by Lanczos, A = M, or G M G^T while the segment preconditioner is
 * active (training targets of the learned preconditioner); BD_ERR_LANCZOS
 * when the tolerance is missed */
int bd_lanczos_inv_sqrt(bd_ctx *ctx, const double *z, double *out, int *iters);

/* ---- ensembles of replicas (no reference counterpart) --------------------
 * A batch advances independent contexts (any sizes, flows, strain rates)
 * concurrently: one host worker thread per replica drives that context's
 * own CUDA stream.  bd_batch_step_lanczos runs bd_step_lanczos(t0, nsteps,
 * with_hop) on every replica and returns when all have finished, with the
 * first non-zero status.  Contexts stay owned by the caller and must outlive
 * the batch; a context must not be used elsewhere while a batch step runs. */
typedef struct bd_batch bd_batch;
int bd_batch_create(bd_ctx *const *ctxs, int n, bd_batch **out);
int bd_batch_step_lanczos(bd_batch *batch, unsigned long t0, int nsteps, int with_hop);
int bd_batch_destroy(bd_batch *batch);
/* Particle-mesh grid for a box of edge L: of the 2^a 3^b 5^c sizes between
 * 1.29 L (the accuracy bound of the default discretisation) and 25 % above,
 * the one with the fastest three-component FFT round trip on the current
 * device (bd_precision for the storage); results are cached per process. */
int bd_autotune_pme_grid(double L, int precision, int *K_out);
/* The default particle-mesh grid bd_create picks for a box of edge L and a
 * real-space cutoff rc (rc <= 0: the default cutoff, the smaller of 10 and
 * 0.43 L): the smallest 2^a 3^b 5^c >= 12.9 L / rc.  Host arithmetic only
 * (no device needed); BD_ERR_ARG for L <= 0 or a grid above 4096. */
int bd_pme_default_grid(double L, double rc, int *K_out);

/* Raw Philox4x32-10 (Salmon et al., SC'11) on the device: block k of out
 * (4 words) is the generator applied to counter ctr[4k..4k+3] under key
 * key[2k..2k+1], for 1 <= n <= 2^20 blocks.  No reference counterpart (the
 * reference's generator is ran1); this is the function behind the
 * library's Philox noise and charge-hop draws, exposed so that it can be
 * checked against the published Random123 known-answer vectors.  Uses the
 * current device and the default stream; allocates and frees a small device
 * buffer. */
int bd_philox4x32_10(const unsigned *ctr, const unsigned *key, unsigned *out, int n);

/* ---- learned preconditioner network (no reference counterpart) ----------
 * Per bead, the BD_MPNN_NEIGHBORS nearest beads within BD_MPNN_CUTOFF
 * (minimum image) feed a three-layer message-passing network of width
 * BD_MPNN_WIDTH (BF16 operands, FP32 accumulation on the tensor cores) whose
 * heads give G_i = a_i (I + sum_j c_ij n_ij n_ij^T), n_ij the unit pair
 * vectors, a_i > 0, |c_ij| <= 1/(2 BD_MPNN_NEIGHBORS).  Training minimises
 * (1/N) sum_i |G_i z_i - u_i|^2 over pairs (z, u = M^-1/2 z), whose minimiser
 * is the diagonal block of M^-1/2.  Parameters are FP32 masters, layout
 * given by bd_mpnn_param_count (W1, b1, W2, b2, W3, W4, b3, wa, ca, wb, cb). */
#define BD_MPNN_NEIGHBORS 12
#define BD_MPNN_WIDTH 64
#define BD_MPNN_RBF 16
#define BD_MPNN_CUTOFF 6.0
size_t bd_mpnn_param_count(void);
int bd_mpnn_set_params(bd_ctx *ctx, const float *w);
int bd_mpnn_get_params(bd_ctx *ctx, float *w);
/* neighbour features of the current configuration (positions and lattice) */
int bd_mpnn_features(bd_ctx *ctx);
/* forward pass: the predicted blocks, 9 N row-major */
int bd_mpnn_predict(bd_ctx *ctx, double *G9);
/* loss and parameter gradient for one pair (z, u) of the current features;
 * the gradient stays on the device unless grad is non-null */
int bd_mpnn_loss_grad(bd_ctx *ctx, const double *z, const double *u, double *loss, float *grad);
/* one Adam step (Kingma and Ba, 2015) with the last gradient */
int bd_mpnn_adam(bd_ctx *ctx, float lr, float beta1, float beta2, float eps, int step);

int bd_step_reference(bd_ctx *ctx, unsigned long t0, int nsteps, int with_hop);

#ifdef __cplusplus
}
#endif
#endif
