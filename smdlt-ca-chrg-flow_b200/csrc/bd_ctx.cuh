// Context layout shared by the bd_b200 translation units.
//
// Device memory layout (all FP64 unless noted):
//   positions rx, ry, rz          SoA, N each (the reference's globals)
//   forces fx, fy, fz             SoA
//   displacement since last neighbour build dxv, dyv, dzv
//   noise R                       3N, interleaved x,y,z per bead (as R[])
//   neighbour rows                N x max_neighbors int32, full list sorted
//                                 ascending; half list = entries > i
//   mobility tiles                packed upper triangle of 32x32-bead tiles,
//                                 each tile 6 x 32 x 32 (xx xy xz yy yz zz)
//   lookup grid                   nt_avg x num_bins x 6
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "bd_internal.cuh"

// Largest Krylov dimension of the Lanczos square root.
constexpr int kMaxKrylov = 400;
// Largest block of the segment preconditioner, in beads.
constexpr int kMaxSegment = BD_PRECOND_MAX_SEGMENT;

struct bd_ctx {
  bd_params p;
  int N, Nb, Nc;
  cudaStream_t stream;
  int device;

  // derived constants
  double rv, r2cut, rnew, qmax2, kappa_d, boxvol, kappas_eff;
  int tp, srpy, sbins, maxnb;
  double strain_ss, strain_interval;
  // lookup grid geometry (initLattice, shear/src/Initialization.c:281-295)
  int nbx, nby, nbz, nhx, nhy, nhz, nbins;
  double bsx, bsy, bsz;

  // step state (host-side mirror)
  unsigned long t, tstart;
  double strain;
  bd::Lat lat;

  // device state
  double *rx, *ry, *rz, *fx, *fy, *fz, *dxv, *dyv, *dzv, *R;
  double *stress;  // 3
  int *err;        // error bits
  int *flag;       // [0] neighbour rebuild due
  int nch;
  int *track, *old, *cflags, *hoplog;  // charges
  double *q;                           // bead charge values (0/1 in reference mode)
  double *dE;                          // charge-hop energy scratch
  bd::Ran1 *rng;
  unsigned long long noise_draws;  // Philox counter: one per bd_get_noise call

  // neighbours
  int *nb_count, *nb_rows, *nb_half;
  int *cell_of, *cell_count, *cell_start, *cell_beads, *cell_cursor;
  int ncell_cap;

  // mobility (packed symmetric tiles)
  int NT;
  size_t ntiles;
  double *Mt;
  float *Mt32;   // FP32 copy of the tiles (BD_PREC_FP32), products accumulated in FP64
  int *tileI;  // tile row index of each packed tile
  double *grid;
  int grid_loaded_mask;
  int *near_pairs, *near_count;
  size_t near_cap;
  double *kvec;
  int kvec_cap, nk;
  double Dtr[3];
  bool hi_built;
  double *rowpart, *colpart;  // matvec partial sums (scratch)
  double *U, *W;              // M F and off-diagonal M R
  double *Ctab;               // (sbins+1) x 3 Nb
  std::vector<double> btab;
  double bt;
  int sbin;

  // Krylov (Lanczos) square root
  int lmax;
  double ltol;
  double *LV;     // (lmax+1) basis vectors, each 3 x NTp SoA (component-major, padded)
  double *Lw;     // work vector, 3 x NTp
  double *Lpart;  // per-block partial dots, (lmax+1) x kDotBlocks
  double *Lh;     // dot results, lmax+1
  double *Lsc;    // device scalars: [0] beta, [1] 1/beta
  double *Lc;     // Ritz combination coefficients, lmax+1
  double *MF;     // M F, 3 x NTp
  double *Yz;     // sqrt(M) z, 3 x NTp
  double *Lt1, *Lt2;  // work vectors of the preconditioned products, 3 x NTp
  double *Lvcur;      // input of the next product (v_j), 3 x NTp
  int *Ljd;           // Lanczos iteration index on the device
  void *lan_graph[2]; // captured iteration (plain, preconditioned), cudaGraphExec_t
  long long lan_graph_launches[2];
  bool use_graphs, capturing;
  long long lan_calls, lan_iters, lan_maxed, lan_negative;
  int lan_last, pre_last;

  // multi-vector Lanczos over a block of steps' noise (bd_step_lanczos with
  // noise_block > 1); vector (j, r) of the basis at BV + (j * nbk + r) * 3 NTp
  int nbk;             // block capacity (1: per-step solves)
  double *BV;          // (lmax+1) x nbk basis vectors
  float *BVs;          // FP32 contexts: their FP32 copy, read by the reorthogonalisation pass
  double *Bw, *Bvcur, *Bt1, *Bt2, *BY;  // nbk x 3 NTp each
  double *BR;          // nbk x 3N noise draws (bead-interleaved)
  double *Bpart;       // 3 x nbk x (lmax+1) x kDotBlocks partial dots
  double *Bh;          // nbk x (lmax+1) first-pass coefficients
  double *Bab;         // alpha, beta: 2 x (lmax+1) x nbk, [j * nbk + r]
  double *Bsc;         // nbk x 2: |z_r|, 1/|z_r|
  double *Bc;          // nbk x (lmax+1) combination coefficients
  int *Bm;             // nbk Krylov dimensions
  int *Bjd;
  int *Bctl;           // device convergence check, k ints each: done, conv, neg, last
                       // checked dimension, consecutive changes known; then the first
                       // dimension to check
  double *Bdh;         // the last eight relative changes per right-hand side
  double *Bpsi;        // quadrature pivots of the device check (k L1 nodes)
  void *blk_while[4];  // whole noise-block solves as one graph (conditional while node),
  int blk_while_key[4];
  long long blk_while_launches[4];
  bool device_krylov;  // convergence checks on the device (default); host QR otherwise
  long long dev_solves, host_fallbacks;
  bool while_failed;   // the conditional graph could not be built: host checks
  double *Bhost;       // pinned host copy of alpha, beta
  void *blk_ev;        // cudaEvent_t of the pending convergence check
  void *blk_graph[4][2];  // captured block iterations (product, orthogonalisation),
  int blk_graph_key[4];   // keyed by (preconditioned, right-hand sides)
  long long blk_graph_launches[4][2];
  int blk_last;        // smallest Krylov dimension of the previous block
  long long blk_runs, blk_products;  // block solves, block iterations run
  long long blk_rhs_products;        // sum over block iterations of their right-hand sides
  // the current block: steps blk_t0 .. blk_t0 + blk_n - 1, of which blk_next
  // are taken; valid while the mobility version and the hop flag it was made
  // with hold.  The generator ran ahead by the untaken draws: Philox counter
  // blk_draw0 at the first draw, ran1 states before each draw in Brng.
  unsigned long blk_t0;
  int blk_n, blk_next, blk_hop;
  long long blk_hiv;
  unsigned long long blk_draw0;
  void *Brng;          // (nbk + 1) bd::Ran1 states
  long long hi_version;  // bumped whenever the mobility or the preconditioner changes

  // CA-TEA sampling (bd_catea.cu)
  double *cb_part;
  int *cb_tileI;
  std::vector<double> cat_brun, cat_crun;
  std::vector<int> cat_gw;

  // parallel charge-hop sweep
  double hop_R;
  int *hop_cells;
  double *hop_de;  // energy change of each charge's last parallel-sweep trial
  unsigned long long hop_sweeps;

  // Ewald Coulomb (bd_coulomb.cu)
  double cw_beta, cw_rc, cw_q2, cw_Q, cw_cell_V;
  double *cw_grid, *cw_bsq, *cw_epart, *cw_energy, *cw_w;
  void *cw_spec;
  int *cw_base, *cw_cell_of, *cw_idx, *cw_count, *cw_start, *cw_cursor;
  int cw_nblk, cw_plan_f, cw_plan_b;

  // block preconditioner of the Lanczos solve
  int pre_kind;       // bd_precond_kind
  int pre_S;          // beads per block
  bool pre_ready;
  double *pre_G, *pre_Gi;  // per block 3S x 3S row-major G and G^-1
  double *pre_B, *pre_Bi;  // learned bead blocks on top of segment blocks
  int *pre_bad;       // blocks replaced by the identity
  size_t pre_cap;
  long long pre_calls, pre_iters, pre_fallbacks;

  // learned preconditioner network (bd_mpnn.cu)
  void *mpnn;
  bool mpnn_ready;

  // smooth-PME mobility (BD_MOB_PME)
  int pmeK, pme_p;
  double pme_rc, pme_alpha, pme_self;
  bool pme_ready;
  bool pme_f32;      // grids, spectra, influence and pair tensors in FP32
  void *pme_grid;    // 3 x K^3 real grids
  void *pme_spec;    // 3 x K*K*(K/2+1) complex spectra
  void *pme_infl;    // 6 x half spectrum influence tensor
  double *pme_bsq;   // |b_d(m)|^2, 3 x K
  double *pme_soff;  // self-block off-diagonal (xy, xz, yz), then per-block partials
  int pme_nblk;      // blocks of the influence kernel
  int *pme_base;     // per bead base grid index, 3 x N
  double *pme_w;     // per bead spline weights, 3 x N x 8
  int pme_plan_f, pme_plan_b;
  int pme_mplan_k[4], pme_mplan_f[4];  // packed-pair transforms for k right-hand sides
  int rl_cap, rl_ncell_cap;  // real-space pair rows
  int *rl_cnt, *rl_rows, *rl_cell_of, *rl_beads, *rl_cell_count, *rl_cell_start, *rl_cursor;
  int *rl_need;      // longest pair row of the last build that overflowed the cap (0: none)
  void *rl_pos;      // lab-frame positions of the last preparation (double4)
  float *pme_vpk;    // FP32 block products: per packed pair and bead the pair's
                     // 6 input values (+2 padding), written by the spread
  void *rl_tt;       // per pair t1 and t2 / r^2 of the real-space tensor (FP64 or FP32)
  double *pme_rsum;  // FP32 block products: real-space sums of every packed pair (6 per bead)
  float4 *rl_w;      // FP32 block products: per pair (t1, w), w = sqrt(|t2| / r^2) d, the sign
                     // of t2 in the lowest mantissa bit of t1
  double pme_cellbuf[19];  // its cell: H, H^-1, volume
  double pme_alpha_ref;    // calcHI's split parameter at that step

  size_t bytes;

  // profiling: CUDA events around selected kernels on the context's stream
  bool prof_on;
  bool prof_products;  // per-product events of noise blocks (host-checked Krylov loop)
  std::vector<cudaEvent_t> prof_ev[BD_PROF_SLOTS][2];
  long long launches;  // kernels launched by the library
};

namespace bd {

void prof_begin(bd_ctx* c, int slot);
void prof_end(bd_ctx* c, int slot);
void prof_clear(bd_ctx* c);

int set_error_from_bits(int bits);
int check(bd_ctx* c);                 // synchronise and fold device error bits
// report a launch error (or an earlier asynchronous one), recording the call
// site for bd_last_error_detail
int launch_ok_at(bd_ctx* c, const char* file, int line);
#define launch_ok(c) ::bd::launch_ok_at((c), __FILE__, __LINE__)
void host_lattice(bd_ctx* c, unsigned long t, Lat* out);
void host_lattice_at(bd_ctx* c, unsigned long t, double dt, int tp, Lat* out);
void rotate_coords(bd_ctx* c, int inverse);  // transformCoords (0) / inverseCoords (1)

// neighbours
int build_neighbors(bd_ctx* c, bool force);
int alloc_neighbors(bd_ctx* c);

// mobility
int alloc_mobility(bd_ctx* c);
int calc_hi(bd_ctx* c);
int update_hi(bd_ctx* c);
int download_mobility(bd_ctx* c, double* M9);
struct VecIn {
  const double* p[3];  // component pointers: x_c(i) = p[c][i*stride]
  int stride;
};
int sym_matvec(bd_ctx* c, int R, const VecIn& v0, const VecIn& v1, double* Y0, double* Y1,
               bool addiag);

// charge hopping
int charge_hop(bd_ctx* c);

// smooth-PME mobility
int pme_prepare(bd_ctx* c, const Lat& l);
int pme_apply(bd_ctx* c, const VecIn& v, double* o0, double* o1, double* o2, int ostride);
// Y_r = M X_r for k vectors in Lanczos layout (3 x NTp), RHS strides xs, ys
int pme_apply_multi(bd_ctx* c, int k, const double* X, size_t xs, double* Y, size_t ys);
int pme_multi_plan(bd_ctx* c, int k);  // creates the batched transforms for k
void pme_free(bd_ctx* c);

// CA-TEA sampling
int ewald_bin(bd_ctx* c, double* eps, std::vector<double>& rowsum);

// Ewald Coulomb
int coulomb_ewald(bd_ctx* c, const Lat& l, const double4* cq);
int coulomb_mesh_potential(bd_ctx* c, const Lat& l, const double4* cq);
int coulomb_quadform(bd_ctx* c, const Lat& l, double* Q6);
void coulomb_free(bd_ctx* c);

// block preconditioner
int precond_build(bd_ctx* c, const Lat& l);
int precond_apply(bd_ctx* c, int which, const double* x, double* y);
int precond_apply_k(bd_ctx* c, int which, int k, const double* x, size_t xs, double* y,
                    size_t ys);
void precond_free(bd_ctx* c);
int mpnn_blocks(bd_ctx* c, const Lat& l, double* G9);
void mpnn_free(bd_ctx* c);

// Krylov square root
void lanczos_graphs_reset(bd_ctx* c);
int alloc_lanczos(bd_ctx* c);
int lanczos_sqrt(bd_ctx* c, const double* zdev_interleaved, bool with_force, int* iters);
void lanczos_blocks_free(bd_ctx* c);
// drops the current noise block and winds the generator back to the draws the
// per-step order has made; every use of the generator outside
// bd_step_lanczos calls it first
void noise_blocks_release(bd_ctx* c);

// noise draw of bd_get_noise into dst (3N, bead-interleaved)
int draw_noise(bd_ctx* c, double* dst);

}  // namespace bd
