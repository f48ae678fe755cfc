// Verlet neighbour rows built by a cell sort on the deformed lattice.
//
// The reference builds its half list with an O(N^2) scan over all pairs,
// keeping j > i with |getNID(i,j)| < rv (shear/src/main26.c:682-707), and
// rebuilds when any bead has moved more than rnew since the last build
// (checkVerlet, shear/src/main26.c:858-869).  Here beads are binned in
// fractional coordinates of the current cell (L1', L2', L e_z in the frame
// the positions are held in), with cell widths of at least rv plus the
// largest extra offset getNID can add to a lattice image (the shear brick
// offset delx).  A pair within rv under getNID is therefore always found in
// the 27-cell stencil, and the getNID test itself is the reference's exact
// arithmetic, so the neighbour set is the reference's bit for bit.  Rows hold
// the full list sorted ascending; the reference's half list is the part of
// each row above i.
//
// The rebuild decision stays on the device: the check kernel raises a flag
// and every build kernel returns at once when it is not raised, so a step
// needs no host round trip.
#include <math.h>

#include <algorithm>

#include "bd_ctx.cuh"

using namespace bd;

struct CellGeom {
  int n1, n2, n3, ncell;
  double L1xp, L2xp, L2yp, L;
};

__global__ void k_check_verlet(const double* __restrict__ dxv, const double* __restrict__ dyv,
                               const double* __restrict__ dzv, int N, double rnew, int* flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool due = false;
  if (i < N) due = sqrt(rr3(dxv[i], dyv[i], dzv[i])) > rnew;
  if (__any_sync(0xffffffffu, due) && (threadIdx.x & 31) == 0) flag[0] = 1;
}

__global__ void k_set_flag(int* flag, int v) { flag[0] = v; }

__device__ __forceinline__ int wrapc(int c, int n) {
  c %= n;
  return c < 0 ? c + n : c;
}

__device__ __forceinline__ int cell_index(const CellGeom& g, double x, double y, double z) {
  double s2 = y / g.L2yp;
  double s1 = (x - s2 * g.L2xp) / g.L1xp;
  double s3 = z / g.L;
  int c1 = wrapc((int)floor((s1 + 0.5) * g.n1), g.n1);
  int c2 = wrapc((int)floor((s2 + 0.5) * g.n2), g.n2);
  int c3 = wrapc((int)floor((s3 + 0.5) * g.n3), g.n3);
  return (c1 * g.n2 + c2) * g.n3 + c3;
}

__global__ void k_cell_count(const int* flag, CellGeom g, const double* __restrict__ rx,
                             const double* __restrict__ ry, const double* __restrict__ rz, int N,
                             int* cell_of, int* cell_count) {
  if (flag[0] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int c = cell_index(g, rx[i], ry[i], rz[i]);
  cell_of[i] = c;
  atomicAdd(&cell_count[c], 1);
}

// Exclusive scan of the cell counts in one block; also clears the counts and
// resets the fill cursors.
__global__ void k_cell_scan(const int* flag, int ncell, int* cell_count, int* cell_start,
                            int* cursor) {
  if (flag[0] == 0) return;
  __shared__ int part[1024];
  int t = threadIdx.x, nt = blockDim.x;
  int per = (ncell + nt - 1) / nt;
  int lo = t * per, hi = min(ncell, lo + per);
  int s = 0;
  for (int c = lo; c < hi; c++) s += cell_count[c];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < nt; o <<= 1) {
    int v = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int base = part[t] - s;
  for (int c = lo; c < hi; c++) {
    cell_start[c] = base;
    cursor[c] = 0;
    base += cell_count[c];
    cell_count[c] = 0;
  }
  if (t == nt - 1) cell_start[ncell] = part[t];
}

__global__ void k_cell_fill(const int* flag, const int* __restrict__ cell_of,
                            const int* __restrict__ cell_start, int* cursor, int* cell_beads,
                            int N) {
  if (flag[0] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int c = cell_of[i];
  int k = atomicAdd(&cursor[c], 1);
  cell_beads[cell_start[c] + k] = i;
}

// One thread per bead: scan the stencil cells, keep j with |getNID(i,j)| < rv,
// sort the row ascending, and zero the bead's displacement since the last
// build (verletlist resets dxv, shear/src/main26.c:685-688).
__global__ void k_nbr_rows(const int* flag, CellGeom g, Lat l, const double* __restrict__ rx,
                           const double* __restrict__ ry, const double* __restrict__ rz, int N,
                           const int* __restrict__ cell_of, const int* __restrict__ cell_start,
                           const int* __restrict__ cell_beads, double rv, int maxnb, int* cnt,
                           int* rows, int* half, double* dxv, double* dyv, double* dzv,
                           int* err) {
  if (flag[0] == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int c = cell_of[i];
  int c3 = c % g.n3, c2 = (c / g.n3) % g.n2, c1 = c / (g.n3 * g.n2);
  int lo1 = g.n1 >= 3 ? -1 : 0, hi1 = g.n1 >= 3 ? 1 : g.n1 - 1;
  int lo2 = g.n2 >= 3 ? -1 : 0, hi2 = g.n2 >= 3 ? 1 : g.n2 - 1;
  int lo3 = g.n3 >= 3 ? -1 : 0, hi3 = g.n3 >= 3 ? 1 : g.n3 - 1;
  int* row = rows + (size_t)i * maxnb;
  int n = 0;
  bool over = false;
  double xi = rx[i], yi = ry[i], zi = rz[i];
  for (int a = lo1; a <= hi1; a++) {
    int d1 = g.n1 >= 3 ? wrapc(c1 + a, g.n1) : a;
    for (int b = lo2; b <= hi2; b++) {
      int d2 = g.n2 >= 3 ? wrapc(c2 + b, g.n2) : b;
      for (int e = lo3; e <= hi3; e++) {
        int d3 = g.n3 >= 3 ? wrapc(c3 + e, g.n3) : e;
        int cc = (d1 * g.n2 + d2) * g.n3 + d3;
        int s0 = cell_start[cc], s1 = cell_start[cc + 1];
        for (int s = s0; s < s1; s++) {
          int j = cell_beads[s];
          if (j == i) continue;
          double vx, vy, vz;
          min_image(l, subx(xi, rx[j]), subx(yi, ry[j]), subx(zi, rz[j]), vx, vy, vz);
          if (sqrt(rr3(vx, vy, vz)) < rv) {
            if (n < maxnb)
              row[n++] = j;
            else
              over = true;
          }
        }
      }
    }
  }
  if (over) atomicOr(err, ERRB_NBR_OVERFLOW);
  for (int a = 1; a < n; a++) {
    int v = row[a], b = a - 1;
    while (b >= 0 && row[b] > v) {
      row[b + 1] = row[b];
      b--;
    }
    row[b + 1] = v;
  }
  int h = 0;
  while (h < n && row[h] < i) h++;
  cnt[i] = n;
  half[i] = h;
  dxv[i] = 0.0;
  dyv[i] = 0.0;
  dzv[i] = 0.0;
}

static inline int nblk(int n, int b) { return (n + b - 1) / b; }

namespace bd {

int alloc_neighbors(bd_ctx* c) {
  int N = c->N;
  double rs = c->rv + c->p.edot * c->tp * c->p.dt + 0.01;
  int m = (int)floor(1.2 * c->p.L / rs) + 2;
  c->ncell_cap = m * m * m;
  size_t nr = (size_t)N * c->maxnb;
  if (cudaMalloc(&c->nb_count, 4 * (size_t)N) != cudaSuccess) return BD_ERR_OOM;
  if (cudaMalloc(&c->nb_half, 4 * (size_t)N) != cudaSuccess) return BD_ERR_OOM;
  if (cudaMalloc(&c->nb_rows, 4 * nr) != cudaSuccess) return BD_ERR_OOM;
  if (cudaMalloc(&c->cell_of, 4 * (size_t)N) != cudaSuccess) return BD_ERR_OOM;
  if (cudaMalloc(&c->cell_beads, 4 * (size_t)N) != cudaSuccess) return BD_ERR_OOM;
  if (cudaMalloc(&c->cell_count, 4 * (size_t)c->ncell_cap) != cudaSuccess) return BD_ERR_OOM;
  if (cudaMalloc(&c->cell_cursor, 4 * (size_t)c->ncell_cap) != cudaSuccess) return BD_ERR_OOM;
  if (cudaMalloc(&c->cell_start, 4 * (size_t)(c->ncell_cap + 1)) != cudaSuccess) return BD_ERR_OOM;
  c->bytes += 4 * (4 * (size_t)N + nr + 3 * (size_t)c->ncell_cap + 1);
  cudaMemsetAsync(c->nb_count, 0, 4 * (size_t)N, c->stream);
  cudaMemsetAsync(c->nb_half, 0, 4 * (size_t)N, c->stream);
  cudaMemsetAsync(c->cell_count, 0, 4 * (size_t)c->ncell_cap, c->stream);
  return BD_OK;
}

// Cell geometry of the current lattice: fractional bins at least rv + delx
// wide in each lattice direction (perpendicular widths of the deformed cell).
static CellGeom cell_geom(bd_ctx* c, const Lat& l) {
  CellGeom g;
  double rs = c->rv + fabs(l.delx) + 1e-6 * l.L;
  double area = l.L1xp * l.L2yp - l.L1yp * l.L2xp;
  double w1 = area / sqrt(l.L2xp * l.L2xp + l.L2yp * l.L2yp);
  double w2 = area / sqrt(l.L1xp * l.L1xp + l.L1yp * l.L1yp);
  double w3 = l.L;
  g.n1 = std::max(1, (int)floor(w1 / rs));
  g.n2 = std::max(1, (int)floor(w2 / rs));
  g.n3 = std::max(1, (int)floor(w3 / rs));
  while ((long)g.n1 * g.n2 * g.n3 > c->ncell_cap) {
    if (g.n1 >= g.n2 && g.n1 >= g.n3)
      g.n1--;
    else if (g.n2 >= g.n3)
      g.n2--;
    else
      g.n3--;
  }
  g.ncell = g.n1 * g.n2 * g.n3;
  g.L1xp = l.L1xp;
  g.L2xp = l.L2xp;
  g.L2yp = l.L2yp;
  g.L = l.L;
  return g;
}

int build_neighbors(bd_ctx* c, bool force) {
  int N = c->N;
  Lat l = c->lat;
  int treal = (int)(c->t % (unsigned long)c->tp);
  l.treal = treal;
  l.delx = c->p.edot * treal * c->p.dt;
  if (force) {
    c->launches++;
    k_set_flag<<<1, 1, 0, c->stream>>>(c->flag, 1);
  } else {
    c->launches++;
    k_check_verlet<<<nblk(N, 256), 256, 0, c->stream>>>(c->dxv, c->dyv, c->dzv, N, c->rnew,
                                                          c->flag);
  }
  CellGeom g = cell_geom(c, l);
  c->launches++;
  k_cell_count<<<nblk(N, 256), 256, 0, c->stream>>>(c->flag, g, c->rx, c->ry, c->rz, N,
                                                    c->cell_of, c->cell_count);
  c->launches++;
  k_cell_scan<<<1, 1024, 0, c->stream>>>(c->flag, g.ncell, c->cell_count, c->cell_start,
                                         c->cell_cursor);
  c->launches++;
  k_cell_fill<<<nblk(N, 256), 256, 0, c->stream>>>(c->flag, c->cell_of, c->cell_start,
                                                   c->cell_cursor, c->cell_beads, N);
  c->launches++;
  k_nbr_rows<<<nblk(N, 128), 128, 0, c->stream>>>(c->flag, g, l, c->rx, c->ry, c->rz, N,
                                                  c->cell_of, c->cell_start, c->cell_beads,
                                                  c->rv, c->maxnb, c->nb_count, c->nb_rows,
                                                  c->nb_half, c->dxv, c->dyv, c->dzv, c->err);
  c->launches++;
  k_set_flag<<<1, 1, 0, c->stream>>>(c->flag, 0);
  return launch_ok(c);
}

}  // namespace bd

extern "C" int bd_download_neighbors(bd_ctx* c, int* counts, int* rows, int maxnb) {
  if (!c || !counts || !rows || maxnb < 1) return BD_ERR_ARG;
  int N = c->N;
  std::vector<int> cnt(N), half(N), r((size_t)N * c->maxnb);
  cudaMemcpyAsync(cnt.data(), c->nb_count, 4 * (size_t)N, cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(half.data(), c->nb_half, 4 * (size_t)N, cudaMemcpyDeviceToHost, c->stream);
  cudaMemcpyAsync(r.data(), c->nb_rows, 4 * r.size(), cudaMemcpyDeviceToHost, c->stream);
  int s = check(c);
  if (s) return s;
  for (int i = 0; i < N; i++) {
    int n = cnt[i] - half[i];
    if (n > maxnb) return BD_ERR_NBR_OVERFLOW;
    counts[i] = n;
    for (int k = 0; k < n; k++) rows[(size_t)i * maxnb + k] = r[(size_t)i * c->maxnb + half[i] + k];
  }
  return BD_OK;
}
