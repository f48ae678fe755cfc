/* Test-only harness around the reference's lookup-table precompute
 * (shear/src/gridHI.c, extensional/src/gridHI.c), compiled from those sources
 * into oracle/_ref/ by oracle/Makefile.  grid_main() is the reference's main
 * renamed; it writes mm/G*.txt relative to the working directory and leaves
 * its tables in the global D, which the getters below copy out at full
 * precision. */
#define main grid_main
#include REF_GRID
#undef main

#include <string.h>

/* nbx nby nbz nhx nhy nhz num_bins origin */
void hg_bins(int *o) {
  o[0] = num_bins_x;
  o[1] = num_bins_y;
  o[2] = num_bins_z;
  o[3] = nhx;
  o[4] = nhy;
  o[5] = nhz;
  o[6] = num_bins;
  o[7] = origin;
}
/* L box_volume bin_size_x bin_size_y bin_size_z dt tp */
void hg_geom(double *o) {
  o[0] = L;
  o[1] = box_volume;
  o[2] = bin_size_x;
  o[3] = bin_size_y;
  o[4] = bin_size_z;
  o[5] = dt;
  o[6] = tp;
}
void hg_D(int nt, double *out) { memcpy(out, D[nt], sizeof(double) * 9 * (size_t)num_bins); }
