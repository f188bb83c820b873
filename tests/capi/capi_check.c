/* A C caller of ScalFMM's C API, unchanged except for the header it includes: reads a particle file
 * (x, y, z, q per particle, .fma or .bfma), runs the Chebyshev FMM through scalfmm_init / scalfmm_build_tree /
 * scalfmm_tree_insert_particles_xyz / scalfmm_set_physical_values / scalfmm_execute_fmm, and writes
 * x, y, z, q, phi, fx, fy, fz per particle.
 *   usage: capi_check IN OUT HEIGHT [mixed]
 * Exit status 0 when every call succeeded. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "b200fmm_capi.h"

int main(int argc, char **argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: %s IN OUT HEIGHT [mixed]\n", argv[0]);
    return 2;
  }
  long long n = 0;
  int nv = 0;
  double width = 0, center[3];
  if (b200fmm_fma_read(argv[1], &n, &nv, &width, center, NULL, 0) != B200FMM_OK || nv < 4) return 3;
  double *in = malloc(sizeof(double) * n * nv);
  if (b200fmm_fma_read(argv[1], &n, &nv, &width, center, in, n * nv) != B200FMM_OK) return 3;
  double *xyz = malloc(sizeof(double) * 3 * n), *q = malloc(sizeof(double) * n);
  for (long long i = 0; i < n; ++i) {
    memcpy(xyz + 3 * i, in + i * nv, 3 * sizeof(double));
    q[i] = in[i * nv + 3];
  }
  scalfmm_handle h = scalfmm_init(chebyshev, multi_thread);
  if (!h) return 4;
  if (argc > 4 && strcmp(argv[4], "mixed") == 0) b200fmm_capi_set_precision(h, B200FMM_MIXED);
  Scalfmm_Cell_Descriptor cells;
  Scalfmm_Leaf_Descriptor leaves;
  memset(&cells, 0, sizeof(cells));
  memset(&leaves, 0, sizeof(leaves));
  scalfmm_build_tree(h, atoi(argv[3]), width, center, cells, leaves);
  scalfmm_tree_insert_particles_xyz(h, (int)n, xyz, BOTH);
  scalfmm_set_physical_values(h, (int)n, q, BOTH);
  scalfmm_execute_fmm(h);
  double *phi = malloc(sizeof(double) * n), *f = malloc(sizeof(double) * 3 * n);
  scalfmm_get_potentials(h, (int)n, phi, TARGET);
  scalfmm_get_forces_xyz(h, (int)n, f, TARGET);
  double timers[16];
  const int nt = scalfmm_get_nb_timers(h);
  scalfmm_get_timers(h, timers);
  printf("timers (s):");
  for (int k = 0; k < nt && k < 16; ++k) printf(" %.3e", timers[k]);
  printf("\n");
  double *out = malloc(sizeof(double) * 8 * n);
  for (long long i = 0; i < n; ++i) {
    memcpy(out + 8 * i, xyz + 3 * i, 3 * sizeof(double));
    out[8 * i + 3] = q[i];
    out[8 * i + 4] = phi[i];
    memcpy(out + 8 * i + 5, f + 3 * i, 3 * sizeof(double));
  }
  const int st = b200fmm_capi_status(h);
  scalfmm_dealloc_handle(h, NULL);
  if (b200fmm_fma_write(argv[2], n, 8, width, center, out) != B200FMM_OK) return 5;
  free(in), free(xyz), free(q), free(phi), free(f), free(out);
  return st == B200FMM_OK ? 0 : 6;
}
