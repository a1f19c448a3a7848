/*
 * Driver for the reference's LevelSetMethod/AdvectMAC.c compiled against
 * shim/mac/mac_levelset.h (test infrastructure; see that header).  Builds the
 * global-index pointer tables the routines read (v2[j][i], v3[k][j][i] and
 * the same for each velocity component) over caller arrays laid out as a grid
 * of extents n at global origin p, x fastest, and calls LevelSetAdvectMAC
 * (2D, n[2] <= 1) or LevelSetAdvectMAC_3D.  Only points the routine updates
 * are written to `out`; the caller pre-fills it.
 */
#include <stdlib.h>

#include "mac_levelset.h"

#define DREF_EXPORT __attribute__((visibility("default")))

/* rows[j] points at global (p.x, j); the table is returned offset so that
 * table[j][i] addresses global (i, j) */
static PetscReal **rows2(double *a, const int n[3], const int p[3], int k, PetscReal **rows) {
  for (int j = 0; j < n[1]; ++j) rows[j] = a + ((size_t)k * n[1] + j) * n[0] - p[0];
  return rows - p[1];
}

static PetscReal ***planes3(double *a, const int n[3], const int p[3], PetscReal **rows, PetscReal ***planes) {
  for (int k = 0; k < n[2]; ++k) planes[k] = rows2(a, n, p, k, rows + (size_t)k * n[1]);
  return planes - p[2];
}

DREF_EXPORT int dref_advect_mac(const int n[3], const int p[3], const double h[3], double *phi, double *u, double *v,
                                double *w, double dt, double *out) {
  const int nz = n[2] > 1 ? n[2] : 1;
  const Coor d = {h[0], h[1], h[2]};
  double *arrays[5] = {phi, out, u, v, w};
  const int na = nz > 1 ? 5 : 4;
  PetscReal **rows = malloc(sizeof(PetscReal *) * (size_t)nz * n[1] * na);
  PetscReal ***planes = malloc(sizeof(PetscReal **) * (size_t)nz * na);
  __typeof__(*(MacGrid)0) gin, gout;
  __typeof__(*(LevelSet)0) lin, lout;
  PetscReal **t2[5];
  PetscReal ***t3[5];
  for (int a = 0; a < na; ++a) {
    if (nz > 1)
      t3[a] = planes3(arrays[a], n, p, rows + (size_t)a * nz * n[1], planes + (size_t)a * nz);
    else
      t2[a] = rows2(arrays[a], n, p, 0, rows + (size_t)a * n[1]);
  }
  gin.p.x = gout.p.x = p[0];
  gin.p.y = gout.p.y = p[1];
  gin.p.z = gout.p.z = nz > 1 ? p[2] : 0;
  gin.n.x = gout.n.x = n[0];
  gin.n.y = gout.n.y = n[1];
  gin.n.z = gout.n.z = nz;
  gin.v2 = nz > 1 ? NULL : t2[0];
  gout.v2 = nz > 1 ? NULL : t2[1];
  gin.v3 = nz > 1 ? t3[0] : NULL;
  gout.v3 = nz > 1 ? t3[1] : NULL;
  lin.g = &gin;
  lout.g = &gout;
  int rc;
  if (nz > 1)
    rc = LevelSetAdvectMAC_3D(&lin, d, dt, t3[2], t3[3], t3[4], &lout);
  else
    rc = LevelSetAdvectMAC(&lin, d, dt, t2[2], t2[3], &lout);
  free(rows);
  free(planes);
  return rc;
}
