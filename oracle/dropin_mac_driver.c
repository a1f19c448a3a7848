/*
 * Test driver linked only into the drop-in library (_ref/libdcell_ref_b200.so):
 * calls the B200 LevelSetAdvectMAC / LevelSetAdvectMAC_3D the way the
 * reference's caller calls the originals (FluidField/tests/testSource.c:
 * 72-84): level sets made by the reference's LevelSetCreate, the face
 * velocities as global-index pointer tables, the step from ls into out.
 * Arrays are grids of extents n at global origin p, x fastest.
 */
#include <stdlib.h>
#include <string.h>

#include "LevelSetMethod.h"

PetscErrorCode LevelSetAdvectMAC(LevelSet ls, Coor d, PetscReal dt, PetscReal **u, PetscReal **v, LevelSet out);
PetscErrorCode LevelSetAdvectMAC_3D(LevelSet ls, Coor d, PetscReal dt, PetscReal ***u, PetscReal ***v,
                                    PetscReal ***w, LevelSet out);

static PetscReal **rows2(double *a, const int n[3], const int p[3], int k, PetscReal **rows) {
  for (int j = 0; j < n[1]; ++j) rows[j] = a + ((size_t)k * n[1] + j) * n[0] - p[0];
  return rows - p[1];
}

__attribute__((visibility("default"))) int ddrop_advect_mac(const int n[3], const int p[3], const double h[3],
                                                            const double *phi, double *u, double *v, double *w,
                                                            double dt, double *out) {
  const int nz = n[2] > 1 ? n[2] : 1;
  const Coor d = {h[0], h[1], h[2]};
  const iCoor pos = {p[0], p[1], nz > 1 ? p[2] : 0}, size = {n[0], n[1], nz};
  const size_t npts = (size_t)n[0] * n[1] * nz;
  LevelSet ls = NULL, nw = NULL;
  int rc = LevelSetCreate(d, pos, size, &ls);
  if (!rc) rc = LevelSetCreate(d, pos, size, &nw);
  if (rc) return rc;
  memcpy(ls->phi->v1, phi, sizeof(double) * npts);
  memcpy(nw->phi->v1, out, sizeof(double) * npts);
  double *arrays[3] = {u, v, w};
  PetscReal **rows = malloc(sizeof(PetscReal *) * (size_t)nz * n[1] * 3);
  PetscReal ***planes = malloc(sizeof(PetscReal **) * (size_t)nz * 3);
  PetscReal **t2[3];
  PetscReal ***t3[3];
  for (int a = 0; a < (nz > 1 ? 3 : 2); ++a) {
    if (nz > 1) {
      PetscReal ***pl = planes + (size_t)a * nz;
      for (int k = 0; k < nz; ++k) pl[k] = rows2(arrays[a], n, p, k, rows + ((size_t)a * nz + k) * n[1]);
      t3[a] = pl - p[2];
    } else {
      t2[a] = rows2(arrays[a], n, p, 0, rows + (size_t)a * n[1]);
    }
  }
  rc = nz > 1 ? LevelSetAdvectMAC_3D(ls, d, dt, t3[0], t3[1], t3[2], nw) : LevelSetAdvectMAC(ls, d, dt, t2[0], t2[1], nw);
  if (!rc) memcpy(out, nw->phi->v1, sizeof(double) * npts);
  free(rows);
  free(planes);
  LevelSetDestroy(ls);
  LevelSetDestroy(nw);
  return rc;
}
