/*
 * Forced-include stand-in for the reference's LevelSetMethod.h, used only to
 * compile its LevelSetMethod/AdvectMAC.c (test infrastructure).
 *
 * That file predates the current struct _LevelSet and struct _Grid: it reads
 * the level set's grid as ls->g and that grid's global-index pointer tables
 * as g->v2 (2D, [j][i]) and g->v3 (3D, [k][j][i]), members the current
 * headers no longer have.  This header defines the real header's include
 * guard, so AdvectMAC.c's own #include "LevelSetMethod.h" adds nothing, and
 * supplies exactly those members plus the grid's p and n; the file then
 * compiles unmodified.
 */
#ifndef DCELL_MAC_LEVELSET_H
#define DCELL_MAC_LEVELSET_H
#define LEVELSETMETHOD_H_
#include "Common.h"

typedef struct {
  iCoor p, n;       /* global index of element 0, extents */
  PetscReal **v2;   /* 2D: v2[j][i] by global index */
  PetscReal ***v3;  /* 3D: v3[k][j][i] by global index */
} *MacGrid;

typedef struct {
  MacGrid g;
} *LevelSet;

PetscErrorCode LevelSetAdvectMAC(LevelSet ls, Coor d, PetscReal dt, PetscReal **u, PetscReal **v, LevelSet out);
PetscErrorCode LevelSetAdvectMAC_3D(LevelSet ls, Coor d, PetscReal dt, PetscReal ***u, PetscReal ***v,
                                    PetscReal ***w, LevelSet out);
#endif
