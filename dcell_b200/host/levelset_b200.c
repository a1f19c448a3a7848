/*
 * levelset_b200.c -- B200 implementation of the reference's level-set
 * transport entry points, for the reference's own C host.
 *
 * Compiled INSIDE adrielb/DCell's build in place of the CPU definitions:
 *   LevelSetAdvectSL, _2D, _3D          (LevelSetMethod/AdvectSL.c:6-89; the
 *                                        whole file is replaced)
 *   LevelSetUpdateIrregularNodeList     (LevelSetMethod/IrregularNodes.c:9-28;
 *                                        the reference's definition is renamed
 *                                        away when IrregularNodes.c is built)
 *   LevelSet_MaxVelocity                (LevelSetMethod/Advect.c:70-111; likewise)
 *   LevelSetReinitialize                (LevelSetMethod/FastMarching.c:11-41; the
 *                                        reference's definition is renamed to
 *                                        LevelSetReinitialize_cpu when
 *                                        FastMarching.c is built, and stays the
 *                                        default)
 * Everything that calls them -- LevelSetAdvectAndReinit, the RK2 half/full
 * steps (AdvectRK2.c), the particle and implicit variants, DCell's ls->Advect
 * slot -- is unchanged and now runs the GPU path.  Fast-marching
 * reinitialisation runs the reference's CPU code unless
 * DCELL_LS_REINIT=gpu selects the GPU's bucketed march (dcell_reinitialize;
 * within 1e-2 cells of the heap, band in grid order).
 *
 * The calls go through the C ABI of libdcell_ls.so (include/dcell_ls.h) with
 * the LevelSet's own FP64 arrays (Grid.v1, band Array data); a process-wide
 * session keeps the device buffers.  Default arithmetic: FP64, linear
 * interpolation, Euler backtrace -- bit-identical to the reference.  The
 * environment selects other modes:
 *   DCELL_DEVICE=<n>                     CUDA device (default 0)
 *   DCELL_LS_PRECISION=f32|f64
 *   DCELL_LS_INTERP=linear|cubic|cubic_separable|cubic_tc
 *   DCELL_LS_BACKTRACE=euler|midpoint
 *   DCELL_LS_REINIT=cpu|gpu                (read at every call)
 * Errors come back as PetscErrorCode through SETERRQ with the library's
 * message; nothing exits.
 */
#include <stdlib.h>
#include <string.h>

#include "LevelSetMethod.h"
#include "LSM_private.h"
#include "dcell_ls.h"

#ifndef PETSC_ERR_LIB
#define PETSC_ERR_LIB 76
#endif

static dcell_session *b200_sess = NULL;
static int b200_interp = DCELL_LINEAR, b200_backtrace = DCELL_EULER, b200_precision = DCELL_F64;

static void b200_config(void) {
  static int done = 0;
  const char *e;
  if (done) return;
  done = 1;
  if ((e = getenv("DCELL_LS_PRECISION")) && !strcmp(e, "f32")) b200_precision = DCELL_F32;
  if ((e = getenv("DCELL_LS_INTERP"))) {
    if (!strcmp(e, "cubic")) b200_interp = DCELL_CUBIC_PLAIN;
    else if (!strcmp(e, "cubic_separable")) b200_interp = DCELL_CUBIC_SEPARABLE;
    else if (!strcmp(e, "cubic_tc")) b200_interp = DCELL_CUBIC_TC;
  }
  if ((e = getenv("DCELL_LS_BACKTRACE")) && !strcmp(e, "midpoint")) b200_backtrace = DCELL_MIDPOINT;
}

#undef __FUNCT__
#define __FUNCT__ "LevelSetB200Session"
static PetscErrorCode LevelSetB200Session(dcell_session **s) {
  PetscFunctionBegin;
  b200_config();
  if (!b200_sess) {
    const char *d = getenv("DCELL_DEVICE");
    int rc = dcell_session_create(d ? atoi(d) : 0, &b200_sess);
    if (rc) SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_session_create: %s", dcell_last_error());
  }
  *s = b200_sess;
  PetscFunctionReturn(0);
}

static void b200_geom(Grid g, dcell_geom *out) {
  out->n[0] = g->n.x;
  out->n[1] = g->n.y;
  out->n[2] = g->is2D ? 1 : g->n.z;
  out->p[0] = g->p.x;
  out->p[1] = g->p.y;
  out->p[2] = g->is2D ? 0 : g->p.z;
  out->h[0] = g->d.x;
  out->h[1] = g->d.y;
  out->h[2] = g->d.z;
}

/* The band as int triples (iCoor is PetscInt x 3; copy when PetscInt != int). */
static const int *b200_band(Array band, int **scratch) {
  *scratch = NULL;
  if (sizeof(PetscInt) == sizeof(int)) return (const int *)ArrayGetData(band);
  {
    int n = ArrayLength(band), i;
    const iCoor *b = (const iCoor *)ArrayGetData(band);
    int *t = (int *)malloc(sizeof(int) * 3 * (size_t)(n > 0 ? n : 1));
    for (i = 0; i < n; ++i) {
      t[3 * i] = (int)b[i].x;
      t[3 * i + 1] = (int)b[i].y;
      t[3 * i + 2] = (int)b[i].z;
    }
    *scratch = t;
    return t;
  }
}

#undef __FUNCT__
#define __FUNCT__ "LevelSetAdvectSL"
PetscErrorCode LevelSetAdvectSL(LevelSet ls, Grid velgrid, PetscReal dt) {
  dcell_session *s;
  dcell_geom g;
  int *tmp, rc;
  const int *band;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  ierr = PetscLogEventBegin(EVENT_LevelSetAdvectSL, 0, 0, 0, 0); CHKERRQ(ierr);
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  if (ls->phi0->SIZE != ls->phi->SIZE || velgrid->SIZE != ls->phi->SIZE * velgrid->dof)
    SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_OUTOFRANGE, "phi0/velgrid do not match phi (GridCopy phi->phi0 first)");
  b200_geom(ls->phi, &g);
  band = b200_band(ls->band, &tmp);
  rc = dcell_ls_advect_sl(s, &g, ls->phi0->v1, velgrid->v1, band, ArrayLength(ls->band), dt, b200_interp,
                          b200_backtrace, b200_precision, ls->phi->v1);
  free(tmp);
  if (rc == DCELL_ERR_DEPARTURE) {
    /* the reference would read outside its arrays here; the GPU path clamped the sample */
    ierr = PetscInfo1(0, "LevelSetAdvectSL: %s\n", dcell_last_error()); CHKERRQ(ierr);
  } else if (rc) {
    SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_advect_sl: %s", dcell_last_error());
  }
  ierr = PetscLogEventEnd(EVENT_LevelSetAdvectSL, 0, 0, 0, 0); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

PetscErrorCode LevelSetAdvectSL_2D(LevelSet ls, Grid velgrid, PetscReal dt) { return LevelSetAdvectSL(ls, velgrid, dt); }
PetscErrorCode LevelSetAdvectSL_3D(LevelSet ls, Grid velgrid, PetscReal dt) { return LevelSetAdvectSL(ls, velgrid, dt); }

#undef __FUNCT__
#define __FUNCT__ "LevelSetUpdateIrregularNodeList"
PetscErrorCode LevelSetUpdateIrregularNodeList(LevelSet ls) {
  dcell_session *s;
  dcell_geom g;
  dcell_irregular_node *buf;
  IrregularNode *nodes;
  int *tmp, rc, count = 0, cap, i;
  const int nb = ArrayLength(ls->band);
  const int *band;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  ierr = PetscLogEventBegin(EVENT_LevelSetUpdateIrregularNodeList, 0, 0, 0, 0); CHKERRQ(ierr);
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  ierr = ArraySetSize(ls->irregularNodes, 0); CHKERRQ(ierr);
  ierr = ArrayZero(ls->irregularNodes); CHKERRQ(ierr);
  b200_geom(ls->phi, &g);
  cap = (ls->phi->is2D ? 5 : 10) * (nb > 0 ? nb : 1); /* per point at most 5 (2D) / 10 (3D) nodes */
  buf = (dcell_irregular_node *)malloc(sizeof(dcell_irregular_node) * (size_t)cap);
  if (!buf) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_MEM, "out of host memory");
  band = b200_band(ls->band, &tmp);
  rc = dcell_ls_update_irregular_nodes(s, &g, ls->phi->v1, band, nb, 0, b200_precision, buf, cap, &count);
  free(tmp);
  if (rc) {
    free(buf);
    SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_update_irregular_nodes: %s", dcell_last_error());
  }
  ierr = ArraySetSize(ls->irregularNodes, count); CHKERRQ(ierr);
  ierr = ArrayZero(ls->irregularNodes); CHKERRQ(ierr);
  nodes = (IrregularNode *)ArrayGetData(ls->irregularNodes);
  for (i = 0; i < count; ++i) {
    IrregularNode *n = &nodes[i];
    const dcell_irregular_node *q = &buf[i];
    n->pos.x = q->pos[0];
    n->pos.y = q->pos[1];
    n->pos.z = q->pos[2];
    n->axis = q->axis;
    n->shift = (VelFace)q->shift;
    n->signCenter = q->signCenter;
    n->signFace = q->signFace;
    n->d = q->d;
    n->X.x = q->X[0];
    n->X.y = q->X[1];
    n->X.z = q->X[2];
    n->op.x = q->op[0];
    n->op.y = q->op[1];
    n->op.z = q->op[2];
  }
  free(buf);
  ierr = PetscLogEventEnd(EVENT_LevelSetUpdateIrregularNodeList, 0, 0, 0, 0); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

#undef __FUNCT__
#define __FUNCT__ "LevelSet_MaxVelocity"
PetscErrorCode LevelSet_MaxVelocity(LevelSet ls, Grid velgrid) {
  dcell_session *s;
  dcell_geom g;
  dcell_irregular_node *buf;
  const int len = ArrayLength(ls->irregularNodes);
  const IrregularNode *nodes = (const IrregularNode *)ArrayGetData(ls->irregularNodes);
  int i, rc;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  b200_geom(ls->phi, &g);
  buf = (dcell_irregular_node *)calloc((size_t)(len > 0 ? len : 1), sizeof(dcell_irregular_node));
  if (!buf) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_MEM, "out of host memory");
  for (i = 0; i < len; ++i) {
    buf[i].pos[0] = nodes[i].pos.x;
    buf[i].pos[1] = nodes[i].pos.y;
    buf[i].pos[2] = nodes[i].pos.z;
  }
  rc = dcell_ls_max_velocity(s, &g, velgrid->v1, buf, len, &ls->maxVel);
  free(buf);
  if (rc) SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_max_velocity: %s", dcell_last_error());
  PetscFunctionReturn(0);
}

/* The reference's own LevelSetReinitialize, renamed at link time. */
PetscErrorCode LevelSetReinitialize_cpu(LevelSet ls);

#undef __FUNCT__
#define __FUNCT__ "LevelSetReinitialize"
PetscErrorCode LevelSetReinitialize(LevelSet ls) {
  dcell_session *s;
  dcell_geom g;
  dcell_irregular_node *buf;
  int *bandbuf, rc, count = 0, i, cap;
  const char *mode = getenv("DCELL_LS_REINIT");
  const int len = ArrayLength(ls->irregularNodes);
  const IrregularNode *nodes;
  iCoor *band;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  if (!mode || strcmp(mode, "gpu")) {
    ierr = LevelSetReinitialize_cpu(ls); CHKERRQ(ierr);
    PetscFunctionReturn(0);
  }
  ierr = PetscLogEventBegin(EVENT_LevelSetReinitialize, 0, 0, 0, 0); CHKERRQ(ierr);
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  ierr = LevelSetResize(ls); CHKERRQ(ierr);  /* as the reference does first (FastMarching.c:25) */
  b200_geom(ls->phi, &g);
  nodes = (const IrregularNode *)ArrayGetData(ls->irregularNodes);
  buf = (dcell_irregular_node *)calloc((size_t)(len > 0 ? len : 1), sizeof(dcell_irregular_node));
  cap = ls->phi->SIZE;
  bandbuf = (int *)malloc(sizeof(int) * 3 * (size_t)(cap > 0 ? cap : 1));
  if (!buf || !bandbuf) {
    free(buf);
    free(bandbuf);
    SETERRQ(PETSC_COMM_SELF, PETSC_ERR_MEM, "out of host memory");
  }
  for (i = 0; i < len; ++i) {
    buf[i].pos[0] = nodes[i].pos.x;
    buf[i].pos[1] = nodes[i].pos.y;
    buf[i].pos[2] = nodes[i].pos.z;
    buf[i].axis = nodes[i].axis;
    buf[i].signCenter = nodes[i].signCenter;
    buf[i].op[0] = nodes[i].op.x;
    buf[i].op[1] = nodes[i].op.y;
    buf[i].op[2] = nodes[i].op.z;
  }
  rc = dcell_ls_reinitialize(s, &g, ls->phi->v1, buf, len, ls->bandWidth, b200_precision, bandbuf, cap, &count);
  free(buf);
  if (rc) {
    free(bandbuf);
    SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_reinitialize: %s", dcell_last_error());
  }
  ierr = ArraySetSize(ls->band, count); CHKERRQ(ierr);
  band = (iCoor *)ArrayGetData(ls->band);
  for (i = 0; i < count; ++i) {
    band[i].x = bandbuf[3 * i];
    band[i].y = bandbuf[3 * i + 1];
    band[i].z = bandbuf[3 * i + 2];
  }
  free(bandbuf);
  ierr = PetscLogEventEnd(EVENT_LevelSetReinitialize, 0, 0, 0, 0); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}
