/*
 * levelset_b200.c -- B200 implementation of the reference's level-set
 * transport entry points, for the reference's own C host.
 *
 * Compiled INSIDE adrielb/DCell's build in place of the CPU definitions:
 *   LevelSetAdvectSL, _2D, _3D          (LevelSetMethod/AdvectSL.c:6-89; the
 *                                        whole file is replaced)
 *   LevelSetAdvectSLRK2HalfStep,
 *   LevelSetAdvectSLRK2FullStep         (LevelSetMethod/AdvectRK2.c:5-26; the
 *                                        reference's definitions are renamed
 *                                        away when AdvectRK2.c is built)
 *   LevelSetUpdateIrregularNodeList     (LevelSetMethod/IrregularNodes.c:9-28;
 *                                        the reference's definition is renamed
 *                                        away when IrregularNodes.c is built)
 *   LevelSet_MaxVelocity                (LevelSetMethod/Advect.c:70-111; likewise)
 *   LevelSetReinitialize                (LevelSetMethod/FastMarching.c:11-41; the
 *                                        reference's definition is renamed to
 *                                        LevelSetReinitialize_cpu when
 *                                        FastMarching.c is built, and stays the
 *                                        default)
 *   LevelSetInitializeParticles, ParticleLS_AdjustRadii,
 *   ParticleLS_ReseedParticles          (LevelSetMethod/ParticleLS.c:6-88,
 *                                        158-185, 202-295)
 *   ParticleLS_AdvectParticles2D/3D,
 *   ParticleLS_ErrorCorrection2D/3D     (ParticleLS2D.c, ParticleLS3D.c; the
 *                                        reference's definitions are renamed
 *                                        away as above)
 *   LevelSetAdvectMAC, _3D              (LevelSetMethod/AdvectMAC.c:18-111; that
 *                                        file is not in the reference's build:
 *                                        it reads ls->g, which the current
 *                                        struct _LevelSet no longer has)
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

/* The node list of the GPU into ls->irregularNodes (the fields the transport
 * path writes; the rest stay zero). */
static PetscErrorCode b200_store_nodes(LevelSet ls, const dcell_irregular_node *buf, int count) {
  IrregularNode *nodes;
  int i;
  PetscErrorCode ierr;

  PetscFunctionBegin;
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
  PetscFunctionReturn(0);
}

#undef __FUNCT__
#define __FUNCT__ "LevelSetUpdateIrregularNodeList"
PetscErrorCode LevelSetUpdateIrregularNodeList(LevelSet ls) {
  dcell_session *s;
  dcell_geom g;
  dcell_irregular_node *buf;
  int *tmp, rc, count = 0, cap;
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
  ierr = b200_store_nodes(ls, buf, count);
  free(buf);
  CHKERRQ(ierr);
  ierr = PetscLogEventEnd(EVENT_LevelSetUpdateIrregularNodeList, 0, 0, 0, 0); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

/* LevelSetAdvectSLRK2HalfStep / FullStep (AdvectRK2.c:5-26): the GridCopy
 * (half step), LevelSetAdvectSL and LevelSetUpdateIrregularNodeList in one
 * library call, phi staying on the device between the advection and the
 * node pass. */
#undef __FUNCT__
#define __FUNCT__ "LevelSetAdvectSLRK2"
static PetscErrorCode b200_rk2(LevelSet ls, Grid velgrid, PetscReal dt, int half) {
  dcell_session *s;
  dcell_geom g;
  dcell_irregular_node *buf;
  int *tmp, rc, count = 0, cap;
  const int nb = ArrayLength(ls->band);
  const int *band;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  if (ls->phi0->SIZE != ls->phi->SIZE || velgrid->SIZE != ls->phi->SIZE * velgrid->dof)
    SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_OUTOFRANGE, "phi0/velgrid do not match phi");
  b200_geom(ls->phi, &g);
  cap = (ls->phi->is2D ? 5 : 10) * (nb > 0 ? nb : 1); /* per point at most 5 (2D) / 10 (3D) nodes */
  buf = (dcell_irregular_node *)malloc(sizeof(dcell_irregular_node) * (size_t)cap);
  if (!buf) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_MEM, "out of host memory");
  band = b200_band(ls->band, &tmp);
  if (half)
    rc = dcell_ls_advect_sl_rk2_half(s, &g, ls->phi0->v1, velgrid->v1, band, nb, dt, b200_interp, b200_backtrace,
                                     b200_precision, ls->phi->v1, 0, buf, cap, &count);
  else
    rc = dcell_ls_advect_sl_rk2_full(s, &g, ls->phi0->v1, velgrid->v1, band, nb, dt, b200_interp, b200_backtrace,
                                     b200_precision, ls->phi->v1, 0, buf, cap, &count);
  free(tmp);
  if (rc == DCELL_ERR_DEPARTURE) {
    /* the reference would read outside its arrays here; the GPU path clamped the sample */
    ierr = PetscInfo1(0, "LevelSetAdvectSLRK2: %s\n", dcell_last_error()); CHKERRQ(ierr);
  } else if (rc) {
    free(buf);
    SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_advect_sl_rk2: %s", dcell_last_error());
  }
  ierr = b200_store_nodes(ls, buf, count);
  free(buf);
  CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

PetscErrorCode LevelSetAdvectSLRK2HalfStep(LevelSet ls, Grid velgrid, PetscReal dt) {
  return b200_rk2(ls, velgrid, dt, 1);
}
PetscErrorCode LevelSetAdvectSLRK2FullStep(LevelSet ls, Grid velgrid, PetscReal dt) {
  return b200_rk2(ls, velgrid, dt, 0);
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

/* LevelSetAdvectMAC / LevelSetAdvectMAC_3D (LevelSetMethod/AdvectMAC.c:
 * 18-111): one first-order conservative upwind step on MAC faces.  The
 * reference routines read the level set's grid as ls->g; with the current
 * struct _LevelSet that grid is ls->phi, and out->phi (same geometry)
 * receives the updated points.  u, v (, w) are the caller's global-index
 * pointer tables (DAVecGetArray of the fluid's face velocities,
 * FluidField/tests/testSource.c:72-84); exactly the face values the step
 * reads are copied out of them. */
PetscErrorCode LevelSetAdvectMAC(LevelSet ls, Coor d, PetscReal dt, PetscReal **u, PetscReal **v, LevelSet out);
PetscErrorCode LevelSetAdvectMAC_3D(LevelSet ls, Coor d, PetscReal dt, PetscReal ***u, PetscReal ***v,
                                    PetscReal ***w, LevelSet out);

/* per axis: the global range [lo, hi] of a component's reads (the updated
 * range [max(p,0), p+n-1), extended by one along the component's own axis) */
static void b200_mac_reads(const dcell_geom *g, int comp, int lo[3], int hi[3]) {
  int a;
  for (a = 0; a < 3; ++a) {
    const int p = g->p[a], n = a < 2 || g->n[2] > 1 ? g->n[a] : 1;
    lo[a] = p < 0 ? 0 : p;
    hi[a] = (a < 2 || g->n[2] > 1) ? p + n - 2 + (a == comp) : 0;
  }
}

#undef __FUNCT__
#define __FUNCT__ "LevelSetAdvectMAC"
static PetscErrorCode b200_advect_mac(LevelSet ls, Coor d, PetscReal dt, PetscReal **u2, PetscReal **v2,
                                      PetscReal ***u3, PetscReal ***v3, PetscReal ***w3, LevelSet out) {
  dcell_session *s;
  dcell_geom g;
  double *buf;
  size_t n;
  int c, i, j, k, rc, lo[3], hi[3];
  const int is3 = u3 != NULL;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  if (out->phi->SIZE != ls->phi->SIZE || out->phi->p.x != ls->phi->p.x || out->phi->p.y != ls->phi->p.y ||
      out->phi->p.z != ls->phi->p.z)
    SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_OUTOFRANGE, "the output level set's grid differs from the input's");
  b200_geom(ls->phi, &g);
  g.h[0] = d.x;
  g.h[1] = d.y;
  g.h[2] = d.z;
  n = (size_t)ls->phi->SIZE;
  buf = (double *)calloc(n * (is3 ? 3 : 2), sizeof(double));
  if (!buf) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_MEM, "out of host memory");
  for (c = 0; c < (is3 ? 3 : 2); ++c) {
    double *dst = buf + (size_t)c * n;
    b200_mac_reads(&g, c, lo, hi);
    for (k = lo[2]; k <= hi[2]; ++k)
      for (j = lo[1]; j <= hi[1]; ++j)
        for (i = lo[0]; i <= hi[0]; ++i) {
          const size_t at = ((size_t)(k - g.p[2]) * g.n[1] + (size_t)(j - g.p[1])) * g.n[0] + (size_t)(i - g.p[0]);
          dst[at] = is3 ? (c == 0 ? u3 : c == 1 ? v3 : w3)[k][j][i] : (c == 0 ? u2 : v2)[j][i];
        }
  }
  rc = dcell_ls_advect_mac(s, &g, ls->phi->v1, buf, buf + n, is3 ? buf + 2 * n : NULL, dt, b200_precision,
                           out->phi->v1);
  free(buf);
  if (rc) SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_advect_mac: %s", dcell_last_error());
  PetscFunctionReturn(0);
}

PetscErrorCode LevelSetAdvectMAC(LevelSet ls, Coor d, PetscReal dt, PetscReal **u, PetscReal **v, LevelSet out) {
  return b200_advect_mac(ls, d, dt, u, v, NULL, NULL, NULL, out);
}

PetscErrorCode LevelSetAdvectMAC_3D(LevelSet ls, Coor d, PetscReal dt, PetscReal ***u, PetscReal ***v,
                                    PetscReal ***w, LevelSet out) {
  return b200_advect_mac(ls, d, dt, NULL, NULL, u, v, w, out);
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

/* ---------------------------------------------------------------------------
 * Particle level set (LevelSetMethod/ParticleLS.c, ParticleLS2D.c,
 * ParticleLS3D.c).  The particle Array's struct _Particle records (X, radius:
 * four doubles) go to the GPU as they are.  Random draws continue the C
 * library's drand48 stream that PETSCRAND48 draws from: its state is read
 * before and written back after each GPU seeding.  Seeding and reseeding are
 * 2D, as the reference's attraction step is; in 3D they return an error.
 */

static void b200_rand48_get(unsigned long long *x) {
  unsigned short t[3] = {0, 0, 0};
  unsigned short *o = seed48(t);
  unsigned short s[3];
  s[0] = o[0];
  s[1] = o[1];
  s[2] = o[2];
  seed48(s);
  *x = (unsigned long long)s[0] | ((unsigned long long)s[1] << 16) | ((unsigned long long)s[2] << 32);
}

static void b200_rand48_set(unsigned long long x) {
  unsigned short s[3];
  s[0] = (unsigned short)(x & 0xFFFF);
  s[1] = (unsigned short)((x >> 16) & 0xFFFF);
  s[2] = (unsigned short)((x >> 32) & 0xFFFF);
  seed48(s);
}

static void b200_pls_params(ParticleLS pls, dcell_pls_params *p) {
  p->r_min = pls->R_MIN;
  p->r_max = pls->R_MAX;
  p->d_init = pls->D_INIT;
  p->g_tol = pls->G_TOL;
  p->e_dist = pls->E_DIST;
  p->s_init = (int)pls->S_INIT;
  p->l_max = pls->L_MAX;
}

#undef __FUNCT__
#define __FUNCT__ "ParticleLS_AdvectParticles"
static PetscErrorCode b200_pls_advect(ParticleLS pls, Coor dh, Grid velgrid, PetscReal dt) {
  dcell_session *s;
  dcell_geom g;
  int rc;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  ierr = PetscLogEventBegin(EVENT_ParticleLS_AdvectParticles, 0, 0, 0, 0); CHKERRQ(ierr);
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  b200_geom(velgrid, &g);
  g.h[0] = dh.x;
  g.h[1] = dh.y;
  g.h[2] = dh.z;
  rc = dcell_ls_pls_advect(s, &g, velgrid->v1, (double *)ArrayGetData(pls->particles), ArrayLength(pls->particles),
                           dt);
  if (rc == DCELL_ERR_DEPARTURE) {
    ierr = PetscInfo1(0, "dcell_ls_pls_advect: %s\n", dcell_last_error()); CHKERRQ(ierr);
  } else if (rc) {
    SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_pls_advect: %s", dcell_last_error());
  }
  ierr = PetscLogEventEnd(EVENT_ParticleLS_AdvectParticles, 0, 0, 0, 0); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

/* ParticleLS_AdvectParticles2D/3D (ParticleLS2D.c:6-36, ParticleLS3D.c:6-36):
 * the velocity grid's own dimension decides (the reference's RK2 steps call
 * the 2D routine in any dimension). */
PetscErrorCode ParticleLS_AdvectParticles2D(ParticleLS pls, Coor dh, Grid velgrid, PetscReal dt) {
  return b200_pls_advect(pls, dh, velgrid, dt);
}
PetscErrorCode ParticleLS_AdvectParticles3D(ParticleLS pls, Coor dh, Grid velgrid, PetscReal dt) {
  return b200_pls_advect(pls, dh, velgrid, dt);
}

#undef __FUNCT__
#define __FUNCT__ "ParticleLS_ErrorCorrection"
static PetscErrorCode b200_pls_correct(ParticleLS pls, LevelSet ls) {
  dcell_session *s;
  dcell_geom g;
  int *bscratch, rc;
  const int *band;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  ierr = PetscLogEventBegin(EVENT_ParticleLS_ErrorCorrection, 0, 0, 0, 0); CHKERRQ(ierr);
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  b200_geom(ls->phi, &g);
  band = b200_band(ls->band, &bscratch);
  rc = dcell_ls_pls_correct(s, &g, ls->phi->v1, band, ArrayLength(ls->band),
                            (const double *)ArrayGetData(pls->particles), ArrayLength(pls->particles));
  free(bscratch);
  if (rc == DCELL_ERR_DEPARTURE) {
    ierr = PetscInfo1(0, "dcell_ls_pls_correct: %s\n", dcell_last_error()); CHKERRQ(ierr);
  } else if (rc) {
    SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_pls_correct: %s", dcell_last_error());
  }
  ierr = PetscLogEventEnd(EVENT_ParticleLS_ErrorCorrection, 0, 0, 0, 0); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

/* ParticleLS_ErrorCorrection2D/3D (ParticleLS2D.c:40-115, ParticleLS3D.c:40-116). */
PetscErrorCode ParticleLS_ErrorCorrection2D(ParticleLS pls, LevelSet ls) { return b200_pls_correct(pls, ls); }
PetscErrorCode ParticleLS_ErrorCorrection3D(ParticleLS pls, LevelSet ls) { return b200_pls_correct(pls, ls); }

/* ParticleLS_AdjustRadii (ParticleLS.c:158-185). */
#undef __FUNCT__
#define __FUNCT__ "ParticleLS_AdjustRadii"
PetscErrorCode ParticleLS_AdjustRadii(ParticleLS pls, LevelSet ls) {
  dcell_session *s;
  dcell_geom g;
  dcell_pls_params prm;
  int rc;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  ierr = PetscLogEventBegin(EVENT_ParticleLS_AdjustRadii, 0, 0, 0, 0); CHKERRQ(ierr);
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  b200_geom(ls->phi, &g);
  b200_pls_params(pls, &prm);
  rc = dcell_ls_pls_adjust_radii(s, &g, ls->phi->v1, (double *)ArrayGetData(pls->particles),
                                 ArrayLength(pls->particles), &prm);
  if (rc) SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_pls_adjust_radii: %s", dcell_last_error());
  ierr = PetscLogEventEnd(EVENT_ParticleLS_AdjustRadii, 0, 0, 0, 0); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

/* Seed (n < 0: LevelSetInitializeParticles' loop) or reseed the particle
 * Array on the GPU, continuing the drand48 stream. */
static PetscErrorCode b200_pls_seed(ParticleLS pls, LevelSet ls, int reseed) {
  dcell_session *s;
  dcell_geom g;
  dcell_pls_params prm;
  int *bscratch, rc;
  const int *band;
  const int nband = ArrayLength(ls->band);
  const int n = reseed ? ArrayLength(pls->particles) : 0;
  long long cap, count = 0;
  unsigned long long rng;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  if (!ls->phi->is2D) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_LIB, "particle seeding is 2D (as the reference's)");
  ierr = LevelSetB200Session(&s); CHKERRQ(ierr);
  b200_geom(ls->phi, &g);
  b200_pls_params(pls, &prm);
  cap = (long long)n + (long long)nband * prm.s_init;
  if (cap >= (1LL << 31)) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_LIB, "too many particles");
  ierr = ArraySetSize(pls->particles, (int)(cap > 0 ? cap : 1)); CHKERRQ(ierr);
  ierr = ArraySetSize(pls->particles, n); CHKERRQ(ierr);  /* room for cap; n live records kept */
  band = b200_band(ls->band, &bscratch);
  b200_rand48_get(&rng);
  rc = reseed ? dcell_ls_pls_reseed(s, &g, ls->phi->v1, band, nband, &prm, &rng,
                                    (double *)ArrayGetData(pls->particles), n, cap, &count)
              : dcell_ls_pls_seed(s, &g, ls->phi->v1, band, nband, &prm, &rng,
                                  (double *)ArrayGetData(pls->particles), cap, &count);
  free(bscratch);
  if (rc && rc != DCELL_ERR_DEPARTURE)
    SETERRQ1(PETSC_COMM_SELF, PETSC_ERR_LIB, "dcell_ls_pls_(re)seed: %s", dcell_last_error());
  b200_rand48_set(rng);
  ierr = ArraySetSize(pls->particles, (int)count); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

/* ParticleLS_ReseedParticles (ParticleLS.c:202-295). */
#undef __FUNCT__
#define __FUNCT__ "ParticleLS_ReseedParticles"
PetscErrorCode ParticleLS_ReseedParticles(ParticleLS pls, LevelSet ls) {
  PetscErrorCode ierr;
  PetscFunctionBegin;
  ierr = PetscLogEventBegin(EVENT_ParticleLS_ReseedParticles, 0, 0, 0, 0); CHKERRQ(ierr);
  ierr = b200_pls_seed(pls, ls, 1); CHKERRQ(ierr);
  ierr = PetscLogEventEnd(EVENT_ParticleLS_ReseedParticles, 0, 0, 0, 0); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}

/* LevelSetInitializeParticles (ParticleLS.c:6-88): the reference's
 * parameters, options and PETSCRAND48 generator, the seeding on the GPU
 * (its AdjustRadii included), the 2D/3D function slots and ls->Advect. */
#undef __FUNCT__
#define __FUNCT__ "LevelSetInitializeParticles"
PetscErrorCode LevelSetInitializeParticles(LevelSet ls) {
  ParticleLS pls;
  PetscErrorCode ierr;

  PetscFunctionBegin;
  ierr = PetscNew(struct _ParticleLS, &ls->pls); CHKERRQ(ierr);
  pls = ls->pls;
  pls->R_MIN = 0.1;
  pls->R_MAX = 0.5;
  pls->D_INIT = 3.0;
  pls->S_INIT = ls->phi->is2D ? 16 : 32;
  pls->L_MAX = 30;
  pls->G_TOL = 1e-3;
  pls->E_DIST = 0.5;
  ierr = PetscOptionsGetReal(0, "-pls_rmin", &pls->R_MIN, 0); CHKERRQ(ierr);
  ierr = PetscOptionsGetReal(0, "-pls_rmax", &pls->R_MAX, 0); CHKERRQ(ierr);
  ierr = PetscOptionsGetReal(0, "-pls_dinit", &pls->D_INIT, 0); CHKERRQ(ierr);
  ierr = PetscOptionsGetInt(0, "-pls_sinit", &pls->S_INIT, 0); CHKERRQ(ierr);
  ierr = PetscOptionsGetReal(0, "-pls_edist", &pls->E_DIST, 0); CHKERRQ(ierr);
  ierr = ArrayCreate("particles", sizeof(struct _Particle), &pls->particles); CHKERRQ(ierr);
  ierr = PetscRandomCreate(PETSC_COMM_WORLD, &pls->rnd); CHKERRQ(ierr);
  ierr = PetscRandomSetType(pls->rnd, PETSCRAND48); CHKERRQ(ierr);
  ierr = b200_pls_seed(pls, ls, 0); CHKERRQ(ierr);
  if (ls->phi->is2D) {
    pls->AdvectParticles = ParticleLS_AdvectParticles2D;
    pls->ErrorCorrection = ParticleLS_ErrorCorrection2D;
  } else {
    pls->AdvectParticles = ParticleLS_AdvectParticles3D;
    pls->ErrorCorrection = ParticleLS_ErrorCorrection3D;
  }
  ls->Advect = LevelSetAdvectPLS;
  ierr = PetscInfo(0, "Particles initialized\n"); CHKERRQ(ierr);
  PetscFunctionReturn(0);
}
