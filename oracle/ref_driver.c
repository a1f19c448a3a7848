/*
 * ctypes-callable driver over the reference's OWN level-set C (compiled from
 * the reference tree against oracle/shim).  Test infrastructure: it loads
 * numpy buffers into the reference's LevelSet / Grid objects, calls the
 * reference functions unchanged and copies the results back out.
 *
 * Reference entry points exercised (paths relative to the reference tree):
 *   LevelSetAdvectSL            LevelSetMethod/AdvectSL.c:6
 *   LevelSetAdvectSLRK2*Step    LevelSetMethod/AdvectRK2.c:5,18
 *   LevelSetUpdateIrregularNodeList  LevelSetMethod/IrregularNodes.c:9
 *   LevelSet_MaxVelocity        LevelSetMethod/Advect.c:70
 *   LevelSetCFLIncrement        LevelSetMethod/Advect.c:54
 *   LevelSetReinitialize        LevelSetMethod/FastMarching.c:11
 *   LevelSetGetVelocity         LevelSetMethod/Advect.c:145 (one-process GA in the shim)
 *   LevelSetInitializeToSphere/Circle  LevelSetMethod/Initializations.c:10,61
 *   Bilinear2D/3D + GridFunction*_Curv/Deriv*  Common/Grid.c:190, Common/Grid3D.c:4
 *   LevelSetDiracDelta2D/3D     LevelSetMethod/NormalDirection.c:36,47
 *   OrthogonalProjection2D/3D   LevelSetMethod/OrthogonalProjection*.c
 *   TricubicInverse.h           (64 Catmull-Rom coefficients of a 4^3 stencil)
 *   particle level set          LevelSetMethod/ParticleLS.c, ParticleLS2D.c, ParticleLS3D.c
 *   GridWrite                   Common/Serialize.c:23 (PETSc binary viewer in the shim)
 *   LevelSetWriteIrregularNodeList  LevelSetMethod/IrregularNodes.c:224
 *   ArrayWrite                  Common/Array.c:134
 */
#include <stdlib.h>
#include <string.h>
#include "LevelSetMethod.h"
#include "LSM_private.h"

#define DREF_EXPORT __attribute__((visibility("default")))

static Coor mkcoor(double x, double y, double z) { Coor c; c.x = x; c.y = y; c.z = z; return c; }
static iCoor mkicoor(int x, int y, int z) { iCoor c; c.x = x; c.y = y; c.z = z; return c; }

DREF_EXPORT void *dref_ls_create(double dx, double dy, double dz, int px, int py, int pz, int nx, int ny, int nz) {
  LevelSet ls = NULL;
  if (LevelSetCreate(mkcoor(dx, dy, dz), mkicoor(px, py, pz), mkicoor(nx, ny, nz), &ls)) return NULL;
  return ls;
}

DREF_EXPORT int dref_ls_destroy(void *h) { return LevelSetDestroy((LevelSet)h); }

/* geometry of phi: p[3], n[3] */
DREF_EXPORT int dref_ls_geometry(void *h, int *p, int *n) {
  LevelSet ls = (LevelSet)h;
  p[0] = ls->phi->p.x; p[1] = ls->phi->p.y; p[2] = ls->phi->p.z;
  n[0] = ls->phi->n.x; n[1] = ls->phi->n.y; n[2] = ls->phi->n.z;
  return ls->phi->SIZE;
}

DREF_EXPORT int dref_ls_set_phi(void *h, const double *src, int which) {
  LevelSet ls = (LevelSet)h;
  Grid g = which ? ls->phi0 : ls->phi;
  if (which && (g->SIZE != ls->phi->SIZE)) {
    int e = GridResize(g, ls->phi->p, ls->phi->n);
    if (e) return e;
  }
  memcpy(g->v1, src, sizeof(double) * (size_t)g->SIZE);
  return 0;
}

DREF_EXPORT int dref_ls_get_phi(void *h, double *dst, int which) {
  LevelSet ls = (LevelSet)h;
  Grid g = which ? ls->phi0 : ls->phi;
  memcpy(dst, g->v1, sizeof(double) * (size_t)g->SIZE);
  return g->SIZE;
}

DREF_EXPORT int dref_ls_set_band(void *h, const int *xyz, int nb) {
  LevelSet ls = (LevelSet)h;
  int e = ArraySetSize(ls->band, nb);
  if (e) return e;
  memcpy(ArrayGetData(ls->band), xyz, sizeof(iCoor) * (size_t)nb);
  return 0;
}

DREF_EXPORT int dref_ls_band_length(void *h) { return ArrayLength(((LevelSet)h)->band); }

DREF_EXPORT int dref_ls_get_band(void *h, int *xyz) {
  LevelSet ls = (LevelSet)h;
  int nb = ArrayLength(ls->band);
  memcpy(xyz, ArrayGetData(ls->band), sizeof(iCoor) * (size_t)nb);
  return nb;
}

DREF_EXPORT double dref_ls_param(void *h, int which) {
  LevelSet ls = (LevelSet)h;
  switch (which) {
    case 0: return ls->bandWidth;
    case 1: return ls->PHI_INF;
    case 2: return ls->CFLcount;
    case 3: return (double)ls->AdvectCount;
    case 4: return ls->maxVel;
    default: return 0.0;
  }
}

/* velocity grid: same p/n as phi, dof 2 (2D) or 3 (3D), dof innermost */
DREF_EXPORT void *dref_vel_create(void *h, const double *src) {
  LevelSet ls = (LevelSet)h;
  Grid phi = ls->phi, vel = NULL;
  int dof = phi->is2D ? 2 : 3;
  if (GridCreate(phi->d, phi->p, phi->n, dof, &vel)) return NULL;
  memcpy(vel->v1, src, sizeof(double) * (size_t)vel->SIZE);
  return vel;
}

DREF_EXPORT int dref_vel_destroy(void *v) { return GridDestroy((Grid)v); }

DREF_EXPORT int dref_advect_sl(void *h, void *vel, double dt) { return LevelSetAdvectSL((LevelSet)h, (Grid)vel, dt); }

DREF_EXPORT int dref_copy_phi_to_phi0(void *h) {
  LevelSet ls = (LevelSet)h;
  return GridCopy(ls->phi, ls->phi0);
}

DREF_EXPORT int dref_rk2_half(void *h, void *vel, double dt) {
  return LevelSetAdvectSLRK2HalfStep((LevelSet)h, (Grid)vel, dt);
}

DREF_EXPORT int dref_rk2_full(void *h, void *vel, double dt) {
  return LevelSetAdvectSLRK2FullStep((LevelSet)h, (Grid)vel, dt);
}

DREF_EXPORT int dref_advect_and_reinit(void *h, void *vel, double dt) {
  return LevelSetAdvectAndReinit((LevelSet)h, (Grid)vel, dt);
}

DREF_EXPORT int dref_cfl_increment(void *h, void *vel, double dt) {
  return LevelSetCFLIncrement((LevelSet)h, (Grid)vel, dt);
}

DREF_EXPORT double dref_max_velocity(void *h, void *vel) {
  LevelSet ls = (LevelSet)h;
  if (LevelSet_MaxVelocity(ls, (Grid)vel)) return -1.0;
  return ls->maxVel;
}

DREF_EXPORT int dref_update_irregular(void *h) {
  LevelSet ls = (LevelSet)h;
  int e = LevelSetUpdateIrregularNodeList(ls);
  if (e) return -e;
  return ArrayLength(ls->irregularNodes);
}

DREF_EXPORT int dref_reinitialize(void *h) { return LevelSetReinitialize((LevelSet)h); }

/* LevelSetGetVelocity (Advect.c:145-192) against the shim's one-process
 * Global Array `global` (dims[ndim], last index the component); writes the
 * level set's velocity grid (its phi box, dof 2/3) to out. */
void dref_ga_set(const double *data, int ndim, const int *dims);
DREF_EXPORT int dref_get_velocity(void *h, const double *global, int ndim, const int *dims, double *out) {
  LevelSet ls = (LevelSet)h;
  Grid velgrid = NULL;
  int e = GridCreate(ls->phi->d, ls->phi->p, ls->phi->n, ls->phi->is2D ? 2 : 3, &velgrid);
  if (e) return e;
  dref_ga_set(global, ndim, dims);
  e = LevelSetGetVelocity(ls, 0, velgrid);
  if (!e) memcpy(out, velgrid->v1, sizeof(double) * (size_t)velgrid->SIZE);
  GridDestroy(velgrid);
  dref_ga_set(NULL, 0, dims);
  return e;
}

/* Irregular node export: 18 doubles per node
 *  0-2 pos.xyz, 3 axis, 4 shift, 5 signCenter, 6 signFace, 7 d,
 *  8-10 X.xyz, 11-13 op.xyz, 14-16 n.xyz, 17 k
 * n and k are the reference IIM surface quantities (IIM/SurfaceQuantities.c:
 * 2D :48-56, 3D :83-89,:111): FD gradient and curvature of phi sampled
 * bilinearly at X, gradient normalised.  Fields a writer did not set stay 0
 * (the reference zeroes the node array first, IrregularNodes.c:16-17). */
DREF_EXPORT int dref_get_irregular(void *h, double *out, int with_surface) {
  LevelSet ls = (LevelSet)h;
  int len = ArrayLength(ls->irregularNodes);
  IrregularNode *nodes = (IrregularNode *)ArrayGetData(ls->irregularNodes);
  Coor dh = ls->phi->d;
  for (int i = 0; i < len; ++i) {
    IrregularNode *n = &nodes[i];
    double *r = out + 18 * (size_t)i;
    r[0] = n->pos.x; r[1] = n->pos.y; r[2] = n->pos.z;
    r[3] = n->axis; r[4] = (int)n->shift; r[5] = n->signCenter; r[6] = n->signFace; r[7] = n->d;
    r[8] = n->X.x; r[9] = n->X.y; r[10] = n->X.z;
    r[11] = n->op.x; r[12] = n->op.y; r[13] = n->op.z;
    r[14] = r[15] = r[16] = r[17] = 0.0;
    if (with_surface) {
      if (ls->phi->is2D) {
        PetscReal **phi;
        GridGet(ls->phi, &phi);
        double nx = Bilinear2D(GridFunction2D_DerivX, phi, dh, n->X.x, n->X.y);
        double ny = Bilinear2D(GridFunction2D_DerivY, phi, dh, n->X.x, n->X.y);
        double hh = sqrt(nx * nx + ny * ny);
        r[14] = nx / hh; r[15] = ny / hh;
        r[17] = Bilinear2D(GridFunction2D_Curv, phi, dh, n->X.x, n->X.y);
      } else {
        PetscReal ***phi;
        GridGet(ls->phi, &phi);
        double nx = Bilinear3D(GridFunction3D_DerivX, phi, dh, n->X);
        double ny = Bilinear3D(GridFunction3D_DerivY, phi, dh, n->X);
        double nz = Bilinear3D(GridFunction3D_DerivZ, phi, dh, n->X);
        double hh = sqrt(nx * nx + ny * ny + nz * nz);
        nx /= hh; ny /= hh; nz /= hh;
        r[14] = nx; r[15] = ny; r[16] = nz;
        r[17] = Bilinear3D(GridFunction3D_Curv, phi, dh, n->X);
      }
    }
  }
  return len;
}

DREF_EXPORT void *dref_init_sphere(double h, double cx, double cy, double cz, double r) {
  LevelSet ls = NULL;
  if (LevelSetInitializeToSphere(mkcoor(h, h, h), mkcoor(cx, cy, cz), r, &ls)) return NULL;
  return ls;
}

DREF_EXPORT void *dref_init_circle(double h, double cx, double cy, double r) {
  LevelSet ls = NULL;
  if (LevelSetInitializeToCircle(mkcoor(h, h, h), mkcoor(cx, cy, 0), r, &ls)) return NULL;
  return ls;
}

/* Point samplers on a standalone phi grid given by the LevelSet's phi. */
DREF_EXPORT double dref_sample(void *h, int fn, double x, double y, double z) {
  LevelSet ls = (LevelSet)h;
  Coor dh = ls->phi->d;
  if (ls->phi->is2D) {
    PetscReal **phi;
    GridGet(ls->phi, &phi);
    switch (fn) {
      case 0: return Bilinear2D(GridFunction2D_Identity, phi, dh, x, y);
      case 1: return Bilinear2D(GridFunction2D_DerivX, phi, dh, x, y);
      case 2: return Bilinear2D(GridFunction2D_DerivY, phi, dh, x, y);
      case 4: return Bilinear2D(GridFunction2D_Curv, phi, dh, x, y);
      case 5: return LevelSetDiracDelta2D(phi, dh, mkcoor(x, y, 0));
      default: return 0.0;
    }
  } else {
    PetscReal ***phi;
    GridGet(ls->phi, &phi);
    Coor X = mkcoor(x, y, z);
    switch (fn) {
      case 0: return Bilinear3D(GridFunction3D_Identity, phi, dh, X);
      case 1: return Bilinear3D(GridFunction3D_DerivX, phi, dh, X);
      case 2: return Bilinear3D(GridFunction3D_DerivY, phi, dh, X);
      case 3: return Bilinear3D(GridFunction3D_DerivZ, phi, dh, X);
      case 4: return Bilinear3D(GridFunction3D_Curv, phi, dh, X);
      case 5: return LevelSetDiracDelta3D(phi, dh, X);
      default: return 0.0;
    }
  }
}

/* Reference MAC velocity interpolation at an arbitrary index-space point. */
DREF_EXPORT int dref_interp_velocity(void *vel, double x, double y, double z, double *out) {
  Grid g = (Grid)vel;
  Coor V, X = mkcoor(x, y, z);
  int e;
  if (g->is2D) {
    PetscReal ***f;
    GridGet(g, &f);
    e = InterpolateVelocity2D(0, f, X, &V);
  } else {
    PetscReal ****f;
    GridGet(g, &f);
    e = InterpolateVelocity3D(0, f, X, &V);
  }
  out[0] = V.x; out[1] = V.y; out[2] = g->is2D ? 0.0 : V.z;
  return e;
}

DREF_EXPORT int dref_ortho3d(const double *phi3_in, const double *phi5_in, double *op_out) {
  double phi3[3][3][3], phi5[5][5][5];
  memcpy(phi3, phi3_in, sizeof(phi3));
  memcpy(phi5, phi5_in, sizeof(phi5));
  Coor op = mkcoor(0, 0, 0);
  int e = OrthogonalProjection3D(phi3, phi5, &op);
  op_out[0] = op.x; op_out[1] = op.y; op_out[2] = op.z;
  return e;
}

DREF_EXPORT int dref_ortho2d(const double *phi3_in, const double *phi5_in, double *op_out) {
  double phi3[3][3], phi5[5][5];
  memcpy(phi3, phi3_in, sizeof(phi3));
  memcpy(phi5, phi5_in, sizeof(phi5));
  Coor op = mkcoor(0, 0, 0);
  int e = OrthogonalProjection2D(phi3, phi5, &op);
  op_out[0] = op.x; op_out[1] = op.y; op_out[2] = 0.0;
  return e;
}

/* The reference's 64 tricubic coefficients for the 4^3 stencil
 * phi[0..3][0..3][0..3] (z, y, x), i.e. TricubicInverse.h evaluated with
 * sub-cell offsets i = j = k = 0 on a 5^3 block whose low corner is the
 * stencil.  Used to pin the oracle's Catmull-Rom operator. */
DREF_EXPORT void dref_tricubic_coefs(const double *stencil64, double *a) {
  double phi[5][5][5];
  int i = 0, j = 0, k = 0;
  memset(phi, 0, sizeof(phi));
  for (int z = 0; z < 4; ++z)
    for (int y = 0; y < 4; ++y)
      for (int x = 0; x < 4; ++x) phi[z][y][x] = stencil64[(z * 4 + y) * 4 + x];
#include "TricubicInverse.h"
  (void)i; (void)j; (void)k;
}

/* ---------------------------------------------------------------------------
 * Particle level set (LevelSetMethod/ParticleLS*.c).  Particles are exchanged
 * as 4 doubles each (struct _Particle: X.x, X.y, X.z, radius). */

/* LevelSetInitializeParticles (ParticleLS.c:6-88): seeds from the band. */
DREF_EXPORT int dref_pls_init(void *h) { return LevelSetInitializeParticles((LevelSet)h); }

/* A particle set with LevelSetInitializeParticles' parameters and function
 * slots but no seeding (its seeding is 2D-only code; 3D particles come from
 * dref_pls_set). */
DREF_EXPORT int dref_pls_create_empty(void *h) {
  LevelSet ls = (LevelSet)h;
  ParticleLS pls;
  int e = PetscNew(struct _ParticleLS, &ls->pls);
  if (e) return e;
  pls = ls->pls;
  pls->R_MIN = 0.1;
  pls->R_MAX = 0.5;
  pls->D_INIT = 3.0;
  pls->S_INIT = ls->phi->is2D ? 16 : 32;
  pls->L_MAX = 30;
  pls->G_TOL = 1e-3;
  pls->E_DIST = 0.5;
  if ((e = ArrayCreate("particles", sizeof(struct _Particle), &pls->particles))) return e;
  if ((e = PetscRandomCreate(PETSC_COMM_WORLD, &pls->rnd))) return e;
  if ((e = PetscRandomSetType(pls->rnd, PETSCRAND48))) return e;
  pls->AdvectParticles = ls->phi->is2D ? ParticleLS_AdvectParticles2D : ParticleLS_AdvectParticles3D;
  pls->ErrorCorrection = ls->phi->is2D ? ParticleLS_ErrorCorrection2D : ParticleLS_ErrorCorrection3D;
  ls->Advect = LevelSetAdvectPLS;
  return 0;
}

/* R_MIN, R_MAX, D_INIT, S_INIT, L_MAX, G_TOL, E_DIST */
DREF_EXPORT int dref_pls_params(void *h, double *out) {
  ParticleLS pls = ((LevelSet)h)->pls;
  if (!pls) return -1;
  out[0] = pls->R_MIN; out[1] = pls->R_MAX; out[2] = pls->D_INIT; out[3] = pls->S_INIT;
  out[4] = pls->L_MAX; out[5] = pls->G_TOL; out[6] = pls->E_DIST;
  return 0;
}

DREF_EXPORT int dref_pls_count(void *h) {
  ParticleLS pls = ((LevelSet)h)->pls;
  return pls ? ArrayLength(pls->particles) : -1;
}

DREF_EXPORT int dref_pls_get(void *h, double *out) {
  ParticleLS pls = ((LevelSet)h)->pls;
  int n = ArrayLength(pls->particles);
  memcpy(out, ArrayGetData(pls->particles), sizeof(struct _Particle) * (size_t)n);
  return n;
}

DREF_EXPORT int dref_pls_set(void *h, const double *src, int n) {
  ParticleLS pls = ((LevelSet)h)->pls;
  int e = ArraySetSize(pls->particles, n);
  if (e) return e;
  memcpy(ArrayGetData(pls->particles), src, sizeof(struct _Particle) * (size_t)n);
  return 0;
}

DREF_EXPORT int dref_pls_advect(void *h, void *vel, double dt) {
  LevelSet ls = (LevelSet)h;
  return ls->pls->AdvectParticles(ls->pls, ls->phi->d, (Grid)vel, dt);
}

DREF_EXPORT int dref_pls_correct(void *h) {
  LevelSet ls = (LevelSet)h;
  return ls->pls->ErrorCorrection(ls->pls, ls);
}

DREF_EXPORT int dref_pls_adjust(void *h) {
  LevelSet ls = (LevelSet)h;
  return ParticleLS_AdjustRadii(ls->pls, ls);
}

DREF_EXPORT int dref_pls_reseed(void *h) {
  LevelSet ls = (LevelSet)h;
  return ParticleLS_ReseedParticles(ls->pls, ls);
}

DREF_EXPORT int dref_pls_step(void *h, void *vel, double dt) { return LevelSetAdvectPLS((LevelSet)h, (Grid)vel, dt); }
DREF_EXPORT int dref_pls_rk2_half(void *h, void *vel, double dt) {
  return LevelSetAdvectPLSRK2HalfStep((LevelSet)h, (Grid)vel, dt);
}
DREF_EXPORT int dref_pls_rk2_full(void *h, void *vel, double dt) {
  return LevelSetAdvectPLSRK2FullStep((LevelSet)h, (Grid)vel, dt);
}

/* the drand48 state (three 16-bit words, least significant first) */
DREF_EXPORT void dref_rand48_get(unsigned short *s) {
  unsigned short tmp[3] = {0, 0, 0};
  unsigned short *old = seed48(tmp);
  s[0] = old[0]; s[1] = old[1]; s[2] = old[2];
  seed48(s);
}
DREF_EXPORT void dref_rand48_set(const unsigned short *s) {
  unsigned short t[3] = {s[0], s[1], s[2]};
  seed48(t);
}

/* ---------------------------------------------------------------------------
 * Output in the reference's file formats, through its own writers. */
void dcell_shim_set_dirs(const char *wd, const char *tmp);

/* directories of DCellGetWorkingDirectory (grids, node lists) and PetscGetTmp (Arrays) */
DREF_EXPORT void dref_set_dirs(const char *wd, const char *tmp) { dcell_shim_set_dirs(wd, tmp); }

/* GridWrite (Common/Serialize.c:23) of a grid, named first (GridSetName,
 * Common/Grid.c:162, which also restarts the grid's .pos / .size files) when
 * its name differs */
static int named_write(Grid g, const char *name, int t) {
  if (strcmp(g->name, name)) {
    int e = GridSetName(g, name);
    if (e) return e;
  }
  return GridWrite(g, t);
}
DREF_EXPORT int dref_grid_write(void *h, const char *name, int t) { return named_write(((LevelSet)h)->phi, name, t); }
/* the same for a velocity grid (dof 2 / 3) */
DREF_EXPORT int dref_vel_write(void *v, const char *name, int t) { return named_write((Grid)v, name, t); }

/* The surface quantities of every irregular node (normal n and curvature k,
 * computed as dref_get_irregular's with_surface export does) stored in the
 * nodes, so that the node-list writer has non-zero values to write. */
DREF_EXPORT int dref_set_surface(void *h) {
  LevelSet ls = (LevelSet)h;
  int len = ArrayLength(ls->irregularNodes);
  double *rows = (double *)malloc(sizeof(double) * 18 * (size_t)(len > 0 ? len : 1));
  if (!rows) return PETSC_ERR_MEM;
  dref_get_irregular(h, rows, 1);
  IrregularNode *nodes = (IrregularNode *)ArrayGetData(ls->irregularNodes);
  for (int i = 0; i < len; ++i) {
    nodes[i].nx = rows[18 * i + 14];
    nodes[i].ny = rows[18 * i + 15];
    nodes[i].nz = rows[18 * i + 16];
    nodes[i].k = rows[18 * i + 17];
  }
  free(rows);
  return len;
}

/* LevelSetWriteIrregularNodeList (IrregularNodes.c:224-246) */
DREF_EXPORT int dref_write_irregular(void *h, int idx) { return LevelSetWriteIrregularNodeList((LevelSet)h, idx); }

/* ArrayWrite (Array.c:134-150) of the particle Array (ParticleLSWriteParticles' call) */
DREF_EXPORT int dref_pls_write(void *h, int t) {
  LevelSet ls = (LevelSet)h;
  if (!ls->pls) return 1;
  return ArrayWrite(ls->pls->particles, t);
}
