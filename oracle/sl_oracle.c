/*
 * FP64 CPU restatement of the level-set transport path -- the ORACLE.
 *
 * Test infrastructure only: tests/, the smoke check and the bench's CPU
 * baseline call it to check or time the CUDA path; the product never does.
 *
 * Every function names the reference code it restates (paths relative to the
 * reference tree).  The linear paths keep the reference's exact floating
 * point operation order (compiled with -ffp-contract=off) so they reproduce
 * the reference bit for bit; tests pin that against the reference compiled
 * from its own sources (oracle/_ref) and against tests/golden fixtures.
 *
 * Grid convention (Common/Grid.c:69-93): a grid covers global indices
 * [p, p+n) per axis, x fastest; a velocity grid has dof values innermost.
 * 2D grids have nz == 1 and pz == 0.  Index gathers are clamped to the grid
 * (the reference reads out of bounds instead; it never does so for band
 * points that sit >= bandWidth+1 cells inside the grid, Resize.c:13-43).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EXPORT __attribute__((visibility("default")))

typedef struct {
  int nx, ny, nz;    /* extents (nz == 1 in 2D) */
  int px, py, pz;    /* global index of element 0 */
  double hx, hy, hz; /* spacing */
} orc_geom;

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static inline size_t gidx(const orc_geom *g, int i, int j, int k) {
  i = clampi(i, g->px, g->px + g->nx - 1);
  j = clampi(j, g->py, g->py + g->ny - 1);
  k = clampi(k, g->pz, g->pz + g->nz - 1);
  return ((size_t)(k - g->pz) * g->ny + (size_t)(j - g->py)) * g->nx + (size_t)(i - g->px);
}

/* Staggering of the MAC components: Common/Common.h:26-30 (Tensor1). */
static const double kStag[3][3] = {{0.5, 0, 0}, {0, 0.5, 0}, {0, 0, 0.5}};

/* InterpolateVelocity3D, Common/InterpolateVelocity.c:35-67 (same order). */
static void interp_vel3d(const orc_geom *g, const double *vel, const double X[3], double V[3]) {
  for (int d = 0; d < 3; ++d) {
    int xs = (int)floor(X[0] + kStag[d][0]);
    int ys = (int)floor(X[1] + kStag[d][1]);
    int zs = (int)floor(X[2] + kStag[d][2]);
    double sx = X[0] - xs + kStag[d][0];
    double sy = X[1] - ys + kStag[d][1];
    double sz = X[2] - zs + kStag[d][2];
    double sum = 0;
    for (int k = 0; k < 2; ++k)
      for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i)
          sum += ((1 - sx) * (1 - i) + i * sx) * ((1 - sy) * (1 - j) + j * sy) * ((1 - sz) * (1 - k) + k * sz) *
                 vel[gidx(g, xs + i, ys + j, zs + k) * 3 + d];
    V[d] = sum;
  }
}

/* InterpolateVelocity2D, Common/InterpolateVelocity.c:7-33. */
static void interp_vel2d(const orc_geom *g, const double *vel, const double X[2], double V[2]) {
  for (int d = 0; d < 2; ++d) {
    int xs = (int)floor(X[0] + kStag[d][0]);
    int ys = (int)floor(X[1] + kStag[d][1]);
    double sx = X[0] - xs + kStag[d][0];
    double sy = X[1] - ys + kStag[d][1];
    double sum = 0;
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i)
        sum += ((1 - sx) * (1 - i) + i * sx) * ((1 - sy) * (1 - j) + j * sy) * vel[gidx(g, xs + i, ys + j, 0) * 2 + d];
    V[d] = sum;
  }
}

/* Bilinear3D with GridFunction3D_Identity, Common/Grid3D.c:4-36
 * (loop order i, j, k with k innermost; weights i*s + (1-i)*(1-s)). */
static double trilinear_ref(const orc_geom *g, const double *f, const double S[3]) {
  int xs = (int)floor(S[0]), ys = (int)floor(S[1]), zs = (int)floor(S[2]);
  double sx = S[0] - xs, sy = S[1] - ys, sz = S[2] - zs, sum = 0.0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k) {
        double xb = i * sx + (1 - i) * (1 - sx);
        double yb = j * sy + (1 - j) * (1 - sy);
        double zb = k * sz + (1 - k) * (1 - sz);
        sum += f[gidx(g, xs + i, ys + j, zs + k)] * xb * yb * zb;
      }
  return sum;
}

/* Bilinear2D with GridFunction2D_Identity, Common/Grid.c:190-217
 * (weights (1 + (2k-1)(2(x-xi)-1)) / 4, x outer loop). */
static double bilinear_ref(const orc_geom *g, const double *f, double x, double y) {
  int xi = (int)floor(x), yi = (int)floor(y);
  double xf = (2. * (x - xi) - 1.), yf = (2. * (y - yi) - 1.), sum = 0.;
  for (int k = 0; k < 2; ++k)
    for (int l = 0; l < 2; ++l) {
      double xb = 1. + (2. * k - 1.) * xf;
      double yb = 1. + (2. * l - 1.) * yf;
      sum += f[gidx(g, xi + k, yi + l, 0)] * xb * yb;
    }
  sum /= 4.;
  return sum;
}

/* ---- Catmull-Rom (Keys a = -1/2) cubic: the operator of the reference's
 * TricubicInverse.h / OrthogonalProjection.c:48-63, which equals the tensor
 * product C (x) C (x) C of this 4x4 matrix (rows: power 0..3, columns:
 * stencil offsets -1..2).  Pinned against the compiled reference header. */
static const double kCR[4][4] = {
    {0, 1, 0, 0}, {-0.5, 0, 0.5, 0}, {1, -2.5, 2, -0.5}, {-0.5, 1.5, -1.5, 0.5}};

/* a[px + 4py + 16pz] = sum C[pz][sz] C[py][sy] C[px][sx] s[sx + 4sy + 16sz] */
ORC_EXPORT void orc_tricubic_coefs(const double *s, double *a) {
  for (int pz = 0; pz < 4; ++pz)
    for (int py = 0; py < 4; ++py)
      for (int px = 0; px < 4; ++px) {
        double acc = 0.0;
        for (int sz = 0; sz < 4; ++sz)
          for (int sy = 0; sy < 4; ++sy)
            for (int sx = 0; sx < 4; ++sx) {
              double w = kCR[pz][sz] * kCR[py][sy] * kCR[px][sx];
              if (w != 0.0) acc += w * s[sx + 4 * sy + 16 * sz];
            }
        a[px + 4 * py + 16 * pz] = acc;
      }
}

ORC_EXPORT void orc_bicubic_coefs(const double *s, double *a) {
  for (int py = 0; py < 4; ++py)
    for (int px = 0; px < 4; ++px) {
      double acc = 0.0;
      for (int sy = 0; sy < 4; ++sy)
        for (int sx = 0; sx < 4; ++sx) {
          double w = kCR[py][sy] * kCR[px][sx];
          if (w != 0.0) acc += w * s[sx + 4 * sy];
        }
      a[px + 4 * py] = acc;
    }
}

/* p, dp/dx, dp/dy, dp/dz of sum a[i+4j+16k] x^i y^j z^k (TricubicInterpolation.h:1-4). */
static void tricubic_eval(const double *a, double x, double y, double z, double *p, double *gx, double *gy,
                          double *gz) {
  double X[4] = {1, x, x * x, x * x * x}, Y[4] = {1, y, y * y, y * y * y}, Z[4] = {1, z, z * z, z * z * z};
  double dX[4] = {0, 1, 2 * x, 3 * x * x}, dY[4] = {0, 1, 2 * y, 3 * y * y}, dZ[4] = {0, 1, 2 * z, 3 * z * z};
  double v = 0, vx = 0, vy = 0, vz = 0;
  for (int k = 0; k < 4; ++k)
    for (int j = 0; j < 4; ++j)
      for (int i = 0; i < 4; ++i) {
        double c = a[i + 4 * j + 16 * k];
        v += c * X[i] * Y[j] * Z[k];
        vx += c * dX[i] * Y[j] * Z[k];
        vy += c * X[i] * dY[j] * Z[k];
        vz += c * X[i] * Y[j] * dZ[k];
      }
  *p = v;
  if (gx) *gx = vx;
  if (gy) *gy = vy;
  if (gz) *gz = vz;
}

static void bicubic_eval(const double *a, double x, double y, double *p, double *gx, double *gy) {
  double X[4] = {1, x, x * x, x * x * x}, Y[4] = {1, y, y * y, y * y * y};
  double dX[4] = {0, 1, 2 * x, 3 * x * x}, dY[4] = {0, 1, 2 * y, 3 * y * y};
  double v = 0, vx = 0, vy = 0;
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) {
      double c = a[i + 4 * j];
      v += c * X[i] * Y[j];
      vx += c * dX[i] * Y[j];
      vy += c * X[i] * dY[j];
    }
  *p = v;
  if (gx) *gx = vx;
  if (gy) *gy = vy;
}

/* Tricubic sample of f at index-space point S: 4^3 stencil around floor(S),
 * 64 coefficients, polynomial at the fractional offset. */
static double tricubic_sample(const orc_geom *g, const double *f, const double S[3]) {
  int c[3];
  double fr[3], s[64], a[64], p;
  for (int d = 0; d < 3; ++d) {
    c[d] = (int)floor(S[d]);
    fr[d] = S[d] - c[d];
  }
  for (int z = 0; z < 4; ++z)
    for (int y = 0; y < 4; ++y)
      for (int x = 0; x < 4; ++x) s[x + 4 * y + 16 * z] = f[gidx(g, c[0] - 1 + x, c[1] - 1 + y, c[2] - 1 + z)];
  orc_tricubic_coefs(s, a);
  tricubic_eval(a, fr[0], fr[1], fr[2], &p, NULL, NULL, NULL);
  return p;
}

static double bicubic_sample(const orc_geom *g, const double *f, double x, double y) {
  int cx = (int)floor(x), cy = (int)floor(y);
  double s[16], a[16], p;
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) s[i + 4 * j] = f[gidx(g, cx - 1 + i, cy - 1 + j, 0)];
  orc_bicubic_coefs(s, a);
  bicubic_eval(a, x - cx, y - cy, &p, NULL, NULL);
  return p;
}

enum { ORC_LINEAR = 0, ORC_CUBIC = 1 };
enum { ORC_EULER = 0, ORC_MIDPOINT = 1 };

/* One SL step over the band (or every grid point when band == NULL).
 * Euler backtrace = LevelSetAdvectSL_2D/_3D, LevelSetMethod/AdvectSL.c:23-89:
 *   V = MAC velocity at the arrival point X;  S = X - V*dt/h  (index space);
 *   phi[X] = interpolant(phi0, S).
 * Midpoint backtrace (new): Xm = X - V(X)*dt/(2h), S = X - V(Xm)*dt/h. */
ORC_EXPORT int orc_sl_step(const orc_geom *g, const double *phi0, const double *vel, double dt, const int *band,
                           int nband, int interp, int backtrace, double *phi) {
  const int is2D = g->nz == 1;
  const long npts = band ? nband : (long)g->nx * g->ny * g->nz;
  for (long b = 0; b < npts; ++b) {
    int xi, yi, zi;
    if (band) {
      xi = band[3 * b]; yi = band[3 * b + 1]; zi = band[3 * b + 2];
    } else {
      xi = g->px + (int)(b % g->nx);
      yi = g->py + (int)((b / g->nx) % g->ny);
      zi = g->pz + (int)(b / ((long)g->nx * g->ny));
    }
    double X[3] = {xi, yi, is2D ? 0.0 : zi}, V[3] = {0, 0, 0}, S[3];
    if (is2D) interp_vel2d(g, vel, X, V); else interp_vel3d(g, vel, X, V);
    if (backtrace == ORC_MIDPOINT) {
      double Xm[3] = {X[0] - V[0] * (0.5 * dt) / g->hx, X[1] - V[1] * (0.5 * dt) / g->hy,
                      is2D ? 0.0 : X[2] - V[2] * (0.5 * dt) / g->hz};
      if (is2D) interp_vel2d(g, vel, Xm, V); else interp_vel3d(g, vel, Xm, V);
    }
    S[0] = X[0] - V[0] * dt / g->hx;
    S[1] = X[1] - V[1] * dt / g->hy;
    S[2] = is2D ? 0.0 : X[2] - V[2] * dt / g->hz;
    double out;
    if (interp == ORC_LINEAR)
      out = is2D ? bilinear_ref(g, phi0, S[0], S[1]) : trilinear_ref(g, phi0, S);
    else
      out = is2D ? bicubic_sample(g, phi0, S[0], S[1]) : tricubic_sample(g, phi0, S);
    phi[gidx(g, xi, yi, zi)] = out;
  }
  return 0;
}

/* MAC velocity at arbitrary index-space points (InterpolateVelocity2D/3D). */
ORC_EXPORT int orc_interp_velocity(const orc_geom *g, const double *vel, const double *X, int n, double *V) {
  for (int i = 0; i < n; ++i) {
    if (g->nz == 1) {
      interp_vel2d(g, vel, X + 3 * i, V + 3 * i);
      V[3 * i + 2] = 0.0;
    } else {
      interp_vel3d(g, vel, X + 3 * i, V + 3 * i);
    }
  }
  return 0;
}

/* ---------------- finite-difference grid functions ----------------------
 * GridFunction2D_* Common/Grid.c:214-254, GridFunction3D_* Grid3D.c:33-108,
 * same operation order.  fn: 0 identity, 1 d/dx, 2 d/dy, 3 d/dz, 4 curvature */
static double gf3(const orc_geom *g, const double *p, int fn, int i, int j, int k) {
#define P(a, b, c) p[gidx(g, (a), (b), (c))]
  const double dx = g->hx, dy = g->hy, dz = g->hz;
  switch (fn) {
    case 0: return P(i, j, k);
    case 1: return (P(i + 1, j, k) - P(i - 1, j, k)) / (2.0 * dx);
    case 2: return (P(i, j + 1, k) - P(i, j - 1, k)) / (2.0 * dy);
    case 3: return (P(i, j, k + 1) - P(i, j, k - 1)) / (2.0 * dz);
    default: {
      double px = (P(i + 1, j, k) - P(i - 1, j, k)) / (2.0 * dx);
      double py = (P(i, j + 1, k) - P(i, j - 1, k)) / (2.0 * dy);
      double pz = (P(i, j, k + 1) - P(i, j, k - 1)) / (2.0 * dz);
      double px2 = px * px, py2 = py * py, pz2 = pz * pz;
      double ppp = px2 + py2 + pz2;
      double pxx = (P(i - 1, j, k) - 2. * P(i, j, k) + P(i + 1, j, k)) / (dx * dx);
      double pyy = (P(i, j - 1, k) - 2. * P(i, j, k) + P(i, j + 1, k)) / (dy * dy);
      double pzz = (P(i, j, k - 1) - 2. * P(i, j, k) + P(i, j, k + 1)) / (dz * dz);
      double pxy = (P(i - 1, j - 1, k) + P(i + 1, j + 1, k) - P(i - 1, j + 1, k) - P(i + 1, j - 1, k)) / (4. * dx * dy);
      double pxz = (P(i - 1, j, k - 1) + P(i + 1, j, k + 1) - P(i - 1, j, k + 1) - P(i + 1, j, k - 1)) / (4. * dx * dz);
      double pyz = (P(i, j - 1, k - 1) + P(i, j + 1, k + 1) - P(i, j - 1, k + 1) - P(i, j + 1, k - 1)) / (4. * dy * dz);
      double c = px2 * (pyy + pzz) + py2 * (pxx + pzz) + pz2 * (pxx + pyy);
      c -= 2. * (px * py * pxy + px * pz * pxz + py * pz * pyz);
      c /= sqrt(ppp * ppp * ppp);
      if (c != c) c = 0;
      return c;
    }
  }
#undef P
}

static double gf2(const orc_geom *g, const double *p, int fn, int i, int j) {
#define P(a, b) p[gidx(g, (a), (b), 0)]
  const double dx = g->hx, dy = g->hy;
  switch (fn) {
    case 0: return P(i, j);
    case 1: return (P(i + 1, j) - P(i - 1, j)) / (2. * dx);
    case 2: return (P(i, j + 1) - P(i, j - 1)) / (2. * dy);
    case 3: return 0.0;
    default: {
      double px = (P(i + 1, j) - P(i - 1, j)) / (2. * dx);
      double py = (P(i, j + 1) - P(i, j - 1)) / (2. * dy);
      double px2 = px * px, py2 = py * py;
      double pxx = (P(i - 1, j) - 2. * P(i, j) + P(i + 1, j)) / (dx * dx);
      double pyy = (P(i, j - 1) - 2. * P(i, j) + P(i, j + 1)) / (dy * dy);
      double pxy = (P(i - 1, j - 1) + P(i + 1, j + 1) - P(i - 1, j + 1) - P(i + 1, j - 1)) / (4. * dx * dy);
      double k = (pxx * py2 - 2. * px * py * pxy + pyy * px2) / sqrt((px2 + py2) * (px2 + py2) * (px2 + py2));
      if (k != k) k = 0;
      return k;
    }
  }
#undef P
}

/* Bilinear3D / Bilinear2D of grid function fn at index-space point X. */
static double sample_gf(const orc_geom *g, const double *p, int fn, const double X[3]) {
  if (g->nz == 1) {
    int xi = (int)floor(X[0]), yi = (int)floor(X[1]);
    double xf = (2. * (X[0] - xi) - 1.), yf = (2. * (X[1] - yi) - 1.), sum = 0.;
    for (int k = 0; k < 2; ++k)
      for (int l = 0; l < 2; ++l) {
        double xb = 1. + (2. * k - 1.) * xf;
        double yb = 1. + (2. * l - 1.) * yf;
        sum += gf2(g, p, fn, xi + k, yi + l) * xb * yb;
      }
    sum /= 4.;
    return sum;
  }
  int xs = (int)floor(X[0]), ys = (int)floor(X[1]), zs = (int)floor(X[2]);
  double sx = X[0] - xs, sy = X[1] - ys, sz = X[2] - zs, sum = 0.0;
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int k = 0; k < 2; ++k) {
        double xb = i * sx + (1 - i) * (1 - sx);
        double yb = j * sy + (1 - j) * (1 - sy);
        double zb = k * sz + (1 - k) * (1 - sz);
        sum += gf3(g, p, fn, xs + i, ys + j, zs + k) * xb * yb * zb;
      }
  return sum;
}

ORC_EXPORT double orc_sample(const orc_geom *g, const double *p, int fn, double x, double y, double z) {
  double X[3] = {x, y, z};
  if (fn == 5) { /* LevelSetDiracDelta2D/3D, LevelSetMethod/NormalDirection.c:36-57 */
    const double eps = 1.5;
    const double phival = sample_gf(g, p, 0, X);
    if (phival < -eps || phival > eps) return 0;
    const double px = sample_gf(g, p, 1, X), py = sample_gf(g, p, 2, X);
    double gradmag;
    if (g->nz == 1) {
      gradmag = sqrt(px * px + py * py);
    } else {
      const double pz = sample_gf(g, p, 3, X);
      gradmag = sqrt(px * px + py * py + pz * pz);
    }
    return gradmag * (1 + cos(3.14159265358979323846264 * phival / eps)) / (2 * eps);
  }
  return sample_gf(g, p, fn, X);
}

/* ---------------- orthogonal projection ---------------------------------- */
#define ORC_MAXREAL 1.7976931348623157e308

/* OrthogonalProjection2D_Linear, LevelSetMethod/OrthogonalProjection.c:175-195 */
static void ortho2d_linear(const double phi[3][3], double op[3], double *mindist) {
  static const int star[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
  *mindist = 2;
  for (int i = 0; i < 4; ++i) {
    int x = star[i][0] + 1, y = star[i][1] + 1;
    if (phi[1][1] * phi[y][x] <= 0) {
      double dist = phi[1][1] / (phi[1][1] - phi[y][x]);
      if (dist < *mindist) {
        *mindist = dist;
        op[0] = dist * star[i][0];
        op[1] = dist * star[i][1];
      }
    }
  }
}

/* OrthogonalProjection2D_Bicubic, OrthogonalProjection.c:30-125: per sub-cell
 * (i,j) in {0,1}^2 a bicubic patch on phi[j..j+3][i..i+3], damped Newton
 * x += d1 + d2/2 from the node corner, TOL 1e-3, <= 20 iterations. */
static void ortho2d_bicubic(const double phi[5][5], double op[3], double *minDist) {
  const double TOL = 1e-3, TOL2 = TOL * TOL;
  const int MAXITER = 20;
  double mindist = ORC_MAXREAL;
  for (int j = 0; j <= 1; ++j)
    for (int i = 0; i <= 1; ++i) {
      double s[16], a[16];
      for (int y = 0; y < 4; ++y)
        for (int x = 0; x < 4; ++x) s[x + 4 * y] = phi[j + y][i + x];
      orc_bicubic_coefs(s, a);
      double x0x = 1 - i, x0y = 1 - j, x = x0x, y = x0y, dist;
      int m;
      for (m = 0; m < MAXITER; ++m) {
        double p, px, py;
        bicubic_eval(a, x, y, &p, &px, &py);
        double pp = px * px + py * py;
        double d1x = -p * px / pp, d1y = -p * py / pp;
        double xp = (x0x - x) * px + (x0y - y) * py;
        double d2x = (x0x - x) - xp / pp * px, d2y = (x0y - y) - xp / pp * py;
        x += d1x + 0.5 * d2x;
        y += d1y + 0.5 * d2y;
        double norm = d1x * d1x + d1y * d1y + d2x * d2x + d2y * d2y;
        if (norm < TOL2) break;
      }
      if (m == MAXITER) dist = ORC_MAXREAL;
      else if (x < -TOL || 1 + TOL < x || y < -TOL || 1 + TOL < y) dist = ORC_MAXREAL;
      else dist = sqrt((x - x0x) * (x - x0x) + (y - x0y) * (y - x0y));
      if (dist < mindist) {
        mindist = dist;
        op[0] = x + i - 1;
        op[1] = y + j - 1;
        op[2] = 0;
      }
    }
  *minDist = mindist;
}

/* OrthogonalProjection2D, OrthogonalProjection.c:6-23 */
ORC_EXPORT void orc_ortho2d(const double *phi3_in, const double *phi5_in, double *op) {
  double phi3[3][3], phi5[5][5], opB[3] = {0, 0, 0}, opL[3] = {0, 0, 0}, dB, dL;
  memcpy(phi3, phi3_in, sizeof(phi3));
  memcpy(phi5, phi5_in, sizeof(phi5));
  ortho2d_bicubic(phi5, opB, &dB);
  ortho2d_linear(phi3, opL, &dL);
  if (dB < dL) memcpy(op, opB, sizeof(opB));
  else { op[0] = opL[0]; op[1] = opL[1]; op[2] = 0; }
}

/* OrthogonalProjection3D_Linear, OrthogonalProjection3D.c:187-208 */
static void ortho3d_linear(const double phi[3][3][3], double op[3]) {
  static const int star[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  double mindist = 2, dist;
  for (int i = 0; i < 6; ++i) {
    int x = star[i][0] + 1, y = star[i][1] + 1, z = star[i][2] + 1;
    if (phi[1][1][1] * phi[z][y][x] <= 0) {
      dist = phi[1][1][1] / (phi[1][1][1] - phi[z][y][x]);
      if (dist < mindist) {
        mindist = dist;
        op[0] = dist * star[i][0];
        op[1] = dist * star[i][1];
        op[2] = dist * star[i][2];
      }
    }
  }
}

/* OrthogonalProjection3D_Quadratic, OrthogonalProjection3D.c:131-183 */
static void ortho3d_quadratic(const double phi[3][3][3], double op[3]) {
  const int i = 1, j = 1, k = 1;
  double p = phi[k][j][i];
  double px = (phi[k][j][i + 1] - phi[k][j][i - 1]) / 2.;
  double py = (phi[k][j + 1][i] - phi[k][j - 1][i]) / 2.;
  double pz = (phi[k + 1][j][i] - phi[k - 1][j][i]) / 2.;
  double px2 = px * px, py2 = py * py, pz2 = pz * pz;
  double pxx = (phi[k][j][i + 1] - 2. * p + phi[k][j][i - 1]);
  double pyy = (phi[k][j + 1][i] - 2. * p + phi[k][j - 1][i]);
  double pzz = (phi[k + 1][j][i] - 2. * p + phi[k - 1][j][i]);
  double pxy = (phi[k][j - 1][i - 1] + phi[k][j + 1][i + 1] - phi[k][j + 1][i - 1] - phi[k][j - 1][i + 1]) / 4.;
  double pxz = (phi[k - 1][j][i - 1] + phi[k + 1][j][i + 1] - phi[k + 1][j][i - 1] - phi[k - 1][j][i + 1]) / 4.;
  double pyz = (phi[k - 1][j - 1][i] + phi[k + 1][j + 1][i] - phi[k + 1][j - 1][i] - phi[k - 1][j + 1][i]) / 4.;
  double pn = sqrt(px2 + py2 + pz2);
  double c = (px2 * pxx + py2 * pyy + pz2 * pzz + 2 * px * py * pxy + 2 * px * pz * pxz + 2 * py * pz * pyz) /
             (px2 + py2 + pz2);
  double a = 0;
  for (int m = 0; m < 5; ++m) {
    double f = p + pn * a + 0.5 * a * a * c;
    double df = pn + a * c;
    a = a - f / df;
  }
  if (fabs(a) < 1) {
    op[0] = a * px / pn;
    op[1] = a * py / pn;
    op[2] = a * pz / pn;
  } else {
    ortho3d_linear(phi, op);
  }
}

/* OrthogonalProjection3D, OrthogonalProjection3D.c:6-127: 8 tricubic
 * sub-cell patches, damped Newton, closest converged in-cell root wins;
 * quadratic (then linear) fallback when none converges. */
ORC_EXPORT void orc_ortho3d(const double *phi3_in, const double *phi5_in, double *op) {
  double phi3[3][3][3], phi5[5][5][5];
  memcpy(phi3, phi3_in, sizeof(phi3));
  memcpy(phi5, phi5_in, sizeof(phi5));
  const double TOL = 1e-3, TOL2 = TOL * TOL;
  const int MAXITER = 20;
  double mindist = ORC_MAXREAL;
  for (int k = 0; k <= 1; ++k)
    for (int j = 0; j <= 1; ++j)
      for (int i = 0; i <= 1; ++i) {
        double s[64], a[64];
        for (int z = 0; z < 4; ++z)
          for (int y = 0; y < 4; ++y)
            for (int x = 0; x < 4; ++x) s[x + 4 * y + 16 * z] = phi5[k + z][j + y][i + x];
        orc_tricubic_coefs(s, a);
        double x0[3] = {1 - i, 1 - j, 1 - k}, x = x0[0], y = x0[1], z = x0[2], dist;
        int m;
        for (m = 0; m < MAXITER; ++m) {
          double p, px, py, pz;
          tricubic_eval(a, x, y, z, &p, &px, &py, &pz);
          double pp = px * px + py * py + pz * pz;
          double d1x = -p * px / pp, d1y = -p * py / pp, d1z = -p * pz / pp;
          double xp = (x0[0] - x) * px + (x0[1] - y) * py + (x0[2] - z) * pz;
          double d2x = (x0[0] - x) - xp / pp * px, d2y = (x0[1] - y) - xp / pp * py, d2z = (x0[2] - z) - xp / pp * pz;
          x += d1x + 0.5 * d2x;
          y += d1y + 0.5 * d2y;
          z += d1z + 0.5 * d2z;
          double norm = d1x * d1x + d1y * d1y + d1z * d1z + d2x * d2x + d2y * d2y + d2z * d2z;
          if (norm < TOL2) break;
        }
        if (m == MAXITER) dist = ORC_MAXREAL;
        else if (x < -TOL || 1 + TOL < x || y < -TOL || 1 + TOL < y || z < -TOL || 1 + TOL < z) dist = ORC_MAXREAL;
        else dist = sqrt((x - x0[0]) * (x - x0[0]) + (y - x0[1]) * (y - x0[1]) + (z - x0[2]) * (z - x0[2]));
        if (dist < mindist) {
          mindist = dist;
          op[0] = x + i - 1;
          op[1] = y + j - 1;
          op[2] = z + k - 1;
        }
      }
  if (fabs(mindist - ORC_MAXREAL) < 1) ortho3d_quadratic(phi3, op);
}

/* ---------------- irregular nodes ----------------------------------------
 * Record layout (18 doubles per node, the same as the reference driver's
 * export):  pos xyz, axis, shift, signCenter, signFace, d, X xyz, op xyz,
 * n xyz, k.  Order = band order, and within one band point the reference's
 * emission order (IrregularNodes.c:69-138 / IrregularNodes3D.c:294-360). */
#define NODE_W 18

static double *node_new(double *out, long *cnt, long cap) {
  if (*cnt >= cap) { (*cnt)++; return NULL; }
  double *r = out + NODE_W * (*cnt)++;
  memset(r, 0, sizeof(double) * NODE_W);
  return r;
}

static const int kFace[4][3] = {{0, 0, 0}, {-1, 0, 0}, {0, -1, 0}, {0, 0, -1}}; /* STAGGERED_GRID */

ORC_EXPORT long orc_irregular_nodes(const orc_geom *g, const double *phi, const int *band, int nband, double *out,
                                    long cap) {
  long cnt = 0;
  const int is2D = g->nz == 1;
  for (int b = 0; b < nband; ++b) {
    const int i = band[3 * b], j = band[3 * b + 1], k = is2D ? 0 : band[3 * b + 2];
    double *n;
    if (is2D) {
      double sten[3][3], local[5][5];
      for (int J = -2; J <= 2; ++J)
        for (int I = -2; I <= 2; ++I) local[J + 2][I + 2] = phi[gidx(g, I + i, J + j, 0)];
      for (int J = -1; J <= 1; ++J)
        for (int I = -1; I <= 1; ++I) sten[J + 1][I + 1] = phi[gidx(g, I + i, J + j, 0)];
      static const int nei[4][2] = {{1, 0}, {-1, 0}, {0, -1}, {0, 1}};
      for (int m = 0; m < 4; ++m) {
        int ni = 1 + nei[m][0], nj = 1 + nei[m][1];
        if (sten[1][1] * sten[nj][ni] <= 0.) {
          if ((n = node_new(out, &cnt, cap))) {
            double op[3] = {0, 0, 0};
            orc_ortho2d(&sten[0][0], &local[0][0], op);
            n[0] = i; n[1] = j; n[2] = band[3 * b + 2];
            n[3] = -1; n[4] = -1; n[5] = sten[1][1] > 0. ? 1 : -1;
            n[11] = op[0]; n[12] = op[1]; n[13] = op[2];
            n[8] = n[0] + op[0]; n[9] = n[1] + op[1];
          }
          break;
        }
      }
      for (int f = 1; f <= 2; ++f) {
        int ni = 1 + kFace[f][0], nj = 1 + kFace[f][1];
        if (sten[1][1] * sten[nj][ni] <= 0.) {
          if ((n = node_new(out, &cnt, cap))) {
            n[7] = sten[1][1] / (sten[1][1] - sten[nj][ni]);
            n[5] = sten[1][1] > 0. ? 1 : -1;
            n[6] = n[7] < 0.5 ? -n[5] : n[5];
            n[0] = i; n[1] = j; n[2] = band[3 * b + 2];
            n[4] = 0; n[3] = f - 1;
            n[8] = n[0] + n[7] * kFace[f][0];
            n[9] = n[1] + n[7] * kFace[f][1];
          }
        }
      }
      /* U-velocity Laplacian (IrregularNodes.c:108-122) */
      double hi = (sten[1][0] + sten[1][1]) / 2., lo = (sten[0][0] + sten[0][1]) / 2.;
      if (hi * lo <= 0.) {
        if ((n = node_new(out, &cnt, cap))) {
          n[7] = hi / (hi - lo);
          n[5] = hi > 0. ? 1 : -1;
          n[6] = n[7] < 0.5 ? -n[5] : n[5];
          n[0] = i; n[1] = j; n[2] = band[3 * b + 2];
          n[4] = 1; n[3] = 1;
          n[8] = n[0] + kFace[1][0] / 2.;
          n[9] = n[1] + kFace[1][1] / 2. - n[7];
        }
      }
      /* V-velocity Laplacian (IrregularNodes.c:124-138) */
      hi = (sten[0][1] + sten[1][1]) / 2.;
      lo = (sten[0][0] + sten[1][0]) / 2.;
      if (hi * lo <= 0.) {
        if ((n = node_new(out, &cnt, cap))) {
          n[7] = hi / (hi - lo);
          n[5] = hi > 0. ? 1 : -1;
          n[6] = n[7] < 0.5 ? -n[5] : n[5];
          n[0] = i; n[1] = j; n[2] = band[3 * b + 2];
          n[4] = 2; n[3] = 0;
          n[8] = n[0] + kFace[2][0] / 2. - n[7];
          n[9] = n[1] + kFace[2][1] / 2.;
        }
      }
    } else {
      double sten[3][3][3], local[5][5][5];
      for (int K = -2; K <= 2; ++K)
        for (int J = -2; J <= 2; ++J)
          for (int I = -2; I <= 2; ++I) local[K + 2][J + 2][I + 2] = phi[gidx(g, I + i, J + j, K + k)];
      for (int K = -1; K <= 1; ++K)
        for (int J = -1; J <= 1; ++J)
          for (int I = -1; I <= 1; ++I) sten[K + 1][J + 1][I + 1] = phi[gidx(g, I + i, J + j, K + k)];
      static const int star[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
      for (int m = 0; m < 6; ++m) {
        int ni = 1 + star[m][0], nj = 1 + star[m][1], nk = 1 + star[m][2];
        if (sten[1][1][1] * sten[nk][nj][ni] <= 0.) {
          if ((n = node_new(out, &cnt, cap))) {
            double op[3] = {0, 0, 0};
            orc_ortho3d(&sten[0][0][0], &local[0][0][0], op);
            n[0] = i; n[1] = j; n[2] = k;
            n[3] = -1; n[4] = -1; n[5] = sten[1][1][1] > 0. ? 1 : -1;
            n[11] = op[0]; n[12] = op[1]; n[13] = op[2];
            n[8] = n[0] + op[0]; n[9] = n[1] + op[1]; n[10] = n[2] + op[2];
          }
          break;
        }
      }
      for (int f = 1; f <= 3; ++f) {
        int ni = 1 + kFace[f][0], nj = 1 + kFace[f][1], nk = 1 + kFace[f][2];
        if (sten[1][1][1] * sten[nk][nj][ni] <= 0.) {
          if ((n = node_new(out, &cnt, cap))) {
            n[7] = sten[1][1][1] / (sten[1][1][1] - sten[nk][nj][ni]);
            n[5] = sten[1][1][1] > 0. ? 1 : -1;
            n[6] = n[7] < 0.5 ? -n[5] : n[5];
            n[0] = i; n[1] = j; n[2] = k;
            n[4] = 0; n[3] = f - 1;
            n[8] = n[0] + n[7] * kFace[f][0];
            n[9] = n[1] + n[7] * kFace[f][1];
            n[10] = n[2] + n[7] * kFace[f][2];
          }
        }
      }
      /* velocity-face nodes (IrregularNodes3D.c:337-360) */
      for (int face = 1; face <= 3; ++face) {
        const int *gg = kFace[face];
        double hi = (sten[1 + gg[2]][1 + gg[1]][1 + gg[0]] + sten[1][1][1]) / 2.;
        for (int axis = 1; axis <= 3; ++axis) {
          if (face == axis) continue;
          const int *lo3 = kFace[axis];
          double lo = (sten[1 + gg[2] + lo3[2]][1 + gg[1] + lo3[1]][1 + gg[0] + lo3[0]] +
                       sten[1 + lo3[2]][1 + lo3[1]][1 + lo3[0]]) / 2.;
          if (hi * lo <= 0.) {
            if ((n = node_new(out, &cnt, cap))) {
              n[7] = hi / (hi - lo);
              if (n[7] != n[7]) n[7] = 0;
              n[5] = hi > 0. ? 1 : -1;
              n[6] = n[7] < 0.5 ? -n[5] : n[5];
              n[0] = i; n[1] = j; n[2] = k;
              n[4] = face; n[3] = axis - 1;
              n[8] = n[0] + kFace[face][0] / 2. + n[7] * kFace[axis][0];
              n[9] = n[1] + kFace[face][1] / 2. + n[7] * kFace[axis][1];
              n[10] = n[2] + kFace[face][2] / 2. + n[7] * kFace[axis][2];
            }
          }
        }
      }
    }
  }
  return cnt;
}

/* Surface quantities at node positions X (IIM/SurfaceQuantities.c 2D:48-56,
 * 3D:83-89,111): normal = normalised bilinear FD gradient, k = bilinear
 * curvature.  Writes fields 14-17 of each record. */
ORC_EXPORT void orc_node_surface(const orc_geom *g, const double *phi, double *nodes, long n) {
  for (long q = 0; q < n; ++q) {
    double *r = nodes + NODE_W * q;
    double X[3] = {r[8], r[9], r[10]};
    if (g->nz == 1) {
      double nx = sample_gf(g, phi, 1, X), ny = sample_gf(g, phi, 2, X);
      double h = sqrt(nx * nx + ny * ny);
      r[14] = nx / h; r[15] = ny / h; r[16] = 0;
    } else {
      double nx = sample_gf(g, phi, 1, X), ny = sample_gf(g, phi, 2, X), nz = sample_gf(g, phi, 3, X);
      double h = sqrt(nx * nx + ny * ny + nz * nz);
      nx /= h; ny /= h; nz /= h;
      r[14] = nx; r[15] = ny; r[16] = nz;
    }
    r[17] = sample_gf(g, phi, 4, X);
  }
}

/* LevelSet_MaxVelocity, LevelSetMethod/Advect.c:70-111: max |V| over the
 * integer positions of the irregular nodes. */
ORC_EXPORT double orc_max_velocity(const orc_geom *g, const double *vel, const double *nodes, long n) {
  double maxv = 0;
  for (long q = 0; q < n; ++q) {
    const double *r = nodes + NODE_W * q;
    double X[3] = {r[0], r[1], r[2]}, V[3] = {0, 0, 0}, mag;
    if (g->nz == 1) {
      interp_vel2d(g, vel, X, V);
      mag = sqrt(V[0] * V[0] + V[1] * V[1]);
    } else {
      interp_vel3d(g, vel, X, V);
      mag = sqrt(V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    }
    maxv = mag > maxv ? mag : maxv;
  }
  return maxv;
}

/* Enclosed volume (area in 2D) through the smoothed Heaviside
 * H_eps(phi) = 0 | 1 | (1 + phi/eps + sin(pi phi/eps)/pi)/2, eps in the units of
 * phi; inside = sum (1 - H) * cell volume.  The integral of the reference's
 * smoothed delta (NormalDirection.c:36-57). */
ORC_EXPORT double orc_volume(const orc_geom *g, const double *phi, double eps) {
  const double pi = 3.14159265358979323846264;
  double cell = g->hx * g->hy * (g->nz == 1 ? 1.0 : g->hz), acc = 0.0;
  size_t npts = (size_t)g->nx * g->ny * g->nz;
  for (size_t q = 0; q < npts; ++q) {
    double p = phi[q], H;
    if (p < -eps) H = 0.0;
    else if (p > eps) H = 1.0;
    else H = 0.5 * (1.0 + p / eps + sin(pi * p / eps) / pi);
    acc += 1.0 - H;
  }
  return acc * cell;
}

/* ---------------------------------------------------------------------------
 * Narrow-band reinitialisation by bucketed fast marching.
 *
 * The reference (LevelSetReinitialize, LevelSetMethod/FastMarching.c:11-41)
 * resets phi to +/-PHI_INF (PHI_INF = bandWidth + 1.5, LevelSet.c:64), seeds
 * the orthogonal-projection irregular nodes (axis == -1) with
 * signCenter * |op| (FMM_InitializeEikonal, :43-89), and marches each side
 * (sign -1, then +1) outwards with a binary heap (FMM_SolveEikonal, :94-146):
 * pop the smallest tentative value, stop past bandWidth, fix it, and push its
 * 4/6 neighbours with the second-order Rickett-Fomel update
 * (FMM_PushNeighbors2D FastMarching2D.c:103-185, FMM_PushNeighbors3D
 * FastMarching3D.c:13-101, AccumulateCoef FastMarching2D.c:33-99).
 *
 * Here the heap is replaced by buckets of width `bucket` (cells): every
 * tentative value below (b+1)*bucket (and <= bandWidth) is fixed together,
 * then the neighbours of the newly fixed points are re-evaluated with the
 * reference's update and keep the smallest value any evaluation gave them.
 * Each evaluation sees what the heap had fixed when it popped the pushing
 * point: the seeds and the marched points whose value is not larger than the
 * pusher's.  A point's update only reads fixed points, so the result does
 * not depend on the order the points of a bucket are handled in: the GPU
 * kernels follow exactly this procedure.  It equals the heap's result except
 * where a point depends on another point of its own bucket or the heap pops
 * out of value order.  Neighbours outside the grid are skipped (the reference reads them
 * out of bounds; its bands stay inside, Resize.c).  The band comes out in
 * grid order (x fastest) instead of the reference's march order.
 * Returns the band length; -1 if an update is not a number (where the
 * reference exits), -2 if a point within the band width was still tentative
 * after the last bucket.
 */
#define FMM_REINIT_TAIL 16

/* AccumulateCoef, FastMarching2D.c:33-99: the one-sided (1st or 2nd order)
 * difference of the upwind side along one axis, p[-3..3] centred on the point. */
static void fmm_accumulate(double bw, const double *p, double *a, double *b, double *c) {
  const double D2p = (3 * p[0] - 4 * p[1] + p[2]) / 2.;
  const double D2m = (3 * p[0] - 4 * p[-1] + p[-2]) / 2.;
  const double D1p = p[0] - p[1];
  const double D1m = p[0] - p[-1];
  double Dm, am, bm, cm, Dp, ap, bp, cp, t;
  if (0 <= p[1] && p[1] < bw && 0 <= p[2] && p[2] < bw && D2p > 0) {
    t = (4 * p[1] - p[2]) / 3;
    ap = 9. / 4.;
    bp = -9. / 2. * t;
    cp = 9. / 4. * t * t;
    Dp = D2p;
  } else if (0 <= p[1] && p[1] < bw && D1p > 0) {
    ap = 1.;
    bp = -2. * p[1];
    cp = p[1] * p[1];
    Dp = D1p;
  } else {
    ap = bp = cp = Dp = 0;
  }
  if (0 <= p[-1] && p[-1] < bw && 0 <= p[-2] && p[-2] < bw && D2m > 0) {
    t = (4 * p[-1] - p[-2]) / 3;
    am = 9. / 4.;
    bm = -9. / 2. * t;
    cm = 9. / 4. * t * t;
    Dm = D2m;
  } else if (0 <= p[-1] && p[-1] < bw && D1m > 0) {
    am = 1;
    bm = -2. * p[-1];
    cm = p[-1] * p[-1];
    Dm = D1m;
  } else {
    am = bm = cm = Dm = 0;
  }
  if (Dm > Dp) {
    *a += am;
    *b += bm;
    *c += cm;
  } else {
    *a += ap;
    *b += bp;
    *c += cp;
  }
}

/* The update of point (i,j,k) from its fixed neighbours on side `sign`
 * (FMM_PushNeighbors3D :40-81 / 2D :126-157): 7-point lines per axis,
 * PHI_INF outside the grid, quadratic a d^2 + b d + c = 0, larger root. */
static double fmm_update(const orc_geom *g, const double *phi, const unsigned char *mark, int i, int j, int k,
                         int sign, double inf, double lim) {
  const int dim = g->nz == 1 ? 2 : 3;
  double a = 0, b = 0, c = -1, line[7];
  for (int ax = 0; ax < dim; ++ax) {
    for (int m = 0; m < 7; ++m) {
      int q[3] = {i, j, k};
      q[ax] += m - 3;
      const int lo = ax == 0 ? g->px : ax == 1 ? g->py : g->pz;
      const int n = ax == 0 ? g->nx : ax == 1 ? g->ny : g->nz;
      if (q[ax] < lo || q[ax] > lo + n - 1) {
        line[m] = inf;
      } else {
        const size_t r = gidx(g, q[0], q[1], q[2]);
        const double v = sign * phi[r];
        line[m] = (mark[r] == 2 && v > lim) ? inf : v;  /* marched later than the pushing point: not yet known */
      }
    }
    fmm_accumulate(inf, line + 3, &a, &b, &c);
  }
  const double disc = sqrt(b * b - 4 * a * c);
  double d1 = (-b + disc) / (2 * a);
  if (d1 != d1) d1 = -b / (2 * a);
  return d1;
}

static const int kStar[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

/* mark: 0 far, 1 tentative (in the list), 2 fixed by the march, 3 seed.
 * The pushes of point (i,j,k) -- value lim on this side -- see what the heap
 * had fixed when it popped that point: the seeds and the marched points of
 * value <= lim. */
static int fmm_relax(const orc_geom *g, double *phi, double *tent, unsigned char *mark, size_t *list, size_t *nlist,
                     int i, int j, int k, int sign, double bw, double inf, double lim) {
  const int nn = g->nz == 1 ? 4 : 6;
  for (int s = 0; s < nn; ++s) {
    const int x = i + kStar[s][0], y = j + kStar[s][1], z = k + kStar[s][2];
    if (x < g->px || x >= g->px + g->nx || y < g->py || y >= g->py + g->ny || z < g->pz || z >= g->pz + g->nz)
      continue;
    const size_t q = gidx(g, x, y, z);
    if (sign * phi[q] < bw) continue;  /* fixed, or the other side */
    const double v = fmm_update(g, phi, mark, x, y, z, sign, inf, lim);
    if (v != v) return -1;
    if (v < tent[q]) tent[q] = v;
    if (mark[q] == 0) {
      mark[q] = 1;
      list[(*nlist)++] = q;
    }
  }
  return 0;
}

ORC_EXPORT long orc_reinit(const orc_geom *g, double *phi, const double *nodes, long nnodes, double bw,
                           double bucket, int *band, long cap) {
  const double inf = bw + 1.5;
  const size_t n = (size_t)g->nx * g->ny * g->nz;
  const int is2d = g->nz == 1;
  unsigned char *mark = calloc(n, 1);
  double *tent = malloc(sizeof(double) * n);
  size_t *list = malloc(sizeof(size_t) * n), *acc = malloc(sizeof(size_t) * n);
  long status = 0;
  for (size_t q = 0; q < n; ++q) phi[q] = phi[q] > 0 ? inf : -inf;  /* FastMarching.c:28-30 */
  for (long r = 0; r < nnodes; ++r) {                                  /* FastMarching.c:57-70 */
    const double *nd = nodes + 18 * r;
    if ((int)nd[3] != -1) continue;
    const size_t q = gidx(g, (int)nd[0], (int)nd[1], (int)nd[2]);
    const double ox = nd[11], oy = nd[12], oz = nd[13];
    phi[q] = nd[5] * (is2d ? sqrt(ox * ox + oy * oy) : sqrt(ox * ox + oy * oy + oz * oz));
    mark[q] = 3;
  }
  for (int sign = -1; sign <= 1 && status == 0; sign += 2) {
    size_t nl = 0;
    for (size_t q = 0; q < n; ++q) {
      tent[q] = HUGE_VAL;
      if (mark[q] == 1) mark[q] = 0;
    }
    for (long r = 0; r < nnodes && status == 0; ++r) {  /* FastMarching.c:72-84 */
      const double *nd = nodes + 18 * r;
      if ((int)nd[3] != -1) continue;
      const int x = (int)nd[0], y = (int)nd[1], z = (int)nd[2];
      if (sign * phi[gidx(g, x, y, z)] >= 0.)
        status = fmm_relax(g, phi, tent, mark, list, &nl, x, y, z, sign, bw, inf, -HUGE_VAL);
    }
    /* a fixed number of buckets: past bandWidth every bucket fixes all that
       is left <= bandWidth, and FMM_REINIT_TAIL more of them let the last
       pushes settle; a point <= bandWidth still tentative after that is an
       error */
    const long nb = (long)ceil(bw / bucket) + FMM_REINIT_TAIL;
    for (long b = 0; b < nb && status == 0; ++b) {
      const double thr = bucket * (double)(b + 1);
      size_t na = 0, keep = 0;
      for (size_t t = 0; t < nl; ++t) {
        const size_t q = list[t];
        const double v = tent[q];
        if (v < thr && v <= bw) {
          phi[q] = sign * v;
          mark[q] = 2;
          acc[na++] = q;
        } else if (v <= bw) {
          list[keep++] = q;
        } else {
          mark[q] = 0;  /* past the band: never fixed unless a later update lowers it */
        }
      }
      nl = keep;
      for (size_t t = 0; t < na && status == 0; ++t) {
        const size_t q = acc[t];
        const int x = g->px + (int)(q % g->nx), y = g->py + (int)((q / g->nx) % g->ny),
                  z = g->pz + (int)(q / ((size_t)g->nx * g->ny));
        status = fmm_relax(g, phi, tent, mark, list, &nl, x, y, z, sign, bw, inf, sign * phi[q]);
      }
    }
    for (size_t t = 0; t < nl && status == 0; ++t)
      if (tent[list[t]] <= bw) status = -2;  /* a point that could still be fixed */
  }
  long count = 0;
  if (status == 0) {
    for (size_t q = 0; q < n; ++q)
      if (mark[q] >= 2) {
        if (count < cap) {
          band[3 * count + 0] = g->px + (int)(q % g->nx);
          band[3 * count + 1] = g->py + (int)((q / g->nx) % g->ny);
          band[3 * count + 2] = g->pz + (int)(q / ((size_t)g->nx * g->ny));
        }
        ++count;
      }
  }
  free(mark);
  free(tent);
  free(list);
  free(acc);
  return status ? status : count;
}

/* ===========================================================================
 * Particle level set (LevelSetMethod/ParticleLS.c, ParticleLS2D.c,
 * ParticleLS3D.c).  Particles are rows of 4 doubles: X.x, X.y, X.z, radius
 * (struct _Particle, LSM_private.h:45-48), positions in global index space.
 * ======================================================================== */

typedef struct {
  double r_min, r_max, d_init, g_tol, e_dist; /* ParticleLS.c:21-27 */
  int s_init, l_max;
} orc_pls_params;

/* PetscSign: 1, 0 or -1 */
static inline double psign(double a) { return a >= 0 ? (a == 0 ? 0 : 1) : -1; }
static inline double pabs(double a) { return a < 0 ? -a : a; }

/* drand48 (POSIX): X <- (0x5DEECE66D X + 0xB) mod 2^48, value X / 2^48 --
 * the stream PETSc's PETSCRAND48 PetscRandomGetValue draws from. */
static double r48(uint64_t *x) {
  *x = (0x5DEECE66DULL * *x + 0xBULL) & 0xFFFFFFFFFFFFULL;
  return (double)*x * (1.0 / 281474976710656.0);
}

/* GridInterpolate2D/3D, Common/Grid.c:351-410 (weights (1-s)(1-i) + i s). */
static double grid_interp(const orc_geom *g, const double *f, const double X[3]) {
  int xs = (int)floor(X[0]), ys = (int)floor(X[1]);
  double sx = X[0] - xs, sy = X[1] - ys, val = 0;
  if (g->nz == 1) {
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i)
        val += ((1 - sx) * (1 - i) + i * sx) * ((1 - sy) * (1 - j) + j * sy) * f[gidx(g, xs + i, ys + j, 0)];
    return val;
  }
  int zs = (int)floor(X[2]);
  double sz = X[2] - zs;
  for (int k = 0; k < 2; ++k)
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i)
        val += ((1 - sx) * (1 - i) + i * sx) * ((1 - sy) * (1 - j) + j * sy) * ((1 - sz) * (1 - k) + k * sz) *
               f[gidx(g, xs + i, ys + j, zs + k)];
  return val;
}

/* Bilinear2D (Common/Grid.c:190-212) of GridFunction2D_Identity / DerivX /
 * DerivY (:214-227): fn 0, 1, 2 as in gf2. */
static double bilinear_gf(const orc_geom *g, const double *p, int fn, double x, double y) {
  int xi = (int)floor(x), yi = (int)floor(y);
  double xf = (2. * (x - xi) - 1.), yf = (2. * (y - yi) - 1.), sum = 0.;
  for (int k = 0; k < 2; ++k)
    for (int l = 0; l < 2; ++l) {
      double xb = 1. + (2. * k - 1.) * xf;
      double yb = 1. + (2. * l - 1.) * yf;
      sum += gf2(g, p, fn, xi + k, yi + l) * xb * yb;
    }
  sum /= 4.;
  return sum;
}

/* ParticleLS_AdvectParticles2D/3D (ParticleLS2D.c:6-36, ParticleLS3D.c:6-36):
 * RK2 midpoint, V1 = U(Xp), X = Xp + dt/2 V1/h, V2 = U(X), Xp += dt V2/h. */
ORC_EXPORT void orc_pls_advect(const orc_geom *g, const double *vel, double *parts, long n, double dt) {
  const int dim = g->nz == 1 ? 2 : 3;
  for (long m = 0; m < n; ++m) {
    double *p = parts + 4 * m, V1[3] = {0, 0, 0}, V2[3] = {0, 0, 0}, X[3];
    if (dim == 2) {
      interp_vel2d(g, vel, p, V1);
      X[0] = p[0] + dt / 2 * V1[0] / g->hx;
      X[1] = p[1] + dt / 2 * V1[1] / g->hy;
      interp_vel2d(g, vel, X, V2);
      p[0] += dt * V2[0] / g->hx;
      p[1] += dt * V2[1] / g->hy;
    } else {
      interp_vel3d(g, vel, p, V1);
      X[0] = p[0] + dt / 2 * V1[0] / g->hx;
      X[1] = p[1] + dt / 2 * V1[1] / g->hy;
      X[2] = p[2] + dt / 2 * V1[2] / g->hz;
      interp_vel3d(g, vel, X, V2);
      p[0] += dt * V2[0] / g->hx;
      p[1] += dt * V2[1] / g->hy;
      p[2] += dt * V2[2] / g->hz;
    }
  }
}

/* ParticleLS_ErrorCorrection2D/3D (ParticleLS2D.c:40-115,
 * ParticleLS3D.c:40-116): phi+ = phi- = phi; every escaped particle (on the
 * wrong side by more than its radius) raises phi+ / lowers phi- at the
 * corners of its cell to sign (sign r - |X - a|); band points take the one
 * of phi+, phi- with the smaller magnitude.  The 3D corner z is floor(X.y),
 * as the reference writes it (ParticleLS3D.c:76).  Corners outside the grid
 * are skipped (the reference writes out of bounds there); returns their
 * number. */
ORC_EXPORT long orc_pls_correct(const orc_geom *g, double *phi, const int *band, long nband, const double *parts,
                                long n) {
  const int dim = g->nz == 1 ? 2 : 3;
  const size_t N = (size_t)g->nx * g->ny * g->nz;
  double *pos = (double *)malloc(N * sizeof(double)), *neg = (double *)malloc(N * sizeof(double));
  long skipped = 0;
  memcpy(pos, phi, N * sizeof(double));
  memcpy(neg, phi, N * sizeof(double));
  for (long m = 0; m < n; ++m) {
    const double *p = parts + 4 * m;
    double dist = grid_interp(g, phi, p);
    double sign = psign(p[3]);
    if (!(sign * dist < 0 && pabs(dist) > pabs(p[3]))) continue;
    int A[3] = {(int)floor(p[0]), (int)floor(p[1]), dim == 3 ? (int)floor(p[1]) : 0};
    for (int k = 0; k < (dim == 3 ? 2 : 1); ++k)
      for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
          int a[3] = {A[0] + i, A[1] + j, A[2] + k};
          if (a[0] < g->px || a[0] >= g->px + g->nx || a[1] < g->py || a[1] >= g->py + g->ny ||
              (dim == 3 && (a[2] < g->pz || a[2] >= g->pz + g->nz))) {
            ++skipped;
            continue;
          }
          double d2 = (p[0] - a[0]) * (p[0] - a[0]) + (p[1] - a[1]) * (p[1] - a[1]);
          if (dim == 3) d2 = d2 + (p[2] - a[2]) * (p[2] - a[2]);
          double phi_p = sign * (sign * p[3] - sqrt(d2));
          size_t q = gidx(g, a[0], a[1], a[2]);
          if (sign > 0)
            pos[q] = phi_p < pos[q] ? pos[q] : phi_p;
          else
            neg[q] = phi_p < neg[q] ? phi_p : neg[q];
        }
  }
  for (long b = 0; b < nband; ++b) {
    size_t q = gidx(g, band[3 * b], band[3 * b + 1], dim == 3 ? band[3 * b + 2] : 0);
    phi[q] = pabs(pos[q]) <= pabs(neg[q]) ? pos[q] : neg[q];
  }
  free(pos);
  free(neg);
  return skipped;
}

/* ParticleLS_AdjustRadii (ParticleLS.c:158-185). */
ORC_EXPORT void orc_pls_adjust(const orc_geom *g, const double *phi, double *parts, long n, const orc_pls_params *prm) {
  for (long m = 0; m < n; ++m) {
    double *p = parts + 4 * m;
    double dist = grid_interp(g, phi, p);
    double sign = psign(p[3]);
    double sphi = sign * dist;
    if (prm->r_min < sphi && sphi < prm->r_max)
      p[3] = sign * sphi;
    else if (sphi > prm->r_max)
      p[3] = sign * prm->r_max;
    else if (sphi < prm->r_min)
      p[3] = sign * prm->r_min;
  }
}

/* ParticleLS_AttractParticleToPhiGoal (ParticleLS.c:108-154), 2D: steps of
 * lambda along the normal towards phi_goal, halving lambda after a step that
 * does not improve; the accepted position is the local Coor X whose z stays
 * 0.  Without convergence in L_MAX steps the radius becomes sign(phi). */
static void pls_attract2(const orc_geom *g, const double *phi, double *p, double goal, const orc_pls_params *prm) {
  double X[3] = {0, 0, 0}, lambda = 1, phi_X = 0;
  double phi_Xp = bilinear_gf(g, phi, 0, p[0], p[1]);
  int l;
  for (l = 0; l < prm->l_max; ++l) {
    double Nx = bilinear_gf(g, phi, 1, p[0], p[1]);
    double Ny = bilinear_gf(g, phi, 2, p[0], p[1]);
    double mag = sqrt(Nx * Nx + Ny * Ny);
    Nx = Nx / mag;
    Ny = Ny / mag;
    double sign = psign(goal - phi_Xp);
    X[0] = p[0] + sign * lambda * Nx;
    X[1] = p[1] + sign * lambda * Ny;
    phi_X = bilinear_gf(g, phi, 0, X[0], X[1]);
    if (pabs(phi_X - goal) > pabs(phi_Xp - goal)) {
      lambda = lambda / 2.;
    } else {
      p[0] = X[0];
      p[1] = X[1];
      p[2] = X[2];
      phi_Xp = phi_X;
    }
    if (pabs(phi_X - goal) < prm->g_tol) break;
  }
  if (l == prm->l_max) {
    phi_X = bilinear_gf(g, phi, 0, p[0], p[1]);
    p[3] = psign(phi_X);
  }
}

/* LevelSetInitializeParticles (ParticleLS.c:6-88), 2D: S_INIT particles in
 * every band cell with |phi| < D_INIT, each from five draws (position x, y,
 * z in the cell, side, |phi_goal| in [R_MIN, D_INIT)), attracted to its
 * phi_goal; then AdjustRadii.  *rng is the drand48 state (in/out).  Returns
 * the number of particles (at most cap are written), -1 for 3D. */
ORC_EXPORT long orc_pls_init(const orc_geom *g, const double *phi, const int *band, long nband,
                             const orc_pls_params *prm, uint64_t *rng, double *out, long cap) {
  if (g->nz != 1) return -1;
  long cnt = 0;
  for (long b = 0; b < nband; ++b) {
    const int bx = band[3 * b], by = band[3 * b + 1], bz = band[3 * b + 2];
    double dist = pabs(phi[gidx(g, bx, by, 0)]);
    if (!(-prm->d_init < dist && dist < prm->d_init)) continue;
    for (int m = 0; m < prm->s_init; ++m, ++cnt) {
      double p[4], sign, goal;
      p[0] = r48(rng);
      p[1] = r48(rng);
      p[2] = r48(rng);
      p[0] += bx - 0.5;
      p[1] += by - 0.5;
      p[2] += bz - 0.5;
      sign = r48(rng);
      sign = sign > 0.5 ? 1 : -1;
      goal = r48(rng);
      goal = (prm->d_init - prm->r_min) * goal + prm->r_min;
      goal *= sign;
      p[3] = sign;
      pls_attract2(g, phi, p, goal, prm);
      if (cnt < cap) memcpy(out + 4 * cnt, p, sizeof p);
    }
  }
  orc_pls_adjust(g, phi, out, cnt < cap ? cnt : cap, prm);
  return cnt;
}

/* ParticleLS_ReseedParticles (ParticleLS.c:202-295), 2D:
 *  1. delete particles farther than D_INIT (E_DIST for escaped ones), each by
 *     moving the last particle into its slot (ArrayDelete1, Common/Array.c:
 *     272-285) and re-examining the slot;
 *  2. count the non-escaped particles per cell floor(X + 1/2) over phi's box
 *     (ArrayGetCoor's linear index; particles whose index falls outside are
 *     not counted -- the reference then increments the previous lookup);
 *  3. append particles, in band order, to every band cell with |phi| <=
 *     D_INIT until it holds S_INIT: three draws for the position, then draws
 *     of phi_goal in [max(-D, phi-0.71), min(D, phi+0.71)) until |phi_goal|
 *     > R_MIN; radius phi_goal; attracted.
 * parts holds n particles and room for cap; *rng is the drand48 state.
 * Returns the new count (> cap: nothing past cap written), -1 for 3D; *uncounted
 * receives the number of particles of step 2 outside the box. */
ORC_EXPORT long orc_pls_reseed(const orc_geom *g, const double *phi, const int *band, long nband,
                               const orc_pls_params *prm, uint64_t *rng, double *parts, long n, long cap,
                               long *uncounted) {
  if (g->nz != 1) return -1;
  for (long i = 0; i < n; ++i) {
    double *p = parts + 4 * i;
    double dist = grid_interp(g, phi, p);
    double sign = psign(p[3]);
    double thres = sign * dist < 0 ? prm->e_dist : prm->d_init;
    if (pabs(dist) > thres) {
      memcpy(p, parts + 4 * (n - 1), 4 * sizeof(double));
      --n;
      --i;
    }
  }
  const long ncell = (long)g->nx * g->ny;
  int *count = (int *)calloc((size_t)ncell, sizeof(int));
  long miss = 0;
  for (long i = 0; i < n; ++i) {
    const double *p = parts + 4 * i;
    double v = grid_interp(g, phi, p);
    if (p[3] * v < 0) continue;
    long cx = (long)floor(p[0] + 0.5), cy = (long)floor(p[1] + 0.5), cz = (long)floor(p[2] + 0.5);
    long idx = (cx - g->px) + (long)g->nx * (cy - g->py) + (long)g->nx * g->ny * (cz - g->pz);
    if (idx < 0 || idx >= ncell) {
      ++miss;
      continue;
    }
    count[idx]++;
  }
  if (uncounted) *uncounted = miss;
  long cnt = n;
  for (long b = 0; b < nband; ++b) {
    const int bx = band[3 * b], by = band[3 * b + 1], bz = band[3 * b + 2];
    double dist = phi[gidx(g, bx, by, 0)];
    if (pabs(dist) > prm->d_init) continue;
    long idx = (bx - g->px) + (long)g->nx * (by - g->py);
    for (int c = count[idx]; c < prm->s_init; ++c, ++cnt) {
      double p[4], goal, phimax, phimin;
      p[0] = r48(rng);
      p[1] = r48(rng);
      p[2] = r48(rng);
      p[0] += bx - 0.5;
      p[1] += by - 0.5;
      p[2] += bz - 0.5;
      for (;;) {
        goal = r48(rng);
        phimax = prm->d_init < dist + 0.71 ? prm->d_init : dist + 0.71;
        phimin = -prm->d_init < dist - 0.71 ? dist - 0.71 : -prm->d_init;
        goal = (phimax - phimin) * goal + phimin;
        if (goal < -prm->r_min || prm->r_min < goal) break;
      }
      p[3] = goal;
      pls_attract2(g, phi, p, goal, prm);
      if (cnt < cap) memcpy(parts + 4 * cnt, p, sizeof p);
    }
  }
  free(count);
  return cnt;
}

/* ------------------------------------------------------------------------
 * First-order conservative upwind step on MAC faces: LevelSetAdvectMAC
 * (2D) and LevelSetAdvectMAC_3D, LevelSetMethod/AdvectMAC.c:18-111.
 *
 * phi, u, v (, w) and out share the grid g; u[i] is the face between cells
 * i-1 and i (v, w likewise along y, z).  Per axis the updated global range is
 * [max(p, 0), p + n - 1) (AdvectMAC.c:30-35, :68-74); at global index 0 and
 * at the range's last point the missing neighbour is extrapolated as
 * 2 phi - (the other neighbour) (:45-48, :83-88).  Each face contributes the
 * upwind product (:50-53, :90-95) and
 *   out = phi + dt * (du / h.x + dv / h.y (+ dw / h.z))    (:55, :97).
 * Points outside the ranges keep their value in out.  The reference reads
 * outside its grid when an axis with a non-empty range has p > 0 or n < 3;
 * those grids return 7 (nothing written).  Returns 0 otherwise.
 * ---------------------------------------------------------------------- */
static inline double mac_at(const orc_geom *g, const double *a, int i, int j, int k) {
  return a[((size_t)(k - g->pz) * g->ny + (size_t)(j - g->py)) * g->nx + (size_t)(i - g->px)];
}

static int mac_range(int p, int n, int *s, int *e) {
  *s = p < 0 ? 0 : p;
  *e = p + n - 1;
  return *e > *s && (p > 0 || n < 3);
}

ORC_EXPORT int orc_advect_mac(const orc_geom *g, const double *phi, const double *u, const double *v,
                              const double *w, double dt, double *out) {
  const int is3 = g->nz > 1;
  int xs, xe, ys, ye, zs = 0, ze = 1;
  int bad = mac_range(g->px, g->nx, &xs, &xe) | mac_range(g->py, g->ny, &ys, &ye);
  if (is3) bad |= mac_range(g->pz, g->nz, &zs, &ze);
  if (bad) return 7;
  for (int k = zs; k < ze; ++k)
    for (int j = ys; j < ye; ++j)
      for (int i = xs; i < xe; ++i) {
        const double p = mac_at(g, phi, i, j, k);
        const double am = i == 0 ? 2 * p - mac_at(g, phi, i + 1, j, k) : mac_at(g, phi, i - 1, j, k);
        const double an = i == xe - 1 ? 2 * p - mac_at(g, phi, i - 1, j, k) : mac_at(g, phi, i + 1, j, k);
        const double bm = j == 0 ? 2 * p - mac_at(g, phi, i, j + 1, k) : mac_at(g, phi, i, j - 1, k);
        const double bn = j == ye - 1 ? 2 * p - mac_at(g, phi, i, j - 1, k) : mac_at(g, phi, i, j + 1, k);
        const double u0 = mac_at(g, u, i, j, k), u1 = mac_at(g, u, i + 1, j, k);
        const double v0 = mac_at(g, v, i, j, k), v1 = mac_at(g, v, i, j + 1, k);
        double du = u0 > 0. ? am * u0 : p * u0;
        double dv = v0 > 0. ? bm * v0 : p * v0;
        du -= u1 > 0. ? p * u1 : an * u1;
        dv -= v1 > 0. ? p * v1 : bn * v1;
        double r;
        if (is3) {
          const double cm = k == 0 ? 2 * p - mac_at(g, phi, i, j, k + 1) : mac_at(g, phi, i, j, k - 1);
          const double cn = k == ze - 1 ? 2 * p - mac_at(g, phi, i, j, k - 1) : mac_at(g, phi, i, j, k + 1);
          const double w0 = mac_at(g, w, i, j, k), w1 = mac_at(g, w, i, j, k + 1);
          double dw = w0 > 0. ? cm * w0 : p * w0;
          dw -= w1 > 0. ? p * w1 : cn * w1;
          r = p + dt * (du / g->hx + dv / g->hy + dw / g->hz);
        } else {
          r = p + dt * (du / g->hx + dv / g->hy);
        }
        out[((size_t)(k - g->pz) * g->ny + (size_t)(j - g->py)) * g->nx + (size_t)(i - g->px)] = r;
      }
  return 0;
}
