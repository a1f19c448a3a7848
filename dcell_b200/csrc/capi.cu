// C ABI of the level-set transport path (include/dcell_ls.h).
//
// Validates arguments, maps them onto the kernel launchers and converts
// device status flags into status codes.  The dcell_ls_* entry points are the
// host-buffer drop-in for the reference's LevelSetAdvectSL,
// LevelSetUpdateIrregularNodeList and LevelSet_MaxVelocity: they copy the
// reference's FP64 arrays in, run the kernels and copy the results back.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "dcell_common.cuh"
#include "dcell_kernels.h"

int launch_tc_gemm_check(const float *A, float *D, int *flags, cudaStream_t st);
int launch_wait_timeout_check(int *result, cudaStream_t st);
static_assert(DCELL_NOALLOC_MAX_BAND == kNoAllocMaxBand, "header and kernel limits differ");

namespace {
thread_local char g_err[1024] = "";
}

extern "C" void dcell_set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  int n = snprintf(g_err, sizeof(g_err), "[dcell %d] ", code);
  if (n < 0) n = 0;
  vsnprintf(g_err + n, sizeof(g_err) - (size_t)n, fmt, ap);
  va_end(ap);
}

#define FAIL(code, ...)                  \
  do {                                   \
    dcell_set_error((code), __VA_ARGS__); \
    return (code);                       \
  } while (0)

static int check_geom(const dcell_geom *g) {
  if (!g) FAIL(DCELL_ERR_ARG, "geometry is NULL");
  if (g->n[0] < 1 || g->n[1] < 1 || g->n[2] < 0)
    FAIL(DCELL_ERR_ARG, "grid extents must be positive (got %d %d %d)", g->n[0], g->n[1], g->n[2]);
  if (!(g->h[0] > 0) || !(g->h[1] > 0) || (g->n[2] > 1 && !(g->h[2] > 0)))
    FAIL(DCELL_ERR_ARG, "grid spacing must be positive");
  const long long n = (long long)g->n[0] * g->n[1] * (g->n[2] > 1 ? g->n[2] : 1);
  if (3 * n >= (1LL << 31)) FAIL(DCELL_ERR_ARG, "grid too large (3 * points must stay below 2^31)");
  return DCELL_OK;
}

static long long grid_points(const dcell_geom *g) {
  return (long long)g->n[0] * g->n[1] * (g->n[2] > 1 ? g->n[2] : 1);
}


extern "C" {

DCELL_API const char *dcell_last_error(void) { return g_err; }
DCELL_API int dcell_version(void) { return DCELL_LS_VERSION; }

DCELL_API int dcell_sl_step(const dcell_geom *g, int dtype, const void *phi0, const void *vel, double dt,
                            const int *band, int nband, int interp, int backtrace, void *phi, int *flags,
                            void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  const bool gather = (interp & DCELL_GATHER_FORM) != 0;
  interp &= ~DCELL_GATHER_FORM;
  if (interp < DCELL_LINEAR || interp > DCELL_CUBIC_TC) FAIL(DCELL_ERR_ARG, "unknown interpolation %d", interp);
  if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
  if (!phi0 || !vel || !phi) FAIL(DCELL_ERR_ARG, "phi0, vel and phi must be device pointers");
  if (band && nband < 0) FAIL(DCELL_ERR_ARG, "nband must be >= 0");
  if (!(dt == dt)) FAIL(DCELL_ERR_NONFINITE, "dt is NaN");
  const dcell::Geom G = dcell::to_geom(g);
  const long long npts = band ? (long long)nband : grid_points(g);
  if (npts == 0) return DCELL_OK;
  cudaStream_t st = (cudaStream_t)stream;
  if (interp == DCELL_LINEAR)
    return launch_sl_linear(G, dtype, phi0, vel, dt, band, npts, backtrace, phi, flags, st, gather);
  if (interp == DCELL_CUBIC_TC) {
    if (dtype != DCELL_F32) FAIL(DCELL_ERR_UNSUPPORTED, "DCELL_CUBIC_TC computes in FP32 only");
    if (G.nz == 1) FAIL(DCELL_ERR_UNSUPPORTED, "DCELL_CUBIC_TC is 3D only");
    return launch_sl_tc(G, (const float *)phi0, (const float *)vel, dt, band, npts, backtrace, (float *)phi, flags,
                        st);
  }
  return launch_sl_cubic(G, dtype, phi0, vel, dt, band, npts, interp, backtrace, phi, flags, st, gather);
}

DCELL_API int dcell_split_bf16(const dcell_geom *g, const float *phi, unsigned int *split, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (!phi || !split) FAIL(DCELL_ERR_ARG, "phi and split are required");
  return launch_split_bf16(phi, split, grid_points(g), (cudaStream_t)stream);
}

DCELL_API int dcell_sl_step_tc_split(const dcell_geom *g, const unsigned int *phi0_split, const float *vel, double dt,
                                     const int *band, int nband, int backtrace, float *phi, unsigned int *phi_split,
                                     int *flags, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (g->n[2] < 2) FAIL(DCELL_ERR_UNSUPPORTED, "the tensor-core step is 3D only");
  if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
  if (!phi0_split || !vel || !phi) FAIL(DCELL_ERR_ARG, "phi0_split, vel and phi must be device pointers");
  if (band && nband < 0) FAIL(DCELL_ERR_ARG, "nband must be >= 0");
  if (!(dt == dt)) FAIL(DCELL_ERR_NONFINITE, "dt is NaN");
  const long long npts = band ? (long long)nband : grid_points(g);
  if (npts == 0) return DCELL_OK;
  return launch_sl_tc_split(dcell::to_geom(g), phi0_split, vel, dt, band, npts, backtrace, phi, phi_split, flags,
                            (cudaStream_t)stream);
}

DCELL_API int dcell_sl_step_tc_split_planes(const dcell_geom *g, const unsigned int *phi0_split, const float *vel,
                                            double dt, int z_begin, int z_end, int backtrace, float *phi,
                                            unsigned int *phi_split, int *flags, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (g->n[2] < 2) FAIL(DCELL_ERR_UNSUPPORTED, "the tensor-core step is 3D only");
  if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
  if (!phi0_split || !vel || !phi) FAIL(DCELL_ERR_ARG, "phi0_split, vel and phi must be device pointers");
  if (!(dt == dt)) FAIL(DCELL_ERR_NONFINITE, "dt is NaN");
  const int nz = g->n[2], bz = tc_slab_planes();
  if (z_begin < 0 || z_end > nz || z_begin > z_end)
    FAIL(DCELL_ERR_ARG, "plane range [%d, %d) outside the grid's %d planes", z_begin, z_end, nz);
  if (z_begin % bz || (z_end % bz && z_end != nz))
    FAIL(DCELL_ERR_ARG, "plane range [%d, %d) not aligned to %d-plane bricks", z_begin, z_end, bz);
  const dcell::Geom G = dcell::to_geom(g);
  if (!tc_brick_applicable(G, phi0_split, vel))
    FAIL(DCELL_ERR_UNSUPPORTED, "plane ranges need the dense brick path (nx %% 4 == 0, 16-byte aligned arrays, "
                                "at least one brick box per axis)");
  if (z_begin == z_end) return DCELL_OK;
  return launch_sl_tc_split_planes(G, phi0_split, vel, dt, backtrace, phi, phi_split, flags, (cudaStream_t)stream,
                                   z_begin / bz, (z_end - z_begin + bz - 1) / bz);
}

DCELL_API int dcell_sl_adjoint(const dcell_geom *g, int dtype, const void *phi0, const void *vel, double dt,
                               int interp, int backtrace, const void *grad_phi, void *grad_phi0, void *grad_vel,
                               void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (g->n[2] < 2) FAIL(DCELL_ERR_UNSUPPORTED, "the adjoint step is 3D only");
  if (interp < DCELL_LINEAR || interp > DCELL_CUBIC_TC) FAIL(DCELL_ERR_ARG, "unknown interpolation %d", interp);
  if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
  if (!phi0 || !vel || !grad_phi || !grad_phi0 || !grad_vel) FAIL(DCELL_ERR_ARG, "all arrays are required");
  if (!(dt == dt)) FAIL(DCELL_ERR_NONFINITE, "dt is NaN");
  return launch_sl_adjoint(dcell::to_geom(g), dtype, phi0, vel, dt, interp, backtrace, grad_phi, grad_phi0, grad_vel,
                           (cudaStream_t)stream);
}

DCELL_API size_t dcell_irregular_nodes_scratch_bytes(int nband) { return irregular_scratch_bytes(nband < 0 ? 0 : nband); }

DCELL_API int dcell_irregular_nodes(const dcell_geom *g, int dtype, const void *phi, const int *band, int nband,
                                    int with_surface, dcell_irregular_node *nodes, int capacity, int *count,
                                    void *scratch, size_t scratch_bytes, int *flags, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (!phi || !count || nband < 0 || (nband > 0 && !band)) FAIL(DCELL_ERR_ARG, "phi, band and count are required");
  if (capacity < 0 || (capacity > 0 && !nodes)) FAIL(DCELL_ERR_ARG, "invalid node buffer");
  if (nband > 0 && (!scratch || scratch_bytes < irregular_scratch_bytes(nband)))
    FAIL(DCELL_ERR_ARG, "scratch must hold %zu bytes", irregular_scratch_bytes(nband));
  return launch_irregular(dcell::to_geom(g), dtype, phi, band, nband, with_surface, nodes, capacity, count, scratch,
                          flags, (cudaStream_t)stream);
}

static int check_field(const int gdims[3], int gdof, int first, int dim) {
  if (!gdims || gdims[0] < 1 || gdims[1] < 1 || gdims[2] < 1) FAIL(DCELL_ERR_ARG, "field extents must be positive");
  if (first < 0 || first + dim > gdof)
    FAIL(DCELL_ERR_ARG, "components %d..%d outside the field's %d", first, first + dim - 1, gdof);
  if ((long long)gdims[0] * gdims[1] * gdims[2] * gdof >= (1LL << 40)) FAIL(DCELL_ERR_ARG, "field too large");
  return DCELL_OK;
}

DCELL_API int dcell_velocity_box(const dcell_geom *g, int dtype, const void *global, const int gdims[3], int gdof,
                                 int first, void *vel, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (!global || !vel) FAIL(DCELL_ERR_ARG, "global and vel are required");
  const int dim = g->n[2] > 1 ? 3 : 2;
  if (dim == 2 && gdims && gdims[2] > 1) FAIL(DCELL_ERR_ARG, "a 2D box needs a 2D field (gdims[2] == 1)");
  if ((rc = check_field(gdims, gdof, first, dim))) return rc;
  return launch_velocity_box(dcell::to_geom(g), dtype, global, gdims, gdof, first, vel, (cudaStream_t)stream);
}

DCELL_API int dcell_velocity_boxes(const dcell_box *boxes, int nboxes, int dim, int dtype, const void *global,
                                   const int gdims[3], int gdof, int first, long long max_points, void *vel,
                                   void *stream) {
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (dim != 2 && dim != 3) FAIL(DCELL_ERR_ARG, "dim must be 2 or 3");
  if (nboxes < 0 || nboxes > 65535 || (nboxes > 0 && (!boxes || !global || !vel)))
    FAIL(DCELL_ERR_ARG, "boxes (at most 65535), global and vel are required");
  if (max_points < 0) FAIL(DCELL_ERR_ARG, "max_points must be >= 0");
  int rc = check_field(gdims, gdof, first, dim);
  if (rc) return rc;
  return launch_velocity_boxes(boxes, nboxes, dim, dtype, global, gdims, gdof, first, max_points, vel,
                               (cudaStream_t)stream);
}

DCELL_API size_t dcell_reinit_scratch_bytes(const dcell_geom *g, int dtype) {
  if (!g) return 0;
  const long long n = (long long)g->n[0] * g->n[1] * (g->n[2] > 1 ? g->n[2] : 1);
  return reinit_scratch_bytes(n, dtype);
}

DCELL_API int dcell_reinitialize(const dcell_geom *g, int dtype, void *phi, const dcell_irregular_node *nodes,
                                 int nnodes, double band_width, double bucket, int *band, int capacity, int *count,
                                 void *scratch, size_t scratch_bytes, int *flags, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (!phi || !count || nnodes < 0 || (nnodes > 0 && !nodes)) FAIL(DCELL_ERR_ARG, "phi, nodes and count are required");
  if (capacity < 0 || (capacity > 0 && !band)) FAIL(DCELL_ERR_ARG, "invalid band buffer");
  if (!(band_width > 0)) FAIL(DCELL_ERR_ARG, "band_width must be positive");
  if (bucket == 0) bucket = 1.0 / 64;
  if (!(bucket > 0) || band_width / bucket > 1e6) FAIL(DCELL_ERR_ARG, "bucket must be positive and not tiny");
  const size_t need = dcell_reinit_scratch_bytes(g, dtype);
  if (!scratch || scratch_bytes < need) FAIL(DCELL_ERR_ARG, "scratch must hold %zu bytes", need);
  if ((uintptr_t)scratch % 256) FAIL(DCELL_ERR_ARG, "scratch must be 256-byte aligned");
  return launch_reinit(dcell::to_geom(g), dtype, phi, nodes, nnodes, band_width, bucket, band, capacity, count,
                       scratch, flags, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Particle level set

DCELL_API void dcell_pls_default_params(int dim, dcell_pls_params *out) {
  if (!out) return;
  out->r_min = 0.1;
  out->r_max = 0.5;
  out->d_init = 3.0;
  out->g_tol = 1e-3;
  out->e_dist = 0.5;
  out->s_init = dim == 3 ? 32 : 16;
  out->l_max = 30;
}

static int check_pls_common(const dcell_geom *g, int dtype, long long n, const void *parts) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (n < 0 || n >= (1LL << 31)) FAIL(DCELL_ERR_ARG, "particle count must be in [0, 2^31)");
  if (n > 0 && !parts) FAIL(DCELL_ERR_ARG, "particles are required");
  return DCELL_OK;
}

static int check_pls_params(const dcell_pls_params *prm) {
  if (!prm) FAIL(DCELL_ERR_ARG, "parameters are required");
  if (prm->s_init < 0 || prm->s_init > 4096 || prm->l_max < 0 || prm->l_max > 100000)
    FAIL(DCELL_ERR_ARG, "s_init must be in [0, 4096] and l_max in [0, 100000]");
  if (!(prm->r_min >= 0) || !(prm->d_init > prm->r_min)) FAIL(DCELL_ERR_ARG, "need 0 <= r_min < d_init");
  return DCELL_OK;
}

DCELL_API int dcell_pls_advect(const dcell_geom *g, int dtype, const void *vel, void *particles, long long n,
                               double dt, int *flags, void *stream) {
  int rc = check_pls_common(g, dtype, n, particles);
  if (rc) return rc;
  if (!vel) FAIL(DCELL_ERR_ARG, "vel is required");
  return launch_pls_advect(dcell::to_geom(g), dtype, vel, particles, n, dt, flags, (cudaStream_t)stream);
}

DCELL_API size_t dcell_pls_correct_scratch_bytes(const dcell_geom *g, int dtype) {
  if (check_geom(g)) return 0;
  return pls_correct_scratch_bytes(grid_points(g), dtype);
}

DCELL_API int dcell_pls_correct(const dcell_geom *g, int dtype, void *phi, const int *band, long long nband,
                                const void *particles, long long n, void *scratch, size_t scratch_bytes, int *flags,
                                void *stream) {
  int rc = check_pls_common(g, dtype, n, particles);
  if (rc) return rc;
  if (!phi || nband < 0 || nband >= (1LL << 31) || (nband > 0 && !band)) FAIL(DCELL_ERR_ARG, "phi and band are required");
  const size_t need = pls_correct_scratch_bytes(grid_points(g), dtype);
  if (!scratch || scratch_bytes < need) FAIL(DCELL_ERR_ARG, "scratch must hold %zu bytes", need);
  if ((uintptr_t)scratch % 256) FAIL(DCELL_ERR_ARG, "scratch must be 256-byte aligned");
  return launch_pls_correct(dcell::to_geom(g), dtype, phi, band, nband, particles, n, scratch, flags,
                            (cudaStream_t)stream);
}

DCELL_API int dcell_pls_adjust_radii(const dcell_geom *g, int dtype, const void *phi, void *particles, long long n,
                                     const dcell_pls_params *prm, int *flags, void *stream) {
  int rc = check_pls_common(g, dtype, n, particles);
  if (rc) return rc;
  if ((rc = check_pls_params(prm))) return rc;
  if (!phi) FAIL(DCELL_ERR_ARG, "phi is required");
  return launch_pls_adjust(dcell::to_geom(g), dtype, phi, particles, n, *prm, flags, (cudaStream_t)stream);
}

DCELL_API size_t dcell_pls_scratch_bytes(const dcell_geom *g, long long nband, long long n) {
  if (check_geom(g) || nband < 0 || n < 0) return 0;
  return pls_scratch_bytes(grid_points(g), nband, n);
}

static int check_pls_seed_args(const dcell_geom *g, int dtype, const void *phi, const int *band, long long nband,
                               const dcell_pls_params *prm, const unsigned long long *rng, const void *parts,
                               long long n, long long capacity, const long long *count, const void *scratch,
                               size_t scratch_bytes) {
  int rc = check_pls_common(g, dtype, n, parts);
  if (rc) return rc;
  if ((rc = check_pls_params(prm))) return rc;
  if (g->n[2] > 1) FAIL(DCELL_ERR_UNSUPPORTED, "particle seeding is 2D (the reference's attraction is 2D code)");
  if (!phi || !rng || !count) FAIL(DCELL_ERR_ARG, "phi, rng and count are required");
  if (nband < 0 || nband * (long long)(prm->s_init > 0 ? prm->s_init : 1) >= (1LL << 31) || (nband > 0 && !band))
    FAIL(DCELL_ERR_ARG, "invalid band");
  if (capacity < 0 || capacity >= (1LL << 31) || (capacity > 0 && !parts)) FAIL(DCELL_ERR_ARG, "invalid particle buffer");
  const size_t need = pls_scratch_bytes(grid_points(g), nband, n);
  if (!scratch || scratch_bytes < need) FAIL(DCELL_ERR_ARG, "scratch must hold %zu bytes", need);
  if ((uintptr_t)scratch % 256) FAIL(DCELL_ERR_ARG, "scratch must be 256-byte aligned");
  return DCELL_OK;
}

DCELL_API int dcell_pls_seed(const dcell_geom *g, int dtype, const void *phi, const int *band, long long nband,
                             const dcell_pls_params *prm, unsigned long long *rng, void *particles, long long capacity,
                             long long *count, void *scratch, size_t scratch_bytes, int *flags, void *stream) {
  int rc = check_pls_seed_args(g, dtype, phi, band, nband, prm, rng, particles, 0, capacity, count, scratch,
                               scratch_bytes);
  if (rc) return rc;
  return launch_pls_seed(dcell::to_geom(g), dtype, phi, band, nband, *prm, rng, particles, capacity, count, scratch,
                         flags, (cudaStream_t)stream);
}

DCELL_API int dcell_pls_reseed(const dcell_geom *g, int dtype, const void *phi, const int *band, long long nband,
                               const dcell_pls_params *prm, unsigned long long *rng, void *particles, long long n,
                               long long capacity, long long *count, void *scratch, size_t scratch_bytes, int *flags,
                               void *stream) {
  int rc = check_pls_seed_args(g, dtype, phi, band, nband, prm, rng, particles, n, capacity, count, scratch,
                               scratch_bytes);
  if (rc) return rc;
  if (n > capacity) FAIL(DCELL_ERR_ARG, "n exceeds the capacity");
  return launch_pls_reseed(dcell::to_geom(g), dtype, phi, band, nband, *prm, rng, particles, n, capacity, count,
                           scratch, flags, (cudaStream_t)stream);
}

DCELL_API int dcell_irregular_nodes_noalloc(const dcell_geom *g, int dtype, const void *phi, const int *band,
                                            int nband, int with_surface, dcell_irregular_node *nodes, int capacity,
                                            int *count, int *flags, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (nband > DCELL_NOALLOC_MAX_BAND)
    FAIL(DCELL_ERR_ARG, "band of %d points exceeds the allocation-free maximum of %d", nband, DCELL_NOALLOC_MAX_BAND);
  if (!phi || !count || nband < 0 || (nband > 0 && !band)) FAIL(DCELL_ERR_ARG, "phi, band and count are required");
  if (capacity < 0 || (capacity > 0 && !nodes)) FAIL(DCELL_ERR_ARG, "invalid node buffer");
  return launch_irregular_noalloc(dcell::to_geom(g), dtype, phi, band, nband, with_surface, nodes, capacity, count,
                                  flags, (cudaStream_t)stream);
}

DCELL_API int dcell_max_velocity(const dcell_geom *g, int dtype, const void *vel, const dcell_irregular_node *nodes,
                                 const int *count, int capacity, double *maxvel, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (!vel || !count || !maxvel || capacity < 0 || (capacity > 0 && !nodes)) FAIL(DCELL_ERR_ARG, "missing pointer");
  return launch_max_velocity(dcell::to_geom(g), dtype, vel, nodes, count, capacity, maxvel, (cudaStream_t)stream);
}

// Updated global range [s, e) of one axis of LevelSetAdvectMAC
// (AdvectMAC.c:30-35, :68-74); false where the reference would read outside
// its grid on that axis (a non-empty range with p > 0 or n < 3).
static bool mac_axis(int p, int n, int *s, int *e) {
  *s = p < 0 ? 0 : p;
  *e = p + n - 1;
  return !(*e > *s && (p > 0 || n < 3));
}

static int mac_ranges(const dcell_geom *g, int range[6]) {
  bool ok = mac_axis(g->p[0], g->n[0], &range[0], &range[1]);
  ok = mac_axis(g->p[1], g->n[1], &range[2], &range[3]) && ok;
  range[4] = 0;
  range[5] = 1;
  if (g->n[2] > 1) ok = mac_axis(g->p[2], g->n[2], &range[4], &range[5]) && ok;
  if (!ok)
    FAIL(DCELL_ERR_UNSUPPORTED,
         "LevelSetAdvectMAC reads outside its grid when an updated axis has origin > 0 or fewer than 3 points");
  return DCELL_OK;
}

DCELL_API int dcell_advect_mac(const dcell_geom *g, int dtype, const void *phi, const void *u, const void *v,
                               const void *w, double dt, void *out, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (!phi || !u || !v || !out || (g->n[2] > 1 && !w)) FAIL(DCELL_ERR_ARG, "phi, u, v, (3D: w) and out are required");
  if (out == phi) FAIL(DCELL_ERR_ARG, "out must not alias phi (the step reads phi's neighbours)");
  if (!(dt == dt)) FAIL(DCELL_ERR_NONFINITE, "dt is NaN");
  int range[6];
  rc = mac_ranges(g, range);
  if (rc) return rc;
  return launch_advect_mac(dcell::to_geom(g), dtype, phi, u, v, g->n[2] > 1 ? w : nullptr, dt, range, out,
                           (cudaStream_t)stream);
}

DCELL_API size_t dcell_volume_scratch_bytes(void) { return volume_scratch_bytes(); }

DCELL_API int dcell_volume(const dcell_geom *g, int dtype, const void *phi, double eps, double *volume, void *scratch,
                           size_t scratch_bytes, void *stream) {
  int rc = check_geom(g);
  if (rc) return rc;
  if (dtype != DCELL_F32 && dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "dtype must be DCELL_F32 or DCELL_F64");
  if (!phi || !volume) FAIL(DCELL_ERR_ARG, "phi and volume are required");
  if (!(eps > 0)) FAIL(DCELL_ERR_ARG, "eps must be positive");
  if (!scratch || scratch_bytes < volume_scratch_bytes())
    FAIL(DCELL_ERR_ARG, "scratch must hold %zu bytes", volume_scratch_bytes());
  return launch_volume(dcell::to_geom(g), dtype, phi, eps, volume, (double *)scratch, (cudaStream_t)stream);
}

DCELL_API int dcell_batch_plan(const dcell_cell *cells, int ncells, int tx, int ty, int tz, dcell_tile *tiles,
                               int capacity, int *ntiles) {
  if (!cells || ncells < 0 || !ntiles || capacity < 0 || (capacity > 0 && !tiles))
    FAIL(DCELL_ERR_ARG, "cells, tiles and ntiles are required");
  if (tx < 1 || ty < 1 || tz < 1) FAIL(DCELL_ERR_ARG, "tile extents must be positive");
  long long k = 0;
  for (int c = 0; c < ncells; ++c) {
    const dcell_cell &C = cells[c];
    if (C.n[0] < 1 || C.n[1] < 1 || C.n[2] < 1 || C.offset < 0) FAIL(DCELL_ERR_ARG, "cell %d has an empty grid", c);
    if (3LL * C.n[0] * C.n[1] * C.n[2] >= (1LL << 31)) FAIL(DCELL_ERR_ARG, "cell %d grid too large", c);
    for (int z = 0; z < C.n[2]; z += tz)
      for (int y = 0; y < C.n[1]; y += ty)
        for (int x = 0; x < C.n[0]; x += tx) {
          if (k < capacity) tiles[k] = dcell_tile{c, x, y, z};
          ++k;
        }
  }
  if (k > (1LL << 31) - 1) FAIL(DCELL_ERR_ARG, "too many tiles");
  *ntiles = (int)k;
  if (k > capacity) FAIL(DCELL_ERR_CAPACITY, "the plan needs %lld tiles, capacity %d", k, capacity);
  return DCELL_OK;
}

DCELL_API int dcell_batch_sl_step(const dcell_cell *cells, int ncells, const dcell_tile *tiles, int ntiles, int tx,
                                  int ty, int tz, int ctas_per_sm, const float *phi0, const float *vel, float *phi,
                                  int interp, int backtrace, int *flags, void *stream) {
  if (!cells || ncells < 0 || ntiles < 0 || (ntiles > 0 && !tiles)) FAIL(DCELL_ERR_ARG, "cells and tiles are required");
  if (!phi0 || !vel || !phi) FAIL(DCELL_ERR_ARG, "phi0, vel and phi must be device pointers");
  if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
  if (tx < 1 || ty < 1 || tz < 1) FAIL(DCELL_ERR_ARG, "tile extents must be positive");
  const int threads = tx * ty * tz;
  cudaStream_t st = (cudaStream_t)stream;
  if (interp == DCELL_CUBIC_TC) {
    if (threads != 128) FAIL(DCELL_ERR_ARG, "DCELL_CUBIC_TC tiles must hold 128 points (got %d)", threads);
    return launch_batch_tc(cells, tiles, ntiles, tx, ty, ctas_per_sm, phi0, vel, backtrace, phi, flags, st);
  }
  if (interp != DCELL_LINEAR && interp != DCELL_CUBIC_PLAIN && interp != DCELL_CUBIC_SEPARABLE)
    FAIL(DCELL_ERR_ARG, "unknown interpolation %d", interp);
  if (threads < 32 || threads > 1024) FAIL(DCELL_ERR_ARG, "tiles must hold 32..1024 points (got %d)", threads);
  return launch_batch_cuda_core(cells, tiles, ntiles, tx, ty, tz, ctas_per_sm, phi0, vel, interp, backtrace, phi,
                                flags, st);
}

DCELL_API int dcell_wait_timeout_check(int *result, void *stream) {
  if (!result) FAIL(DCELL_ERR_ARG, "result is required");
  return launch_wait_timeout_check(result, (cudaStream_t)stream);
}

DCELL_API int dcell_batch_sl_step_tc_split(const dcell_cell *cells, int ncells, const dcell_tile *bricks,
                                           int nbricks, const unsigned int *phi0_split, const float *vel,
                                           int backtrace, float *phi, unsigned int *phi_split, int *flags,
                                           void *stream) {
  if (ncells < 0 || nbricks < 0) FAIL(DCELL_ERR_ARG, "ncells and nbricks must be >= 0");
  if (nbricks > 0 && (!cells || !bricks || !phi0_split || !vel || !phi || !phi_split))
    FAIL(DCELL_ERR_ARG, "cells, bricks, phi0_split, vel, phi and phi_split are required");
  if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
  return launch_batch_brick(cells, bricks, nbricks, phi0_split, vel, backtrace, phi, phi_split, flags,
                            (cudaStream_t)stream);
}

DCELL_API size_t dcell_batch_tma_maps_bytes(int ncells) { return ncells > 0 ? (size_t)ncells * 256 : 0; }

DCELL_API int dcell_batch_tma_maps(const dcell_cell *cells, int ncells, const unsigned int *phi0_split,
                                   const float *vel, void *maps, void *stream) {
  if (ncells < 0) FAIL(DCELL_ERR_ARG, "ncells must be >= 0");
  if (ncells == 0) return DCELL_OK;
  if (!cells || !phi0_split || !vel || !maps) FAIL(DCELL_ERR_ARG, "cells, phi0_split, vel and maps are required");
  if (((uintptr_t)maps % 64) || ((uintptr_t)phi0_split % 16) || ((uintptr_t)vel % 16))
    FAIL(DCELL_ERR_ARG, "maps must be 64-byte aligned, phi0_split and vel 16-byte aligned");
  std::vector<unsigned char> host((size_t)ncells * 256);
  int rc = batch_tma_maps_host(cells, ncells, phi0_split, vel, host.data());
  if (rc) return rc;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(maps, host.data(), host.size(), cudaMemcpyHostToDevice, (cudaStream_t)stream));
  DCELL_CUDA_CHECK(cudaStreamSynchronize((cudaStream_t)stream));  // the staging vector goes out of scope
  return DCELL_OK;
}

DCELL_API int dcell_batch_sl_step_tc_split_tma(const dcell_cell *cells, int ncells, const dcell_tile *bricks,
                                               int nbricks, const void *maps, const unsigned int *phi0_split,
                                               const float *vel, int backtrace, float *phi, unsigned int *phi_split,
                                               int *flags, void *stream) {
  if (ncells < 0 || nbricks < 0) FAIL(DCELL_ERR_ARG, "ncells and nbricks must be >= 0");
  if (nbricks > 0 && (!cells || !bricks || !maps || !phi0_split || !vel || !phi || !phi_split))
    FAIL(DCELL_ERR_ARG, "cells, bricks, maps, phi0_split, vel, phi and phi_split are required");
  if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
  return launch_batch_brick_tma(cells, bricks, nbricks, maps, phi0_split, vel, backtrace, phi, phi_split, flags,
                                (cudaStream_t)stream);
}

DCELL_API int dcell_tc_gemm_check(const float *a, float *d, int *flags, void *stream) {
  if (!a || !d) FAIL(DCELL_ERR_ARG, "a and d are required");
  return launch_tc_gemm_check(a, d, flags, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Host-buffer session
struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  int ensure(size_t bytes) {
    if (bytes <= cap) return DCELL_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      FAIL(DCELL_ERR_NOMEM, "cudaMalloc of %zu bytes failed", bytes);
    }
    cap = bytes;
    return DCELL_OK;
  }
  // grow to `bytes`, keeping the first `keep` bytes (copied on `st`)
  int grow_keep(size_t bytes, size_t keep, cudaStream_t st) {
    if (bytes <= cap) return DCELL_OK;
    void *q = nullptr;
    if (cudaMalloc(&q, bytes) != cudaSuccess) {
      cudaGetLastError();
      FAIL(DCELL_ERR_NOMEM, "cudaMalloc of %zu bytes failed", bytes);
    }
    if (p && keep) DCELL_CUDA_CHECK(cudaMemcpyAsync(q, p, keep < cap ? keep : cap, cudaMemcpyDeviceToDevice, st));
    if (p) {
      cudaStreamSynchronize(st);
      cudaFree(p);
    }
    p = q;
    cap = bytes;
    return DCELL_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// A level set kept on the device across steps (dcell_ls_resident_*): phi
// (two buffers, stepped ping-pong) in the set precision, its packed split
// words for the FP32 tensor-core step, the band, the irregular nodes of the
// current phi, the velocity of the last step.
struct Resident {
  bool on = false;
  dcell_geom g{};
  int precision = DCELL_F64;
  int cur = 0;          // phi[cur] / split[cur] hold the level set
  bool split_ok = false;  // split[cur] is the split of phi[cur]
  int nband = 0, ncap = 0;
  DevBuf phi[2], split[2], vel, vel64, band, nodes, scratch, small;
  bool nodes_pending = false;   // the irregular nodes of phi[cur] are due (the node pass of the last step)
  bool reinit_pending = false;  // a step triggered the reinitialisation; it runs before the level set is next used
  double reinit_bw = 0.0;       // its band width
  int *reinit_hv = nullptr;     // pinned: its flags, -, band points
  cudaEvent_t reinit_ev = nullptr;
};

struct dcell_session {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t h2d = nullptr, d2h = nullptr;  // copy streams of the pipelined dense step
  std::vector<cudaEvent_t> ev_in, ev_out;
  DevBuf gates;
  DevBuf phi0_64, vel_64, phi_64, phi0_32, vel_32, phi_32, stage32, band, vals, nodes, scratch, small, parts, split;
  std::vector<double> host_vals;
  Resident res;
};

#define ENSURE(buf, bytes)             \
  do {                                 \
    int _r = (buf).ensure(bytes);      \
    if (_r) return _r;                 \
  } while (0)

static int session_flags_status(dcell_session *s, int flags) {
  if (flags & DCELL_FLAG_WAIT_TIMEOUT) FAIL(DCELL_ERR_TIMEOUT, "a device-side wait timed out");
  if (flags & DCELL_FLAG_CAPACITY) FAIL(DCELL_ERR_CAPACITY, "node capacity exceeded");
  if (flags & DCELL_FLAG_BAD_BAND) FAIL(DCELL_ERR_ARG, "a band entry lies outside the grid");
  if (flags & DCELL_FLAG_NONFINITE) FAIL(DCELL_ERR_NONFINITE, "a fast-marching update is not a number");
  if (flags & DCELL_FLAG_UNSETTLED)
    FAIL(DCELL_ERR_UNSUPPORTED, "fast marching left points tentative after its last bucket");
  if (flags & DCELL_FLAG_DEPARTURE_CLAMPED)
    FAIL(DCELL_ERR_DEPARTURE, "a departure point left the grid; its sample was clamped to the grid");
  if (flags & DCELL_FLAG_PARTICLE_OUTSIDE)
    FAIL(DCELL_ERR_DEPARTURE, "a particle's stencil or cell left the grid (clamped or skipped)");
  (void)s;
  return DCELL_OK;
}

static size_t band_index(const dcell_geom *g, const int *b) {
  const int nz = g->n[2] > 1 ? g->n[2] : 1;
  const int x = b[0] - g->p[0], y = b[1] - g->p[1], z = nz == 1 ? 0 : b[2] - g->p[2];
  return ((size_t)z * g->n[1] + (size_t)y) * g->n[0] + (size_t)x;
}

static int check_band_host(const dcell_geom *g, const int *band, int nband) {
  const int nz = g->n[2] > 1 ? g->n[2] : 1;
  for (int b = 0; b < nband; ++b) {
    const int *c = band + 3 * b;
    if (c[0] < g->p[0] || c[0] >= g->p[0] + g->n[0] || c[1] < g->p[1] || c[1] >= g->p[1] + g->n[1] ||
        (nz > 1 && (c[2] < g->p[2] || c[2] >= g->p[2] + nz)))
      FAIL(DCELL_ERR_ARG, "band entry %d (%d,%d,%d) lies outside the grid", b, c[0], c[1], c[2]);
  }
  return DCELL_OK;
}

extern "C" {

DCELL_API int dcell_session_create(int device, dcell_session **out) {
  if (!out) FAIL(DCELL_ERR_ARG, "out is NULL");
  *out = nullptr;
  DCELL_CUDA_CHECK(cudaSetDevice(device));
  dcell_session *s = new dcell_session();
  s->device = device;
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete s;
    FAIL(DCELL_ERR_CUDA, "cudaStreamCreate failed");
  }
  int rc = s->small.ensure(256);
  if (rc) {
    cudaStreamDestroy(s->stream);
    delete s;
    return rc;
  }
  *out = s;
  return DCELL_OK;
}

DCELL_API int dcell_session_destroy(dcell_session *s) {
  if (!s) return DCELL_OK;
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->stream);
  for (DevBuf *b : {&s->phi0_64, &s->vel_64, &s->phi_64, &s->phi0_32, &s->vel_32, &s->phi_32, &s->stage32, &s->band, &s->vals,
                    &s->nodes, &s->scratch, &s->small, &s->parts, &s->split, &s->gates})
    b->release();
  Resident &r = s->res;
  for (DevBuf *b : {&r.phi[0], &r.phi[1], &r.split[0], &r.split[1], &r.vel, &r.vel64, &r.band, &r.nodes, &r.scratch,
                    &r.small})
    b->release();
  if (r.reinit_hv) cudaFreeHost(r.reinit_hv);
  if (r.reinit_ev) cudaEventDestroy(r.reinit_ev);
  for (cudaEvent_t e : s->ev_in) cudaEventDestroy(e);
  for (cudaEvent_t e : s->ev_out) cudaEventDestroy(e);
  if (s->h2d) cudaStreamDestroy(s->h2d);
  if (s->d2h) cudaStreamDestroy(s->d2h);
  cudaStreamDestroy(s->stream);
  delete s;
  return DCELL_OK;
}

// The dense FP32 tensor-core step on host arrays, pipelined over z-slabs:
// the inputs go up in plane chunks on one copy stream (converted to FP32 and
// split on arrival), slab k is stepped once the planes up to its top + kHalo
// are on the device, and its result comes down on a second copy stream while
// later chunks still go up.  A slab launch runs only if max |w| dt / h_z over
// the planes present is at most kHalo - 3 (every departure stencil then lies
// in them); otherwise it leaves its slab, and once all inputs are present
// the whole grid is stepped again and copied down (identical results either
// way: the same kernel on the same inputs).
// Slabs and halo of the z-slab pipelines: a slab's step starts once the
// planes up to its top + kPipeHalo are on the device, and runs only if max
// |w| dt / h_z over those planes is at most kPipeHalo - 3.
constexpr int kPipeHalo = 6, kPipeSlabs = 8;

// the session's two copy streams and kPipeSlabs events per direction
static int ensure_copy_streams(dcell_session *s) {
  if (!s->h2d) {
    DCELL_CUDA_CHECK(cudaStreamCreateWithFlags(&s->h2d, cudaStreamNonBlocking));
    DCELL_CUDA_CHECK(cudaStreamCreateWithFlags(&s->d2h, cudaStreamNonBlocking));
  }
  while ((int)s->ev_in.size() < kPipeSlabs) {
    cudaEvent_t a, b;
    DCELL_CUDA_CHECK(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    DCELL_CUDA_CHECK(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
    s->ev_in.push_back(a);
    s->ev_out.push_back(b);
  }
  return DCELL_OK;
}

static int ls_advect_tc_pipelined(dcell_session *s, const dcell_geom *g, const double *phi0, const double *vel,
                                  double dt, int backtrace, double *phi) {
  constexpr int kHalo = kPipeHalo, kSlabs = kPipeSlabs;
  const dcell::Geom G = dcell::to_geom(g);
  const long long plane = (long long)G.nx * G.ny, n = plane * G.nz;
  cudaStream_t st = s->stream;
  int rc;
  if ((rc = ensure_copy_streams(s))) return rc;
  ENSURE(s->phi0_64, n * sizeof(double));
  ENSURE(s->vel_64, n * 3 * sizeof(double));
  ENSURE(s->phi_64, n * sizeof(double));
  ENSURE(s->vel_32, n * 3 * sizeof(float));
  ENSURE(s->phi0_32, n * sizeof(float));
  ENSURE(s->phi_32, n * sizeof(float));
  ENSURE(s->split, n * sizeof(uint32_t));
  ENSURE(s->gates, kSlabs * sizeof(int));
  int *dflags = (int *)s->small.p, *gates = (int *)s->gates.p;
  double *p64 = (double *)s->phi0_64.p, *v64 = (double *)s->vel_64.p, *o64 = (double *)s->phi_64.p;
  float *p32 = (float *)s->phi0_32.p, *v32 = (float *)s->vel_32.p, *o32 = (float *)s->phi_32.p;
  uint32_t *w = (uint32_t *)s->split.p;
  // every stream starts after the work this session queued before
  cudaEvent_t start = s->ev_out[kSlabs - 1];
  DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, sizeof(int), st));
  DCELL_CUDA_CHECK(cudaMemsetAsync(gates, 0, kSlabs * sizeof(int), st));
  DCELL_CUDA_CHECK(cudaEventRecord(start, st));
  DCELL_CUDA_CHECK(cudaStreamWaitEvent(s->h2d, start, 0));
  const int BZ = tc_slab_planes();
  const int nbz = (G.nz + BZ - 1) / BZ, per = (nbz + kSlabs - 1) / kSlabs;
  int have = 0, gated = 0, nslab = 0;  // planes present on the device, planes in the gate's max
  for (int k = 0; k < kSlabs; ++k) {
    const int b0 = k * per, b1 = b0 + per < nbz ? b0 + per : nbz;
    if (b0 >= b1) break;
    const int z0 = b0 * BZ, z1 = b1 * BZ < G.nz ? b1 * BZ : G.nz;
    const int need = z1 + kHalo < G.nz ? z1 + kHalo : G.nz;
    if (need > have) {  // the next chunk of planes: up, to FP32, split
      const long long o = have * plane, m = (need - have) * plane;
      DCELL_CUDA_CHECK(cudaMemcpyAsync(p64 + o, phi0 + o, m * sizeof(double), cudaMemcpyHostToDevice, s->h2d));
      DCELL_CUDA_CHECK(
          cudaMemcpyAsync(v64 + 3 * o, vel + 3 * o, 3 * m * sizeof(double), cudaMemcpyHostToDevice, s->h2d));
      if ((rc = launch_convert(p64 + o, DCELL_F64, p32 + o, DCELL_F32, m, s->h2d))) return rc;
      if ((rc = launch_convert(v64 + 3 * o, DCELL_F64, v32 + 3 * o, DCELL_F32, 3 * m, s->h2d))) return rc;
      if ((rc = launch_split_bf16(p32 + o, w + o, m, s->h2d))) return rc;
      have = need;
    }
    DCELL_CUDA_CHECK(cudaEventRecord(s->ev_in[k], s->h2d));
    DCELL_CUDA_CHECK(cudaStreamWaitEvent(st, s->ev_in[k], 0));
    // the gate: max |w| over every plane present bounds the departures of
    // this slab (a running max: each chunk's planes once)
    if (have > gated) {
      if ((rc = launch_max_abs_component(v32 + 3 * gated * plane, (have - gated) * plane, 3, 2, gates, st)))
        return rc;
      gated = have;
    }
    TcSlab slab;
    slab.bz0 = b0;
    slab.nbz = b1 - b0;
    slab.gate_maxw = gates;
    slab.gate_limit = (float)(kHalo - 3);
    if ((rc = launch_sl_tc_slab(G, w, v32, dt, backtrace, o32, nullptr, dflags, st, slab))) return rc;
    const long long oz = z0 * plane, mz = (z1 - z0) * plane;
    if ((rc = launch_convert(o32 + oz, DCELL_F32, o64 + oz, DCELL_F64, mz, st))) return rc;
    DCELL_CUDA_CHECK(cudaEventRecord(s->ev_out[k], st));
    DCELL_CUDA_CHECK(cudaStreamWaitEvent(s->d2h, s->ev_out[k], 0));
    DCELL_CUDA_CHECK(cudaMemcpyAsync(phi + oz, o64 + oz, mz * sizeof(double), cudaMemcpyDeviceToHost, s->d2h));
    ++nslab;
  }
  DCELL_CUDA_CHECK(cudaStreamSynchronize(s->h2d));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(s->d2h));
  int hf = 0;
  DCELL_CUDA_CHECK(cudaMemcpy(&hf, dflags, sizeof(int), cudaMemcpyDeviceToHost));
  if (hf & dcell::FLAG_PIPELINE_REDO) {  // a slab was left: step the whole grid with every plane present
    DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, sizeof(int), st));
    if ((rc = launch_sl_tc_split(G, w, v32, dt, nullptr, n, backtrace, o32, nullptr, dflags, st))) return rc;
    if ((rc = launch_convert(o32, DCELL_F32, o64, DCELL_F64, n, st))) return rc;
    DCELL_CUDA_CHECK(cudaMemcpyAsync(phi, o64, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    DCELL_CUDA_CHECK(cudaMemcpyAsync(&hf, dflags, sizeof(int), cudaMemcpyDeviceToHost, st));
    DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  }
  (void)nslab;
  return session_flags_status(s, hf & ~dcell::FLAG_PIPELINE_REDO);
}

DCELL_API int dcell_ls_advect_sl(dcell_session *s, const dcell_geom *g, const double *phi0, const double *vel,
                                 const int *band, int nband, double dt, int interp, int backtrace, int precision,
                                 double *phi) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_geom(g);
  if (rc) return rc;
  if (!phi0 || !vel || !phi) FAIL(DCELL_ERR_ARG, "phi0, vel and phi are required");
  if (precision != DCELL_F32 && precision != DCELL_F64) FAIL(DCELL_ERR_ARG, "precision must be F32 or F64");
  if (band && nband < 0) FAIL(DCELL_ERR_ARG, "nband must be >= 0");
  if (band) {
    rc = check_band_host(g, band, nband);
    if (rc) return rc;
  }
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  if (precision == DCELL_F32 && interp == DCELL_CUBIC_TC && !band && g->n[2] > 1) {
    if (!(dt == dt)) FAIL(DCELL_ERR_NONFINITE, "dt is NaN");
    if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
    const dcell::Geom G = dcell::to_geom(g);
    if (G.nz >= 4 * tc_slab_planes() && tc_brick_applicable(G, (const void *)256, (const void *)256))
      return ls_advect_tc_pipelined(s, g, phi0, vel, dt, backtrace, phi);
  }
  const long long n = grid_points(g);
  const int dof = g->n[2] > 1 ? 3 : 2;
  const long long npts = band ? nband : n;
  cudaStream_t st = s->stream;
  ENSURE(s->phi0_64, n * sizeof(double));
  ENSURE(s->vel_64, n * dof * sizeof(double));
  int *dflags = (int *)s->small.p;
  DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, sizeof(int), st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi0_64.p, phi0, n * sizeof(double), cudaMemcpyHostToDevice, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->vel_64.p, vel, n * dof * sizeof(double), cudaMemcpyHostToDevice, st));
  const int *dband = nullptr;
  if (band && nband > 0) {
    ENSURE(s->band, (size_t)nband * 3 * sizeof(int));
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->band.p, band, (size_t)nband * 3 * sizeof(int), cudaMemcpyHostToDevice, st));
    dband = (const int *)s->band.p;
  }
  const void *dphi0 = s->phi0_64.p, *dvel = s->vel_64.p;
  void *dphi;
  int dtype = precision;
  if (precision == DCELL_F32) {
    ENSURE(s->phi0_32, n * sizeof(float));
    ENSURE(s->vel_32, n * dof * sizeof(float));
    ENSURE(s->phi_32, n * sizeof(float));
    if ((rc = launch_convert(s->phi0_64.p, DCELL_F64, s->phi0_32.p, DCELL_F32, n, st))) return rc;
    if ((rc = launch_convert(s->vel_64.p, DCELL_F64, s->vel_32.p, DCELL_F32, n * dof, st))) return rc;
    dphi0 = s->phi0_32.p;
    dvel = s->vel_32.p;
    dphi = s->phi_32.p;
  } else {
    ENSURE(s->phi_64, n * sizeof(double));
    dphi = s->phi_64.p;
  }
  if (npts > 0) {
    const dcell::Geom G = dcell::to_geom(g);
    if (precision == DCELL_F32 && interp == DCELL_CUBIC_TC && !band && G.nz > 1) {
      // dense tensor-core step: split phi0 into packed BF16 words and run the
      // split-state stepper (TMA bricks where the grid allows)
      if (!(dt == dt)) FAIL(DCELL_ERR_NONFINITE, "dt is NaN");
      ENSURE(s->split, n * sizeof(uint32_t));
      if ((rc = launch_split_bf16((const float *)dphi0, (uint32_t *)s->split.p, n, st))) return rc;
      rc = launch_sl_tc_split(G, (const uint32_t *)s->split.p, (const float *)dvel, dt, nullptr, n, backtrace,
                              (float *)dphi, nullptr, dflags, st);
    } else {
      rc = dcell_sl_step(g, dtype, dphi0, dvel, dt, dband, band ? nband : 0, interp, backtrace, dphi, dflags, st);
    }
    if (rc) return rc;
  }
  // results back: band values (gathered) or the whole grid
  if (band) {
    if (nband > 0) {
      ENSURE(s->vals, (size_t)nband * sizeof(double));
      if (precision == DCELL_F32) {
        // gather the FP32 band values, then widen them into vals
        ENSURE(s->stage32, (size_t)nband * sizeof(float));
        float *stage = (float *)s->stage32.p;
        if ((rc = launch_gather_band(dcell::to_geom(g), DCELL_F32, s->phi_32.p, dband, nband, stage, st))) return rc;
        if ((rc = launch_convert(stage, DCELL_F32, s->vals.p, DCELL_F64, nband, st))) return rc;
      } else {
        if ((rc = launch_gather_band(dcell::to_geom(g), DCELL_F64, s->phi_64.p, dband, nband, s->vals.p, st)))
          return rc;
      }
      s->host_vals.resize((size_t)nband);
      DCELL_CUDA_CHECK(cudaMemcpyAsync(s->host_vals.data(), s->vals.p, (size_t)nband * sizeof(double),
                                       cudaMemcpyDeviceToHost, st));
    }
  } else {
    if (precision == DCELL_F32) {
      if ((rc = launch_convert(s->phi_32.p, DCELL_F32, s->phi0_64.p, DCELL_F64, n, st))) return rc;
      DCELL_CUDA_CHECK(cudaMemcpyAsync(phi, s->phi0_64.p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    } else {
      DCELL_CUDA_CHECK(cudaMemcpyAsync(phi, s->phi_64.p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
  }
  int hflags = 0;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(&hflags, dflags, sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  if (band)
    for (int b = 0; b < nband; ++b) phi[band_index(g, band + 3 * b)] = s->host_vals[(size_t)b];
  return session_flags_status(s, hflags);
}

// One substep of LevelSetAdvectSLRK2HalfStep / FullStep (AdvectRK2.c:5-26):
// (half: phi0 <- phi, GridCopy), phi <- SL(phi0) at the band points (or
// everywhere), then the irregular-node list of the new phi -- the same device
// paths as dcell_ls_advect_sl followed by dcell_ls_update_irregular_nodes, with
// phi staying on the device between them.
static int ls_rk2(dcell_session *s, const dcell_geom *g, int half, double *phi0, const double *vel,
                  const int *band, int nband, double dt, int interp, int backtrace, int precision, double *phi,
                  int with_surface, dcell_irregular_node *nodes, int capacity, int *count) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_geom(g);
  if (rc) return rc;
  if (!phi0 || !vel || !phi || !count) FAIL(DCELL_ERR_ARG, "phi0, vel, phi and count are required");
  if (precision != DCELL_F32 && precision != DCELL_F64) FAIL(DCELL_ERR_ARG, "precision must be F32 or F64");
  if (nband < 0 || (nband > 0 && !band)) FAIL(DCELL_ERR_ARG, "invalid band");
  if (capacity < 0 || (capacity > 0 && !nodes)) FAIL(DCELL_ERR_ARG, "invalid node buffer");
  if (interp < DCELL_LINEAR || interp > DCELL_CUBIC_TC) FAIL(DCELL_ERR_ARG, "unknown interpolation %d", interp);
  if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
  if (!(dt == dt)) FAIL(DCELL_ERR_NONFINITE, "dt is NaN");
  if ((rc = check_band_host(g, band, nband))) return rc;
  const long long n = grid_points(g);
  const int dof = g->n[2] > 1 ? 3 : 2;
  const bool dense = band == nullptr;
  if (half) memcpy(phi0, phi, (size_t)n * sizeof(double));  // GridCopy(ls->phi, ls->phi0)
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  ENSURE(s->phi0_64, n * sizeof(double));
  ENSURE(s->vel_64, n * dof * sizeof(double));
  ENSURE(s->phi_64, n * sizeof(double));
  int *dflags = (int *)s->small.p, *dcount = dflags + 1;
  DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, 2 * sizeof(int), st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi0_64.p, phi0, n * sizeof(double), cudaMemcpyHostToDevice, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->vel_64.p, vel, n * dof * sizeof(double), cudaMemcpyHostToDevice, st));
  // phi before the step: the points off the band keep it
  if (!dense) {
    if (half)
      DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi_64.p, s->phi0_64.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    else
      DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi_64.p, phi, n * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  const int *dband = nullptr;
  if (nband > 0) {
    ENSURE(s->band, (size_t)nband * 3 * sizeof(int));
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->band.p, band, (size_t)nband * 3 * sizeof(int), cudaMemcpyHostToDevice, st));
    dband = (const int *)s->band.p;
  }
  const void *dphi0 = s->phi0_64.p, *dvel = s->vel_64.p;
  void *dphi = s->phi_64.p;
  if (precision == DCELL_F32) {
    ENSURE(s->phi0_32, n * sizeof(float));
    ENSURE(s->vel_32, n * dof * sizeof(float));
    ENSURE(s->phi_32, n * sizeof(float));
    if ((rc = launch_convert(s->phi0_64.p, DCELL_F64, s->phi0_32.p, DCELL_F32, n, st))) return rc;
    if ((rc = launch_convert(s->vel_64.p, DCELL_F64, s->vel_32.p, DCELL_F32, n * dof, st))) return rc;
    if (!dense && (rc = launch_convert(s->phi_64.p, DCELL_F64, s->phi_32.p, DCELL_F32, n, st))) return rc;
    dphi0 = s->phi0_32.p;
    dvel = s->vel_32.p;
    dphi = s->phi_32.p;
  }
  const dcell::Geom G = dcell::to_geom(g);
  if (!dense && nband == 0) {
    // nothing to advect
  } else if (precision == DCELL_F32 && interp == DCELL_CUBIC_TC && dense && G.nz > 1) {
    ENSURE(s->split, n * sizeof(uint32_t));  // split-state step, as dcell_ls_advect_sl
    if ((rc = launch_split_bf16((const float *)dphi0, (uint32_t *)s->split.p, n, st))) return rc;
    if ((rc = launch_sl_tc_split(G, (const uint32_t *)s->split.p, (const float *)dvel, dt, nullptr, n, backtrace,
                                 (float *)dphi, nullptr, dflags, st)))
      return rc;
  } else if ((rc = dcell_sl_step(g, precision, dphi0, dvel, dt, dband, nband, interp, backtrace, dphi, dflags, st))) {
    return rc;
  }
  // the node list of the new phi, on the device copy
  const size_t sb = irregular_scratch_bytes(nband);
  ENSURE(s->scratch, sb);
  ENSURE(s->nodes, (size_t)(capacity > 0 ? capacity : 1) * sizeof(dcell_irregular_node));
  rc = dcell_irregular_nodes(g, precision, dphi, dband, nband, with_surface, (dcell_irregular_node *)s->nodes.p,
                             capacity, dcount, s->scratch.p, sb, dflags, st);
  if (rc) return rc;
  // phi back: the band values (gathered, widened) or the whole grid
  if (!dense) {
    if (nband > 0) {
      ENSURE(s->vals, (size_t)nband * sizeof(double));
      if (precision == DCELL_F32) {
        ENSURE(s->stage32, (size_t)nband * sizeof(float));
        if ((rc = launch_gather_band(G, DCELL_F32, dphi, dband, nband, s->stage32.p, st))) return rc;
        if ((rc = launch_convert(s->stage32.p, DCELL_F32, s->vals.p, DCELL_F64, nband, st))) return rc;
      } else if ((rc = launch_gather_band(G, DCELL_F64, dphi, dband, nband, s->vals.p, st))) {
        return rc;
      }
      s->host_vals.resize((size_t)nband);
      DCELL_CUDA_CHECK(cudaMemcpyAsync(s->host_vals.data(), s->vals.p, (size_t)nband * sizeof(double),
                                       cudaMemcpyDeviceToHost, st));
    }
  } else {
    if (precision == DCELL_F32) {
      if ((rc = launch_convert(dphi, DCELL_F32, s->phi0_64.p, DCELL_F64, n, st))) return rc;
      DCELL_CUDA_CHECK(cudaMemcpyAsync(phi, s->phi0_64.p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    } else {
      DCELL_CUDA_CHECK(cudaMemcpyAsync(phi, dphi, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
  }
  int hv[2] = {0, 0};
  DCELL_CUDA_CHECK(cudaMemcpyAsync(hv, dflags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  if (!dense)
    for (int b = 0; b < nband; ++b) phi[band_index(g, band + 3 * b)] = s->host_vals[(size_t)b];
  *count = hv[1];
  const int ncopy = hv[1] < capacity ? hv[1] : capacity;
  if (ncopy > 0)
    DCELL_CUDA_CHECK(cudaMemcpy(nodes, s->nodes.p, (size_t)ncopy * sizeof(dcell_irregular_node), cudaMemcpyDeviceToHost));
  return session_flags_status(s, hv[0]);
}

DCELL_API int dcell_ls_advect_sl_rk2_half(dcell_session *s, const dcell_geom *g, double *phi0, const double *vel,
                                          const int *band, int nband, double dt, int interp, int backtrace,
                                          int precision, double *phi, int with_surface, dcell_irregular_node *nodes,
                                          int capacity, int *count) {
  return ls_rk2(s, g, 1, phi0, vel, band, nband, dt, interp, backtrace, precision, phi, with_surface, nodes,
                capacity, count);
}

DCELL_API int dcell_ls_advect_sl_rk2_full(dcell_session *s, const dcell_geom *g, const double *phi0,
                                          const double *vel, const int *band, int nband, double dt, int interp,
                                          int backtrace, int precision, double *phi, int with_surface,
                                          dcell_irregular_node *nodes, int capacity, int *count) {
  return ls_rk2(s, g, 0, const_cast<double *>(phi0), vel, band, nband, dt, interp, backtrace, precision, phi,
                with_surface, nodes, capacity, count);
}

DCELL_API int dcell_ls_update_irregular_nodes(dcell_session *s, const dcell_geom *g, const double *phi,
                                              const int *band, int nband, int with_surface, int precision,
                                              dcell_irregular_node *nodes, int capacity, int *count) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_geom(g);
  if (rc) return rc;
  if (!phi || !count || nband < 0 || (nband > 0 && !band)) FAIL(DCELL_ERR_ARG, "phi, band and count are required");
  if (capacity < 0 || (capacity > 0 && !nodes)) FAIL(DCELL_ERR_ARG, "invalid node buffer");
  if (precision != DCELL_F32 && precision != DCELL_F64) FAIL(DCELL_ERR_ARG, "precision must be F32 or F64");
  if ((rc = check_band_host(g, band, nband))) return rc;
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long n = grid_points(g);
  ENSURE(s->phi_64, n * sizeof(double));
  int *dflags = (int *)s->small.p;
  int *dcount = dflags + 1;
  DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, 2 * sizeof(int), st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi_64.p, phi, n * sizeof(double), cudaMemcpyHostToDevice, st));
  const void *dphi = s->phi_64.p;
  if (precision == DCELL_F32) {
    ENSURE(s->phi_32, n * sizeof(float));
    if ((rc = launch_convert(s->phi_64.p, DCELL_F64, s->phi_32.p, DCELL_F32, n, st))) return rc;
    dphi = s->phi_32.p;
  }
  if (nband > 0) {
    ENSURE(s->band, (size_t)nband * 3 * sizeof(int));
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->band.p, band, (size_t)nband * 3 * sizeof(int), cudaMemcpyHostToDevice, st));
  }
  const size_t sb = irregular_scratch_bytes(nband);
  ENSURE(s->scratch, sb);
  ENSURE(s->nodes, (size_t)(capacity > 0 ? capacity : 1) * sizeof(dcell_irregular_node));
  rc = dcell_irregular_nodes(g, precision, dphi, (const int *)s->band.p, nband, with_surface,
                             (dcell_irregular_node *)s->nodes.p, capacity, dcount, s->scratch.p, sb, dflags, st);
  if (rc) return rc;
  int hv[2] = {0, 0};
  DCELL_CUDA_CHECK(cudaMemcpyAsync(hv, dflags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  *count = hv[1];
  const int ncopy = hv[1] < capacity ? hv[1] : capacity;
  if (ncopy > 0)
    DCELL_CUDA_CHECK(cudaMemcpy(nodes, s->nodes.p, (size_t)ncopy * sizeof(dcell_irregular_node), cudaMemcpyDeviceToHost));
  return session_flags_status(s, hv[0]);
}

DCELL_API int dcell_ls_reinitialize(dcell_session *s, const dcell_geom *g, double *phi,
                                    const dcell_irregular_node *nodes, int nnodes, double band_width, int precision,
                                    int *band, int capacity, int *count) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_geom(g);
  if (rc) return rc;
  if (!phi || !count || nnodes < 0 || (nnodes > 0 && !nodes)) FAIL(DCELL_ERR_ARG, "phi, nodes and count are required");
  if (capacity < 0 || (capacity > 0 && !band)) FAIL(DCELL_ERR_ARG, "invalid band buffer");
  if (precision != DCELL_F32 && precision != DCELL_F64) FAIL(DCELL_ERR_ARG, "precision must be F32 or F64");
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long n = grid_points(g);
  ENSURE(s->phi_64, n * sizeof(double));
  int *dflags = (int *)s->small.p;
  int *dcount = dflags + 1;
  DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, 2 * sizeof(int), st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi_64.p, phi, n * sizeof(double), cudaMemcpyHostToDevice, st));
  void *dphi = s->phi_64.p;
  if (precision == DCELL_F32) {
    ENSURE(s->phi_32, n * sizeof(float));
    if ((rc = launch_convert(s->phi_64.p, DCELL_F64, s->phi_32.p, DCELL_F32, n, st))) return rc;
    dphi = s->phi_32.p;
  }
  ENSURE(s->nodes, (size_t)(nnodes > 0 ? nnodes : 1) * sizeof(dcell_irregular_node));
  if (nnodes > 0)
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->nodes.p, nodes, (size_t)nnodes * sizeof(dcell_irregular_node),
                                     cudaMemcpyHostToDevice, st));
  const size_t sb = dcell_reinit_scratch_bytes(g, precision);
  ENSURE(s->scratch, sb);
  ENSURE(s->band, (size_t)(capacity > 0 ? capacity : 1) * 3 * sizeof(int));
  rc = dcell_reinitialize(g, precision, dphi, (const dcell_irregular_node *)s->nodes.p, nnodes, band_width, 0.0,
                          (int *)s->band.p, capacity, dcount, s->scratch.p, sb, dflags, st);
  if (rc) return rc;
  if (precision == DCELL_F32 && (rc = launch_convert(s->phi_32.p, DCELL_F32, s->phi_64.p, DCELL_F64, n, st)))
    return rc;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(phi, s->phi_64.p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  int hv[2] = {0, 0};
  DCELL_CUDA_CHECK(cudaMemcpyAsync(hv, dflags, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  *count = hv[1];
  const int ncopy = hv[1] < capacity ? hv[1] : capacity;
  if (ncopy > 0)
    DCELL_CUDA_CHECK(cudaMemcpy(band, s->band.p, (size_t)ncopy * 3 * sizeof(int), cudaMemcpyDeviceToHost));
  return session_flags_status(s, hv[0]);
}

DCELL_API int dcell_ls_max_velocity(dcell_session *s, const dcell_geom *g, const double *vel,
                                    const dcell_irregular_node *nodes, int count, double *maxvel) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_geom(g);
  if (rc) return rc;
  if (!vel || !maxvel || count < 0 || (count > 0 && !nodes)) FAIL(DCELL_ERR_ARG, "vel, nodes and maxvel are required");
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long n = grid_points(g);
  const int dof = g->n[2] > 1 ? 3 : 2;
  ENSURE(s->vel_64, n * dof * sizeof(double));
  ENSURE(s->nodes, (size_t)(count > 0 ? count : 1) * sizeof(dcell_irregular_node));
  int *dcount = (int *)s->small.p + 1;
  double *dmax = (double *)((char *)s->small.p + 64);
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->vel_64.p, vel, n * dof * sizeof(double), cudaMemcpyHostToDevice, st));
  if (count > 0)
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->nodes.p, nodes, (size_t)count * sizeof(dcell_irregular_node),
                                     cudaMemcpyHostToDevice, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(dcount, &count, sizeof(int), cudaMemcpyHostToDevice, st));
  rc = dcell_max_velocity(g, DCELL_F64, s->vel_64.p, (const dcell_irregular_node *)s->nodes.p, dcount, count, dmax, st);
  if (rc) return rc;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(maxvel, dmax, sizeof(double), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  return DCELL_OK;
}

DCELL_API int dcell_ls_advect_mac(dcell_session *s, const dcell_geom *g, const double *phi, const double *u,
                                  const double *v, const double *w, double dt, int precision, double *out) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_geom(g);
  if (rc) return rc;
  const bool is3 = g->n[2] > 1;
  if (!phi || !u || !v || !out || (is3 && !w)) FAIL(DCELL_ERR_ARG, "phi, u, v, (3D: w) and out are required");
  if (precision != DCELL_F32 && precision != DCELL_F64) FAIL(DCELL_ERR_ARG, "precision must be DCELL_F32 or DCELL_F64");
  int range[6];
  rc = mac_ranges(g, range);
  if (rc) return rc;
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long n = grid_points(g);
  const size_t b64 = (size_t)n * sizeof(double);
  const int ncomp = is3 ? 3 : 2;
  ENSURE(s->phi_64, b64);
  ENSURE(s->phi0_64, b64);
  ENSURE(s->vel_64, b64 * ncomp);
  double *dphi = (double *)s->phi_64.p, *dout = (double *)s->phi0_64.p, *dvel = (double *)s->vel_64.p;
  const double *comp[3] = {u, v, w};
  DCELL_CUDA_CHECK(cudaMemcpyAsync(dphi, phi, b64, cudaMemcpyHostToDevice, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(dout, out, b64, cudaMemcpyHostToDevice, st));
  for (int c = 0; c < ncomp; ++c)
    DCELL_CUDA_CHECK(cudaMemcpyAsync(dvel + c * n, comp[c], b64, cudaMemcpyHostToDevice, st));
  if (precision == DCELL_F64) {
    rc = dcell_advect_mac(g, DCELL_F64, dphi, dvel, dvel + n, is3 ? dvel + 2 * n : nullptr, dt, dout, st);
    if (rc) return rc;
  } else {  // FP32 arithmetic on converted copies
    const size_t b32 = (size_t)n * sizeof(float);
    ENSURE(s->phi_32, b32);
    ENSURE(s->phi0_32, b32);
    ENSURE(s->vel_32, b32 * ncomp);
    float *fphi = (float *)s->phi_32.p, *fout = (float *)s->phi0_32.p, *fvel = (float *)s->vel_32.p;
    if ((rc = launch_convert(dphi, DCELL_F64, fphi, DCELL_F32, n, st)) ||
        (rc = launch_convert(dout, DCELL_F64, fout, DCELL_F32, n, st)) ||
        (rc = launch_convert(dvel, DCELL_F64, fvel, DCELL_F32, n * ncomp, st)))
      return rc;
    rc = dcell_advect_mac(g, DCELL_F32, fphi, fvel, fvel + n, is3 ? fvel + 2 * n : nullptr, dt, fout, st);
    if (rc) return rc;
    if ((rc = launch_convert(fout, DCELL_F32, dout, DCELL_F64, n, st))) return rc;
  }
  DCELL_CUDA_CHECK(cudaMemcpyAsync(out, dout, b64, cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  return DCELL_OK;
}

// Particle level set on host arrays: particles and phi are copied in and
// out around the device entry points on the session's stream.
DCELL_API int dcell_ls_pls_advect(dcell_session *s, const dcell_geom *g, const double *vel, double *particles,
                                  long long n, double dt) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_pls_common(g, DCELL_F64, n, particles);
  if (rc) return rc;
  if (!vel) FAIL(DCELL_ERR_ARG, "vel is required");
  if (n == 0) return DCELL_OK;
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long np = grid_points(g);
  const int dof = g->n[2] > 1 ? 3 : 2;
  ENSURE(s->vel_64, np * dof * sizeof(double));
  ENSURE(s->parts, (size_t)n * 4 * sizeof(double));
  int *dflags = (int *)s->small.p;
  DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, sizeof(int), st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->vel_64.p, vel, np * dof * sizeof(double), cudaMemcpyHostToDevice, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->parts.p, particles, n * 4 * sizeof(double), cudaMemcpyHostToDevice, st));
  if ((rc = dcell_pls_advect(g, DCELL_F64, s->vel_64.p, s->parts.p, n, dt, dflags, st))) return rc;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(particles, s->parts.p, n * 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  int hf = 0;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(&hf, dflags, sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  return session_flags_status(s, hf);
}

DCELL_API int dcell_ls_pls_correct(dcell_session *s, const dcell_geom *g, double *phi, const int *band, int nband,
                                   const double *particles, long long n) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_pls_common(g, DCELL_F64, n, particles);
  if (rc) return rc;
  if (!phi || nband < 0 || (nband > 0 && !band)) FAIL(DCELL_ERR_ARG, "phi and band are required");
  if ((rc = check_band_host(g, band, nband))) return rc;
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long np = grid_points(g);
  ENSURE(s->phi_64, np * sizeof(double));
  ENSURE(s->parts, (size_t)(n > 0 ? n : 1) * 4 * sizeof(double));
  ENSURE(s->band, (size_t)(nband > 0 ? nband : 1) * 3 * sizeof(int));
  const size_t sb = pls_correct_scratch_bytes(np, DCELL_F64);
  ENSURE(s->scratch, sb);
  int *dflags = (int *)s->small.p;
  DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, sizeof(int), st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi_64.p, phi, np * sizeof(double), cudaMemcpyHostToDevice, st));
  if (n > 0)
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->parts.p, particles, n * 4 * sizeof(double), cudaMemcpyHostToDevice, st));
  if (nband > 0)
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->band.p, band, (size_t)nband * 3 * sizeof(int), cudaMemcpyHostToDevice, st));
  if ((rc = dcell_pls_correct(g, DCELL_F64, s->phi_64.p, (const int *)s->band.p, nband, s->parts.p, n, s->scratch.p,
                              sb, dflags, st)))
    return rc;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(phi, s->phi_64.p, np * sizeof(double), cudaMemcpyDeviceToHost, st));
  int hf = 0;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(&hf, dflags, sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  return session_flags_status(s, hf);
}

DCELL_API int dcell_ls_pls_adjust_radii(dcell_session *s, const dcell_geom *g, const double *phi, double *particles,
                                        long long n, const dcell_pls_params *prm) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_pls_common(g, DCELL_F64, n, particles);
  if (rc) return rc;
  if ((rc = check_pls_params(prm))) return rc;
  if (!phi) FAIL(DCELL_ERR_ARG, "phi is required");
  if (n == 0) return DCELL_OK;
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long np = grid_points(g);
  ENSURE(s->phi_64, np * sizeof(double));
  ENSURE(s->parts, (size_t)n * 4 * sizeof(double));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi_64.p, phi, np * sizeof(double), cudaMemcpyHostToDevice, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->parts.p, particles, n * 4 * sizeof(double), cudaMemcpyHostToDevice, st));
  if ((rc = dcell_pls_adjust_radii(g, DCELL_F64, s->phi_64.p, s->parts.p, n, prm, nullptr, st))) return rc;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(particles, s->parts.p, n * 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  return DCELL_OK;
}

// Seed (n < 0) or reseed n particles on host arrays.
static int ls_pls_seed_common(dcell_session *s, const dcell_geom *g, const double *phi, const int *band, int nband,
                              const dcell_pls_params *prm, unsigned long long *rng, double *particles, long long n,
                              long long capacity, long long *count) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  if (!rng || !count) FAIL(DCELL_ERR_ARG, "rng and count are required");
  int rc = check_pls_common(g, DCELL_F64, n > 0 ? n : 0, particles);
  if (rc) return rc;
  if ((rc = check_pls_params(prm))) return rc;
  if (!phi || nband < 0 || (nband > 0 && !band)) FAIL(DCELL_ERR_ARG, "phi and band are required");
  if (capacity < (n > 0 ? n : 0) || (capacity > 0 && !particles)) FAIL(DCELL_ERR_ARG, "invalid particle buffer");
  if ((rc = check_band_host(g, band, nband))) return rc;
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long np = grid_points(g);
  const long long nn = n > 0 ? n : 0;
  ENSURE(s->phi_64, np * sizeof(double));
  ENSURE(s->parts, (size_t)(capacity > 0 ? capacity : 1) * 4 * sizeof(double));
  ENSURE(s->band, (size_t)(nband > 0 ? nband : 1) * 3 * sizeof(int));
  const size_t sb = pls_scratch_bytes(np, nband, nn);
  ENSURE(s->scratch, sb);
  int *dflags = (int *)s->small.p;
  unsigned long long *drng = (unsigned long long *)((char *)s->small.p + 128);
  long long *dcount = (long long *)((char *)s->small.p + 136);
  DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, sizeof(int), st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(drng, rng, sizeof(unsigned long long), cudaMemcpyHostToDevice, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi_64.p, phi, np * sizeof(double), cudaMemcpyHostToDevice, st));
  if (nn > 0)
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->parts.p, particles, nn * 4 * sizeof(double), cudaMemcpyHostToDevice, st));
  if (nband > 0)
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->band.p, band, (size_t)nband * 3 * sizeof(int), cudaMemcpyHostToDevice, st));
  rc = n < 0 ? dcell_pls_seed(g, DCELL_F64, s->phi_64.p, (const int *)s->band.p, nband, prm, drng, s->parts.p,
                              capacity, dcount, s->scratch.p, sb, dflags, st)
             : dcell_pls_reseed(g, DCELL_F64, s->phi_64.p, (const int *)s->band.p, nband, prm, drng, s->parts.p, nn,
                                capacity, dcount, s->scratch.p, sb, dflags, st);
  if (rc) return rc;
  long long hc = 0;
  int hf = 0;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(&hc, dcount, sizeof(long long), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(rng, drng, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(&hf, dflags, sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  *count = hc;
  const long long ncopy = hc < capacity ? hc : capacity;
  if (ncopy > 0)
    DCELL_CUDA_CHECK(cudaMemcpy(particles, s->parts.p, ncopy * 4 * sizeof(double), cudaMemcpyDeviceToHost));
  return session_flags_status(s, hf);
}

DCELL_API int dcell_ls_pls_seed(dcell_session *s, const dcell_geom *g, const double *phi, const int *band, int nband,
                                const dcell_pls_params *prm, unsigned long long *rng, double *particles,
                                long long capacity, long long *count) {
  return ls_pls_seed_common(s, g, phi, band, nband, prm, rng, particles, -1, capacity, count);
}

DCELL_API int dcell_ls_pls_reseed(dcell_session *s, const dcell_geom *g, const double *phi, const int *band,
                                  int nband, const dcell_pls_params *prm, unsigned long long *rng, double *particles,
                                  long long n, long long capacity, long long *count) {
  if (n < 0) FAIL(DCELL_ERR_ARG, "n must be >= 0");
  return ls_pls_seed_common(s, g, phi, band, nband, prm, rng, particles, n, capacity, count);
}

// ---------------------------------------------------------------------------
// Device-resident level set: LevelSetAdvectAndReinit (Advect.c:33-50) step
// after step with phi, its band and irregular nodes kept on the device.

static bool same_geom(const dcell_geom *a, const dcell_geom *b) {
  return a->n[0] == b->n[0] && a->n[1] == b->n[1] && a->n[2] == b->n[2] && a->p[0] == b->p[0] &&
         a->p[1] == b->p[1] && a->p[2] == b->p[2] && a->h[0] == b->h[0] && a->h[1] == b->h[1] && a->h[2] == b->h[2];
}

// The irregular nodes of phi[cur] over the band (LevelSetUpdateIrregularNodeList);
// the count stays on the device (small + 4).
static int resident_nodes(dcell_session *s) {
  Resident &r = s->res;
  cudaStream_t st = s->stream;
  int *dflags = (int *)r.small.p, *dcount = dflags + 1;
  const size_t sb = irregular_scratch_bytes(r.nband);
  ENSURE(r.scratch, sb);
  return dcell_irregular_nodes(&r.g, r.precision, r.phi[r.cur].p, (const int *)r.band.p, r.nband, 0,
                               (dcell_irregular_node *)r.nodes.p, r.ncap, dcount, r.scratch.p, sb, dflags, st);
}

// Node capacity for a band of nband points (sign changes at a band point's
// faces and its projection node), grown keeping the current nodes (the next
// step's max |V| reads them), with a quarter of headroom so that a band that
// grows a little after a reinitialisation does not reallocate every time;
// the band buffer holds any band of the grid.
static int resident_sizes(dcell_session *s, int nband) {
  Resident &r = s->res;
  const long long n = grid_points(&r.g);
  const long long most = 8LL * n + 1024;
  const long long need = std::min<long long>(8LL * nband + 1024, most);
  if (need > r.ncap) {
    const int want = (int)std::min<long long>(need + need / 4, most);
    int rc = r.nodes.grow_keep((size_t)want * sizeof(dcell_irregular_node),
                               (size_t)r.ncap * sizeof(dcell_irregular_node), s->stream);
    if (rc) return rc;
    r.ncap = want;
  }
  ENSURE(r.band, (size_t)(n > 0 ? n : 1) * 3 * sizeof(int));
  ENSURE(r.small, 256);
  return DCELL_OK;
}

// The node pass a step leaves due (LevelSetUpdateIrregularNodeList of the
// new level set), enqueued on the session stream: the next call runs it
// first, under its velocity upload, before the max |V| and a
// reinitialisation read the nodes.
static int resident_nodes_due(dcell_session *s) {
  Resident &r = s->res;
  if (!r.nodes_pending) return DCELL_OK;
  r.nodes_pending = false;
  return resident_nodes(s);
}

// LevelSetReinitialize on the device (the bucketed march, band width bw),
// seeded by the current irregular nodes, enqueued on the session stream with
// its counters copied back behind it; reinit_ev marks the end.  The session
// stream holds nothing else of this call yet, so reading the node count is
// a short wait.
static int resident_reinit_enqueue(dcell_session *s, double bw) {
  Resident &r = s->res;
  cudaStream_t st = s->stream;
  const dcell_geom *g = &r.g;
  const long long n = grid_points(g);
  int *dflags = (int *)r.small.p, *dcount = dflags + 1;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(r.reinit_hv, dcount, sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  int nn = r.reinit_hv[0];
  if (nn > r.ncap) nn = r.ncap;
  const size_t sb = dcell_reinit_scratch_bytes(g, r.precision);
  ENSURE(r.scratch, sb);
  int rc = dcell_reinitialize(g, r.precision, r.phi[r.cur].p, (const dcell_irregular_node *)r.nodes.p, nn, bw, 0.0,
                              (int *)r.band.p, (int)n, dflags + 2, r.scratch.p, sb, dflags, st);
  if (rc) return rc;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(r.reinit_hv, dflags, 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaEventRecord(r.reinit_ev, st));
  r.split_ok = false;
  r.reinit_pending = false;
  return DCELL_OK;
}

// Waits for the enqueued reinitialisation alone (later work on the stream
// may still run), takes its band and grows the node buffer for it.
static int resident_reinit_finish(dcell_session *s) {
  Resident &r = s->res;
  DCELL_CUDA_CHECK(cudaEventSynchronize(r.reinit_ev));
  int rc = session_flags_status(s, r.reinit_hv[0] & ~DCELL_FLAG_DEPARTURE_CLAMPED);
  if (rc) return rc;
  r.nband = r.reinit_hv[2];
  return resident_sizes(s, r.nband);
}

DCELL_API int dcell_ls_resident_set(dcell_session *s, const dcell_geom *g, const double *phi, const int *band,
                                    int nband, int precision) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  int rc = check_geom(g);
  if (rc) return rc;
  if (!phi || (nband > 0 && !band) || nband < 0) FAIL(DCELL_ERR_ARG, "phi (and band when nband > 0) are required");
  if (precision != DCELL_F32 && precision != DCELL_F64) FAIL(DCELL_ERR_ARG, "precision must be F32 or F64");
  if (nband > 0 && (rc = check_band_host(g, band, nband))) return rc;
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  Resident &r = s->res;
  r.on = false;
  r.nodes_pending = false;
  r.reinit_pending = false;
  if (!r.reinit_hv) DCELL_CUDA_CHECK(cudaMallocHost((void **)&r.reinit_hv, 4 * sizeof(int)));
  if (!r.reinit_ev) DCELL_CUDA_CHECK(cudaEventCreateWithFlags(&r.reinit_ev, cudaEventDisableTiming));
  r.g = *g;
  r.precision = precision;
  r.cur = 0;
  r.nband = nband;
  r.ncap = 0;
  const long long n = grid_points(g);
  cudaStream_t st = s->stream;
  const size_t es = precision == DCELL_F32 ? sizeof(float) : sizeof(double);
  ENSURE(r.phi[0], n * es);
  ENSURE(r.phi[1], n * es);
  if ((rc = resident_sizes(s, nband))) return rc;
  if (precision == DCELL_F32) {
    ENSURE(s->phi_64, n * sizeof(double));
    DCELL_CUDA_CHECK(cudaMemcpyAsync(s->phi_64.p, phi, n * sizeof(double), cudaMemcpyHostToDevice, st));
    if ((rc = launch_convert(s->phi_64.p, DCELL_F64, r.phi[0].p, DCELL_F32, n, st))) return rc;
  } else {
    DCELL_CUDA_CHECK(cudaMemcpyAsync(r.phi[0].p, phi, n * sizeof(double), cudaMemcpyHostToDevice, st));
  }
  if (nband > 0)
    DCELL_CUDA_CHECK(cudaMemcpyAsync(r.band.p, band, (size_t)nband * 3 * sizeof(int), cudaMemcpyHostToDevice, st));
  r.split_ok = false;
  DCELL_CUDA_CHECK(cudaMemsetAsync(r.small.p, 0, 256, st));
  if ((rc = resident_nodes(s))) return rc;
  int hf = 0;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(&hf, r.small.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  r.on = true;
  return session_flags_status(s, hf);
}

DCELL_API int dcell_ls_resident_advect_and_reinit(dcell_session *s, const dcell_geom *g, const void *vel,
                                                  int vel_dtype, double dt, int interp, int backtrace, int dense,
                                                  dcell_ls_loop *loop) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  Resident &r = s->res;
  if (!r.on) FAIL(DCELL_ERR_ARG, "no resident level set: call dcell_ls_resident_set first");
  if (!g || !same_geom(g, &r.g)) FAIL(DCELL_ERR_ARG, "geometry differs from the resident level set's");
  if (!vel || !loop) FAIL(DCELL_ERR_ARG, "vel and loop are required");
  if (vel_dtype != DCELL_F32 && vel_dtype != DCELL_F64) FAIL(DCELL_ERR_ARG, "vel_dtype must be F32 or F64");
  if (interp < DCELL_LINEAR || interp > DCELL_CUBIC_TC) FAIL(DCELL_ERR_ARG, "unknown interpolation %d", interp);
  if (backtrace != DCELL_EULER && backtrace != DCELL_MIDPOINT) FAIL(DCELL_ERR_ARG, "unknown backtrace %d", backtrace);
  if (!(dt == dt)) FAIL(DCELL_ERR_NONFINITE, "dt is NaN");
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long n = grid_points(g);
  const int dof = g->n[2] > 1 ? 3 : 2;
  const dcell::Geom G = dcell::to_geom(g);
  int rc;
  int *dflags = (int *)r.small.p, *dcount = dflags + 1;
  double *dmax = (double *)((char *)r.small.p + 64);
  DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, sizeof(int), st));
  // the reinitialisation the last step triggered runs first; with the
  // pipelined upload below it overlaps this step's velocity copy
  // the velocity upload (on the copy stream, when pipelined) needs only the
  // session's earlier work done, not this call's reinitialisation
  if ((rc = ensure_copy_streams(s))) return rc;
  cudaEvent_t start = s->ev_out[kPipeSlabs - 1];
  DCELL_CUDA_CHECK(cudaEventRecord(start, st));
  if ((rc = resident_nodes_due(s))) return rc;  // the last step's node pass
  bool reinit_open = r.reinit_pending;  // enqueued, its band not yet taken
  if (reinit_open && (rc = resident_reinit_enqueue(s, r.reinit_bw))) return rc;
  if (reinit_open && !dense) {  // the band step below needs the new band first
    if ((rc = resident_reinit_finish(s))) return rc;
    reinit_open = false;
  }
  const size_t ves = r.precision == DCELL_F32 ? sizeof(float) : sizeof(double);
  const size_t ies = vel_dtype == DCELL_F32 ? sizeof(float) : sizeof(double);
  ENSURE(r.vel, n * dof * ves);
  if (vel_dtype != r.precision) ENSURE(r.vel64, n * dof * ies);
  const int cur = r.cur, nxt = 1 - cur;
  const bool use_band = !dense && r.nband > 0;
  const bool dense_tc = r.precision == DCELL_F32 && interp == DCELL_CUBIC_TC && !use_band && G.nz > 1;
  // The dense tensor-core step on deep grids overlaps the velocity upload:
  // plane chunks go up on the copy stream and each z-slab is stepped once
  // the planes it can read are present (the gate of ls_advect_tc_pipelined:
  // a slab whose departures could reach planes not yet present is left, and
  // the whole grid is stepped again below).
  const bool pipelined = dense_tc && G.nz >= 4 * tc_slab_planes() &&
                         tc_brick_applicable(G, (const void *)256, (const void *)256);
  bool redo_possible = false;
  if (pipelined) {
    ENSURE(r.split[0], n * sizeof(uint32_t));
    ENSURE(r.split[1], n * sizeof(uint32_t));
    ENSURE(s->gates, kPipeSlabs * sizeof(int));
    int *gates = (int *)s->gates.p;
    if (!r.split_ok && (rc = launch_split_bf16((const float *)r.phi[cur].p, (uint32_t *)r.split[cur].p, n, st)))
      return rc;
    DCELL_CUDA_CHECK(cudaMemsetAsync(gates, 0, kPipeSlabs * sizeof(int), st));
    DCELL_CUDA_CHECK(cudaStreamWaitEvent(s->h2d, start, 0));
    const long long plane = (long long)G.nx * G.ny;
    const int BZ = tc_slab_planes(), nbz = (G.nz + BZ - 1) / BZ, per = (nbz + kPipeSlabs - 1) / kPipeSlabs;
    float *v32 = (float *)r.vel.p;
    int have = 0, gated = 0;  // planes present on the device, planes in the gate's max
    for (int k = 0; k < kPipeSlabs; ++k) {
      const int b0 = k * per, b1 = b0 + per < nbz ? b0 + per : nbz;
      if (b0 >= b1) break;
      const int z1 = b1 * BZ < G.nz ? b1 * BZ : G.nz;
      const int need = z1 + kPipeHalo < G.nz ? z1 + kPipeHalo : G.nz;
      if (need > have) {  // the next chunk of velocity planes
        const long long o = have * plane * dof, m = (need - have) * plane * dof;
        if (vel_dtype == r.precision) {
          DCELL_CUDA_CHECK(cudaMemcpyAsync(v32 + o, (const float *)vel + o, m * sizeof(float), cudaMemcpyHostToDevice,
                                           s->h2d));
        } else {
          double *v64 = (double *)r.vel64.p;
          DCELL_CUDA_CHECK(cudaMemcpyAsync(v64 + o, (const double *)vel + o, m * sizeof(double),
                                           cudaMemcpyHostToDevice, s->h2d));
          if ((rc = launch_convert(v64 + o, DCELL_F64, v32 + o, DCELL_F32, m, s->h2d))) return rc;
        }
        have = need;
      }
      DCELL_CUDA_CHECK(cudaEventRecord(s->ev_in[k], s->h2d));
      DCELL_CUDA_CHECK(cudaStreamWaitEvent(st, s->ev_in[k], 0));
      if (have > gated) {  // the gate's running max over the planes present
        if ((rc = launch_max_abs_component(v32 + 3 * gated * plane, (have - gated) * plane, 3, 2, gates, st)))
          return rc;
        gated = have;
      }
      TcSlab slab;
      slab.bz0 = b0;
      slab.nbz = b1 - b0;
      slab.gate_maxw = gates;
      slab.gate_limit = (float)(kPipeHalo - 3);
      if ((rc = launch_sl_tc_slab(G, (const uint32_t *)r.split[cur].p, v32, dt, backtrace, (float *)r.phi[nxt].p,
                                  (uint32_t *)r.split[nxt].p, dflags, st, slab)))
        return rc;
    }
    // the last slab waited for the last chunk: every velocity plane is present on st from here
    redo_possible = true;
    r.split_ok = true;
  }
  if (reinit_open) {  // its band sizes the node pass (and the upload, when pipelined, is already on its way)
    if ((rc = resident_reinit_finish(s))) return rc;
    reinit_open = false;
  }
  if (!pipelined) {
    // the step's velocity (the only per-step upload)
    if (vel_dtype == r.precision) {
      DCELL_CUDA_CHECK(cudaMemcpyAsync(r.vel.p, vel, n * dof * ves, cudaMemcpyHostToDevice, st));
    } else {
      DCELL_CUDA_CHECK(cudaMemcpyAsync(r.vel64.p, vel, n * dof * ies, cudaMemcpyHostToDevice, st));
      if ((rc = launch_convert(r.vel64.p, vel_dtype, r.vel.p, r.precision, n * dof, st))) return rc;
    }
  }
  // LevelSetCFLIncrement (Advect.c:54-66) needs max |V| at the current
  // nodes; the reference takes it after the advection, from the nodes of the
  // level set before this step -- the same nodes, queued here (before the
  // node pass of the new level set overwrites them)
  if ((rc = dcell_max_velocity(g, r.precision, r.vel.p, (const dcell_irregular_node *)r.nodes.p, dcount, r.ncap, dmax,
                               st)))
    return rc;
  // GridCopy (phi0 <- phi) and the SL step: phi[nxt] from phi[cur]
  if (pipelined) {
    rc = DCELL_OK;  // stepped above
  } else if (dense_tc) {
    ENSURE(r.split[0], n * sizeof(uint32_t));
    ENSURE(r.split[1], n * sizeof(uint32_t));
    if (!r.split_ok && (rc = launch_split_bf16((const float *)r.phi[cur].p, (uint32_t *)r.split[cur].p, n, st)))
      return rc;
    rc = launch_sl_tc_split(G, (const uint32_t *)r.split[cur].p, (const float *)r.vel.p, dt, nullptr, n, backtrace,
                            (float *)r.phi[nxt].p, (uint32_t *)r.split[nxt].p, dflags, st);
    r.split_ok = true;
  } else {
    if (use_band)  // band points only: the others keep phi's values
      DCELL_CUDA_CHECK(cudaMemcpyAsync(r.phi[nxt].p, r.phi[cur].p, n * ves, cudaMemcpyDeviceToDevice, st));
    rc = dcell_sl_step(g, r.precision, r.phi[cur].p, r.vel.p, dt, use_band ? (const int *)r.band.p : nullptr,
                       use_band ? r.nband : 0, interp, backtrace, r.phi[nxt].p, dflags, st);
    r.split_ok = false;
  }
  if (rc) return rc;
  r.cur = nxt;
  // LevelSetUpdateIrregularNodeList of the new phi: due, it runs first in the
  // next call (under its upload) or before a reinitialisation
  r.nodes_pending = true;
  double maxvel = 0.0;
  int hf = 0;
  DCELL_CUDA_CHECK(cudaMemcpyAsync(&maxvel, dmax, sizeof(double), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaMemcpyAsync(&hf, dflags, sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  if (redo_possible && (hf & dcell::FLAG_PIPELINE_REDO)) {
    // a slab was left: step the whole grid with every plane present (the
    // same kernel on the same inputs)
    DCELL_CUDA_CHECK(cudaMemsetAsync(dflags, 0, sizeof(int), st));
    if ((rc = launch_sl_tc_split(G, (const uint32_t *)r.split[cur].p, (const float *)r.vel.p, dt, nullptr, n,
                                 backtrace, (float *)r.phi[nxt].p, (uint32_t *)r.split[nxt].p, dflags, st)))
      return rc;
    DCELL_CUDA_CHECK(cudaMemcpyAsync(&hf, dflags, sizeof(int), cudaMemcpyDeviceToHost, st));
    DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  }
  hf &= ~dcell::FLAG_PIPELINE_REDO;
  if ((rc = session_flags_status(s, hf & ~DCELL_FLAG_DEPARTURE_CLAMPED))) return rc;
  loop->maxVel = maxvel;
  loop->CFLcount += dt * maxvel / g->h[0];
  loop->AdvectCount++;
  loop->reinitialized = 0;
  if (loop->AdvectCount > loop->AdvectThres || loop->CFLcount > loop->CFLthres) {
    // LevelSetReinitialize (the device's bucketed march, new band), from
    // this step's nodes: it runs before the level set is next used -- at the
    // start of the next call, under its velocity upload, or in
    // dcell_ls_resident_get
    loop->CFLcount = 0;
    loop->AdvectCount = 0;
    r.reinit_pending = true;
    r.reinit_bw = loop->bandWidth;
    loop->reinitialized = 1;
  }
  loop->band = r.nband;
  return (hf & DCELL_FLAG_DEPARTURE_CLAMPED) && use_band
             ? (dcell_set_error(DCELL_ERR_DEPARTURE, "a departure point left the grid; its sample was clamped"),
                DCELL_ERR_DEPARTURE)
             : DCELL_OK;
}

DCELL_API int dcell_ls_resident_get(dcell_session *s, const dcell_geom *g, double *phi, int *band, int capacity,
                                    int *nband) {
  if (!s) FAIL(DCELL_ERR_ARG, "session is NULL");
  Resident &r = s->res;
  if (!r.on) FAIL(DCELL_ERR_ARG, "no resident level set: call dcell_ls_resident_set first");
  if (!g || !same_geom(g, &r.g)) FAIL(DCELL_ERR_ARG, "geometry differs from the resident level set's");
  if (capacity < 0 || (capacity > 0 && !band)) FAIL(DCELL_ERR_ARG, "invalid band buffer");
  DCELL_CUDA_CHECK(cudaSetDevice(s->device));
  cudaStream_t st = s->stream;
  const long long n = grid_points(g);
  int rc;
  if (r.reinit_pending) {  // the reinitialisation the last step triggered, from that step's nodes
    if ((rc = resident_nodes_due(s)) || (rc = resident_reinit_enqueue(s, r.reinit_bw)) ||
        (rc = resident_reinit_finish(s)))
      return rc;
  }
  if (phi) {
    if (r.precision == DCELL_F32) {
      ENSURE(s->phi_64, n * sizeof(double));
      if ((rc = launch_convert(r.phi[r.cur].p, DCELL_F32, s->phi_64.p, DCELL_F64, n, st))) return rc;
      DCELL_CUDA_CHECK(cudaMemcpyAsync(phi, s->phi_64.p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    } else {
      DCELL_CUDA_CHECK(cudaMemcpyAsync(phi, r.phi[r.cur].p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
  }
  const int ncopy = r.nband < capacity ? r.nband : capacity;
  if (ncopy > 0)
    DCELL_CUDA_CHECK(cudaMemcpyAsync(band, r.band.p, (size_t)ncopy * 3 * sizeof(int), cudaMemcpyDeviceToHost, st));
  DCELL_CUDA_CHECK(cudaStreamSynchronize(st));
  if (nband) *nband = r.nband;
  return DCELL_OK;
}

}  // extern "C"
