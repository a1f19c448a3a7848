/*
 * dcell_ls.h -- C ABI of the B200 (sm_100a) level-set transport path.
 *
 * Drop-in boundary for adrielb/DCell's LevelSetMethod hot path.  Plain C
 * types, plain pointers and sizes; no C++ or torch types.  All functions
 * return a status (DCELL_OK == 0, like the reference's PetscErrorCode) and
 * never exit; dcell_last_error() gives the message of the last failure on
 * the calling thread.
 *
 * Two layers:
 *  - device-resident entry points (dcell_sl_step, dcell_irregular_nodes, ...)
 *    take DEVICE pointers and a cudaStream_t (passed as void*), enqueue work
 *    and return without synchronising;
 *  - host-buffer entry points (dcell_ls_*) take the reference's own FP64
 *    host arrays (Grid.v1, Array data of LevelSet.band) through a session,
 *    copy in, compute, copy out and synchronise -- what a LevelSet C host
 *    calls from LevelSetAdvectSL & co.
 *
 * Grid convention (reference Common/Grid.c:69-93, Common/Grid.h:8-22): a grid
 * covers global indices [p, p+n) per axis, x fastest; velocity grids keep dof
 * (2 or 3) values innermost, u at x-face i-1/2, v at y-face j-1/2, w at z-face
 * k-1/2 (Common/Common.h:26-30, Tensor1).  2D grids have n[2] <= 1.  The band
 * is an array of iCoor {x, y, z} int triples in GLOBAL indices
 * (LevelSetMethod.h:23, Common/Common.h:22-24).
 */
#ifndef DCELL_LS_H_
#define DCELL_LS_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DCELL_LS_VERSION 1

#if defined(__GNUC__)
#define DCELL_API __attribute__((visibility("default")))
#else
#define DCELL_API
#endif

/* status codes (reference: PetscErrorCode, 0 = success) */
enum {
  DCELL_OK = 0,
  DCELL_ERR_ARG = 1,          /* invalid argument (SETERRQ ... ARG_OUTOFRANGE in Array.c:92-95) */
  DCELL_ERR_CUDA = 2,         /* CUDA runtime error */
  DCELL_ERR_DEPARTURE = 3,    /* a departure point left the grid (sample clamped) */
  DCELL_ERR_NONFINITE = 4,    /* non-finite input or result */
  DCELL_ERR_TIMEOUT = 5,      /* a bounded device-side wait gave up */
  DCELL_ERR_CAPACITY = 6,     /* caller buffer too small */
  DCELL_ERR_UNSUPPORTED = 7,  /* combination not implemented */
  DCELL_ERR_NOMEM = 8         /* device allocation failed */
};

enum { DCELL_F32 = 0, DCELL_F64 = 1 };

/* reconstruction at the departure point */
enum {
  DCELL_LINEAR = 0,          /* reference Bilinear2D/Bilinear3D (Grid.c:190, Grid3D.c:4) */
  DCELL_CUBIC_PLAIN = 1,     /* Catmull-Rom, 64 (16) coefficients by the 1331 (121) non-zeros
                                of TricubicInverse.h (OrthogonalProjection.c:48-63 in 2D) */
  DCELL_CUBIC_SEPARABLE = 2, /* same interpolant as 3 (2) passes of 4-tap filters */
  DCELL_CUBIC_TC = 3         /* same interpolant, coefficient solve as a split-BF16 tcgen05
                                GEMM with FP32 accumulation (3D, FP32 only) */
};

/* OR'ed into interp: run the global-gather form of DCELL_LINEAR /
 * DCELL_CUBIC_PLAIN / DCELL_CUBIC_SEPARABLE on a dense FP32 3D grid (one
 * thread per point, every value gathered from global memory) instead of its
 * shared-memory-staged form (TMA z-march for LINEAR, TMA bricks for the two
 * cubic forms).  Both forms give the same results; the flag exists to compare
 * their data paths. */
#define DCELL_GATHER_FORM 0x100

/* departure-point backtrace */
enum {
  DCELL_EULER = 0,    /* S = X - V(X) dt/h, V at the arrival point (AdvectSL.c:44-47, :78-82) */
  DCELL_MIDPOINT = 1  /* Xm = X - V(X) dt/(2h);  S = X - V(Xm) dt/h */
};

/* Grid geometry: the n / p / d fields of struct _Grid (Grid.h:8-22). */
typedef struct dcell_geom {
  int n[3];
  int p[3];
  double h[3];
} dcell_geom;

/* One irregular node: the fields of struct _IrregularNode
 * (LevelSetMethod.h:29-54) that the transport path writes. */
typedef struct dcell_irregular_node {
  int pos[3];      /* node index (global) */
  int axis;        /* 0/1/2 or -1 for an orthogonal-projection node */
  int shift;       /* VelFace: CELL_CENTER 0, U_FACE 1, V_FACE 2, W_FACE 3; -1 for projection nodes */
  int signCenter;
  int signFace;
  int pad;
  double d;        /* crossing fraction along the axis */
  double X[3];     /* index-space position of the interface point */
  double op[3];    /* orthogonal projection relative to pos (projection nodes) */
  double n[3];     /* unit normal at X (with_surface) */
  double k;        /* curvature at X (with_surface) */
} dcell_irregular_node;

/* A box of a level set on the global index grid, packed at `offset` points
 * into a batch buffer (velocity acquisition of many cells). */
typedef struct dcell_box {
  long long offset; /* first point of the box in the packed output */
  int p[3];         /* global index of the box's first point */
  int n[3];         /* extents (n[2] == 1 in 2D) */
} dcell_box;

/* Text of the last error on this thread ("" if none). */
DCELL_API const char *dcell_last_error(void);
DCELL_API int dcell_version(void);

/* ------------------------------------------------------------------------
 * Device-resident entry points
 * ---------------------------------------------------------------------- */

/* One semi-Lagrangian step: for each band point X (or every grid point when
 * band == NULL), phi[X] = interp(phi0, S(X)).
 * Replaces LevelSetAdvectSL / _2D / _3D (LevelSetMethod/AdvectSL.c:6-89).
 * phi0, phi: dtype grids of n[0]*n[1]*n[2] values; vel: dtype, dof innermost;
 * band: int32 [nband][3] or NULL; dt is the step the velocity is multiplied
 * by (fold any scalar time factor of the field into it).  phi is written at
 * the updated points only.  Samples outside the grid are clamped to it: for a
 * dense step (band == NULL) that is the boundary condition (constant
 * extrapolation at the domain edge); for a band step it means the band came
 * too close to the grid edge (the reference would read out of bounds) and
 * DCELL_FLAG_DEPARTURE_CLAMPED is raised.  Band entries outside the grid are
 * skipped and raise DCELL_FLAG_BAD_BAND.  Grids are limited to
 * 3 * points < 2^31.  flags (optional int on the device) receives
 * DCELL_FLAG_* bits.  DCELL_CUBIC_TC requires dtype F32 and a 3D
 * grid.  Dense FP32 3D grids with nx % 4 == 0 and 16-byte aligned arrays run
 * the shared-memory-staged forms unless interp carries DCELL_GATHER_FORM. */
#define DCELL_FLAG_DEPARTURE_CLAMPED 1
#define DCELL_FLAG_NONFINITE 2
#define DCELL_FLAG_CAPACITY 4
#define DCELL_FLAG_WAIT_TIMEOUT 8
#define DCELL_FLAG_BAD_BAND 16
#define DCELL_FLAG_UNSETTLED 32 /* reinitialisation: points still tentative after its last bucket */
#define DCELL_FLAG_PARTICLE_OUTSIDE 64 /* a particle's stencil or cell left the grid (clamped / skipped) */
DCELL_API int dcell_sl_step(const dcell_geom *g, int dtype, const void *phi0, const void *vel, double dt, const int *band,
                  int nband, int interp, int backtrace, void *phi, int *flags, void *stream);

/* Split-BF16 state of an FP32 grid: split[i] holds bf16 hi = RN(phi[i]) in
 * its low 16 bits and bf16 lo = RN(phi[i] - hi) in its high 16 bits. */
DCELL_API int dcell_split_bf16(const dcell_geom *g, const float *phi, unsigned int *split, void *stream);

/* DCELL_CUBIC_TC step on a split-state level set: the stencil operands come
 * from phi0_split (as made by dcell_split_bf16 or by a previous step), so the
 * kernel forms the tensor-core A rows with byte permutes instead of per-entry
 * conversions.  Writes phi (FP32) and, when phi_split != NULL, its split --
 * the next step's input.  Same interpolant, backtrace, band and flag rules as
 * dcell_sl_step; 3D only. */
DCELL_API int dcell_sl_step_tc_split(const dcell_geom *g, const unsigned int *phi0_split, const float *vel, double dt,
                                     const int *band, int nband, int backtrace, float *phi, unsigned int *phi_split,
                                     int *flags, void *stream);

/* dcell_sl_step_tc_split on the arrival planes [z_begin, z_end) only (dense
 * grid, no band): the form a z-slab owner uses to step its interior planes
 * while its halo planes are still in flight, then the planes next to the
 * halos.  z_begin and z_end are multiples of the brick depth, 8 planes (z_end
 * may also be nz); the brick path must apply (nx % 4 == 0, 16-byte aligned
 * arrays, a grid at least one brick box wide per axis), else
 * DCELL_ERR_UNSUPPORTED.  Planes outside the range are not written.  No
 * reference counterpart: the reference never splits one level set. */
DCELL_API int dcell_sl_step_tc_split_planes(const dcell_geom *g, const unsigned int *phi0_split, const float *vel,
                                            double dt, int z_begin, int z_end, int backtrace, float *phi,
                                            unsigned int *phi_split, int *flags, void *stream);

/* Adjoint of one dense 3D SL step (dcell_sl_step with band == NULL): given
 * grad_phi = dL/dphi, ACCUMULATES dL/dphi0 into grad_phi0 and dL/dvel into
 * grad_vel (same layouts as phi0 / vel; zero them first for a fresh
 * gradient).  The transpose of the interpolation weights is scattered with
 * global atomics; the velocity sensitivity goes through the departure point
 * (and, for DCELL_MIDPOINT, through the midpoint).  interp DCELL_LINEAR or
 * any cubic mode (they share one interpolant).  No counterpart in the
 * reference, which has no derivatives. */
DCELL_API int dcell_sl_adjoint(const dcell_geom *g, int dtype, const void *phi0, const void *vel, double dt,
                               int interp, int backtrace, const void *grad_phi, void *grad_phi0, void *grad_vel,
                               void *stream);

/* Irregular-node pass over the band: replaces LevelSetUpdateIrregularNodeList
 * (LevelSetMethod/IrregularNodes.c:9-141, IrregularNodes3D.c:6-117) including
 * OrthogonalProjection2D/3D (OrthogonalProjection*.c).  Nodes are written in
 * the reference's order (band order; per point: projection node, cell-face
 * nodes, velocity-face nodes).  With with_surface != 0 also fills n and k as
 * IIMUpdateSurfaceQuantities_2D/3D does (IIM/SurfaceQuantities.c:48-56,
 * :83-89, :111).  *count (device int) receives the total node count even if
 * it exceeds capacity (then DCELL_FLAG_CAPACITY is raised).  scratch is a
 * device buffer of at least dcell_irregular_nodes_scratch_bytes(nband). */
DCELL_API size_t dcell_irregular_nodes_scratch_bytes(int nband);
DCELL_API int dcell_irregular_nodes(const dcell_geom *g, int dtype, const void *phi, const int *band, int nband,
                          int with_surface, dcell_irregular_node *nodes, int capacity, int *count, void *scratch,
                          size_t scratch_bytes, int *flags, void *stream);

/* Narrow-band reinitialisation of phi to the signed distance (cell units):
 * replaces LevelSetReinitialize (LevelSetMethod/FastMarching.c:11-41) after
 * its LevelSetResize, i.e. FMM_InitializeEikonal / FMM_SolveEikonal
 * (FastMarching.c:43-146) with the second-order update of
 * FMM_PushNeighbors2D/3D and AccumulateCoef (FastMarching2D.c:33-185,
 * FastMarching3D.c:13-101).  phi (device, dtype) is overwritten: band points
 * get the marched distance, all others +/-PHI_INF = +/-(band_width + 1.5).
 * nodes / nnodes: the irregular nodes of phi (device, as dcell_irregular_nodes
 * writes them); those with axis == -1 seed the march with signCenter * |op|.
 * The heap is replaced by buckets of width `bucket` cells (0: 1/64): all
 * tentative values of a bucket are fixed together, so results differ from
 * the heap's where a point depends on another of its own bucket (measured
 * against the reference: mean 5e-5, max 1e-2 cells).  band (device int32
 * [capacity][3], global indices) receives the fixed points in grid order (x
 * fastest) -- the reference lists them in march order; *count (device int)
 * their number (DCELL_FLAG_CAPACITY if above capacity).  A non-finite update
 * raises DCELL_FLAG_NONFINITE (the reference exits), points still tentative
 * after the last bucket DCELL_FLAG_UNSETTLED.  scratch: a device buffer of at
 * least dcell_reinit_scratch_bytes(g, dtype). */
DCELL_API size_t dcell_reinit_scratch_bytes(const dcell_geom *g, int dtype);
DCELL_API int dcell_reinitialize(const dcell_geom *g, int dtype, void *phi, const dcell_irregular_node *nodes,
                                 int nnodes, double band_width, double bucket, int *band, int capacity, int *count,
                                 void *scratch, size_t scratch_bytes, int *flags, void *stream);

/* Velocity acquisition: replaces LevelSetGetVelocity
 * (LevelSetMethod/Advect.c:145-192), i.e. GridResize of the velocity grid to
 * the phi box (which zeroes it, Common/Grid.c:146) and NGA_Get of the part of
 * the box inside the fluid's Global Array.  global: device array of the
 * fluid's field, [gdims[2]][gdims[1]][gdims[0]][gdof] (3D) or
 * [gdims[1]][gdims[0]][gdof] (2D, gdims[2] = 1), components in VelFace order
 * (CELL_CENTER, U_FACE, V_FACE, W_FACE); components first .. first+dim-1
 * (first = 1: U_FACE..) are copied.  vel: device array of the box (the
 * extents and global origin of g; h unused), dim components innermost; box
 * points outside the field get 0. */
DCELL_API int dcell_velocity_box(const dcell_geom *g, int dtype, const void *global, const int gdims[3], int gdof,
                                 int first, void *vel, void *stream);
/* The same for nboxes boxes (device array) in one launch, box b written at
 * boxes[b].offset * dim of vel; max_points bounds the largest box (sizes the
 * launch).  dim 2 or 3; nboxes <= 65535. */
DCELL_API int dcell_velocity_boxes(const dcell_box *boxes, int nboxes, int dim, int dtype, const void *global,
                                   const int gdims[3], int gdof, int first, long long max_points, void *vel,
                                   void *stream);

/* Allocation-free variant of dcell_irregular_nodes.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory -- a
 * host whose device memory is all owned by another runtime's allocator or a
 * fixed-size pool, or one that must not call cudaMalloc because that call can
 * synchronise the device and stall its other streams.  Same inputs, outputs
 * and results as dcell_irregular_nodes, but it takes no scratch: the scan
 * scratch lives in a static array of the library (about 4 MiB, held on every
 * GPU that loads the library until the process exits).  Limits and rules:
 *   - nband <= DCELL_NOALLOC_MAX_BAND, else DCELL_ERR_ARG and no work;
 *   - the first call on a device (made with that device current) looks up the
 *     array's device address; make that first call before any stream capture;
 *   - that address is kept per device number for the life of the process:
 *     make every call from the device's primary context (the CUDA runtime's
 *     own), and do not call cudaDeviceReset between calls -- a reset or
 *     another context would leave the kept address pointing elsewhere;
 *   - all calls on a device share the array, so calls that overlap on the GPU
 *     (different streams, or a second call before the first one finished)
 *     race; serialise them;
 *   - it allocates nothing (no cudaMalloc, cudaFree or allocating library
 *     call).  The caller still provides nodes, count and flags. */
#define DCELL_NOALLOC_MAX_BAND (1 << 20)
DCELL_API int dcell_irregular_nodes_noalloc(const dcell_geom *g, int dtype, const void *phi, const int *band,
                                            int nband, int with_surface, dcell_irregular_node *nodes, int capacity,
                                            int *count, int *flags, void *stream);

/* max |V| over the integer positions of the irregular nodes
 * (LevelSet_MaxVelocity, LevelSetMethod/Advect.c:70-111).  count and maxvel
 * are device pointers; *maxvel is overwritten. */
DCELL_API int dcell_max_velocity(const dcell_geom *g, int dtype, const void *vel, const dcell_irregular_node *nodes,
                       const int *count, int capacity, double *maxvel, void *stream);

/* Enclosed volume (2D: area) sum (1 - H_eps(phi)) * cell volume with the
 * smoothed Heaviside whose derivative is the reference's smoothed delta
 * (LevelSetDiracDelta2D/3D, NormalDirection.c:36-57); FP64 accumulation,
 * deterministic.  *volume is a device double.  scratch: at least
 * dcell_volume_scratch_bytes() bytes. */
DCELL_API size_t dcell_volume_scratch_bytes(void);
DCELL_API int dcell_volume(const dcell_geom *g, int dtype, const void *phi, double eps, double *volume, void *scratch,
                 size_t scratch_bytes, void *stream);

/* ------------------------------------------------------------------------
 * Particle level set (LevelSetMethod/ParticleLS.c, ParticleLS2D.c,
 * ParticleLS3D.c).  Particles are device records of four values of the
 * dtype: X.x, X.y, X.z in global index space and the signed radius, i.e.
 * struct _Particle (LevelSetMethod/LSM_private.h:45-48).  Random draws follow
 * the reference's PETSCRAND48 stream, the C library's drand48: rng holds the
 * 48-bit state X (X <- 0x5DEECE66D X + 0xB mod 2^48, value X / 2^48); srand48
 * (0x12345678), PETSc's default seed, gives 0x12345678330E.
 * ---------------------------------------------------------------------- */

/* LevelSetInitializeParticles' parameters (ParticleLS.c:21-27). */
typedef struct dcell_pls_params {
  double r_min, r_max; /* particle radius bounds: 0.1, 0.5 */
  double d_init;       /* seeding band |phi| < d_init: 3 */
  double g_tol;        /* attraction tolerance: 1e-3 */
  double e_dist;       /* escaped particles farther than this are deleted: 0.5 */
  int s_init;          /* particles per cell: 16 (2D), 32 (3D) */
  int l_max;           /* attraction steps: 30 */
} dcell_pls_params;
DCELL_API void dcell_pls_default_params(int dim, dcell_pls_params *out);

/* ParticleLS_AdvectParticles2D/3D (ParticleLS2D.c:6-36, ParticleLS3D.c:6-36):
 * RK2 midpoint with the MAC velocity interpolation of InterpolateVelocity*.
 * vel: the velocity grid of g (dof 2/3 innermost).  Stencils outside the
 * grid are clamped and raise DCELL_FLAG_PARTICLE_OUTSIDE. */
DCELL_API int dcell_pls_advect(const dcell_geom *g, int dtype, const void *vel, void *particles, long long n,
                               double dt, int *flags, void *stream);

/* ParticleLS_ErrorCorrection2D/3D (ParticleLS2D.c:40-115,
 * ParticleLS3D.c:40-116): escaped particles correct phi at the band points.
 * The 3D cell corner z is floor(X.y), as the reference computes it
 * (ParticleLS3D.c:76).  Corners outside the grid are skipped (the reference
 * writes out of bounds) and raise DCELL_FLAG_PARTICLE_OUTSIDE.  Several
 * escaped particles giving a corner exactly +0 and -0 may leave the other
 * zero than the reference's particle order would.  scratch: at least
 * dcell_pls_correct_scratch_bytes(g, dtype) bytes. */
DCELL_API size_t dcell_pls_correct_scratch_bytes(const dcell_geom *g, int dtype);
DCELL_API int dcell_pls_correct(const dcell_geom *g, int dtype, void *phi, const int *band, long long nband,
                                const void *particles, long long n, void *scratch, size_t scratch_bytes, int *flags,
                                void *stream);

/* ParticleLS_AdjustRadii (ParticleLS.c:158-185). */
DCELL_API int dcell_pls_adjust_radii(const dcell_geom *g, int dtype, const void *phi, void *particles, long long n,
                                     const dcell_pls_params *prm, int *flags, void *stream);

/* LevelSetInitializeParticles' seeding (ParticleLS.c:36-75, 2D): s_init
 * particles in every band cell with |phi| < d_init, five draws each from
 * *rng (device, advanced), attracted to their phi goal, then AdjustRadii.
 * *count (device) = the number seeded; records past capacity are not written
 * (DCELL_FLAG_CAPACITY).  scratch: dcell_pls_scratch_bytes(g, nband, 0). */
DCELL_API size_t dcell_pls_scratch_bytes(const dcell_geom *g, long long nband, long long n);
DCELL_API int dcell_pls_seed(const dcell_geom *g, int dtype, const void *phi, const int *band, long long nband,
                             const dcell_pls_params *prm, unsigned long long *rng, void *particles, long long capacity,
                             long long *count, void *scratch, size_t scratch_bytes, int *flags, void *stream);

/* ParticleLS_ReseedParticles (ParticleLS.c:202-295, 2D) on n particles:
 * deletion in the reference's order (the last particle moves into a deleted
 * slot), per-cell counts of the non-escaped particles, and new particles in
 * band order for cells below s_init (draws from *rng, attracted).  *count
 * (device) = the new number; records past capacity are not written
 * (DCELL_FLAG_CAPACITY).  Particles whose cell lies outside phi's box are not
 * counted (DCELL_FLAG_PARTICLE_OUTSIDE; the reference counts them against the
 * previous lookup).  scratch: dcell_pls_scratch_bytes(g, nband, n). */
DCELL_API int dcell_pls_reseed(const dcell_geom *g, int dtype, const void *phi, const int *band, long long nband,
                               const dcell_pls_params *prm, unsigned long long *rng, void *particles, long long n,
                               long long capacity, long long *count, void *scratch, size_t scratch_bytes, int *flags,
                               void *stream);

/* ------------------------------------------------------------------------
 * Batched cells: many DCells' level sets of uneven sizes in one launch
 * (the reference advances them one after another per rank,
 * DWorld/DCellsArray.c:50-102).
 * ---------------------------------------------------------------------- */

/* One cell of a packed batch.  Its phi occupies elements
 * [offset, offset + n0*n1*n2) of the packed phi arrays (x fastest) and its
 * MAC velocity elements [3*offset, 3*(offset + n0*n1*n2)) of the packed
 * velocity array.  The grid edge is the cell's domain boundary (samples
 * outside are clamped).  dt is this cell's step. */
typedef struct dcell_cell {
  long long offset;
  int n[3];
  int pad; /* 0, or the padded row length of dcell_batch_sl_step_tc_split_tma's packing */
  double h[3];
  double dt;
} dcell_cell;

/* A tile: the box [x0, x0+tx) x [y0, y0+ty) x [z0, z0+tz) of cell `cell`,
 * clipped to the cell's grid. */
typedef struct dcell_tile {
  int cell;
  int x0, y0, z0;
} dcell_tile;

/* Host-only: cover every point of every cell by tiles of tx*ty*tz points,
 * cell by cell, z, y, x.  *ntiles receives the number needed even when it
 * exceeds capacity (then DCELL_ERR_CAPACITY). */
DCELL_API int dcell_batch_plan(const dcell_cell *cells, int ncells, int tx, int ty, int tz, dcell_tile *tiles,
                               int capacity, int *ntiles);

/* One SL step of every cell of the batch in ONE persistent launch over the
 * tile queue (device arrays cells, tiles; FP32 phi0/vel/phi packed as
 * above).  interp: DCELL_CUBIC_TC needs tx*ty*tz == 128; the CUDA-core
 * modes need tx*ty*tz in [32, 1024].  ctas_per_sm (1..4 for TC, 1..8
 * otherwise) sets the persistent grid; it and the tile shape are what the
 * autotuner of dcell_b200.batch chooses. */
DCELL_API int dcell_batch_sl_step(const dcell_cell *cells, int ncells, const dcell_tile *tiles, int ntiles, int tx,
                                  int ty, int tz, int ctas_per_sm, const float *phi0, const float *vel, float *phi,
                                  int interp, int backtrace, int *flags, void *stream);

/* The split-state tensor-core step (dcell_sl_step_tc_split) of every cell
 * of a batch in ONE persistent launch over bricks of 32 x 4 x 8 points:
 * bricks = dcell_batch_plan(cells, ncells, 32, 4, 8, ...) as a device array;
 * phi0_split (packed split words), vel, phi and phi_split (the next step's
 * input) packed as for dcell_batch_sl_step.  Every cell gets the bits
 * dcell_sl_step_tc_split gives it alone (cells of any shape: the brick boxes
 * are staged with copies clamped to the cell, the edge replication of the
 * single-grid kernel).  3D cells, FP32. */
DCELL_API int dcell_batch_sl_step_tc_split(const dcell_cell *cells, int ncells, const dcell_tile *bricks,
                                           int nbricks, const unsigned int *phi0_split, const float *vel,
                                           int backtrace, float *phi, unsigned int *phi_split, int *flags,
                                           void *stream);

/* The same batched split-state step with the boxes staged by TMA (the dense
 * kernel's data path), for cells packed with padded rows: cell.pad = the
 * row length in points (a multiple of 4, >= n[0]; its extra columns hold
 * copies of the cell's last column in phi0_split and vel), cell.offset a
 * multiple of 4.  maps: dcell_batch_tma_maps_bytes(ncells) bytes of device
 * memory filled by dcell_batch_tma_maps for these very phi0_split and vel
 * arrays (a tensor map per cell and array; build once per buffer pair).  The
 * step writes every real point with the bits dcell_sl_step_tc_split gives the
 * unpadded cell, and the pad columns with copies of the new last column, so
 * its output feeds the next step.  No reference counterpart (batching). */
DCELL_API size_t dcell_batch_tma_maps_bytes(int ncells);
DCELL_API int dcell_batch_tma_maps(const dcell_cell *cells, int ncells, const unsigned int *phi0_split,
                                   const float *vel, void *maps, void *stream);
DCELL_API int dcell_batch_sl_step_tc_split_tma(const dcell_cell *cells, int ncells, const dcell_tile *bricks,
                                               int nbricks, const void *maps, const unsigned int *phi0_split,
                                               const float *vel, int backtrace, float *phi, unsigned int *phi_split,
                                               int *flags, void *stream);

/* One explicit first-order conservative upwind step of phi on MAC faces:
 * LevelSetAdvectMAC (2D) / LevelSetAdvectMAC_3D, LevelSetMethod/AdvectMAC.c:
 * 18-111 (replaces them; the reference routines read the level set's grid
 * through members the current struct _LevelSet no longer has).  phi, u, v,
 * w (3D only; NULL in 2D) and out are device arrays on the grid g, x
 * fastest; u at (i, j, k) is the face between cells i-1 and i (v, w likewise
 * along y, z).  Per axis the updated global range is [max(p, 0), p + n - 1);
 * at global index 0 and at the range's last point the missing neighbour is
 * extrapolated as 2 phi - (the other neighbour), and
 *   out = phi + dt (du / h.x + dv / h.y (+ dw / h.z))
 * with each face's upwind product.  Points outside the ranges are not
 * written (the reference leaves its output level set's other values); out
 * must not alias phi.  The reference reads outside its grid when an updated
 * axis has p > 0 or n < 3: such grids return DCELL_ERR_UNSUPPORTED and
 * nothing is written.  DCELL_F64 gives the reference's bits. */
DCELL_API int dcell_advect_mac(const dcell_geom *g, int dtype, const void *phi, const void *u, const void *v,
                               const void *w, double dt, void *out, void *stream);

/* ------------------------------------------------------------------------
 * Host-buffer drop-in entry points (reference FP64 layout)
 * ---------------------------------------------------------------------- */
typedef struct dcell_session dcell_session;

/* A session owns device mirrors (grow-only) and a stream on one device. */
DCELL_API int dcell_session_create(int device, dcell_session **out);
DCELL_API int dcell_session_destroy(dcell_session *s);

/* LevelSetAdvectSL(ls, velgrid, dt) with ls->phi0->v1 = phi0, velgrid->v1 =
 * vel, ls->band = band and ls->phi->v1 = phi (updated in place at the band
 * points, or everywhere when band == NULL).  precision: DCELL_F64 computes in
 * FP64 (the reference's arithmetic, bit-identical for DCELL_LINEAR +
 * DCELL_EULER), DCELL_F32 in FP32.  DCELL_F32 + DCELL_CUBIC_TC on a dense 3D
 * grid runs the split-state step (phi0 carried as BF16 hi + lo, 2^-17
 * relative; dcell_sl_step_tc_split) pipelined with the copies: z-slabs are
 * stepped while later planes are still going up and finished slabs come
 * down.  Returns DCELL_ERR_DEPARTURE (after writing the clamped result) if a
 * departure point left the grid. */
DCELL_API int dcell_ls_advect_sl(dcell_session *s, const dcell_geom *g, const double *phi0, const double *vel, const int *band,
                       int nband, double dt, int interp, int backtrace, int precision, double *phi);

/* Device-resident level set: the reference's LevelSetAdvectAndReinit loop
 * (LevelSetMethod/Advect.c:33-50, called once per time step by DCell's
 * ls->Advect slot) without the round trip of phi through host memory.
 * dcell_ls_resident_set uploads phi (reference Grid layout, FP64 host) and
 * its band once and computes its irregular nodes; each
 * dcell_ls_resident_advect_and_reinit call then uploads only the step's
 * velocity (host, FP32 or FP64 by vel_dtype: FP32 halves the bytes) and runs
 * on the device GridCopy (phi0 <- phi), LevelSetAdvectSL (dense when `dense`
 * or no band, else the band points), LevelSetCFLIncrement (max |V| over the
 * irregular nodes of the level set before the step, Advect.c:54-111),
 * LevelSetUpdateIrregularNodeList, and, when loop->AdvectCount >
 * loop->AdvectThres or loop->CFLcount > loop->CFLthres, the reinitialisation
 * (dcell_reinitialize's bucketed march, band width loop->bandWidth) that
 * replaces phi's band; the counters live in `loop` as in struct _LevelSet.
 * The node pass of the step's new level set, and the reinitialisation a
 * step triggers (loop->reinitialized = 1), run before their results are
 * next used -- first thing in the next call, where they overlap that step's
 * velocity upload, or (the reinitialisation) in dcell_ls_resident_get -- so
 * loop->band reports the band before the reinitialisation and an error of
 * the node pass is returned by the next call; the results are those of
 * running both at the end of the step.
 * dcell_ls_resident_get downloads phi (FP64) and the band where the host
 * needs them (output, or a CPU fast marching instead of the device one).
 * precision: the arithmetic (DCELL_F32 with DCELL_CUBIC_TC on a dense 3D grid
 * carries the split state between steps, as dcell_sl_step_tc_split; on grids
 * of at least 32 planes the velocity then goes up in plane chunks while
 * z-slabs already step, with the bits of the unpipelined step).  One
 * resident level set per session; dcell_ls_resident_set replaces it. */
typedef struct dcell_ls_loop {
  double CFLcount, CFLthres, maxVel, bandWidth; /* struct _LevelSet's fields (LevelSetMethod.h:10-26) */
  int AdvectCount, AdvectThres;
  int reinitialized; /* out: 1 when this step triggered the reinitialisation */
  int band;          /* out: band points after the step (before a reinitialisation it triggered) */
} dcell_ls_loop;
DCELL_API int dcell_ls_resident_set(dcell_session *s, const dcell_geom *g, const double *phi, const int *band,
                                    int nband, int precision);
DCELL_API int dcell_ls_resident_advect_and_reinit(dcell_session *s, const dcell_geom *g, const void *vel,
                                                  int vel_dtype, double dt, int interp, int backtrace, int dense,
                                                  dcell_ls_loop *loop);
DCELL_API int dcell_ls_resident_get(dcell_session *s, const dcell_geom *g, double *phi, int *band, int capacity,
                                    int *nband);

/* LevelSetAdvectSLRK2HalfStep / LevelSetAdvectSLRK2FullStep (AdvectRK2.c:
 * 5-26) on host arrays in one call each: the half step first copies phi into
 * phi0 (GridCopy), then both advect phi from phi0 as dcell_ls_advect_sl does
 * (same arguments, same device paths, same results) and rebuild the
 * irregular-node list of the new phi as dcell_ls_update_irregular_nodes does,
 * with phi kept on the device between the two.  The status is that of the
 * pair (DCELL_ERR_DEPARTURE after writing phi and the nodes, as
 * dcell_ls_advect_sl). */
DCELL_API int dcell_ls_advect_sl_rk2_half(dcell_session *s, const dcell_geom *g, double *phi0, const double *vel,
                                          const int *band, int nband, double dt, int interp, int backtrace,
                                          int precision, double *phi, int with_surface, dcell_irregular_node *nodes,
                                          int capacity, int *count);
DCELL_API int dcell_ls_advect_sl_rk2_full(dcell_session *s, const dcell_geom *g, const double *phi0,
                                          const double *vel, const int *band, int nband, double dt, int interp,
                                          int backtrace, int precision, double *phi, int with_surface,
                                          dcell_irregular_node *nodes, int capacity, int *count);

/* LevelSetUpdateIrregularNodeList(ls) on host phi; *count = node count. */
DCELL_API int dcell_ls_update_irregular_nodes(dcell_session *s, const dcell_geom *g, const double *phi, const int *band,
                                    int nband, int with_surface, int precision, dcell_irregular_node *nodes,
                                    int capacity, int *count);

/* LevelSetReinitialize(ls) after its LevelSetResize, on host arrays (see
 * dcell_reinitialize): phi (FP64 host grid, overwritten), the irregular nodes
 * of phi (as dcell_ls_update_irregular_nodes returns them; only axis, pos,
 * signCenter and op are read), band_width = ls->bandWidth.  band (host int
 * [capacity][3]) receives the new band in grid order, *count its length.
 * precision: the arithmetic, DCELL_F64 or DCELL_F32. */
DCELL_API int dcell_ls_reinitialize(dcell_session *s, const dcell_geom *g, double *phi, const dcell_irregular_node *nodes,
                                    int nnodes, double band_width, int precision, int *band, int capacity, int *count);

/* LevelSetAdvectMAC / LevelSetAdvectMAC_3D on host FP64 arrays (see
 * dcell_advect_mac; w is NULL in 2D): out is read and updated in place at the
 * updated points.  precision: the arithmetic, DCELL_F64 (the reference's
 * bits) or DCELL_F32. */
DCELL_API int dcell_ls_advect_mac(dcell_session *s, const dcell_geom *g, const double *phi, const double *u,
                                  const double *v, const double *w, double dt, int precision, double *out);

/* LevelSet_MaxVelocity(ls, velgrid) on host arrays. */
DCELL_API int dcell_ls_max_velocity(dcell_session *s, const dcell_geom *g, const double *vel,
                          const dcell_irregular_node *nodes, int count, double *maxvel);

/* The particle level set on host arrays (FP64, the reference's layout):
 * particles are ls->pls->particles' struct _Particle records.  rng is the
 * drand48 state (in/out).  Seed and reseed write at most capacity records
 * and return DCELL_ERR_CAPACITY when *count exceeds it. */
DCELL_API int dcell_ls_pls_advect(dcell_session *s, const dcell_geom *g, const double *vel, double *particles,
                                  long long n, double dt);
DCELL_API int dcell_ls_pls_correct(dcell_session *s, const dcell_geom *g, double *phi, const int *band, int nband,
                                   const double *particles, long long n);
DCELL_API int dcell_ls_pls_adjust_radii(dcell_session *s, const dcell_geom *g, const double *phi, double *particles,
                                        long long n, const dcell_pls_params *prm);
DCELL_API int dcell_ls_pls_seed(dcell_session *s, const dcell_geom *g, const double *phi, const int *band, int nband,
                                const dcell_pls_params *prm, unsigned long long *rng, double *particles,
                                long long capacity, long long *count);
DCELL_API int dcell_ls_pls_reseed(dcell_session *s, const dcell_geom *g, const double *phi, const int *band,
                                  int nband, const dcell_pls_params *prm, unsigned long long *rng, double *particles,
                                  long long n, long long capacity, long long *count);

/* ------------------------------------------------------------------------
 * Output in the reference's file formats, written asynchronously
 * ---------------------------------------------------------------------- */
typedef struct dcell_writer dcell_writer;

/* A writer with a background thread; dir receives grids and node lists,
 * tmpdir (NULL: $PETSC_TMP, else /tmp) the particle arrays, as PetscGetTmp
 * directs the reference's ArrayWrite.  Device writes use `device`. */
DCELL_API int dcell_writer_create(const char *dir, const char *tmpdir, int device, dcell_writer **out);
/* Waits for every pending write; returns the first error since the last flush. */
DCELL_API int dcell_writer_flush(dcell_writer *w);
DCELL_API int dcell_writer_destroy(dcell_writer *w);

/* GridWrite (Common/Serialize.c:23-55): <dir>/<name>.<t+10000>.Real64 in
 * PETSc's binary Vec format (big-endian int32 class id 1211214, int32
 * length, FP64 values; FP32 data is widened), its .info companion
 * ("-vecload_block_size <dof>" for dof > 1), and one line "px py [pz]" /
 * "nx ny [nz]" appended to <dir>/<name>.pos / .size (truncated by this
 * writer's first write).  data: the grid's dof values per point on the device
 * (dcell_writer_grid; snapshotted on `stream`, the caller may overwrite it
 * once the stream passes this call) or FP64 on the host. */
DCELL_API int dcell_writer_grid(dcell_writer *w, const char *name, int t, const dcell_geom *g, int dof, int dtype,
                                const void *data, void *stream);
DCELL_API int dcell_writer_grid_host(dcell_writer *w, const char *name, int t, const dcell_geom *g, int dof,
                                     const double *data);

/* LevelSetWriteIrregularNodeList (LevelSetMethod/IrregularNodes.c:145-246):
 * <dir>/<name>.irregNode.<idx+10000>.array, big-endian FP64 rows -- 2D: X,
 * pos, n, f1, fa1, k, f1_n, f1_nn (11) for nodes with axis != -1; 3D: X, pos,
 * n, k and the 13 IIM quantities (23) for every node.  IIM quantities this
 * path does not compute are 0.  count is a device int (dcell_irregular_nodes'
 * output) for the device form. */
DCELL_API int dcell_writer_irregular_nodes(dcell_writer *w, const char *name, int idx, int dim,
                                           const dcell_irregular_node *nodes, const int *count, int capacity,
                                           void *stream);
DCELL_API int dcell_writer_irregular_nodes_host(dcell_writer *w, const char *name, int idx, int dim,
                                                const dcell_irregular_node *nodes, int count);

/* ArrayWrite of the particle Array (Common/Array.c:133-150, via
 * ParticleLSWriteParticles, ParticleLS.c:190-198): <tmpdir>/<name>.<t+10000>.array,
 * the n records as native FP64 (FP32 data is widened). */
DCELL_API int dcell_writer_particles(dcell_writer *w, const char *name, int t, const void *particles, long long n,
                                     int dtype, void *stream);
DCELL_API int dcell_writer_particles_host(dcell_writer *w, const char *name, int t, const double *particles,
                                          long long n);

/* ------------------------------------------------------------------------
 * Diagnostics
 * ---------------------------------------------------------------------- */

/* D = bf16(A) * M^T on the tensor-core path of DCELL_CUBIC_TC, where M is
 * the 64x64 Catmull-Rom operator of TricubicInverse.h; A (128 x 64) and D
 * (128 x 64) are row-major FP32 device arrays.  Checks the MMA operand
 * layouts on the running GPU against a host product. */
DCELL_API int dcell_tc_gemm_check(const float *a, float *d, int *flags, void *stream);

/* The give-up path of the device-side waits: one thread waits, with both
 * bounded mbarrier waits the tensor-core kernels use (polling, then
 * suspending), on a phase that nothing completes.  *result (a device int)
 * receives 1 if the polling wait gave up, + 2 if the suspending one did
 * (3 expected, within about a second); the context stays usable. */
DCELL_API int dcell_wait_timeout_check(int *result, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DCELL_LS_H_ */
