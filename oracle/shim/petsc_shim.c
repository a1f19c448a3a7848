/*
 * Implementation of the PETSc / GA stand-in declared in petsc.h and ga.h.
 * Test infrastructure only: it lets the reference's own level-set C compile
 * and run so its FP64 results can serve as the oracle.
 */
#include <stdarg.h>

#include "petsc.h"
#include "ga.h"

int dcell_shim_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, "[reference error %d] ", code);
  vfprintf(stderr, fmt, ap);
  fprintf(stderr, "\n");
  va_end(ap);
  return code;
}

int dcell_shim_malloc(size_t bytes, void **out) {
  *out = malloc(bytes ? bytes : 1);
  return *out ? 0 : PETSC_ERR_MEM;
}

int dcell_shim_calloc(size_t bytes, void **out) {
  *out = calloc(1, bytes ? bytes : 1);
  return *out ? 0 : PETSC_ERR_MEM;
}

PetscErrorCode VecCreateSeqWithArray(MPI_Comm c, PetscInt bs, PetscInt n, const PetscScalar *a, Vec *v) {
  (void)c;
  Vec x = (Vec)calloc(1, sizeof(*x));
  if (!x) return PETSC_ERR_MEM;
  x->array = (PetscScalar *)a;
  x->n = n;
  x->bs = bs;
  *v = x;
  return 0;
}

PetscErrorCode VecDestroy(Vec *v) {
  if (v && *v) {
    free(*v);
    *v = NULL;
  }
  return 0;
}

PetscErrorCode VecZeroEntries(Vec v) {
  memset(v->array, 0, sizeof(PetscScalar) * (size_t)v->n);
  return 0;
}

PetscErrorCode VecSet(Vec v, PetscScalar s) {
  for (PetscInt i = 0; i < v->n; ++i) v->array[i] = s;
  return 0;
}

PetscErrorCode VecCopy(Vec x, Vec y) {
  if (x->n != y->n) return dcell_shim_error(60, "VecCopy: sizes %d != %d", x->n, y->n);
  memmove(y->array, x->array, sizeof(PetscScalar) * (size_t)x->n);
  return 0;
}

PetscErrorCode VecView(Vec v, PetscViewer w) {
  (void)v;
  (void)w;
  return 0;
}

/* 2-d table: one block holding m row pointers; a[i] = array + (i-ms)*n - ns. */
PetscErrorCode VecGetArray2d(Vec x, PetscInt m, PetscInt n, PetscInt ms, PetscInt ns, PetscScalar ***a) {
  PetscScalar **rows = (PetscScalar **)malloc(sizeof(PetscScalar *) * (size_t)(m > 0 ? m : 1));
  if (!rows) return PETSC_ERR_MEM;
  for (PetscInt i = 0; i < m; ++i) rows[i] = x->array + (ptrdiff_t)i * n - ns;
  *a = rows - ms;
  return 0;
}

PetscErrorCode VecRestoreArray2d(Vec x, PetscInt m, PetscInt n, PetscInt ms, PetscInt ns, PetscScalar ***a) {
  (void)x; (void)m; (void)n; (void)ns;
  if (*a) free(*a + ms);
  *a = NULL;
  return 0;
}

/* 3-d table: one block = [m plane pointers][m*n row pointers]. */
PetscErrorCode VecGetArray3d(Vec x, PetscInt m, PetscInt n, PetscInt p, PetscInt ms, PetscInt ns, PetscInt ps,
                             PetscScalar ****a) {
  size_t np = (size_t)(m > 0 ? m : 1), nr = (size_t)(m * n > 0 ? m * n : 1);
  void **blk = (void **)malloc(sizeof(void *) * (np + nr));
  if (!blk) return PETSC_ERR_MEM;
  PetscScalar ***planes = (PetscScalar ***)blk;
  PetscScalar **rows = (PetscScalar **)(blk + np);
  for (PetscInt i = 0; i < m; ++i) {
    for (PetscInt j = 0; j < n; ++j) rows[i * n + j] = x->array + ((ptrdiff_t)i * n + j) * p - ps;
    planes[i] = rows + (ptrdiff_t)i * n - ns;
  }
  *a = planes - ms;
  return 0;
}

PetscErrorCode VecRestoreArray3d(Vec x, PetscInt m, PetscInt n, PetscInt p, PetscInt ms, PetscInt ns,
                                 PetscInt ps, PetscScalar ****a) {
  (void)x; (void)m; (void)n; (void)p; (void)ns; (void)ps;
  if (*a) free(*a + ms);
  *a = NULL;
  return 0;
}

/* 4-d table: one block = [m][m*n][m*n*p] pointers. */
PetscErrorCode VecGetArray4d(Vec x, PetscInt m, PetscInt n, PetscInt p, PetscInt q, PetscInt ms, PetscInt ns,
                             PetscInt ps, PetscInt qs, PetscScalar *****a) {
  size_t n1 = (size_t)(m > 0 ? m : 1), n2 = (size_t)(m * n > 0 ? m * n : 1),
         n3 = (size_t)(m * n * p > 0 ? m * n * p : 1);
  void **blk = (void **)malloc(sizeof(void *) * (n1 + n2 + n3));
  if (!blk) return PETSC_ERR_MEM;
  PetscScalar ****l1 = (PetscScalar ****)blk;
  PetscScalar ***l2 = (PetscScalar ***)(blk + n1);
  PetscScalar **l3 = (PetscScalar **)(blk + n1 + n2);
  for (PetscInt i = 0; i < m; ++i) {
    for (PetscInt j = 0; j < n; ++j) {
      for (PetscInt k = 0; k < p; ++k)
        l3[(i * n + j) * p + k] = x->array + (((ptrdiff_t)i * n + j) * p + k) * q - qs;
      l2[i * n + j] = l3 + ((ptrdiff_t)i * n + j) * p - ps;
    }
    l1[i] = l2 + (ptrdiff_t)i * n - ns;
  }
  *a = l1 - ms;
  return 0;
}

PetscErrorCode VecRestoreArray4d(Vec x, PetscInt m, PetscInt n, PetscInt p, PetscInt q, PetscInt ms,
                                 PetscInt ns, PetscInt ps, PetscInt qs, PetscScalar *****a) {
  (void)x; (void)m; (void)n; (void)p; (void)q; (void)ns; (void)ps; (void)qs;
  if (*a) free(*a + ms);
  *a = NULL;
  return 0;
}

PetscErrorCode PetscViewerDestroy(PetscViewer *v) { if (v) *v = NULL; return 0; }
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm c, const char *name, PetscFileMode m, PetscViewer *v) {
  (void)c; (void)name; (void)m; *v = NULL; return 0;
}
PetscErrorCode PetscViewerASCIIOpen(MPI_Comm c, const char *name, PetscViewer *v) {
  (void)c; (void)name; *v = NULL; return 0;
}
PetscErrorCode PetscViewerASCIIPrintf(PetscViewer v, const char *fmt, ...) { (void)v; (void)fmt; return 0; }
PetscErrorCode PetscViewerBinaryWrite(PetscViewer v, void *d, PetscInt n, PetscDataType t, PetscBool tmp) {
  (void)v; (void)d; (void)n; (void)t; (void)tmp; return 0;
}
PetscErrorCode PetscGetTmp(MPI_Comm c, char *dir, size_t len) { (void)c; snprintf(dir, len, "/tmp"); return 0; }
PetscErrorCode PetscGetWorkingDirectory(char *dir, size_t len) { snprintf(dir, len, "."); return 0; }
PetscErrorCode PetscBinaryOpen(const char *name, PetscFileMode m, int *fd) { (void)name; (void)m; *fd = -1; return 0; }
PetscErrorCode PetscBinaryWrite(int fd, void *p, PetscInt n, PetscDataType t, PetscBool tmp) {
  (void)fd; (void)p; (void)n; (void)t; (void)tmp; return 0;
}
PetscErrorCode PetscBinaryClose(int fd) { (void)fd; return 0; }
PetscErrorCode MatView(Mat m, PetscViewer v) { (void)m; (void)v; return 0; }
int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return 0; }

/* A one-process Global Array: one double array with dims[ndim] (row major,
 * last index fastest), registered by the driver (dref_ga_set).  NGA_Get
 * copies the patch [lo, hi] (inclusive) into buf, whose trailing extents are
 * ld[0..ndim-2] (Global Arrays' NGA_Get contract; an empty patch copies
 * nothing); NGA_Inquire reports the dims.  Enough for LevelSetGetVelocity
 * (Advect.c:145-192) to run as written. */
static const double *shim_ga_data = NULL;
static int shim_ga_ndim = 0, shim_ga_dims[4] = {0, 0, 0, 0};

void dref_ga_set(const double *data, int ndim, const int *dims) {
  shim_ga_data = data;
  shim_ga_ndim = ndim;
  for (int i = 0; i < 4; ++i) shim_ga_dims[i] = i < ndim ? dims[i] : 0;
}

void NGA_Get(int g_a, int lo[], int hi[], void *buf, int ld[]) {
  (void)g_a;
  double *out = (double *)buf;
  const int nd = shim_ga_ndim;
  if (!shim_ga_data || nd < 2) {
    fprintf(stderr, "[oracle shim] NGA_Get without a registered array\n");
    return;
  }
  int idx[4] = {0, 0, 0, 0};
  for (int d = 0; d < nd; ++d) {
    if (hi[d] < lo[d]) return; /* empty patch */
    idx[d] = lo[d];
  }
  for (;;) {
    size_t src = 0, dst = 0;
    for (int d = 0; d < nd; ++d) {
      src = src * (size_t)shim_ga_dims[d] + (size_t)idx[d];
      dst = d == 0 ? (size_t)(idx[0] - lo[0]) : dst * (size_t)ld[d - 1] + (size_t)(idx[d] - lo[d]);
    }
    out[dst] = shim_ga_data[src];
    int d = nd - 1;
    while (d >= 0 && ++idx[d] > hi[d]) {
      idx[d] = lo[d];
      --d;
    }
    if (d < 0) break;
  }
}
void NGA_Inquire(int g_a, int *type, int *ndim, int dims[]) {
  (void)g_a;
  *type = 0;
  *ndim = shim_ga_ndim;
  for (int i = 0; i < 4; ++i) dims[i] = shim_ga_dims[i];
}

/* PETSCRAND48: the C library's drand48 (POSIX: X <- (0x5DEECE66D X + 0xB)
 * mod 2^48, value X / 2^48), seeded with srand48 when the type is set. */
struct dcell_shim_random {
  long seed;
};

PetscErrorCode PetscRandomCreate(MPI_Comm c, PetscRandom *r) {
  int rank = 0;
  (void)c;
  MPI_Comm_rank(c, &rank);
  *r = (PetscRandom)calloc(1, sizeof(struct dcell_shim_random));
  if (!*r) return PETSC_ERR_MEM;
  (*r)->seed = 0x12345678 + 76543 * rank;
  return 0;
}
PetscErrorCode PetscRandomSetType(PetscRandom r, PetscRandomType t) {
  if (strcmp(t, PETSCRAND48)) return dcell_shim_error(PETSC_ERR_ARG_OUTOFRANGE, "random type %s", t);
  srand48(r->seed);
  return 0;
}
PetscErrorCode PetscRandomGetValue(PetscRandom r, PetscScalar *v) {
  (void)r;
  *v = drand48();
  return 0;
}
PetscErrorCode PetscRandomDestroy(PetscRandom *r) {
  free(*r);
  *r = NULL;
  return 0;
}

/* Symbols referenced by the compiled files but defined in subsystems the
 * oracle does not build (GA gather glue, file output). */
typedef struct _Array *Array;
PetscErrorCode GAGather(int ga, Array c, Array v) { (void)ga; (void)c; (void)v; return 1; }
PetscErrorCode DCellGetWorkingDirectory(char *wd) { strcpy(wd, "."); return 0; }
typedef struct _Grid *Grid;
PetscErrorCode GridWrite(Grid g, int t) { (void)g; (void)t; return 0; }
