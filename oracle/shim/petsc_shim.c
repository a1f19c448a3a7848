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

/* File viewers.  PETSc is absent, so its binary format is restated from its
 * documentation: big-endian values; a Vec is the class id 1211214 (int32),
 * its length (int32), then its values; a binary viewer opened for writing
 * creates `<name>.info` beside the file, into which VecView writes
 * "-vecload_block_size <bs>" for a block size above one. */
struct dcell_shim_viewer {
  FILE *f;    /* the file */
  FILE *info; /* binary viewers: <name>.info */
  int binary;
};

static void put_be(FILE *f, const void *p, size_t elem, size_t n) {
  const unsigned char *b = (const unsigned char *)p;
  for (size_t i = 0; i < n; ++i)
    for (size_t k = 0; k < elem; ++k) fputc(b[i * elem + (elem - 1 - k)], f);
}

PetscErrorCode VecView(Vec v, PetscViewer w) {
  struct dcell_shim_viewer *sv = (struct dcell_shim_viewer *)w;
  if (!sv || !sv->binary) return 0;
  const int head[2] = {1211214, v->n};
  put_be(sv->f, head, sizeof(int), 2);
  put_be(sv->f, v->array, sizeof(double), (size_t)v->n);
  if (v->bs > 1 && sv->info) fprintf(sv->info, "-vecload_block_size %d\n", v->bs);
  return ferror(sv->f) ? dcell_shim_error(66, "VecView: write failed") : 0;
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

PetscErrorCode PetscViewerDestroy(PetscViewer *v) {
  if (v && *v) {
    struct dcell_shim_viewer *sv = (struct dcell_shim_viewer *)*v;
    if (sv->f) fclose(sv->f);
    if (sv->info) fclose(sv->info);
    free(sv);
  }
  if (v) *v = NULL;
  return 0;
}
static PetscErrorCode open_viewer(const char *name, int binary, PetscViewer *v) {
  struct dcell_shim_viewer *sv = (struct dcell_shim_viewer *)calloc(1, sizeof(*sv));
  if (!sv) return PETSC_ERR_MEM;
  sv->binary = binary;
  sv->f = fopen(name, binary ? "wb" : "w");
  if (!sv->f) {
    free(sv);
    return dcell_shim_error(65, "cannot open %s", name);
  }
  if (binary) {
    char info[PETSC_MAX_PATH_LEN];
    snprintf(info, sizeof info, "%s.info", name);
    sv->info = fopen(info, "w");
  }
  *v = sv;
  return 0;
}
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm c, const char *name, PetscFileMode m, PetscViewer *v) {
  (void)c;
  if (m != FILE_MODE_WRITE) return dcell_shim_error(56, "PetscViewerBinaryOpen: only FILE_MODE_WRITE is supported");
  return open_viewer(name, 1, v);
}
PetscErrorCode PetscViewerASCIIOpen(MPI_Comm c, const char *name, PetscViewer *v) {
  (void)c;
  return open_viewer(name, 0, v);
}
PetscErrorCode PetscViewerASCIIPrintf(PetscViewer v, const char *fmt, ...) {
  struct dcell_shim_viewer *sv = (struct dcell_shim_viewer *)v;
  if (!sv) return 0;
  va_list ap;
  va_start(ap, fmt);
  vfprintf(sv->f, fmt, ap);
  va_end(ap);
  fflush(sv->f);
  return 0;
}
PetscErrorCode PetscViewerBinaryWrite(PetscViewer v, void *d, PetscInt n, PetscDataType t, PetscBool tmp) {
  struct dcell_shim_viewer *sv = (struct dcell_shim_viewer *)v;
  (void)tmp;
  if (!sv) return 0;
  if (t == PETSC_DOUBLE) put_be(sv->f, d, sizeof(double), (size_t)n);
  else if (t == PETSC_INT) put_be(sv->f, d, sizeof(int), (size_t)n);
  else fwrite(d, 1, (size_t)n, sv->f);
  return 0;
}
/* Output directories of the reference's writers: DCellGetWorkingDirectory
 * (grids, node lists) and PetscGetTmp (Array files); set by the driver. */
static char g_wd[PETSC_MAX_PATH_LEN] = ".";
static char g_tmp[PETSC_MAX_PATH_LEN] = "/tmp";
void dcell_shim_set_dirs(const char *wd, const char *tmp) {
  if (wd) snprintf(g_wd, sizeof g_wd, "%s", wd);
  if (tmp) snprintf(g_tmp, sizeof g_tmp, "%s", tmp);
}
PetscErrorCode PetscGetTmp(MPI_Comm c, char *dir, size_t len) { (void)c; snprintf(dir, len, "%s", g_tmp); return 0; }
PetscErrorCode PetscGetWorkingDirectory(char *dir, size_t len) { snprintf(dir, len, "%s", g_wd); return 0; }
/* PetscBinaryOpen / Write / Close over a FILE * kept in a small table. */
static FILE *g_bin[16];
PetscErrorCode PetscBinaryOpen(const char *name, PetscFileMode m, int *fd) {
  if (m != FILE_MODE_WRITE) return dcell_shim_error(56, "PetscBinaryOpen: only FILE_MODE_WRITE is supported");
  for (int i = 0; i < 16; ++i)
    if (!g_bin[i]) {
      g_bin[i] = fopen(name, "wb");
      if (!g_bin[i]) return dcell_shim_error(65, "cannot open %s", name);
      *fd = i;
      return 0;
    }
  return dcell_shim_error(55, "PetscBinaryOpen: too many open files");
}
PetscErrorCode PetscBinaryWrite(int fd, void *p, PetscInt n, PetscDataType t, PetscBool tmp) {
  (void)tmp;
  if (fd < 0 || fd >= 16 || !g_bin[fd]) return dcell_shim_error(62, "PetscBinaryWrite: bad descriptor");
  if (t == PETSC_DOUBLE) put_be(g_bin[fd], p, sizeof(double), (size_t)n);
  else if (t == PETSC_INT) put_be(g_bin[fd], p, sizeof(int), (size_t)n);
  else fwrite(p, 1, (size_t)n, g_bin[fd]);
  return 0;
}
PetscErrorCode PetscBinaryClose(int fd) {
  if (fd >= 0 && fd < 16 && g_bin[fd]) {
    fclose(g_bin[fd]);
    g_bin[fd] = NULL;
  }
  return 0;
}
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
/* The reference's own DCellGetWorkingDirectory (Common/Serialize.c:9-19)
 * caches the directory in a `static const` array, which gcc places in
 * read-only memory; its object's definition is weakened at link time and this
 * one, returning the same directory (PetscGetWorkingDirectory's), is used. */
PetscErrorCode DCellGetWorkingDirectory(char *wd) { return PetscGetWorkingDirectory(wd, PETSC_MAX_PATH_LEN); }
