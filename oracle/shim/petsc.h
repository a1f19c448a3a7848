/*
 * Minimal PETSc stand-in used ONLY to compile the reference's level-set hot
 * path (LevelSetMethod/, Common/) on a machine without PETSc, GA or MPI.
 *
 * This is test infrastructure for the oracle: it supplies the container and
 * bookkeeping vocabulary the reference uses (PetscReal = double, Vec backed by
 * a caller array, offset N-d pointer tables, error macros, no-op logging and
 * options).  None of the reference's arithmetic goes through it, so results of
 * the compiled reference are the reference's own FP64 results.
 *
 * Semantics restated from PETSc's public documentation:
 *  - VecGetArrayNd(x, m, n, ..., mstart, nstart, ..., &a) returns a table with
 *    a[i][j]... == array[((i-mstart)*n + (j-nstart))...], i.e. row-major with
 *    the LAST index fastest and per-axis start offsets.
 *  - PetscFree(p) frees and zeroes p.
 *  - CHKERRQ(e) returns e from the calling function when e != 0.
 */
#ifndef DCELL_ORACLE_PETSC_SHIM_H
#define DCELL_ORACLE_PETSC_SHIM_H

#include <float.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef double PetscReal;
typedef double PetscScalar;
typedef int PetscInt;
typedef int PetscErrorCode;
typedef int PetscLogEvent;
typedef int PetscClassId;
typedef int MPI_Comm;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef enum { PETSC_INT = 0, PETSC_DOUBLE = 1, PETSC_CHAR = 2 } PetscDataType;
typedef enum { FILE_MODE_READ = 0, FILE_MODE_WRITE = 1, FILE_MODE_APPEND = 2 } PetscFileMode;

typedef struct dcell_shim_vec {
  PetscScalar *array;
  PetscInt n;
  PetscInt bs;
} *Vec;
typedef void *Mat;
typedef void *DM;
typedef void *PetscViewer;
typedef struct dcell_shim_random *PetscRandom;
typedef const char *PetscRandomType;
#define PETSCRAND48 "rand48"

#define PETSC_COMM_SELF 0
#define PETSC_COMM_WORLD 1
#define PETSC_MAX_PATH_LEN 4096
#define PETSC_PI 3.14159265358979323846264
#define PETSC_MAX_REAL DBL_MAX
#define PETSC_ERR_ARG_OUTOFRANGE 63
#define PETSC_ERR_MEM 55
#define PETSC_DECIDE (-1)

int dcell_shim_error(int code, const char *fmt, ...);
int dcell_shim_malloc(size_t bytes, void **out);
int dcell_shim_calloc(size_t bytes, void **out);

#define PetscFunctionBegin
#define PetscFunctionReturn(x) return (x)
#define CHKERRQ(e) do { if (e) return (e); } while (0)
#define CHKMEMQ
#define SETERRQ(c, n, s) return dcell_shim_error((n), "%s", (s))
#define SETERRQ1(c, n, ...) return dcell_shim_error((n), __VA_ARGS__)
#define SETERRQ2(c, n, ...) return dcell_shim_error((n), __VA_ARGS__)
#define SETERRQ3(c, n, ...) return dcell_shim_error((n), __VA_ARGS__)

#define PetscMalloc(sz, pp) dcell_shim_malloc((size_t)(sz), (void **)(pp))
#define PetscNew(type, pp) dcell_shim_calloc(sizeof(type), (void **)(pp))
#define PetscFree(p) ((p) ? (free(p), (p) = 0, 0) : 0)
#define PetscMemzero(p, n) (memset((p), 0, (size_t)(n)), 0)
#define PetscMemcpy(d, s, n) (memcpy((d), (s), (size_t)(n)), 0)
#define PetscStrcpy(d, s) (strcpy((d), (s)), 0)
#define PetscSNPrintf(b, l, ...) (snprintf((b), (size_t)(l), __VA_ARGS__), 0)

#define PetscSqr(x) ((x) * (x))
#define PetscSqrtScalar(x) sqrt(x)
#define PetscAbs(x) (((x) < 0) ? -(x) : (x))
#define PetscMax(a, b) (((a) < (b)) ? (b) : (a))
#define PetscMin(a, b) (((a) < (b)) ? (a) : (b))
#define PetscSign(a) (((a) >= 0) ? ((a) == 0 ? 0 : 1) : -1)

/* logging, info and options: accepted and ignored */
#define PetscInfo(o, ...) 0
#define PetscInfo1(o, ...) 0
#define PetscInfo2(o, ...) 0
#define PetscInfo3(o, ...) 0
#define PetscInfo4(o, ...) 0
#define PetscInfo5(o, ...) 0
#define PetscLogEventRegister(name, cls, ev) (*(ev) = 0, 0)
#define PetscLogEventBegin(e, a, b, c, d) 0
#define PetscLogEventEnd(e, a, b, c, d) 0
#define PetscOptionsGetReal(pre, name, val, flg) 0
#define PetscOptionsGetInt(pre, name, val, flg) 0
#define PetscOptionsGetBool(pre, name, val, flg) 0

/* vectors */
PetscErrorCode VecCreateSeqWithArray(MPI_Comm c, PetscInt bs, PetscInt n, const PetscScalar *a, Vec *v);
PetscErrorCode VecDestroy(Vec *v);
PetscErrorCode VecZeroEntries(Vec v);
PetscErrorCode VecSet(Vec v, PetscScalar s);
PetscErrorCode VecCopy(Vec x, Vec y);
PetscErrorCode VecView(Vec v, PetscViewer w);
PetscErrorCode VecGetArray2d(Vec x, PetscInt m, PetscInt n, PetscInt ms, PetscInt ns, PetscScalar ***a);
PetscErrorCode VecRestoreArray2d(Vec x, PetscInt m, PetscInt n, PetscInt ms, PetscInt ns, PetscScalar ***a);
PetscErrorCode VecGetArray3d(Vec x, PetscInt m, PetscInt n, PetscInt p, PetscInt ms, PetscInt ns, PetscInt ps,
                             PetscScalar ****a);
PetscErrorCode VecRestoreArray3d(Vec x, PetscInt m, PetscInt n, PetscInt p, PetscInt ms, PetscInt ns,
                                 PetscInt ps, PetscScalar ****a);
PetscErrorCode VecGetArray4d(Vec x, PetscInt m, PetscInt n, PetscInt p, PetscInt q, PetscInt ms, PetscInt ns,
                             PetscInt ps, PetscInt qs, PetscScalar *****a);
PetscErrorCode VecRestoreArray4d(Vec x, PetscInt m, PetscInt n, PetscInt p, PetscInt q, PetscInt ms,
                                 PetscInt ns, PetscInt ps, PetscInt qs, PetscScalar *****a);

/* random numbers: PETSCRAND48 draws from the C library's drand48 stream
 * (one global state, seeded by srand48(seed) when the type is set; the
 * default seed is 0x12345678 + 76543 * rank), values in [0, 1). */
PetscErrorCode PetscRandomCreate(MPI_Comm c, PetscRandom *r);
PetscErrorCode PetscRandomSetType(PetscRandom r, PetscRandomType t);
PetscErrorCode PetscRandomGetValue(PetscRandom r, PetscScalar *v);
PetscErrorCode PetscRandomDestroy(PetscRandom *r);

/* viewers and files: the oracle never writes files */
PetscErrorCode PetscViewerDestroy(PetscViewer *v);
PetscErrorCode PetscViewerBinaryOpen(MPI_Comm c, const char *name, PetscFileMode m, PetscViewer *v);
PetscErrorCode PetscViewerASCIIOpen(MPI_Comm c, const char *name, PetscViewer *v);
PetscErrorCode PetscViewerASCIIPrintf(PetscViewer v, const char *fmt, ...);
PetscErrorCode PetscViewerBinaryWrite(PetscViewer v, void *data, PetscInt n, PetscDataType t, PetscBool istemp);
PetscErrorCode PetscGetTmp(MPI_Comm c, char *dir, size_t len);
PetscErrorCode PetscGetWorkingDirectory(char *dir, size_t len);
PetscErrorCode PetscBinaryOpen(const char *name, PetscFileMode m, int *fd);
PetscErrorCode PetscBinaryWrite(int fd, void *p, PetscInt n, PetscDataType t, PetscBool istemp);
PetscErrorCode PetscBinaryClose(int fd);
PetscErrorCode MatView(Mat m, PetscViewer v);
int MPI_Comm_rank(MPI_Comm c, int *rank);

#endif /* DCELL_ORACLE_PETSC_SHIM_H */
