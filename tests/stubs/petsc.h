/* Minimal declarations of the PETSc API subset used by vpfhf_b200/petsc/VFMech_gpu.c and
 * the reference headers it includes -- for a compile-only check of the adapter where PETSc
 * is not installed (tests/test_petsc_adapter.py).  Not an implementation. */
#ifndef VFGPU_TEST_PETSC_STUB_H
#define VFGPU_TEST_PETSC_STUB_H
#include <stdio.h>
typedef double PetscReal;
typedef double PetscScalar;
typedef int PetscInt;
typedef int PetscMPIInt;
typedef int PetscErrorCode;
typedef enum { PETSC_FALSE, PETSC_TRUE } PetscBool;
typedef int MPI_Comm;
typedef struct _p_Vec *Vec;
typedef struct _p_Mat *Mat;
typedef struct _p_DM *DM;
typedef struct _p_SNES *SNES;
typedef struct _p_KSP *KSP;
typedef struct _p_PC *PC;
typedef struct _p_TS *TS;
typedef struct _p_IS *IS;
typedef struct _p_PetscViewer *PetscViewer;
typedef struct _p_PetscOptions *PetscOptions;
#define PETSC_MAX_PATH_LEN 4096
#define PETSC_COMM_WORLD 0
#define PETSC_COMM_SELF 1
#define PETSC_ERR_SUP 56
#define PETSC_ERR_LIB 76
#define PETSC_PI 3.14159265358979323846
#define SETERRQ(c, n, s) return (n)
#define SETERRQ2(c, n, s, a, b) return (n)
#define CHKERRQ(e) do { if (e) return (e); } while (0)
#define PetscFunctionBegin
#define PetscFunctionReturn(x) return (x)
int MPI_Comm_size(MPI_Comm, PetscMPIInt *);
PetscErrorCode DMDAGetInfo(DM, PetscInt *, PetscInt *, PetscInt *, PetscInt *, PetscInt *,
                           PetscInt *, PetscInt *, PetscInt *, PetscInt *, void *, void *, void *,
                           void *);
PetscErrorCode DMDAGetBoundingBox(DM, PetscReal[], PetscReal[]);
PetscErrorCode VecGetArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar **);
PetscErrorCode VecGetArray(Vec, PetscScalar **);
PetscErrorCode VecRestoreArray(Vec, PetscScalar **);
PetscErrorCode VecMin(Vec, PetscInt *, PetscReal *);
PetscErrorCode VecMax(Vec, PetscInt *, PetscReal *);
PetscErrorCode PetscPrintf(MPI_Comm, const char[], ...);
PetscErrorCode PetscMalloc(size_t, void *);
PetscErrorCode PetscFree(void *);
PetscErrorCode PetscOptionsGetInt(PetscOptions, const char[], const char[], PetscInt *, PetscBool *);
#endif
