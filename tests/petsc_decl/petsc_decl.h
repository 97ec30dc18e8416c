/* petsc_decl.h -- declarations only (no definitions) of the part of PETSc's public C API
 * that fr_sdg_b200/petsc/frsdg_petsc.cpp uses, with PETSc 3.21's signatures as its manual
 * pages give them, so that the adapter can be type-checked and compiled to an object
 * without a PETSc installation.  Test infrastructure: nothing links against it. */
#pragma once
#include <stddef.h>

typedef int PetscErrorCode;
typedef int PetscMPIInt;
typedef int PetscInt;
typedef double PetscReal;
typedef double PetscScalar;
typedef enum { PETSC_FALSE, PETSC_TRUE } PetscBool;
typedef const char* VecType;
typedef struct _p_PetscObject* PetscObject;
typedef struct _p_Vec* Vec;
typedef struct _p_Mat* Mat;
typedef struct _p_DM* DM;
typedef struct _p_TS* TS;
typedef struct _p_PC* PC;
typedef struct _p_ompi_comm* MPI_Comm;

#define PETSC_SUCCESS ((PetscErrorCode)0)
enum { PETSC_ERR_SUP = 56, PETSC_ERR_ARG_WRONG = 62, PETSC_ERR_ARG_INCOMP = 75, PETSC_ERR_LIB = 76 };
extern MPI_Comm PETSC_COMM_SELF_decl;
#define PETSC_COMM_SELF PETSC_COMM_SELF_decl

PetscErrorCode PetscError(MPI_Comm, int, const char*, const char*, PetscErrorCode, int, const char*, ...);
#define PetscFunctionBeginUser do { } while (0)
#define PetscFunctionReturn(x) return (x)
#define PetscCall(x) do { PetscErrorCode ierr_ = (x); if (ierr_) return ierr_; } while (0)
#define SETERRQ(comm, code, ...) return PetscError(comm, __LINE__, __func__, __FILE__, code, 1, __VA_ARGS__)

typedef enum { INSERT_VALUES = 1 } InsertMode;
typedef enum { DM_BOUNDARY_NONE, DM_BOUNDARY_GHOSTED, DM_BOUNDARY_MIRROR, DM_BOUNDARY_PERIODIC,
               DM_BOUNDARY_TWIST } DMBoundaryType;
typedef enum { DMDA_STENCIL_STAR, DMDA_STENCIL_BOX } DMDAStencilType;
typedef enum { MATOP_MULT = 3 } MatOperation;

PetscErrorCode PetscObjectGetComm(PetscObject, MPI_Comm*);
int MPI_Comm_size(MPI_Comm, int*);

PetscErrorCode VecGetLocalSize(Vec, PetscInt*);
PetscErrorCode VecGetSize(Vec, PetscInt*);
PetscErrorCode VecGetArrayRead(Vec, const PetscScalar**);
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar**);
PetscErrorCode VecGetArray(Vec, PetscScalar**);
PetscErrorCode VecRestoreArray(Vec, PetscScalar**);
PetscErrorCode VecGetArrayWrite(Vec, PetscScalar**);
PetscErrorCode VecRestoreArrayWrite(Vec, PetscScalar**);
PetscErrorCode VecCUDAGetArrayRead(Vec, const PetscScalar**);
PetscErrorCode VecCUDARestoreArrayRead(Vec, const PetscScalar**);
PetscErrorCode VecCUDAGetArray(Vec, PetscScalar**);
PetscErrorCode VecCUDARestoreArray(Vec, PetscScalar**);
PetscErrorCode VecCUDAGetArrayWrite(Vec, PetscScalar**);
PetscErrorCode VecCUDARestoreArrayWrite(Vec, PetscScalar**);

PetscErrorCode DMGetVecType(DM, VecType*);
PetscErrorCode DMGetLocalVector(DM, Vec*);
PetscErrorCode DMRestoreLocalVector(DM, Vec*);
PetscErrorCode DMGlobalToLocalBegin(DM, Vec, InsertMode, Vec);
PetscErrorCode DMGlobalToLocalEnd(DM, Vec, InsertMode, Vec);
PetscErrorCode DMDAGetInfo(DM, PetscInt*, PetscInt*, PetscInt*, PetscInt*, PetscInt*, PetscInt*, PetscInt*,
                           PetscInt*, PetscInt*, DMBoundaryType*, DMBoundaryType*, DMBoundaryType*,
                           DMDAStencilType*);
PetscErrorCode DMDAGetCorners(DM, PetscInt*, PetscInt*, PetscInt*, PetscInt*, PetscInt*, PetscInt*);
PetscErrorCode DMDAGetGhostCorners(DM, PetscInt*, PetscInt*, PetscInt*, PetscInt*, PetscInt*, PetscInt*);

PetscErrorCode MatCreateShell(MPI_Comm, PetscInt, PetscInt, PetscInt, PetscInt, void*, Mat*);
PetscErrorCode MatShellSetOperation(Mat, MatOperation, void (*)(void));
PetscErrorCode MatShellGetContext(Mat, void*);
PetscErrorCode MatDestroy(Mat*);

PetscErrorCode PCShellGetContext(PC, void*);

PetscErrorCode TSGetTime(TS, PetscReal*);
PetscErrorCode TSGetSolution(TS, Vec*);
PetscErrorCode TSGetApplicationContext(TS, void*);
PetscErrorCode TSSetApplicationContext(TS, void*);
PetscErrorCode TSSetRHSFunction(TS, Vec, PetscErrorCode (*)(TS, PetscReal, Vec, Vec, void*), void*);
PetscErrorCode TSSetIFunction(TS, Vec, PetscErrorCode (*)(TS, PetscReal, Vec, Vec, Vec, void*), void*);
PetscErrorCode TSSetIJacobian(TS, Mat, Mat, PetscErrorCode (*)(TS, PetscReal, Vec, Vec, PetscReal, Mat, Mat, void*),
                              void*);
PetscErrorCode TSSetPostStep(TS, PetscErrorCode (*)(TS));
PetscErrorCode TSSetPostEvaluate(TS, PetscErrorCode (*)(TS));
PetscErrorCode TSSetTransientVariable(TS, PetscErrorCode (*)(TS, Vec, Vec, void*), void*);
