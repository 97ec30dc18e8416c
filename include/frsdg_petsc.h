/* frsdg_petsc.h -- the PETSc callbacks of fr_sdg's PetscSolver over libfrsdg.
 *
 * fr_sdg registers static callbacks on its TS in include/petsc_solver_impl.hpp:
 * TSSetRHSFunction (600) with rhs_func (657-670), TSSetIFunction (572) with
 * fun_implicit (626-655), TSSetTransientVariable (575) with primitive_to_conservative
 * (719-727), TSSetIJacobian (215) with pre_jv_eval (223-248) on a MatShell whose
 * MATOP_MULT (212) is matmult (250-432), and TSSetPostStep (586-607) with
 * apply_stabilization (683-702).  The functions below have the same signatures and
 * meaning; their bodies unwrap the Vecs and call the library.  Compile
 * fr_sdg_b200/petsc/frsdg_petsc.cpp inside fr_sdg (PETSc headers, the CUDA runtime and
 * libfrsdg on the link line).
 *
 * Vecs: CUDA Vecs (-dm_vec_type cuda) for every callback; host Vecs only for the
 * right-hand side of a single-rank DMDA (frsdg_rhs_host).  Work is enqueued on the
 * stream set with FrsdgPetscSetStream (default: the legacy default stream, which is
 * PETSc's default PETSC_STREAM_GLOBAL_BLOCKING device context).
 *
 * Ranks: a single-rank DMDA passes the Vec arrays straight through.  A 2D DMDA split
 * in rows only (-da_processors_x 1) runs each rank's row block through a row window
 * (frsdg_set_row_window): the owned rows of the global Vec plus one ghost element row
 * per neighbour, taken from the DMDA's ghosted local Vec (DMGlobalToLocal, the
 * reference's VecType::Local view), are staged into a device buffer of the adapter.
 * Other decompositions return PETSC_ERR_SUP. */
#pragma once
#include <petscdmda.h>
#include <petscts.h>

#include "frsdg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct FrsdgPetsc_* FrsdgPetsc;

/* A handle for the DMDA `da` (fr_sdg's PetscSolver::dmda, dof = n_eqs (p+1)^dim,
 * stencil width 1) and the configuration the options describe; checks that cfg's mesh
 * matches the DMDA's. */
PetscErrorCode FrsdgPetscCreate(DM da, const frsdg_config* cfg, FrsdgPetsc* out);
PetscErrorCode FrsdgPetscDestroy(FrsdgPetsc* c);
PetscErrorCode FrsdgPetscSetStream(FrsdgPetsc c, void* cuda_stream);
frsdg_handle* FrsdgPetscHandle(FrsdgPetsc c);

/* The registrations of PetscSolver::setup_ts (549-612): implicit -> IFunction,
 * TransientVariable (cfg.cond_sys), a MatShell Jacobian (JacobianMult) set with
 * IJacobian as both operator and preconditioning matrix; explicit -> RHSFunction.
 * When the configuration filters, limits or applies the positivity limiter, PostStep
 * is registered -- as TSSetPostEvaluate instead for an implicit TS with
 * post_evaluate (the reference's -do_post_ts false branch, 592-596).  Sets c as the
 * TS application context. */
PetscErrorCode FrsdgPetscSetUpTS(TS ts, FrsdgPetsc c, PetscBool implicit, PetscBool post_evaluate);

PetscErrorCode FrsdgPetscRHSFunction(TS ts, PetscReal t, Vec U, Vec rhs, void* ctx);
PetscErrorCode FrsdgPetscIFunction(TS ts, PetscReal t, Vec U, Vec U_t, Vec F, void* ctx);
PetscErrorCode FrsdgPetscTransientVariable(TS ts, Vec prim, Vec cons, void* ctx);
PetscErrorCode FrsdgPetscIJacobian(TS ts, PetscReal t, Vec U, Vec U_t, PetscReal sigma, Mat J, Mat P, void* ctx);
PetscErrorCode FrsdgPetscJacobianMult(Mat J, Vec v, Vec out);
PetscErrorCode FrsdgPetscPostStep(TS ts);

/* PCSHELL callbacks (single-rank DMDA, p <= 5): element block-Jacobi of the implicit
 * Jacobian at the state and shift of the last FrsdgPetscIJacobian (frsdg_pc_setup /
 * frsdg_pc_apply); PCShellSetContext(pc, c). */
PetscErrorCode FrsdgPetscPCSetUp(PC pc);
PetscErrorCode FrsdgPetscPCApply(PC pc, Vec r, Vec z);

#ifdef __cplusplus
}
#endif
