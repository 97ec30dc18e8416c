// frsdg_petsc.cpp -- fr_sdg's PETSc TS callbacks (include/petsc_solver_impl.hpp of the
// reference) over libfrsdg's C ABI; the interface and its conventions are described in
// include/frsdg_petsc.h.  Compiled inside fr_sdg, against PETSc, the CUDA runtime and
// libfrsdg.
#include "frsdg_petsc.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <new>

namespace
{
// device staging buffers of the adapter
enum Stage
{
    ST_U = 0,    // residual input (ghosted row block)
    ST_JAC = 1,  // the Jacobian's base state, kept from IJacobian to the last JacobianMult
    ST_DIR = 2,  // JacobianMult direction (ghosted row block)
    ST_OUT = 3,  // post-step and change-of-variables output (row block)
    ST_COUNT = 4
};
} // namespace

struct FrsdgPetsc_
{
    frsdg_handle* h = nullptr;
    frsdg_config  cfg{};
    DM            da = nullptr;
    MPI_Comm      comm{};
    cudaStream_t  stream = nullptr;
    bool          device = true;     // CUDA Vecs
    bool          windowed = false;  // a row block of a 2D DMDA split over ranks in rows
    PetscInt      dim = 0, Nx = 0, Ny = 0, dof = 0;
    PetscInt      ys = 0, ym = 0;    // owned element rows [ys, ys + ym)
    PetscInt      gys = 0, gxs = 0, gxm = 0;  // ghosted local Vec: first row, first column, columns
    PetscInt      lo = 0, hi = 0;    // ghost rows staged below / above the owned rows (0 or 1)
    size_t        row = 0;           // doubles per element row, Nx dof
    size_t        n_local = 0;       // doubles of this rank's part of a global Vec
    size_t        n_stage = 0;       // doubles of one staging buffer
    double*       st[ST_COUNT] = {};
    Mat           J = nullptr;
    PetscReal     jac_t = 0.0, jac_sigma = 0.0;
    bool          jac_ready = false;
};

#define FRSDG_PETSC_CALL(x)                                                                                    \
    do                                                                                                         \
    {                                                                                                          \
        if ((x) != FRSDG_OK) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_LIB, "libfrsdg: %s", frsdg_last_error());     \
    } while (0)

#define FRSDG_CUDA_CALL(x, what)                                                                               \
    do                                                                                                         \
    {                                                                                                          \
        const cudaError_t e_ = (x);                                                                            \
        if (e_ != cudaSuccess)                                                                                 \
            SETERRQ(PETSC_COMM_SELF, PETSC_ERR_LIB, "%s: %s", what, cudaGetErrorString(e_));                   \
    } while (0)

namespace
{
// Rows [lo, lo + ym) of a window are the first ym rows of an owned-rows-only array f:
// the library reads and writes outputs (and the per-node inputs U_t, r) only at its
// computed rows, so the window's row 0 sits lo rows before f.  Computed as an address.
double* window_view(const FrsdgPetsc c, double* f)
{
    return reinterpret_cast<double*>(reinterpret_cast<uintptr_t>(f) - sizeof(double) * size_t(c->lo) * c->row);
}
const double* window_view(const FrsdgPetsc c, const double* f)
{
    return window_view(c, const_cast<double*>(f));
}

// dst (rows lo + ym + hi of the window) <- the owned rows of the global Vec g and the
// ghost rows of its DMDA local copy (the reference's VecType::Local view), one strided
// device copy out of the ghosted local Vec.
PetscErrorCode stage_ghosted(FrsdgPetsc c, Vec g, double* dst)
{
    PetscFunctionBeginUser;
    Vec l;
    PetscCall(DMGetLocalVector(c->da, &l));
    PetscCall(DMGlobalToLocalBegin(c->da, g, INSERT_VALUES, l));
    PetscCall(DMGlobalToLocalEnd(c->da, g, INSERT_VALUES, l));
    const PetscScalar* b;
    PetscCall(VecCUDAGetArrayRead(l, &b));
    const size_t lrow = size_t(c->gxm) * size_t(c->dof);     // doubles per local row
    const size_t col0 = size_t(0 - c->gxs) * size_t(c->dof);  // element column 0 in a local row
    const double* src = b + size_t(c->ys - c->lo - c->gys) * lrow + col0;
    const cudaError_t e = cudaMemcpy2DAsync(dst, sizeof(double) * c->row, src, sizeof(double) * lrow,
                                            sizeof(double) * c->row, size_t(c->lo + c->ym + c->hi),
                                            cudaMemcpyDeviceToDevice, c->stream);
    PetscCall(VecCUDARestoreArrayRead(l, &b));
    PetscCall(DMRestoreLocalVector(c->da, &l));
    FRSDG_CUDA_CALL(e, "staging the ghosted row block");
    PetscFunctionReturn(PETSC_SUCCESS);
}

// dst (window rows, owned rows at lo) <- the owned rows of the global Vec g
PetscErrorCode stage_owned(FrsdgPetsc c, Vec g, double* dst)
{
    PetscFunctionBeginUser;
    const PetscScalar* a;
    PetscCall(VecCUDAGetArrayRead(g, &a));
    const cudaError_t e = cudaMemcpyAsync(dst + size_t(c->lo) * c->row, a, sizeof(double) * c->n_local,
                                          cudaMemcpyDeviceToDevice, c->stream);
    PetscCall(VecCUDARestoreArrayRead(g, &a));
    FRSDG_CUDA_CALL(e, "staging the owned rows");
    PetscFunctionReturn(PETSC_SUCCESS);
}

// the owned rows of the window buffer src -> the global Vec g
PetscErrorCode unstage_owned(FrsdgPetsc c, const double* src, Vec g)
{
    PetscFunctionBeginUser;
    PetscScalar* a;
    PetscCall(VecCUDAGetArrayWrite(g, &a));
    const cudaError_t e = cudaMemcpyAsync(a, src + size_t(c->lo) * c->row, sizeof(double) * c->n_local,
                                          cudaMemcpyDeviceToDevice, c->stream);
    PetscCall(VecCUDARestoreArrayWrite(g, &a));
    FRSDG_CUDA_CALL(e, "writing the owned rows");
    PetscFunctionReturn(PETSC_SUCCESS);
}

PetscErrorCode need_device(const FrsdgPetsc c, const char* what)
{
    if (!c->device)
        SETERRQ(PETSC_COMM_SELF, PETSC_ERR_SUP, "%s needs CUDA Vecs (-dm_vec_type cuda)", what);
    return PETSC_SUCCESS;
}
} // namespace

extern "C" {

PetscErrorCode FrsdgPetscCreate(DM da, const frsdg_config* cfg, FrsdgPetsc* out)
{
    PetscFunctionBeginUser;
    if (!da || !cfg || !out) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_WRONG, "FrsdgPetscCreate: null argument");
    PetscInt dim, M, N, m, n, dof, s;
    DMBoundaryType bx, by;
    PetscCall(DMDAGetInfo(da, &dim, &M, &N, nullptr, &m, &n, nullptr, &dof, &s, &bx, &by, nullptr, nullptr));
    const PetscInt np = cfg->poly_deg + 1;
    if (dim != cfg->dim || M != cfg->n_elems[0] || (dim == 2 && N != cfg->n_elems[1]) ||
        dof != (dim == 2 ? 4 * np * np : 3 * np) || s != 1)
        SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_INCOMP,
                "FrsdgPetscCreate: the DMDA (dim, elements, dof, stencil width) does not match the configuration");
    if ((bx == DM_BOUNDARY_PERIODIC) != (cfg->bc[FRSDG_LEFT].kind == FRSDG_BC_PERIODIC) ||
        (dim == 2 && (by == DM_BOUNDARY_PERIODIC) != (cfg->bc[FRSDG_BOTTOM].kind == FRSDG_BC_PERIODIC)))
        SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_INCOMP,
                "FrsdgPetscCreate: periodic DMDA directions and periodic boundary kinds differ");

    VecType vt;
    PetscCall(DMGetVecType(da, &vt));
    MPI_Comm comm;
    PetscCall(PetscObjectGetComm(reinterpret_cast<PetscObject>(da), &comm));
    int size = 1;
    MPI_Comm_size(comm, &size);
    PetscInt xs, ys, zs, xm, ym, zm, gxs, gys, gzs, gxm, gym, gzm;
    PetscCall(DMDAGetCorners(da, &xs, &ys, &zs, &xm, &ym, &zm));
    PetscCall(DMDAGetGhostCorners(da, &gxs, &gys, &gzs, &gxm, &gym, &gzm));
    const bool device = vt && std::strstr(vt, "cuda") != nullptr;
    if (dim == 1) ym = 1;
    PetscInt lo = 0, hi = 0;
    if (size > 1)
    {
        if (dim != 2 || m != 1 || xs != 0 || xm != M)
            SETERRQ(PETSC_COMM_SELF, PETSC_ERR_SUP,
                    "libfrsdg runs a multi-rank DMDA only in 2D, split in rows (-da_processors_x 1)");
        if (!device) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_SUP, "a multi-rank DMDA needs CUDA Vecs (-dm_vec_type cuda)");
        const bool per_y = by == DM_BOUNDARY_PERIODIC;
        lo = (ys > 0 || per_y) ? 1 : 0;
        hi = (ys + ym < N || per_y) ? 1 : 0;
        if (gys > ys - lo || gys + gym < ys + ym + hi || gxs > 0 || gxs + gxm < M)
            SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_INCOMP, "the DMDA's local Vec lacks the ghost rows");
    }

    FrsdgPetsc c = new (std::nothrow) FrsdgPetsc_;
    if (!c) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_LIB, "FrsdgPetscCreate: out of host memory");
    c->cfg = *cfg;
    c->da = da;
    c->comm = comm;
    c->device = device;
    c->windowed = size > 1;
    c->dim = dim;
    c->Nx = M;
    c->Ny = dim == 2 ? N : 1;
    c->dof = dof;
    c->row = size_t(M) * size_t(dof);
    c->ys = ys;
    c->ym = ym;
    c->gys = gys;
    c->gxs = gxs;
    c->gxm = gxm;
    c->lo = lo;
    c->hi = hi;
    c->n_local = size_t(xm) * size_t(ym) * size_t(dof);
    if (frsdg_create(cfg, &c->h) != FRSDG_OK)
    {
        delete c;
        SETERRQ(PETSC_COMM_SELF, PETSC_ERR_LIB, "libfrsdg: %s", frsdg_last_error());
    }
    *out = c;
    if (c->windowed)
        FRSDG_PETSC_CALL(frsdg_set_row_window(c->h, int(c->ys - c->lo), int(c->lo + c->ym + c->hi), int(c->lo),
                                              int(c->lo + c->ym)));
    if (c->device)
    {
        c->n_stage = c->windowed ? size_t(c->lo + c->ym + c->hi) * c->row : c->n_local;
        for (int k = 0; k < ST_COUNT; ++k)
        {
            if (!c->windowed && k != ST_JAC) continue;  // a single rank reads the Vec arrays in place
            void* p = nullptr;
            FRSDG_CUDA_CALL(cudaMalloc(&p, sizeof(double) * c->n_stage), "staging buffers");
            c->st[k] = static_cast<double*>(p);
            FRSDG_CUDA_CALL(cudaMemset(p, 0, sizeof(double) * c->n_stage), "staging buffers");
        }
    }
    PetscFunctionReturn(PETSC_SUCCESS);
}

PetscErrorCode FrsdgPetscDestroy(FrsdgPetsc* pc)
{
    PetscFunctionBeginUser;
    if (!pc || !*pc) PetscFunctionReturn(PETSC_SUCCESS);
    FrsdgPetsc c = *pc;
    if (c->J) PetscCall(MatDestroy(&c->J));
    for (double*& p : c->st)
        if (p) cudaFree(p);
    if (c->h) frsdg_destroy(c->h);
    delete c;
    *pc = nullptr;
    PetscFunctionReturn(PETSC_SUCCESS);
}

PetscErrorCode FrsdgPetscSetStream(FrsdgPetsc c, void* cuda_stream)
{
    c->stream = static_cast<cudaStream_t>(cuda_stream);
    return PETSC_SUCCESS;
}

frsdg_handle* FrsdgPetscHandle(FrsdgPetsc c) { return c ? c->h : nullptr; }

// PetscSolver::rhs_func (petsc_solver_impl.hpp:657-670): rhs = -R(U)
PetscErrorCode FrsdgPetscRHSFunction(TS, PetscReal t, Vec U, Vec rhs, void* ctx)
{
    PetscFunctionBeginUser;
    FrsdgPetsc c = static_cast<FrsdgPetsc>(ctx);
    if (!c->device)
    {
        // host Vecs (single rank): staged through the handle's device buffers
        const PetscScalar* u;
        PetscScalar* f;
        PetscCall(VecGetArrayRead(U, &u));
        PetscCall(VecGetArrayWrite(rhs, &f));
        const int rc = frsdg_rhs_host(c->h, t, u, f, c->stream);
        PetscCall(VecRestoreArrayWrite(rhs, &f));
        PetscCall(VecRestoreArrayRead(U, &u));
        FRSDG_PETSC_CALL(rc);
        PetscFunctionReturn(PETSC_SUCCESS);
    }
    PetscScalar* f;
    if (c->windowed)
    {
        PetscCall(stage_ghosted(c, U, c->st[ST_U]));
        PetscCall(VecCUDAGetArrayWrite(rhs, &f));
        const int rc = frsdg_rhs(c->h, t, c->st[ST_U], window_view(c, f), c->stream);
        PetscCall(VecCUDARestoreArrayWrite(rhs, &f));
        FRSDG_PETSC_CALL(rc);
        PetscFunctionReturn(PETSC_SUCCESS);
    }
    const PetscScalar* u;
    PetscCall(VecCUDAGetArrayRead(U, &u));
    PetscCall(VecCUDAGetArrayWrite(rhs, &f));
    const int rc = frsdg_rhs(c->h, t, u, f, c->stream);
    PetscCall(VecCUDARestoreArrayWrite(rhs, &f));
    PetscCall(VecCUDARestoreArrayRead(U, &u));
    FRSDG_PETSC_CALL(rc);
    PetscFunctionReturn(PETSC_SUCCESS);
}

// PetscSolver::fun_implicit (626-655): F = U_t + R(M(U)) at the TS's time
PetscErrorCode FrsdgPetscIFunction(TS ts, PetscReal, Vec U, Vec U_t, Vec F, void* ctx)
{
    PetscFunctionBeginUser;
    FrsdgPetsc c = static_cast<FrsdgPetsc>(ctx);
    PetscCall(need_device(c, "FrsdgPetscIFunction"));
    PetscReal t;
    PetscCall(TSGetTime(ts, &t));
    const PetscScalar *u = nullptr, *ut;
    PetscScalar* f;
    if (c->windowed)
        PetscCall(stage_ghosted(c, U, c->st[ST_U]));
    else
        PetscCall(VecCUDAGetArrayRead(U, &u));
    PetscCall(VecCUDAGetArrayRead(U_t, &ut));
    PetscCall(VecCUDAGetArrayWrite(F, &f));
    const int rc = c->windowed ? frsdg_ifunction(c->h, t, c->st[ST_U], window_view(c, ut), window_view(c, f), c->stream)
                               : frsdg_ifunction(c->h, t, u, ut, f, c->stream);
    PetscCall(VecCUDARestoreArrayWrite(F, &f));
    PetscCall(VecCUDARestoreArrayRead(U_t, &ut));
    if (!c->windowed) PetscCall(VecCUDARestoreArrayRead(U, &u));
    FRSDG_PETSC_CALL(rc);
    PetscFunctionReturn(PETSC_SUCCESS);
}

// PetscSolver::primitive_to_conservative (719-727), the TS transient variable
PetscErrorCode FrsdgPetscTransientVariable(TS, Vec prim, Vec cons, void* ctx)
{
    PetscFunctionBeginUser;
    FrsdgPetsc c = static_cast<FrsdgPetsc>(ctx);
    PetscCall(need_device(c, "FrsdgPetscTransientVariable"));
    if (c->windowed)
    {
        // elementwise over the whole window: run it on the staged rows, keep the owned ones
        PetscCall(stage_owned(c, prim, c->st[ST_U]));
        FRSDG_PETSC_CALL(frsdg_prim_to_cons(c->h, c->st[ST_U], c->st[ST_OUT], c->stream));
        PetscCall(unstage_owned(c, c->st[ST_OUT], cons));
        PetscFunctionReturn(PETSC_SUCCESS);
    }
    const PetscScalar* a;
    PetscScalar* b;
    PetscCall(VecCUDAGetArrayRead(prim, &a));
    PetscCall(VecCUDAGetArrayWrite(cons, &b));
    const int rc = frsdg_prim_to_cons(c->h, a, b, c->stream);
    PetscCall(VecCUDARestoreArrayWrite(cons, &b));
    PetscCall(VecCUDARestoreArrayRead(prim, &a));
    FRSDG_PETSC_CALL(rc);
    PetscFunctionReturn(PETSC_SUCCESS);
}

// ComplexStepJacobianStrategy::pre_jv_eval (223-248): the state and shift of the
// following products, kept in the adapter's buffer until the next call
PetscErrorCode FrsdgPetscIJacobian(TS ts, PetscReal, Vec U, Vec, PetscReal sigma, Mat, Mat, void* ctx)
{
    PetscFunctionBeginUser;
    FrsdgPetsc c = static_cast<FrsdgPetsc>(ctx);
    PetscCall(need_device(c, "FrsdgPetscIJacobian"));
    PetscReal t;
    PetscCall(TSGetTime(ts, &t));
    if (c->windowed)
        PetscCall(stage_ghosted(c, U, c->st[ST_JAC]));
    else
        PetscCall(stage_owned(c, U, c->st[ST_JAC]));
    FRSDG_PETSC_CALL(frsdg_jvp_prepare(c->h, t, sigma, c->st[ST_JAC]));
    c->jac_t = t;
    c->jac_sigma = sigma;
    c->jac_ready = true;
    PetscFunctionReturn(PETSC_SUCCESS);
}

// ComplexStepJacobianStrategy::matmult (250-432), the MatShell's MATOP_MULT
PetscErrorCode FrsdgPetscJacobianMult(Mat J, Vec v, Vec out)
{
    PetscFunctionBeginUser;
    FrsdgPetsc c;
    PetscCall(MatShellGetContext(J, &c));
    if (!c->jac_ready) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_WRONG, "FrsdgPetscJacobianMult before FrsdgPetscIJacobian");
    PetscScalar* o;
    if (c->windowed)
    {
        PetscCall(stage_ghosted(c, v, c->st[ST_DIR]));
        PetscCall(VecCUDAGetArrayWrite(out, &o));
        const int rc = frsdg_jvp(c->h, c->st[ST_DIR], window_view(c, o), c->stream);
        PetscCall(VecCUDARestoreArrayWrite(out, &o));
        FRSDG_PETSC_CALL(rc);
        PetscFunctionReturn(PETSC_SUCCESS);
    }
    const PetscScalar* vv;
    PetscCall(VecCUDAGetArrayRead(v, &vv));
    PetscCall(VecCUDAGetArrayWrite(out, &o));
    const int rc = frsdg_jvp(c->h, vv, o, c->stream);
    PetscCall(VecCUDARestoreArrayWrite(out, &o));
    PetscCall(VecCUDARestoreArrayRead(v, &vv));
    FRSDG_PETSC_CALL(rc);
    PetscFunctionReturn(PETSC_SUCCESS);
}

// PetscSolver::apply_stabilization (683-702): limit the TS solution in place
PetscErrorCode FrsdgPetscPostStep(TS ts)
{
    PetscFunctionBeginUser;
    FrsdgPetsc c;
    PetscCall(TSGetApplicationContext(ts, &c));
    PetscCall(need_device(c, "FrsdgPetscPostStep"));
    Vec U;
    PetscCall(TSGetSolution(ts, &U));
    if (c->windowed)
    {
        PetscCall(stage_ghosted(c, U, c->st[ST_U]));
        FRSDG_PETSC_CALL(frsdg_post_step_to(c->h, c->st[ST_U], c->st[ST_OUT], c->stream));
        PetscCall(unstage_owned(c, c->st[ST_OUT], U));
        PetscFunctionReturn(PETSC_SUCCESS);
    }
    PetscScalar* u;
    PetscCall(VecCUDAGetArray(U, &u));
    const int rc = frsdg_post_step(c->h, u, c->stream);
    PetscCall(VecCUDARestoreArray(U, &u));
    FRSDG_PETSC_CALL(rc);
    PetscFunctionReturn(PETSC_SUCCESS);
}

PetscErrorCode FrsdgPetscPCSetUp(PC pc)
{
    PetscFunctionBeginUser;
    FrsdgPetsc c;
    PetscCall(PCShellGetContext(pc, &c));
    if (c->windowed) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_SUP, "FrsdgPetscPCSetUp: single-rank DMDAs only");
    if (!c->jac_ready) SETERRQ(PETSC_COMM_SELF, PETSC_ERR_ARG_WRONG, "FrsdgPetscPCSetUp before FrsdgPetscIJacobian");
    FRSDG_PETSC_CALL(frsdg_pc_setup(c->h, c->jac_t, c->jac_sigma, c->st[ST_JAC], c->stream));
    PetscFunctionReturn(PETSC_SUCCESS);
}

PetscErrorCode FrsdgPetscPCApply(PC pc, Vec r, Vec z)
{
    PetscFunctionBeginUser;
    FrsdgPetsc c;
    PetscCall(PCShellGetContext(pc, &c));
    const PetscScalar* rr;
    PetscScalar* zz;
    PetscCall(VecCUDAGetArrayRead(r, &rr));
    PetscCall(VecCUDAGetArrayWrite(z, &zz));
    const int rc = frsdg_pc_apply(c->h, rr, zz, c->stream);
    PetscCall(VecCUDARestoreArrayWrite(z, &zz));
    PetscCall(VecCUDARestoreArrayRead(r, &rr));
    FRSDG_PETSC_CALL(rc);
    PetscFunctionReturn(PETSC_SUCCESS);
}

// PetscSolver::setup_ts (549-612), the callback registrations
PetscErrorCode FrsdgPetscSetUpTS(TS ts, FrsdgPetsc c, PetscBool implicit, PetscBool post_evaluate)
{
    PetscFunctionBeginUser;
    PetscCall(TSSetApplicationContext(ts, c));
    const bool stab = c->cfg.apply_filter || c->cfg.apply_weno || c->cfg.pp_limit;
    if (implicit)
    {
        PetscCall(TSSetIFunction(ts, nullptr, FrsdgPetscIFunction, c));
        if (c->cfg.cond_sys) PetscCall(TSSetTransientVariable(ts, FrsdgPetscTransientVariable, c));
        const PetscInt n_loc = PetscInt(c->n_local);
        const PetscInt n_glob = c->Nx * c->Ny * c->dof;
        if (!c->J)
        {
            PetscCall(MatCreateShell(c->comm, n_loc, n_loc, n_glob, n_glob, c, &c->J));
            PetscCall(MatShellSetOperation(c->J, MATOP_MULT, reinterpret_cast<void (*)(void)>(FrsdgPetscJacobianMult)));
        }
        PetscCall(TSSetIJacobian(ts, c->J, c->J, FrsdgPetscIJacobian, c));
        if (stab)
        {
            if (post_evaluate)
                PetscCall(TSSetPostEvaluate(ts, FrsdgPetscPostStep));
            else
                PetscCall(TSSetPostStep(ts, FrsdgPetscPostStep));
        }
    }
    else
    {
        PetscCall(TSSetRHSFunction(ts, nullptr, FrsdgPetscRHSFunction, c));
        if (stab) PetscCall(TSSetPostStep(ts, FrsdgPetscPostStep));
    }
    PetscFunctionReturn(PETSC_SUCCESS);
}

} // extern "C"
