/*
 * frsdg.h -- C ABI of the B200 Flux Reconstruction residual library (libfrsdg.so).
 *
 * The library replaces the hot path of fr_sdg's PETSc time-stepping callbacks:
 * the FR spatial residual of the compressible Euler equations, its complex-step
 * Jacobian-vector product, the post-step stabilisation and the change of
 * variables.  Every entry point takes plain pointers and sizes; no PETSc, CUDA
 * or torch type appears in a signature.  Streams are passed as `void*`
 * (a cudaStream_t, NULL = legacy default stream).
 *
 * Vector layout (the DMDA natural ordering of a single-rank PETSc Vec,
 * include/vec_dof_view.hpp:102-117 and include/physics_impl_2D.hpp:13-35):
 *   2D: element (i,j) starts at ((j*Nx + i) * ndofs), ndofs = 4*n*n, and inside an
 *       element value (eq, k, l) sits at ((l*n + k)*4 + eq)   [node-major AoS]
 *   1D: element e starts at (e * ndofs), ndofs = 3*n, and inside an element value
 *       (eq, node) sits at (eq*n + node)                        [SoA]
 * with n = poly_deg + 1 GLL points per direction.
 *
 * Every function returns 0 (FRSDG_OK) on success or a negative FRSDG_ERR_* code;
 * frsdg_last_error() gives a one-line description of the last failure on the
 * calling thread.  Device pointers must be 16-byte aligned.  A handle is not
 * thread safe: use one handle per host thread.  Hot calls (residual, rhs,
 * ifunction, jvp, post_step, prim_to_cons) allocate nothing; every workspace is
 * allocated by frsdg_create.
 */
#ifndef FRSDG_H
#define FRSDG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FRSDG_ABI_VERSION 2

/* ---- status codes (PETSc-style: 0 = success) ---------------------------- */
enum {
    FRSDG_OK             = 0,
    FRSDG_ERR_ARG        = -1, /* invalid argument or configuration */
    FRSDG_ERR_CUDA       = -2, /* a CUDA runtime call failed */
    FRSDG_ERR_NOMEM      = -3, /* device allocation failed in frsdg_create */
    FRSDG_ERR_UNSUPPORTED = -4, /* configuration valid but not built in */
    FRSDG_ERR_NODEVICE   = -5  /* no CUDA device visible */
};

/* ---- policy enums (runtime stand-ins for the reference's compile-time traits,
 *      include/physics_evaluator.hpp:37-52) ------------------------------- */
enum { FRSDG_GAS_IDEAL = 0, FRSDG_GAS_VDW = 1 };              /* gas_models.hpp:56-158 */
enum { FRSDG_RUSANOV = 0, FRSDG_HLLC = 1 };                    /* riemann_solver.hpp:13-17 */
enum { FRSDG_COORD_CARTESIAN = 0, FRSDG_COORD_RADIAL = 1 };    /* macro_and_libc.hpp:154-159 */

/* Geometry policies (geometry_models.hpp:61-195, tests/bump.cpp:13-171):
 *  CARTESIAN     x = Lx*csi, y = Ly*eta
 *  DELAVAL       GeometryDeLavalNozzle2D with the straight-line profile (h=0.5, h'=0)
 *  WALL_PROFILE  x = x0 + Lx*csi, y = h(x)*(1-eta) + Ly*eta with a wall profile h(x)
 *                chosen by geom_profile (wedges of tests/bump.cpp and
 *                tests/boundary_conforming.cpp, or a Gaussian bump)
 *  SINE_WARP     x = Lx*csi + A sin(2 pi csi) sin(2 pi eta), same displacement on y */
enum {
    FRSDG_GEOM_CARTESIAN    = 0,
    FRSDG_GEOM_DELAVAL      = 1,
    FRSDG_GEOM_WALL_PROFILE = 2,
    FRSDG_GEOM_SINE_WARP    = 3
};
enum {
    FRSDG_PROFILE_FLAT        = 0, /* h = 0 */
    FRSDG_PROFILE_WEDGE_BUMP  = 1, /* tests/bump.cpp:29-119 (5 zones, returns -h) */
    FRSDG_PROFILE_WEDGE_BC    = 2, /* tests/boundary_conforming.cpp:28-67 (3 zones) */
    FRSDG_PROFILE_GAUSS_BUMP  = 3  /* h = A exp(-k x^2), geom_params[1]=A, [2]=k */
};

/* Boundary faces, in the reference's Direction order (boundary_conditions.hpp:17-23). */
enum { FRSDG_LEFT = 0, FRSDG_RIGHT = 1, FRSDG_TOP = 2, FRSDG_BOTTOM = 3 };

/* Boundary kinds.  OUTFLOW, WALL and PERIODIC are the reference's native binders
 * (boundary_conditions.hpp:296-323) and keep the imaginary part in the complex
 * step; every other kind stands for a user lambda (bind_lambda, 270-294) and,
 * like it, sees only the real part of the interior state in the complex step. */
enum {
    FRSDG_BC_OUTFLOW         = 0, /* ghost = interior */
    FRSDG_BC_WALL            = 1, /* flip the momentum component of the face axis */
    FRSDG_BC_PERIODIC        = 2, /* wrap to the opposite element (both faces of an axis) */
    FRSDG_BC_DIRICHLET       = 3, /* ghost = state[0..3] (conservative) */
    FRSDG_BC_SLIP_WALL       = 4, /* reflect velocity about the face normal (tests/bump.cpp:250-272) */
    FRSDG_BC_VORTEX          = 5, /* exact isentropic vortex (factory.hpp:311-352, 504-511);
                                     params: u0, v0, beta, r_v, l */
    FRSDG_BC_SUBSONIC_INFLOW = 6, /* total pressure / temperature inflow; params: p0, T0, R, angle */
    FRSDG_BC_PRESSURE_OUTLET = 7  /* static pressure outlet; params: p_out */
};

typedef struct frsdg_bc {
    int32_t kind;
    int32_t pad_;
    double  state[4];  /* conservative ghost for DIRICHLET (1D uses state[0..2]) */
    double  params[6];
} frsdg_bc;

/* Mirror of the ConfigOptions fields the hot path reads (parser.hpp:45-191),
 * plus the policy choices the reference fixes at compile time. */
typedef struct frsdg_config {
    int32_t dim;             /* 1 or 2 */
    int32_t poly_deg;        /* p, 1..9 (n = p+1 GLL points per direction) */
    int32_t n_elems[2];      /* Nx, Ny (Ny ignored in 1D) */
    double  box_length[2];   /* Lx, Ly */
    double  radau_corr;      /* VCJH c (0 = nodal DG) */
    int32_t gas_law;         /* FRSDG_GAS_* */
    int32_t riemann;         /* FRSDG_RUSANOV / FRSDG_HLLC */
    double  gamma, R_spec, vdw_a, vdw_b;
    int32_t coord_sys;       /* FRSDG_COORD_* (RADIAL: 1D only) */
    int32_t geometry;        /* FRSDG_GEOM_* (2D only) */
    int32_t geom_profile;    /* FRSDG_PROFILE_* for WALL_PROFILE */
    int32_t pad0_;
    double  geom_params[4];  /* WALL_PROFILE: [0]=x0; SINE_WARP: [0]=amplitude */
    frsdg_bc bc[4];          /* indexed by FRSDG_LEFT..FRSDG_BOTTOM (1D: LEFT, RIGHT) */
    /* stabilisation (filter.hpp:393-759) */
    int32_t apply_filter;
    int32_t filt_cut_off;    /* default 2 */
    int32_t filt_strength;   /* default 32 */
    int32_t apply_weno;
    double  filt_alpha;      /* default 36 */
    double  weno_gamma;      /* default 0.998 */
    double  shock_theta;     /* default 1 */
    double  shock_threshold; /* default 0.8 */
    int32_t cond_sys;        /* -solve_positive_preserving: unknowns (log rho, u, [v], log e) */
    int32_t jvp_exact_bc;    /* 0 (default): the complex-step JVP and Jacobian blocks see the
                                boundary ghosts of user-lambda boundary kinds (slip wall, Dirichlet,
                                vortex, subsonic inflow, pressure outlet) as constants, as the
                                reference does (boundary_conditions.hpp:276-293); 1: they are
                                differentiated too (exact Jacobian; 2D only) */
    double  csd_eps;         /* complex-step h (reference: 1e-7, petsc_solver_impl.hpp:179) */
    /* positivity-preserving limiter (no counterpart in the reference): 1 = the
     * scaling limiter of Zhang and Shu (J. Comput. Phys. 229, 2010) after the
     * post-step stabilisation, and on every Runge-Kutta stage when frsdg_pp_limit is
     * called there; cell averages by GLL quadrature, floor eps = min(pp_eps, rho_bar,
     * p_bar).  Default 0 (off), pp_eps 1e-13. */
    int32_t pp_limit;
    /* FP32 residual of the mixed form (frsdg_residual_f32, frsdg_rk_stage_mixed, the
     * FRSDG_STAGE_MIXED stages) at p = 4 to 7 (no counterpart in the reference): 1 = its
     * derivative contractions run on the tensor cores (tcgen05, operands split into
     * TF32 high and low parts, FP32 accumulation), 0 = FP32 FMAs on the CUDA cores.
     * Other orders, FP64 and complex residuals and batch launches ignore it. */
    int32_t mixed_tc;
    double  pp_eps;
} frsdg_config;

typedef struct frsdg_handle frsdg_handle;

/* Library identity and errors. */
int         frsdg_abi_version(void);
const char* frsdg_last_error(void);

/* Fill *cfg with the reference defaults (parser.hpp:45-91, 257-275). */
int frsdg_config_default(frsdg_config* cfg);

/* Build a handle on the current CUDA device: reference element (GLL nodes,
 * differentiation matrix, VCJH correction derivatives), filter matrices, cached
 * curved metrics and face normals, boundary data and all workspaces.
 * Replaces PhysicsEvaluator's constructor (physics_evaluator.hpp:188-201) and
 * PetscSolver::setup_dmda/setup_ts (petsc_solver_impl.hpp:492-612). */
int frsdg_create(const frsdg_config* cfg, frsdg_handle** out);
int frsdg_destroy(frsdg_handle* h);

/* Number of doubles in one solution vector (Nx*Ny*4*n*n or Nx*3*n). */
int frsdg_n_dofs(const frsdg_handle* h, int64_t* n);

/* R(U): PhysicsEvaluator::residual_kernel<double> (physics_impl_2D.hpp:646-902,
 * physics_impl_1D.hpp:9-94).  U and R are device pointers. */
int frsdg_residual(frsdg_handle* h, double t, const double* U, double* R, void* stream);

/* rhs = -R(U): PetscSolver::rhs_func (petsc_solver_impl.hpp:657-670). */
int frsdg_rhs(frsdg_handle* h, double t, const double* U, double* rhs, void* stream);

/* F = U_t + R(M(U)): PetscSolver::fun_implicit (petsc_solver_impl.hpp:626-655);
 * M = prim->cons when cond_sys, identity otherwise. */
int frsdg_ifunction(frsdg_handle* h, double t, const double* U, const double* U_t,
                    double* F, void* stream);

/* Snapshot (t, sigma, U) for later frsdg_jvp calls:
 * ComplexStepJacobianStrategy::pre_jv_eval (petsc_solver_impl.hpp:223-248).
 * U must stay valid until the next frsdg_jvp_prepare. */
int frsdg_jvp_prepare(frsdg_handle* h, double t, double sigma, const double* U);

/* JV = sigma*Im(M(U+ihV))/h + Im(R(M(U+ihV)))/h, h = cfg.csd_eps:
 * ComplexStepJacobianStrategy::matmult (petsc_solver_impl.hpp:250-432). */
int frsdg_jvp(frsdg_handle* h, const double* V, double* JV, void* stream);

/* Row window for domain decomposition (2D; the reference's DMDA ghosted local view,
 * physics_impl_2D.hpp:646-902, with the halo width one element row).  After this call
 * every vector argument of the handle holds `rows` element rows of the mesh starting
 * at global row `row_base` (DMDA layout within them); rows [row_begin, row_end) are
 * computed and written, the others are ghost rows the caller fills from the
 * neighbouring partitions before each call (one row below and above is read).  Sides
 * without a ghost row must be the mesh's non-periodic edge; on a periodic mesh both
 * sides need ghost rows (row_base may be -1).  Geometry is looked up at global rows.
 * rows = 0 restores the whole-mesh view. */
int frsdg_set_row_window(frsdg_handle* h, int row_base, int rows, int row_begin, int row_end);

/* Mixed precision (2D; no reference counterpart -- the reference computes in FP64
 * only).  frsdg_residual_f32: R = residual_kernel evaluated in FP32 on an FP32 state.
 * frsdg_rk_stage_mixed: frsdg_rk_stage on the FP64 stage input Us with the residual in
 * FP32 arithmetic: every node's density, velocities, internal energy, pressure and sound
 * speed are recovered from the FP64 state in FP64 (so that pressures near vacuum keep
 * their sign) and rounded to FP32; fluxes, Riemann solves and derivative contractions
 * run in FP32; the stage combination is FP64:
 *   out = alpha*A + beta*B + gamma*rhs(Us),  acc += delta*rhs
 * (A, B, acc may be NULL).  No change of variables. */
int frsdg_residual_f32(frsdg_handle* h, double t, const float* U32, float* R32, void* stream);
int frsdg_rk_stage_mixed(frsdg_handle* h, double t, const double* Us, const double* A, double alpha,
                         const double* B, double beta, double gamma, double* out, double* acc,
                         double delta, void* stream);

/* One Runge-Kutta stage with the element-local work that follows it fused in (no
 * reference counterpart: the reference runs the post-step as a separate pass after
 * TSStep, petsc_solver_impl.hpp:683-702).  out = alpha*A + beta*B + gamma*rhs(Us) and
 * acc += delta*rhs as in frsdg_rk_stage, then per flag:
 *   FRSDG_STAGE_MIXED      the residual of frsdg_rk_stage_mixed (2D, no change of variables);
 *   FRSDG_STAGE_LIMIT      out = the positivity limiter applied to out (cfg.pp_limit);
 *   FRSDG_STAGE_POST_STEP  out = frsdg_post_step applied to out (the spectral filter of
 *                          cfg.apply_filter, then the limiter of cfg.pp_limit) -- the last
 *                          stage of a step.
 * With FRSDG_STAGE_POST_STEP in 2D, when the post-step is element-local (the filter,
 * the limiter, or nothing; not the WENO limiter alone, which reads neighbours), this is
 * ONE launch: each CTA finishes its elements' stage values in shared memory, filters
 * and limits them there and writes out once.  Otherwise (1D, WENO, and the limiter
 * alone, which is faster as its own pass) it runs the stage and then the separate
 * passes.  Results equal the unfused sequence's up to rounding.  out may alias A (the
 * state updated in place) but not Us. */
enum { FRSDG_STAGE_MIXED = 1, FRSDG_STAGE_LIMIT = 2, FRSDG_STAGE_POST_STEP = 4 };
int frsdg_rk_stage_fused(frsdg_handle* h, double t, const double* Us, const double* A, double alpha,
                         const double* B, double beta, double gamma, double* out, double* acc,
                         double delta, int32_t flags, void* stream);

/* Element-diagonal blocks of the implicit Jacobian J = sigma*dM/dU + dR(M(U))/dU at
 * (t, U), by complex step (h = cfg.csd_eps) with element colouring, in one launch:
 * the preconditioner's part of ComplexStepJacobianStrategy::pre_jv_eval
 * (petsc_solver_impl.hpp:223-248), which assembles its preconditioner by DMDA-coloured
 * finite differences (MatFDColoringApply, 72-95, 244).  Elements of one colour share
 * no face, so seeding DOF d of every element of colour c gives column d of each such
 * element's block.  blocks: nelem * nd * nd doubles (nd = 4 (p+1)^2), block e
 * column-major: blocks[(e*nd + col)*nd + row].  2D only. */
int frsdg_jac_blocks(frsdg_handle* h, double t, double sigma, const double* U,
                     double* blocks, void* stream);

/* Block-Jacobi preconditioner for the Newton-Krylov solve (the PCSetUp / PCApply
 * pair PETSc runs on the coloured Jacobian): frsdg_pc_setup computes the blocks of
 * frsdg_jac_blocks into handle-owned storage (allocated by the first call:
 * nelem*nd*nd doubles and as many floats), inverts each block in FP64 with partial
 * pivoting, keeps the inverses in FP32, synchronises the stream and fails with
 * FRSDG_ERR_ARG on a zero pivot; p <= 5.  frsdg_pc_apply: z_e = inv(J_ee) r_e for
 * every element (z must not alias r). */
int frsdg_pc_setup(frsdg_handle* h, double t, double sigma, const double* U, void* stream);

/* All five blocks of every element row of the same Jacobian (the element and its four
 * face neighbours) from one complex-step launch with the distance-2 colouring
 * (i + 2 j) mod 5: blocks5: nelem * 5 * nd * nd doubles, block (e, s) column-major at
 * ((e*5 + s)*nd + col)*nd + row, s = 0 self, 1 right, 2 top, 3 bottom, 4 left (zero where
 * the neighbour does not exist).  2D, whole mesh; periodic directions need a multiple of
 * 5 elements. */
int frsdg_jac_blocks5(frsdg_handle* h, double t, double sigma, const double* U,
                      double* blocks5, void* stream);

/* Red-black block Gauss-Seidel preconditioner from those blocks (non-periodic 2D
 * meshes, p <= 5): frsdg_pc_setup_gs computes them into handle-owned storage (first call
 * allocates 5 nelem nd^2 doubles and 5 nelem nd^2 floats), inverts the diagonal blocks
 * (FP64, partial pivoting, kept in FP32), keeps the couplings in FP32 and makes
 * frsdg_pc_apply run one symmetric sweep: red z = D^-1 r; black z = D^-1 (r - J z_red);
 * red z -= D^-1 J z_black.  Synchronises the stream; FRSDG_ERR_ARG on a zero pivot. */
int frsdg_pc_setup_gs(frsdg_handle* h, double t, double sigma, const double* U, void* stream);
int frsdg_pc_apply(frsdg_handle* h, const double* r, double* z, void* stream);

/* Restarted GMRES on the device: the Krylov solver PETSc's KSPGMRES runs for every
 * Newton system of the implicit path (petsc_solver_impl.hpp:549-612; the reference
 * leaves it to PETSc), without a host round trip per iteration.  All arrays are device
 * memory; nothing is allocated.
 * frsdg_gmres_work_doubles: size (in doubles) of the scratch array `work` for vectors
 *   of n entries.
 * frsdg_gmres_arnoldi: Arnoldi step j (0 <= j < 256) on the basis V[0..j] (row i of V at
 *   V + i*ldv, n entries each): w <- w - V h by classical Gram-Schmidt, repeated once
 *   when the first pass leaves ||w||^2 below half its value; column j of the row-major
 *   Hessenberg H (leading dimension ldh > j, j + 2 rows) gets h and ||w||, then the
 *   previous Givens rotations (cs, sn) and a new one that zeroes H[j+1][j]; the
 *   least-squares residual vector g turns with it (|g[j+1]| is the new residual norm);
 *   *inv_hn = 1/||w|| (0 when w vanished), the scale of the next basis vector.
 * frsdg_gmres_solve: y = R^-1 g on the first k columns of the rotated H (back
 *   substitution; a zero diagonal leaves y at 0 there).
 * Reductions run in a fixed order: repeated calls give identical results. */
int64_t frsdg_gmres_work_doubles(int64_t n);
int frsdg_gmres_arnoldi(const double* V, int64_t ldv, int32_t j, double* w, int64_t n, double* H, int32_t ldh,
                        double* cs, double* sn, double* g, double* inv_hn, double* work, void* stream);
int frsdg_gmres_solve(const double* H, int32_t ldh, const double* g, int32_t k, double* y, void* stream);

/* One explicit Runge-Kutta stage fused into the residual pass:
 *   out = alpha*A + beta*B + gamma*rhs(Us),   acc += delta*rhs(Us)   (rhs = -R)
 * A, B and acc may be NULL (the term is dropped).  out must not alias Us (the
 * residual reads neighbouring elements of Us while out is written); A, B and acc may
 * alias each other or out.  SSP-RK3 and classic RK4 are sequences of such stages;
 * the reference delegates them to PETSc TS (petsc_solver_impl.hpp:549-612). */
int frsdg_rk_stage(frsdg_handle* h, double t, const double* Us, const double* A, double alpha,
                   const double* B, double beta, double gamma, double* out, double* acc, double delta,
                   void* stream);

/* In-place post-step stabilisation U <- limit(U) (spectral filter, WENO with
 * shock sensor): PetscSolver::apply_stabilization (petsc_solver_impl.hpp:683-702). */
int frsdg_post_step(frsdg_handle* h, double* U, void* stream);

/* Out-of-place post-step: dst = limit(src), src left unchanged; src and dst must not
 * alias (frsdg_post_step on dst with src's values gives the same result).  It has no
 * counterpart in the reference: a time integrator that writes its last stage to a
 * separate buffer limits it into the state directly, without the device copy of the
 * state that the in-place call makes for the WENO limiter. */
int frsdg_post_step_to(frsdg_handle* h, const double* src, double* dst, void* stream);

/* Positivity-preserving limiter on U in place (no counterpart in the reference):
 * per element, scale the density about its cell average until rho >= eps, then the
 * whole state until p >= eps (Zhang and Shu, J. Comput. Phys. 229 (2010) 8918-8934),
 * eps = min(cfg.pp_eps, rho_bar, p_bar); elements already admissible are left
 * untouched.  U32 (2D, may be NULL): an FP32 copy of U refreshed where U changes (for
 * callers that keep one for frsdg_residual_f32).  Does nothing unless cfg.pp_limit.  frsdg_post_step and
 * frsdg_post_step_to apply it after the stabilisation themselves; a time integrator
 * calls it on the output of every Runge-Kutta stage. */
int frsdg_pp_limit(frsdg_handle* h, double* U, float* U32, void* stream);

/* cons = M(prim): PetscSolver::primitive_to_conservative (petsc_solver_impl.hpp:719-727). */
int frsdg_prim_to_cons(frsdg_handle* h, const double* prim, double* cons, void* stream);

/* rhs = -R(U) with U and rhs in host memory; the copies to and from the device
 * use handle-owned staging buffers on `stream` and the call returns after the
 * result is in host memory.  For callers whose PETSc Vecs live on the host. */
int frsdg_rhs_host(frsdg_handle* h, double t, const double* U_host, double* rhs_host,
                   void* stream);

/* Device-side health word: number of nodes seen with a non-positive or
 * non-finite density by the residual calls since the previous frsdg_status call
 * (0 = healthy); the count restarts at zero.  Synchronises the handle's last
 * stream. */
int frsdg_status(frsdg_handle* h, int64_t* bad_nodes);

/* ---- batches of independent instances (no counterpart in the reference, which
 * runs one problem per process) -------------------------------------------------
 * A batch advances `count` 2D instances -- handles on the current device with affine
 * geometry, no row window and no change of variables -- by SSP-RK3 from t = 0 to their
 * own t_end with their own time step dt (the last step clipped to land on t_end, like
 * TS_EXACTFINALTIME_MATCHSTEP, petsc_solver_impl.hpp:556), each followed by its
 * handle's post-step (stabilisation and positivity limiter; the limiter also acts on
 * every stage output when cfg.pp_limit).  states[i] is instance i's device state,
 * advanced in place; the handles and states must outlive the batch.  mixed = 1: the
 * stages of frsdg_rk_stage_mixed (FP32 residual arithmetic, node primitives recovered
 * from the FP64 stage inputs in FP64, stage sums in FP64).
 * Instances sharing order, gas law, flux and VCJH correction form a group; one step is
 * one residual-and-stage launch per group and stage over the concatenated tiles of the
 * group's instances, one limiter launch per group and stage, one post-step launch per
 * group and one clock update: no host work per instance.  The first step or run times
 * the candidate tiles and persistent-CTA counts of every group with CUDA events and
 * keeps the fastest (cached per device, order, gas law, flux, precision and size).
 * frsdg_batch_step enqueues one step; frsdg_batch_run captures one step into a CUDA graph
 * and replays it until every instance has reached t_end (or max_steps > 0 steps),
 * reading the device's count of active instances every 16 steps, and returns the
 * number of steps taken.  Each handle's health word counts its instance's bad nodes.
 * dt_scale (may be NULL: fixed steps dt[i]): adaptive steps -- after every step,
 * dt = dt_scale[i] / max(|v| + c) over the instance's state (a CFL number times the
 * element size), which keeps the positivity limiter's CFL bound when near-vacuum nodes
 * raise the wave speed; dt[i] is the first step. */
typedef struct frsdg_batch frsdg_batch;
int frsdg_batch_create(frsdg_handle* const* handles, int32_t count, double* const* states, const double* dt,
                       const double* dt_scale, const double* t_end, int32_t mixed, frsdg_batch** out);
int frsdg_batch_step(frsdg_batch* b, void* stream);
int frsdg_batch_run(frsdg_batch* b, int64_t max_steps, int64_t* steps, void* stream);
/* current time of every instance (t[count]), whether it is still active and the steps it
 * has taken (active, steps: may be NULL).  With adaptive steps an instance whose step
 * would fall below 1e-3 of its initial dt (a state whose wave speed blew up) stops:
 * inactive with t < t_end. */
int frsdg_batch_times(const frsdg_batch* b, double* t, int32_t* active, int64_t* steps);
/* number of groups, and the autotuner's choice for one: order n, tile variant (0: the
 * tuned shape, 1: half its element rows), persistent CTAs of the stage launch, tiles,
 * and the stage launch time that decided it (ms) */
int frsdg_batch_groups(const frsdg_batch* b, int32_t* groups);
int frsdg_batch_tuning(const frsdg_batch* b, int32_t group, int32_t* order, int32_t* variant, int32_t* grid,
                       int32_t* tiles, float* stage_ms);
int frsdg_batch_destroy(frsdg_batch* b);

/* Add to the health word the nodes of U whose density is not positive and finite
 * (read back by frsdg_status).  The residual calls count the states they read; this
 * check covers a state that no residual has read yet, such as the output of the last
 * stage of a step: the time integrator's step rejection (the reference leaves it to
 * PETSc, -ts_max_reject, tools/c-vcjh_test.py:100-105) reads both. */
int frsdg_check_state(frsdg_handle* h, const double* U, void* stream);

/* The library's device FP64 reciprocal (op 0) and square root (op 1) -- a
 * single-precision seed refined by Newton steps, used throughout the residual --
 * applied elementwise to the device array x[0..n) into y, for validation against
 * IEEE division and sqrt.  Ops 2 and 3: the same in the deferred form of the residual's
 * node and face passes (the fast path, redone with ops 0 / 1 when the input lies
 * outside its range; equal to ops 0 / 1).  Ops 4 and 5: the FP32 reciprocal and square
 * root of the FP32 residual, on x rounded to float (results widened to double).  No
 * handle needed. */
int frsdg_device_math(int32_t op, const double* x, double* y, int64_t n, void* stream);

/* The split-precision tensor-core contraction of the FP32 residual on its own, for
 * validation (no counterpart in the reference; it stands for the derivative sums of
 * compute_volume_term, physics_impl_2D.hpp:320-354): out[l][k] = sum_m D[k][m]
 * v[l][m] for `lines` lines of n (2..8) FP32 values, D an n x n FP64 matrix, all
 * device arrays.  Values and D are split into TF32 high and low parts and multiplied
 * by tcgen05 MMAs with FP32 accumulation.  Synchronises the stream; returns
 * FRSDG_ERR_CUDA if the MMA completion wait gave up. */
int frsdg_tc_lines(int32_t n, const float* v, const double* D, float* out, int64_t lines, void* stream);

/* Largest solution (in doubles) frsdg_post_step_static accepts: 4,194,304 (32 MiB
 * of scratch held on every device that loads the library). */
#define FRSDG_POST_STEP_STATIC_MAX_DOFS 4194304

/* frsdg_post_step for callers that must not allocate device memory (for example
 * while a CUDA stream is being captured into a graph, where cudaMalloc is not
 * allowed, or under a memory manager that owns every allocation).  It has no
 * counterpart in the reference.  It takes the configuration instead of a handle
 * and allocates nothing: the copy the WENO limiter reads from is a fixed device
 * array of FRSDG_POST_STEP_STATIC_MAX_DOFS doubles inside the library; larger
 * solutions are rejected with FRSDG_ERR_ARG.  The first call in each CUDA context
 * looks up that array's device address, so make the first call outside any stream
 * capture.  Calls share the array: calls that overlap on the GPU (different
 * streams, or different host threads) race and must be ordered by the caller.
 * Every call rebuilds the small operators (filter matrix, differentiation matrix,
 * GLL weights) on the host from the configuration -- a few microseconds of host work
 * per call for p <= 9 -- and passes them by value to the kernel; a caller that
 * limits the same configuration often and may allocate should keep a handle and
 * call frsdg_post_step instead.
 * Results equal frsdg_post_step's for the same configuration and input. */
int frsdg_post_step_static(const frsdg_config* cfg, double* U, void* stream);

/* PETSc binary Vec records, the file format of `-ts_monitor_solution binary:<file>`
 * (options read by TSSetFromOptions, petsc_solver_impl.hpp:557; the record is
 * written by PETSc's VecView) that the reference's tools read back
 * (tools/plot.py:109-129, tools/check_iso_vortex.py:215-233).  One record = the
 * class id 1211214 and the length n as big-endian integers of index_bytes bytes
 * (4, or 8 for PETSc built with 64-bit indices), then n big-endian doubles.
 *
 * frsdg_petsc_vec_record_bytes: the record's size in bytes; FRSDG_ERR_ARG for
 * index_bytes other than 4 or 8, or n > 2^31-1 with index_bytes = 4.
 * frsdg_petsc_vec_pack: writes the record of the device vector x[0..n) into the
 * device buffer out (record_bytes long) on `stream`, asynchronously; x and out
 * 8-byte aligned.  A writer appends the bytes to the file as they are. */
int frsdg_petsc_vec_record_bytes(int64_t n, int32_t index_bytes, int64_t* bytes);
int frsdg_petsc_vec_pack(const double* x, int64_t n, int32_t index_bytes, void* out, void* stream);

/* Host-only set-up operators, usable without a GPU.
 * Reference element: GLL (reference_element.hpp:50-147) and CachedElementData
 * (cached_computations.hpp:8-137).  Arrays: nodes[n], weights[n], D[n*n]
 * (row-major D(i,j)), dL[n], dR[n] with n = p+1. */
int frsdg_reference_element(int32_t p, double radau_corr, double* nodes, double* weights,
                            double* D, double* dL, double* dR);

/* Spectral filter matrix V diag(sigma) V^-1 (filter.hpp:451-484), row-major n*n. */
int frsdg_filter_matrix(int32_t p, int32_t cut_off, int32_t strength, double alpha,
                        double* F);

#ifdef __cplusplus
}
#endif
#endif /* FRSDG_H */
