// handle.hpp -- the frsdg_handle behind the C ABI (include/frsdg.h), shared by the
// translation units that implement entry points on handles (capi.cu, batch.cu).
//
// The handle plays the role of the reference's PhysicsEvaluator + PetscSolver pair
// (physics_evaluator.hpp:158-318, petsc_solver_impl.hpp:444-755): it owns the reference
// element, the filter, the cached curved metrics, the boundary data and every workspace.
#pragma once
#include "../../include/frsdg.h"
#include "frsdg_internal.hpp"
#include "pplimit.hpp"
#include "setup_ops.hpp"
#include "stab.hpp"

#include <cuda_runtime.h>

struct frsdg_handle
{
    frsdg_config cfg{};
    int          n = 0, Nx = 0, Ny = 0, ndofs = 0;
    int64_t      ntot = 0, nelem = 0;
    int          geo = frsdg::GEO_AFFINE;
    frsdg::RefElem      re;
    frsdg::Fr2dArgs     a2{};   // template of the 2D launch arguments
    frsdg::Fr1dArgs     a1{};
    frsdg::StabArgs     st{};
    double*      d_metrics = nullptr;
    double*      d_xnorm = nullptr;
    double*      d_ynorm = nullptr;
    double*      d_bxy = nullptr;
    double*      d_detJ = nullptr;   // positivity limiter on curved meshes: detJ per node
    frsdg::PPArgs       pp{};               // template of the positivity limiter's launch
    frsdg::PostArgs*    d_post = nullptr;   // 2D: operands of the fused stage epilogue
    double*      d_work = nullptr;   // post-step source copy (WENO)
    double*      d_stage = nullptr;  // host-buffer staging (2 * ntot), allocated on first use
    unsigned long long* d_bad = nullptr;
    double*      d_blocks = nullptr;  // preconditioner: element-diagonal Jacobian blocks (FP64)
    float*       d_inv = nullptr;     // and their inverses (FP32); both allocated by the first frsdg_pc_setup
    unsigned long long* d_singular = nullptr;
    double*      d_blocks5 = nullptr; // block Gauss-Seidel: the five blocks of every element row (FP64)
    float*       d_off = nullptr;     // and the four off-diagonal ones in FP32; allocated by frsdg_pc_setup_gs
    int          pc_kind = 0;         // 0 none, 1 block Jacobi, 2 block Gauss-Seidel
    double       jvp_t = 0.0, jvp_sigma = 1.0;
    const double* jvp_U = nullptr;
    cudaStream_t last = nullptr;
    int          device = 0;
    // row window (frsdg_set_row_window); win_rows == 0: the vectors are the whole mesh
    int          win_rows = 0, win_base = 0, win_begin = 0, win_end = 0;
    // frsdg_rhs_host pipeline: upload / compute / download streams and their events
#ifdef FRSDG_HOST_CHUNKS
    static constexpr int kHostChunks = FRSDG_HOST_CHUNKS;  // tuning builds
#else
    static constexpr int kHostChunks = 32;  // at most; at least 4 element rows per chunk
#endif
    cudaStream_t hst[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t  hev[2 * kHostChunks + 2] = {};
};
