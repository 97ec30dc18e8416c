// frsdg_internal.hpp -- structures shared by the C-ABI host code and the kernels.
#pragma once
#include "../../include/frsdg.h"

#include <cstdint>
#include <cuda_runtime.h>

namespace frsdg
{

constexpr int kMaxN = 10;  // p <= 9
constexpr int kThreads = 256;

// Output forms of one residual pass (the PETSc callback each one serves).
enum Mode : int
{
    MODE_RESIDUAL = 0, // R(U)                      residual_kernel<double>
    MODE_RHS      = 1, // -R(U)                     rhs_func
    MODE_IFUNC    = 2, // U_t + R(M(U))             fun_implicit
    MODE_JVP      = 3, // sigma Im(u)/h + Im(R)/h   ComplexStepJacobianStrategy::matmult
    MODE_STAGE    = 4, // out = alpha A + beta B + gamma rhs, acc += delta rhs (rhs = -R): one RK stage
    MODE_JAC      = 5  // element-diagonal blocks of sigma dM/dU + dR(M(U))/dU, coloured complex step
};

// Explicit Runge-Kutta stage fused into the residual's output pass.
struct StageArgs
{
    const double* A;   // may be null (term dropped)
    const double* B;   // may be null
    double*       acc; // may be null
    double alpha, beta, gamma, delta;
    float*        out32; // may be null: FP32 copy of out (the next stage's input in mixed precision)
};

// Geometry classes of the 2D kernel: constant diagonal metrics (Cartesian and the
// straight de Laval channel) or cached per-node metrics and per-face normals.
enum GeoClass : int
{
    GEO_AFFINE = 0,
    GEO_CURVED = 1
};

struct BcDev
{
    int32_t kind;
    int32_t pad_;
    double  state[4];
    double  params[6];
};

// Small per-handle operators: differentiation matrix, VCJH correction derivatives.
struct Ops
{
    double D[kMaxN * kMaxN];
    double dL[kMaxN];
    double dR[kMaxN];
    double csi[kMaxN];
    float  Df[kMaxN * kMaxN];  // FP32 copies for the single-precision residual
    float  dLf[kMaxN];
    float  dRf[kMaxN];
    double F[kMaxN * kMaxN];   // spectral filter matrix (the stage epilogue's post-step)
};

// Operator entries in the arithmetic type T of a residual instantiation.
template <class T> __device__ __forceinline__ T opD(const Ops& o, int i);
template <> __device__ __forceinline__ double opD<double>(const Ops& o, int i) { return o.D[i]; }
template <> __device__ __forceinline__ float opD<float>(const Ops& o, int i) { return o.Df[i]; }
template <class T> __device__ __forceinline__ T opL(const Ops& o, int i);
template <> __device__ __forceinline__ double opL<double>(const Ops& o, int i) { return o.dL[i]; }
template <> __device__ __forceinline__ float opL<float>(const Ops& o, int i) { return o.dLf[i]; }
template <class T> __device__ __forceinline__ T opR(const Ops& o, int i);
template <> __device__ __forceinline__ double opR<double>(const Ops& o, int i) { return o.dR[i]; }
template <> __device__ __forceinline__ float opR<float>(const Ops& o, int i) { return o.dRf[i]; }

struct GasParams
{
    double gamma, a, b;
};

// Stage epilogue of the 2D residual kernel (MODE_STAGE): element-local work fused into
// the stage that produces a state, in this order -- the spectral filter of the
// post-step (the whole-element form of stab2d_tile's filter branch), the positivity
// limiter (pplimit.cuh), and the largest |v| + c of the result (adaptive time steps).
enum : int
{
    POST_FILTER = 1,
    POST_PP = 2,
    POST_AMAX = 4
};
struct PostArgs
{
    double w[kMaxN];           // GLL weights (the filter matrix is Ops::F)
    double pp_eps;             // the limiter's floor (cfg.pp_eps)
    const double* detJ;        // per-node detJ [global element][node] (curved meshes), or null
    unsigned long long* amax;  // POST_AMAX: atomicMax target (bits of a positive double)
};

struct Fr2dArgs
{
    int    Nx, Ny, per_x, per_y;
    GasParams gas;
    double xi_x, xi_y, eta_x, eta_y, scale_x, scale_y; // GEO_AFFINE
    const double* metrics;                              // GEO_CURVED: [elem][node][4] xi_x, xi_y, eta_x, eta_y
    const double* xnorm;                                // GEO_CURVED: [(j*(Nx+1)+I)*n + l][2]
    const double* ynorm;                                // GEO_CURVED: [(J*Nx+i)*n + k][2]
    const double* bxy[4];                               // boundary face points [idx][2], by direction
    BcDev  bc[4];
    double Lx, Ly;
    double t;
    int    mode, cond_sys;
    const double* U;   // state (primitive when cond_sys)
    const double* W;   // JVP: direction V; IFUNC: U_t
    void*  out;        // double* (float* for the FP32 residual)
    double h, inv_h, sigma;
    unsigned long long* bad;
    StageArgs st;
    int    nd;         // DOFs per element, 4 n^2
    int    out_f32;    // residual written as float (FP32 instantiation)
    // row window (domain decomposition): the vectors hold Ny element rows starting at
    // global row row_base; rows [row_begin, row_end) are computed, the others are ghosts
    int    row_base, row_begin, row_end;
    int    exact_bc;   // complex scalars: differentiate the user-lambda boundary kinds too
    int    jac_cmode;  // MODE_JAC colouring: 0 checkerboard, 1 three-colour cycles (odd periodic),
                       // 2 distance-2 colouring (i + 2 j) mod 5 for all five blocks of an element row
    int    in_f64;     // FP32 instantiation: U is an FP64 state, node primitives recovered in FP64
    int    tc;         // FP32 instantiation at n = 5, 6: derivative contractions on the tensor cores
    Ops    ops;
    // (after the operators: a batch launch sets these per stage, not per instance)
    int    post;       // MODE_STAGE: element-local post-processing of the stage output (POST_*)
    int    pad_post_;
    const PostArgs* pa;  // its operands (device memory) when post != 0
};

// ---- batches of instances (batch.cu) ----------------------------------------
// Clock of one instance of a batch: the device-side time loop of frsdg_batch_run.
// One step takes h = dt, or the remainder t_end - t when a full step would overshoot
// (by more than 1e-14 relative), and the instance stays active while t < t_end.
struct BatchClock
{
    double t, dt, t_end;
    int    active, adaptive;
    // adaptive: after every step dt = dt_scale / max(|v| + c) over the instance's
    // state (amax, the bit pattern of that positive double, gathered by the limiter
    // pass of the state)
    double dt_scale;
    unsigned long long amax;
    long long steps;   // steps taken
    // adaptive: an instance whose step falls below dt_floor (a blown-up state's wave
    // speed) stops where it is -- inactive before t_end -- instead of crawling on
    double dt_floor;
};

__host__ __device__ inline double batch_step_size(const BatchClock& c)
{
    const double tol = 1e-14 * (c.t_end > 1.0 ? c.t_end : (c.t_end < -1.0 ? -c.t_end : 1.0));
    return c.t + c.dt <= c.t_end + tol ? c.dt : c.t_end - c.t;
}

// One instance of a batch group: its residual launch template (the operators are the
// group's) and its state and stage buffers.
struct BatchInst2D
{
    Fr2dArgs a;
    double*  U;       // state
    double*  b[3];    // SSP-RK3 stage outputs (b[2]: the last, limited into U by the post-step)
    int      inst;    // batch index (clock)
    int      fused_step;  // the post-step is the last stage's epilogue, which writes U
    int      post[3];     // stage epilogue of each stage (Fr2dArgs::post)
    int      pad_;
    const PostArgs* pa;   // its operands
};

struct Fr2dBatchArgs
{
    Ops ops;
    const BatchInst2D* inst;
    const BatchClock*  clock;
    const int4*        tiles;  // (instance in group, bx, by, -)
    int ntiles;
    int stage;                 // SSP-RK3 stage 0, 1, 2
    int mixed;
};

// Colour of element (gi, gj) for the coloured Jacobian: no two elements sharing a
// face have the same colour.  Checkerboard, or, when a periodic direction has an
// odd number of elements, (i mod 2 | 2 for the last) + 3 (j mod 2 | 2 for the last).
__host__ __device__ inline int elem_colour(int cmode, int Nx, int Ny, int per_x, int per_y, int gi, int gj)
{
    if (cmode == 0) return (gi + gj) & 1;
    if (cmode == 2) return (gi + 2 * gj) % 5;
    const int cx = (per_x && (Nx & 1) && gi == Nx - 1) ? 2 : (gi & 1);
    const int cy = (per_y && (Ny & 1) && gj == Ny - 1) ? 2 : (gj & 1);
    return cx + 3 * cy;
}

struct Fr1dArgs
{
    int    N, per;
    GasParams gas;
    double inv_jac, h_elem;
    int    radial;
    BcDev  bc[2];
    double t;
    int    mode, cond_sys;
    const double* U;
    const double* W;
    void*  out;
    double h, inv_h, sigma;
    unsigned long long* bad;
    StageArgs st;
    Ops    ops;
};

// Tile of elements per CTA of the 2D kernel: TX along x (contiguous in memory)
// by TY along y, about 100-400 nodes per tile, for the FP64 (words = 1), complex
// (words = 2) and FP32 (f32) residuals.  face_tiles() selects the shapes sized by
// face points (with the block size and register cap chosen in residual2d.cuh);
// the others keep one thread per tile node.
// FRSDG_TX / FRSDG_TY override the shape for tuning builds.
__host__ __device__ constexpr bool face_tiles(int n, int words, bool f32)
{
    return words == 1 && (f32 ? (n == 5 || n == 6) : n >= 5);
}
__host__ __device__ constexpr int tile_x(int n, int words, bool f32)
{
#ifdef FRSDG_TX
    return FRSDG_TX;
#else
    if (face_tiles(n, words, f32)) return n == 5 ? 4 : 2;
    return n <= 2 ? 8 : n <= 3 ? 8 : n <= 4 ? 4 : n <= 6 ? 4 : 2;
#endif
}
__host__ __device__ constexpr int tile_y(int n, int words, bool f32)
{
#ifdef FRSDG_TY
    return FRSDG_TY;
#else
    if (face_tiles(n, words, f32)) return n == 5 ? 2 : n == 6 ? 4 : n <= 9 ? 2 : 1;
    return n <= 2 ? 8 : n <= 3 ? 4 : n <= 4 ? 4 : n <= 6 ? 2 : n <= 9 ? 2 : 1;
#endif
}

// Launchers (one translation unit per polynomial order).
template <class S, int N> cudaError_t launch_fr2d(int gas, int riem, int geo, const Fr2dArgs& a, cudaStream_t s);
template <class S, int N> cudaError_t launch_fr1d(int gas, int riem, const Fr1dArgs& a, cudaStream_t s);
template <class S, int N>
cudaError_t launch_fr2d_batch(int gas, int riem, int var, const Fr2dBatchArgs& b, int grid, cudaStream_t s,
                              int* occupancy);

// Stage combination alpha A + beta B + gamma rhs at index idx (rhs = -r), with the
// accumulator update acc += delta rhs.
__device__ __forceinline__ double stage_value(const StageArgs& st, int64_t idx, double r)
{
    const double v = -r;
    double o = 0.0;
    if (st.A) o = st.alpha * __ldg(st.A + idx);
    if (st.B) o = o + st.beta * __ldg(st.B + idx);
    if (st.acc) st.acc[idx] = st.acc[idx] + st.delta * v;
    return o + st.gamma * v;
}

// Output of one real residual value r = R at index idx in the requested form.
__device__ __forceinline__ void store_residual(int mode, const double* W, const StageArgs& st, double* out,
                                               int64_t idx, double r)
{
    if (mode == MODE_RHS) out[idx] = -r;
    else if (mode == MODE_IFUNC) out[idx] = __ldg(W + idx) + r;
    else if (mode == MODE_STAGE)
    {
        const double ov = stage_value(st, idx, r);
        out[idx] = ov;
        if (st.out32) st.out32[idx] = static_cast<float>(ov);
    }
    else out[idx] = r;
}

} // namespace frsdg
