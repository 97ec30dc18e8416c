// pplimit.cu -- positivity-preserving scaling limiter (Zhang and Shu, "On
// positivity-preserving high order discontinuous Galerkin schemes for compressible
// Euler equations on rectangular meshes", J. Comput. Phys. 229 (2010) 8918-8934,
// sec. 3), per element, in place:
//   Ubar = GLL-quadrature cell average (weights w_k w_l detJ_kl in 2D, w_k in 1D),
//   eps = min(eps0, rho_bar, p_bar); elements with an inadmissible average are kept;
//   1. rho_min < eps:  rho <- rho_bar + theta1 (rho - rho_bar),
//                      theta1 = (rho_bar - eps) / (rho_bar - rho_min);
//   2. U <- Ubar + theta2 (U - Ubar), theta2 = min over nodes with p < eps of the
//      point t of the segment Ubar -> U_q with pressure eps (60 bisection steps,
//      keeping the admissible end).
// It has no counterpart in the reference.  Elements that need no limiting are not
// written back, so the pass reads the state once and writes only limited elements.
//
// 2D: one warp per element (lanes over its nodes, shuffles for the cell sums and
// the minima); 1D: one thread per element.
#include "pplimit.hpp"
#include "device_math.cuh"

#include <cuda_runtime.h>

namespace frsdg
{
namespace
{

__device__ __forceinline__ double pp_gas_pressure(const PPArgs& a, double rho, double e)
{
    if (a.gas_law == FRSDG_GAS_IDEAL) return (a.gas.gamma - 1.0) * rho * e;
    const double covol = 1.0 - a.gas.b * rho;
    const double cvT = e + a.gas.a * rho;
    return ((a.gas.gamma - 1.0) * rho * cvT) / covol - a.gas.a * rho * rho;
}

template <int NV> __device__ __forceinline__ double pp_pressure(const PPArgs& a, const double* u)
{
    double m2 = 0.0;
#pragma unroll
    for (int c = 1; c < NV - 1; ++c) m2 += u[c] * u[c];
    const double rho = u[0];
    const double e = (u[NV - 1] - 0.5 * m2 / rho) / rho;
    return pp_gas_pressure(a, rho, e);
}

// |v| + c of a node (the sound speed of the configured gas law, c^2 clamped at 0)
__device__ __forceinline__ double node_wave_speed(const PPArgs& a, const double* u)
{
    const double rho = u[0];
    const double vx = u[1] / rho, vy = u[2] / rho;
    const double e = u[3] / rho - 0.5 * (vx * vx + vy * vy);
    double c2;
    if (a.gas_law == FRSDG_GAS_IDEAL) c2 = a.gas.gamma * (a.gas.gamma - 1.0) * e;
    else
    {
        const double cov = 1.0 - a.gas.b * rho, gm1 = a.gas.gamma - 1.0;
        c2 = (a.gas.gamma * gm1 * (e + a.gas.a * rho)) / (cov * cov) +
             (gm1 * a.gas.a * rho * (2.0 - a.gas.b * rho)) / (cov * cov) - 2.0 * a.gas.a * rho;
    }
    return sqrt(vx * vx + vy * vy) + sqrt(fmax(c2, 0.0));
}

template <int NV>
__device__ __forceinline__ double pp_segment_root(const PPArgs& a, const double* ub, const double* uq, double eps)
{
    double lo = 0.0, hi = 1.0, s[NV];
    for (int it = 0; it < 60; ++it)
    {
        const double mid = 0.5 * (lo + hi);
#pragma unroll
        for (int c = 0; c < NV; ++c) s[c] = ub[c] + mid * (uq[c] - ub[c]);
        if (s[0] > 0.0 && pp_pressure<NV>(a, s) >= eps) lo = mid;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// One element of a 2D state, limited by one warp: base / base32 point at the element's
// values (base32 may be null), e_glob is its global index for the cached detJ;
// refresh32: write the FP32 copy even when the element is admissible.
template <int N>
__device__ __forceinline__ void pp_element2d(const PPArgs& a, double* base, float* base32, int64_t e_glob,
                                             bool limit, bool refresh32, unsigned long long* amax = nullptr)
{
    constexpr int NQ = N * N, R = (NQ + 31) / 32;
    const int lane = threadIdx.x & 31;
    double u[R][4], W[R];
    double wsum = 0.0, ub[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        const int q = lane + 32 * r;
        W[r] = 0.0;
        u[r][0] = u[r][1] = u[r][2] = u[r][3] = 0.0;
        if (q < NQ)
        {
            const double2 x0 = *reinterpret_cast<const double2*>(base + q * 4);
            const double2 x1 = *reinterpret_cast<const double2*>(base + q * 4 + 2);
            u[r][0] = x0.x; u[r][1] = x0.y; u[r][2] = x1.x; u[r][3] = x1.y;
            W[r] = a.w[q % N] * a.w[q / N] * (a.detJ ? __ldg(a.detJ + e_glob * NQ + q) : 1.0);
        }
        wsum += W[r];
#pragma unroll
        for (int c = 0; c < 4; ++c) ub[c] += W[r] * u[r][c];
    }
    wsum = warp_sum(wsum);
#pragma unroll
    for (int c = 0; c < 4; ++c) ub[c] = warp_sum(ub[c]) / wsum;
    const double pb = pp_pressure<4>(a, ub);
    bool touched = false;
    // the limiter acts when enabled and the cell average is admissible (uniform across the warp)
    if (limit && ub[0] > 0.0 && pb > 0.0)
    {
        const double eps = fmin(a.eps0, fmin(ub[0], pb));
        double rmin = 1e300;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (lane + 32 * r < NQ) rmin = fmin(rmin, u[r][0]);
        rmin = warp_min(rmin);
        if (rmin < eps)
        {
            const double th1 = (ub[0] - eps) / (ub[0] - rmin);
#pragma unroll
            for (int r = 0; r < R; ++r) u[r][0] = ub[0] + th1 * (u[r][0] - ub[0]);
            touched = true;
        }
        double th2 = 1.0;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (lane + 32 * r < NQ && !(pp_pressure<4>(a, u[r]) >= eps)) th2 = fmin(th2, pp_segment_root<4>(a, ub, u[r], eps));
        th2 = warp_min(th2);
        if (th2 < 1.0)
        {
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) u[r][c] = ub[c] + th2 * (u[r][c] - ub[c]);
            touched = true;
        }
    }
    if (amax)
    {
        // the largest |v| + c of the (limited) element, for the next adaptive time step
        double w = 0.0;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (lane + 32 * r < NQ) w = fmax(w, node_wave_speed(a, u[r]));
        w = -warp_min(-w);
        if (lane == 0 && w > 0.0 && w < 1e300) atomicMax(amax, static_cast<unsigned long long>(__double_as_longlong(w)));
    }
    if (!touched && !refresh32) return;
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        const int q = lane + 32 * r;
        if (q >= NQ) continue;
        if (touched)
        {
            *reinterpret_cast<double2*>(base + q * 4) = make_double2(u[r][0], u[r][1]);
            *reinterpret_cast<double2*>(base + q * 4 + 2) = make_double2(u[r][2], u[r][3]);
        }
        if (base32)
            *reinterpret_cast<float4*>(base32 + q * 4) =
                make_float4(float(u[r][0]), float(u[r][1]), float(u[r][2]), float(u[r][3]));
    }
}

template <int N> __global__ void __launch_bounds__(256) pp_limit2d_kernel(const PPArgs a)
{
    constexpr int NQ = N * N;
    const int64_t e = int64_t(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32;
    if (e >= a.nelem) return;  // whole warps leave together
    // the element's global row, for the cached detJ of a curved mesh (row windows wrap)
    const int64_t j_loc = e / a.Nx;
    const int64_t j_glob = ((j_loc + a.row_base) % a.Ny + a.Ny) % a.Ny;
    const int64_t e_glob = j_glob * a.Nx + (e - j_loc * a.Nx);
    pp_element2d<N>(a, a.U + e * (4 * NQ), a.U32 ? a.U32 + e * (4 * NQ) : nullptr, e_glob, true, false);
}

template <int N> __global__ void __launch_bounds__(256) pp_batch_kernel(const PPBatchArgs b)
{
    constexpr int NQ = N * N;
    const int64_t g = int64_t(blockIdx.x) * (blockDim.x / 32) + threadIdx.x / 32;
    if (g >= b.nelem) return;  // whole warps leave together
    int lo = 0, hi = b.ninst;  // instance i with elem_begin[i] <= g < elem_begin[i + 1]
    while (hi - lo > 1)
    {
        const int mid = (lo + hi) / 2;
        if (b.elem_begin[mid] <= g) lo = mid;
        else hi = mid;
    }
    const BatchInst2D& in = b.binst[lo];
    if (!b.clock[in.inst].active) return;
    const PPArgs& a = b.inst[lo];
    const int64_t e = g - b.elem_begin[lo];
    // slots 0-2: the stage outputs; 3: the state after the post-step
    double* buf = b.slot == 3 ? in.U : in.b[b.slot];
    const bool limit = a.enabled != 0;
    if (!limit && !(b.slot == 3 && b.clock[in.inst].adaptive)) return;
    // the state after the post-step also yields the instance's wave speed (adaptive dt)
    unsigned long long* amax = b.slot == 3 && b.clock[in.inst].adaptive ? &b.clock[in.inst].amax : nullptr;
    pp_element2d<N>(a, buf + e * (4 * NQ), nullptr, 0, limit, false, amax);
}

__global__ void batch_clock_kernel(BatchClock* clock, int count, int* active_count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count)
    {
        BatchClock c = clock[i];
        if (c.active)
        {
            const double h = batch_step_size(c);
            c.t = h == c.dt ? c.t + c.dt : c.t_end;
            ++c.steps;
            const double tol = 1e-14 * (c.t_end > 1.0 ? c.t_end : (c.t_end < -1.0 ? -c.t_end : 1.0));
            c.active = c.t < c.t_end - tol;
            if (c.adaptive)
            {
                const double w = __longlong_as_double(static_cast<long long>(c.amax));
                if (c.amax && w > 0.0) c.dt = c.dt_scale / w;
                c.amax = 0ull;
            }
            clock[i] = c;
        }
        if (c.active && active_count) atomicAdd(active_count, 1);
    }
}

template <int N> __global__ void __launch_bounds__(128) pp_limit1d_kernel(const PPArgs a)
{
    const int64_t e = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (e >= a.nelem) return;
    double* u = a.U + e * (3 * N);
    double wsum = 0.0, ub[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < N; ++q)
    {
        wsum += a.w[q];
        for (int c = 0; c < 3; ++c) ub[c] += a.w[q] * u[c * N + q];
    }
    for (int c = 0; c < 3; ++c) ub[c] /= wsum;
    const double pb = pp_pressure<3>(a, ub);
    if (!(ub[0] > 0.0) || !(pb > 0.0)) return;
    const double eps = fmin(a.eps0, fmin(ub[0], pb));
    double rmin = u[0];
    for (int q = 1; q < N; ++q) rmin = fmin(rmin, u[q]);
    if (rmin < eps)
    {
        const double th1 = (ub[0] - eps) / (ub[0] - rmin);
        for (int q = 0; q < N; ++q) u[q] = ub[0] + th1 * (u[q] - ub[0]);
    }
    double th2 = 1.0;
    for (int q = 0; q < N; ++q)
    {
        const double uq[3] = {u[q], u[N + q], u[2 * N + q]};
        if (!(pp_pressure<3>(a, uq) >= eps)) th2 = fmin(th2, pp_segment_root<3>(a, ub, uq, eps));
    }
    if (th2 < 1.0)
        for (int q = 0; q < N; ++q)
            for (int c = 0; c < 3; ++c) u[c * N + q] = ub[c] + th2 * (u[c * N + q] - ub[c]);
}

template <int N> cudaError_t launch_pp_batch_n(const PPBatchArgs& b, cudaStream_t s)
{
    if (b.nelem <= 0) return cudaSuccess;
    pp_batch_kernel<N><<<unsigned((b.nelem + 7) / 8), 256, 0, s>>>(b);
    return cudaGetLastError();
}

template <int N> cudaError_t launch_n(const PPArgs& a, cudaStream_t s)
{
    if (a.nelem <= 0) return cudaSuccess;
    if (a.dim == 2)
    {
        const int64_t blocks = (a.nelem + 7) / 8;
        pp_limit2d_kernel<N><<<unsigned(blocks), 256, 0, s>>>(a);
    }
    else
    {
        const int64_t blocks = (a.nelem + 127) / 128;
        pp_limit1d_kernel<N><<<unsigned(blocks), 128, 0, s>>>(a);
    }
    return cudaGetLastError();
}

// Health check of a state: nodes whose density is not positive and finite, added to
// the handle's health word (one atomic per warp that found any).
__global__ void __launch_bounds__(256) check_density_kernel(const double* U, int64_t nodes, int stride_node,
                                                            int stride_elem, int per_elem, unsigned long long* bad)
{
    const int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    bool b = false;
    if (q < nodes)
    {
        const int64_t e = q / per_elem, k = q - e * per_elem;
        const double rho = __ldg(U + e * stride_elem + k * stride_node);
        b = !(rho > 0.0) || !(rho < 1e308);
    }
    const unsigned m = __ballot_sync(0xffffffffu, b);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(bad, (unsigned long long)__popc(m));
}

// The library's device reciprocal and square root (device_math.cuh), elementwise, for
// validation against IEEE division and sqrt.
__global__ void device_math_kernel(int op, const double* x, double* y, int64_t n)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    y[i] = op == 0 ? s_rcp(x[i]) : s_sqrt(x[i]);
}

} // namespace

cudaError_t launch_pp_batch(int n, const PPBatchArgs& b, cudaStream_t s)
{
    switch (n)
    {
        case 2: return launch_pp_batch_n<2>(b, s);
        case 3: return launch_pp_batch_n<3>(b, s);
        case 4: return launch_pp_batch_n<4>(b, s);
        case 5: return launch_pp_batch_n<5>(b, s);
        case 6: return launch_pp_batch_n<6>(b, s);
        case 7: return launch_pp_batch_n<7>(b, s);
        case 8: return launch_pp_batch_n<8>(b, s);
        case 9: return launch_pp_batch_n<9>(b, s);
        case 10: return launch_pp_batch_n<10>(b, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batch_clock(BatchClock* clock, int count, int* active_count, cudaStream_t s)
{
    if (count <= 0) return cudaSuccess;
    batch_clock_kernel<<<(count + 255) / 256, 256, 0, s>>>(clock, count, active_count);
    return cudaGetLastError();
}

cudaError_t launch_check_density(int dim, int n, int64_t nelem, const double* U, unsigned long long* bad,
                                 cudaStream_t s)
{
    const int per_elem = dim == 2 ? n * n : n;
    const int64_t nodes = nelem * per_elem;
    if (nodes <= 0) return cudaSuccess;
    // 2D: density of node q at q*4 (node-major AoS); 1D: eq 0 of element e at e*3n + k
    const int stride_node = dim == 2 ? 4 : 1, stride_elem = dim == 2 ? 4 * n * n : 3 * n;
    check_density_kernel<<<unsigned((nodes + 255) / 256), 256, 0, s>>>(U, nodes, stride_node, stride_elem,
                                                                        per_elem, bad);
    return cudaGetLastError();
}

cudaError_t launch_device_math(int op, const double* x, double* y, int64_t n, cudaStream_t s)
{
    if (n <= 0) return cudaSuccess;
    device_math_kernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(op, x, y, n);
    return cudaGetLastError();
}

cudaError_t launch_pp_limit(const PPArgs& a, cudaStream_t s)
{
    switch (a.n)
    {
        case 2: return launch_n<2>(a, s);
        case 3: return launch_n<3>(a, s);
        case 4: return launch_n<4>(a, s);
        case 5: return launch_n<5>(a, s);
        case 6: return launch_n<6>(a, s);
        case 7: return launch_n<7>(a, s);
        case 8: return launch_n<8>(a, s);
        case 9: return launch_n<9>(a, s);
        case 10: return launch_n<10>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace frsdg
