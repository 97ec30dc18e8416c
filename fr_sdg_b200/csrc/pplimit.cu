// pplimit.cu -- the positivity-preserving scaling limiter's kernels (the per-element
// limiter itself is in pplimit.cuh).  Elements that need no limiting are not written
// back, so a pass reads the state once and writes only limited elements.
//
// 2D: one warp per element (lanes over its nodes, shuffles for the cell sums and
// the minima); 1D: one thread per element.
#include "pplimit.hpp"
#include "pplimit.cuh"
#include "device_math.cuh"

#include <cuda_runtime.h>

namespace frsdg
{
namespace
{
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
    if (a.fused && b.slot >= 2) return;  // its last stage's epilogue is the post-step
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
                if (!(c.dt >= c.dt_floor)) c.active = 0;  // stalled (also a NaN step)
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
// validation against IEEE division and sqrt: op 0 / 1 the checked FP64 functions;
// 2 / 3 the deferred form the residual's node and face passes use (fast path, redone
// with the checked function when the input left the fast range); 4 / 5 the FP32 fast
// forms of the mixed residual (MathDeferred on float, redone with the IEEE operations),
// on x rounded to float, the result widened to double.
__global__ void device_math_kernel(int op, const double* x, double* y, int64_t n)
{
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = x[i];
    unsigned bad = 0;
    const MathDeferred md{bad};
    double r;
    switch (op)
    {
        case 0: r = s_rcp(v); break;
        case 1: r = s_sqrt(v); break;
        case 2: r = md.rcp(v); if (bad) r = s_rcp(v); break;
        case 3: r = md.sqrt(v); if (bad) r = s_sqrt(v); break;
        case 4:
        {
            const float f = static_cast<float>(v);
            float q = md.rcp(f);
            if (bad) q = s_rcp(f);
            r = q;
            break;
        }
        default:
        {
            const float f = static_cast<float>(v);
            float q = md.sqrt(f);
            if (bad) q = s_sqrt(f);
            r = q;
            break;
        }
    }
    y[i] = r;
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
