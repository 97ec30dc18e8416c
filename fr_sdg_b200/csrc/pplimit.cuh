// pplimit.cuh -- the per-element positivity-preserving scaling limiter (Zhang and Shu,
// "On positivity-preserving high order discontinuous Galerkin schemes for compressible
// Euler equations on rectangular meshes", J. Comput. Phys. 229 (2010) 8918-8934,
// sec. 3), shared by the limiter kernels (pplimit.cu) and the fused stage epilogue of
// the residual kernel (residual2d.cuh):
//   Ubar = GLL-quadrature cell average (weights w_k w_l detJ_kl in 2D, w_k in 1D),
//   eps = min(eps0, rho_bar, p_bar); elements with an inadmissible average are kept;
//   1. rho_min < eps:  rho <- rho_bar + theta1 (rho - rho_bar),
//                      theta1 = (rho_bar - eps) / (rho_bar - rho_min);
//   2. U <- Ubar + theta2 (U - Ubar), theta2 = min over nodes with p < eps of the
//      point t of the segment Ubar -> U_q with pressure eps (60 bisection steps,
//      keeping the admissible end).
// It has no counterpart in the reference.  The argument type PA provides gas_law, gas,
// eps0, w[] (GLL weights) and detJ (per-node Jacobian determinants, or null).
#pragma once
#include "device_math.cuh"
#include "frsdg_internal.hpp"

namespace frsdg
{

// The limiter's view of a stage epilogue's arguments (PostArgs and the kernel's gas)
struct PPView
{
    int           gas_law;
    GasParams     gas;
    double        eps0;
    const double* w;
    const double* detJ;
};


template <class PA> __device__ __forceinline__ double pp_gas_pressure(const PA& a, double rho, double e)
{
    if (a.gas_law == FRSDG_GAS_IDEAL) return (a.gas.gamma - 1.0) * rho * e;
    const double covol = 1.0 - a.gas.b * rho;
    const double cvT = e + a.gas.a * rho;
    return ((a.gas.gamma - 1.0) * rho * cvT) / covol - a.gas.a * rho * rho;
}

template <int NV, class PA> __device__ __forceinline__ double pp_pressure(const PA& a, const double* u)
{
    double m2 = 0.0;
#pragma unroll
    for (int c = 1; c < NV - 1; ++c) m2 += u[c] * u[c];
    const double rho = u[0];
    const double e = (u[NV - 1] - 0.5 * m2 / rho) / rho;
    return pp_gas_pressure(a, rho, e);
}

// |v| + c of a node (the sound speed of the configured gas law, c^2 clamped at 0)
template <class PA> __device__ __forceinline__ double node_wave_speed(const PA& a, const double* u)
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

// The same quantities with reciprocals (device_math.cuh: within 2 ulp of the
// quotients): the screen that lets admissible elements skip the limiter, and the wave
// speed of the adaptive time step, where rounding is immaterial.
template <class PA, class M = MathChecked>
__device__ __forceinline__ double pp_pressure_fast(const PA& a, const double* u, const M& m = M{})
{
    const double ir = m.rcp(u[0]);
    const double rho_e = u[3] - 0.5 * (u[1] * u[1] + u[2] * u[2]) * ir;  // rho e
    if (a.gas_law == FRSDG_GAS_IDEAL) return (a.gas.gamma - 1.0) * rho_e;
    const double rho = u[0];
    return ((a.gas.gamma - 1.0) * (rho_e + a.gas.a * rho * rho)) * m.rcp(1.0 - a.gas.b * rho) - a.gas.a * rho * rho;
}
template <class PA> __device__ __forceinline__ double node_wave_speed_fast(const PA& a, const double* u)
{
    const double rho = u[0], ir = s_rcp(rho);
    const double vx = u[1] * ir, vy = u[2] * ir;
    const double v2 = vx * vx + vy * vy;
    const double e = u[3] * ir - 0.5 * v2;
    double c2;
    if (a.gas_law == FRSDG_GAS_IDEAL) c2 = a.gas.gamma * (a.gas.gamma - 1.0) * e;
    else
    {
        const double cov = 1.0 - a.gas.b * rho, gm1 = a.gas.gamma - 1.0, ic2 = s_rcp(cov * cov);
        c2 = (a.gas.gamma * gm1 * (e + a.gas.a * rho)) * ic2 + (gm1 * a.gas.a * rho * (2.0 - a.gas.b * rho)) * ic2 -
             2.0 * a.gas.a * rho;
    }
    return s_sqrt(v2) + s_sqrt(fmax(c2, 0.0));
}

template <int NV, class PA>
__device__ __forceinline__ double pp_segment_root(const PA& a, const double* ub, const double* uq, double eps)
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

__device__ __forceinline__ double pp_warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double pp_warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// One element of a 2D state, limited by one warp: base / base32 point at the element's
// values (base32 may be null), e_glob is its global index for the cached detJ;
// refresh32: write the FP32 copy even when the element is admissible.
template <int N, class PA>
__device__ __forceinline__ void pp_element2d(const PA& a, double* base, float* base32, int64_t e_glob,
                                             bool limit, bool refresh32, unsigned long long* amax = nullptr)
{
    constexpr int NQ = N * N, R = (NQ + 31) / 32;
    const int lane = threadIdx.x & 31;
    double u[R][4], W[R];
    double wsum = 0.0, ub[4] = {0.0, 0.0, 0.0, 0.0};
    // screen: an element whose nodes all have density and pressure above eps0 is left
    // as it is (eps <= eps0), so it needs no cell average (nodes within 1e-10 of the
    // floor take the exact path)
    // (the pressures' reciprocals with deferred range checks: one redo of the screen when
    // an input left the fast range, instead of a branch per reciprocal; the same result)
    bool clear = true;
    unsigned bad = 0;
    const double thr = a.eps0 * (1.0 + 1e-10);
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        const int q = lane + 32 * r;
        u[r][0] = u[r][1] = u[r][2] = u[r][3] = 0.0;
        if (q < NQ)
        {
            const double2 x0 = *reinterpret_cast<const double2*>(base + q * 4);
            const double2 x1 = *reinterpret_cast<const double2*>(base + q * 4 + 2);
            u[r][0] = x0.x; u[r][1] = x0.y; u[r][2] = x1.x; u[r][3] = x1.y;
            clear = clear && u[r][0] > thr && pp_pressure_fast(a, u[r], MathDeferred{bad}) > thr;
        }
    }
    if (bad)
    {
        clear = true;
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (lane + 32 * r < NQ) clear = clear && u[r][0] > thr && pp_pressure_fast(a, u[r]) > thr;
    }
    if (__all_sync(0xffffffffu, clear || !limit))
    {
        if (amax)
        {
            double w = 0.0;
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (lane + 32 * r < NQ) w = fmax(w, node_wave_speed_fast(a, u[r]));
            w = -pp_warp_min(-w);
            if (lane == 0 && w > 0.0 && w < 1e300)
                atomicMax(amax, static_cast<unsigned long long>(__double_as_longlong(w)));
        }
        if (refresh32 && base32)
        {
#pragma unroll
            for (int r = 0; r < R; ++r)
            {
                const int q = lane + 32 * r;
                if (q < NQ)
                    *reinterpret_cast<float4*>(base32 + q * 4) =
                        make_float4(float(u[r][0]), float(u[r][1]), float(u[r][2]), float(u[r][3]));
            }
        }
        return;
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
    {
        const int q = lane + 32 * r;
        W[r] = q < NQ ? a.w[q % N] * a.w[q / N] * (a.detJ ? __ldg(a.detJ + e_glob * NQ + q) : 1.0) : 0.0;
        wsum += W[r];
#pragma unroll
        for (int c = 0; c < 4; ++c) ub[c] += W[r] * u[r][c];
    }
    wsum = pp_warp_sum(wsum);
#pragma unroll
    for (int c = 0; c < 4; ++c) ub[c] = pp_warp_sum(ub[c]) / wsum;
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
        rmin = pp_warp_min(rmin);
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
        th2 = pp_warp_min(th2);
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
            if (lane + 32 * r < NQ) w = fmax(w, node_wave_speed_fast(a, u[r]));
        w = -pp_warp_min(-w);
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

} // namespace frsdg
