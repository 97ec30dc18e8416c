// physics.cuh -- gas laws, Euler fluxes, Riemann solvers and boundary states on
// the device, for one node or one face point.
//
// Formulas and operation order follow the fr_sdg reference:
//   smooth_abs/max/min, wrap_positive   include/macro_and_libc.hpp:80-138
//   IdealGas / VanDerWaals              include/gas_models.hpp:56-158
//   make_state, fluxes                  include/riemann_solver.hpp:20-66
//   Rusanov / HLLC (1D, 2D)             include/riemann_solver.hpp:87-349
//   boundary binders                    include/boundary_conditions.hpp:59-151, 239-323
// Divisions by the same denominator are taken as one reciprocal and products,
// which moves results by at most a few ulps against the reference.
#pragma once
#include "device_math.cuh"
#include "frsdg_internal.hpp"

namespace frsdg
{

template <class S> __device__ __forceinline__ S cs(double v) { return S(v); }
template <> __device__ __forceinline__ float cs<float>(double v) { return static_cast<float>(v); }

// macro_and_libc.hpp:80-113
template <class S, class M = MathChecked> __device__ __forceinline__ S smooth_abs(S v, const M& m = M{})
{
    const S eps = cs<S>(1e-7);
    return m.sqrt(v * v + eps * eps) - eps;
}
template <class S, class M = MathChecked> __device__ __forceinline__ S smooth_max(S a, S b, const M& m = M{})
{
    return cs<S>(0.5) * (a + b + smooth_abs(a - b, m));
}
template <class S, class M = MathChecked> __device__ __forceinline__ S smooth_min(S a, S b, const M& m = M{})
{
    return cs<S>(0.5) * (a + b - smooth_abs(a - b, m));
}

// gas_models.hpp:56-87 (GAS == 0) and 89-158 (GAS == 1)
template <int GAS, class S> __device__ __forceinline__ S gas_pressure(const GasParams& g, S rho, S e)
{
    if constexpr (GAS == FRSDG_GAS_IDEAL)
        return (cs<S>(g.gamma) - cs<S>(1.0)) * rho * e;
    else
    {
        const S covol = cs<S>(1.0) - cs<S>(g.b) * rho;
        const S cvT   = e + cs<S>(g.a) * rho;
        const S p_id  = ((cs<S>(g.gamma) - cs<S>(1.0)) * rho * cvT) * s_rcp(covol);
        return p_id - cs<S>(g.a) * rho * rho;
    }
}
// sound speed with the pressure already known (ideal: sqrt(gamma p / rho))
template <int GAS, class S>
__device__ __forceinline__ S gas_sound_speed(const GasParams& g, S rho, S inv_rho, S e, S p)
{
    if constexpr (GAS == FRSDG_GAS_IDEAL)
        return s_sqrt(cs<S>(g.gamma) * p * inv_rho);
    else
    {
        const S covol     = cs<S>(1.0) - cs<S>(g.b) * rho;
        const S inv_dsq   = s_rcp(covol * covol);
        const S thermal   = e + cs<S>(g.a) * rho;
        const S gm1       = cs<S>(g.gamma) - cs<S>(1.0);
        const S term1     = (cs<S>(g.gamma) * gm1 * thermal) * inv_dsq;
        const S term2     = (gm1 * cs<S>(g.a) * rho * (cs<S>(2.0) - cs<S>(g.b) * rho)) * inv_dsq;
        const S term3     = cs<S>(2.0) * cs<S>(g.a) * rho;
        return s_sqrt(term1 + term2 - term3);
    }
}

// Primitive view of one 2D node: wrapped density and its inverse, velocities,
// specific internal energy (make_state of riemann_solver.hpp:29-37) and pressure.
template <class S> struct Prim2
{
    S rho, inv_rho, u, v, e, p;
};

template <int GAS, class S> __device__ __forceinline__ Prim2<S> prim2(const GasParams& g, const S U[4])
{
    Prim2<S> q;
    q.rho     = s_wrap_positive(U[0]);
    q.inv_rho = s_rcp(q.rho);
    q.u       = U[1] * q.inv_rho;
    q.v       = U[2] * q.inv_rho;
    const S E = s_wrap_positive(U[3]);
    q.e       = E * q.inv_rho - cs<S>(0.5) * (q.u * q.u + q.v * q.v);
    q.p       = gas_pressure<GAS>(g, q.rho, q.e);
    return q;
}

// euler_fluxes_2d_w_p (riemann_solver.hpp:48-66)
template <class S>
__device__ __forceinline__ void fluxes2(const S U[4], const Prim2<S>& q, S F[4], S G[4])
{
    const S rEp = U[3] + q.p;
    const S ruv = U[1] * q.v;
    F[0] = U[1];
    F[1] = U[1] * q.u + q.p;
    F[2] = ruv;
    F[3] = q.u * rEp;
    G[0] = U[2];
    G[1] = ruv;
    G[2] = U[2] * q.v + q.p;
    G[3] = q.v * rEp;
}

// RiemannSolver2D<Rusanov> (riemann_solver.hpp:189-247) and <HLLC> (249-349)
template <int RIEM, int GAS, class S>
__device__ __forceinline__ void riemann2(const GasParams& g, const S UL[4], const S UR[4], double nx_, double ny_,
                                         S Fs[4])
{
    using real    = typename scalar_traits<S>::real;
    const real nx = static_cast<real>(nx_), ny = static_cast<real>(ny_);
    const Prim2<S> L = prim2<GAS>(g, UL);
    const Prim2<S> R = prim2<GAS>(g, UR);
    const S unL = L.u * nx + L.v * ny;
    const S utL = -L.u * ny + L.v * nx;
    const S unR = R.u * nx + R.v * ny;
    const S utR = -R.u * ny + R.v * nx;
    const S cL  = gas_sound_speed<GAS>(g, L.rho, L.inv_rho, L.e, L.p);
    const S cR  = gas_sound_speed<GAS>(g, R.rho, R.inv_rho, R.e, R.p);
    const S FL0 = UL[0] * unL, FL1 = UL[0] * unL * unL + L.p, FL2 = UL[0] * unL * utL, FL3 = (UL[3] + L.p) * unL;
    const S FR0 = UR[0] * unR, FR1 = UR[0] * unR * unR + R.p, FR2 = UR[0] * unR * utR, FR3 = (UR[3] + R.p) * unR;
    S f0, f1, f2, f3;
    if constexpr (RIEM == FRSDG_RUSANOV)
    {
        const S smax = smooth_max(smooth_abs(unL) + cL, smooth_abs(unR) + cR);
        const S h    = cs<S>(0.5);
        f0 = h * (FL0 + FR0) - h * smax * (UR[0] - UL[0]);
        f1 = h * (FL1 + FR1) - h * smax * (UR[0] * unR - UL[0] * unL);
        f2 = h * (FL2 + FR2) - h * smax * (UR[0] * utR - UL[0] * utL);
        f3 = h * (FL3 + FR3) - h * smax * (UR[3] - UL[3]);
    }
    else
    {
        const S sL = smooth_min(unL - cL, unR - cR);
        const S sR = smooth_max(unL + cL, unR + cR);
        const S rhoL_diff = UL[0] * (sL - unL);
        const S rhoR_diff = UR[0] * (sR - unR);
        const S sM = (R.p - L.p + unL * rhoL_diff - unR * rhoR_diff) * s_rcp(rhoL_diff - rhoR_diff);
        // One star state, the side chosen by the sign of sM, then the HLLC sampling
        // of riemann_solver.hpp:314-341 expressed as selects.
        const bool left = s_branch(sM) >= 0.0;
        const S    K0 = left ? UL[0] : UR[0];
        const S    K3 = left ? UL[3] : UR[3];
        const S    sK = left ? sL : sR;
        const S    unK = left ? unL : unR;
        const S    utK = left ? utL : utR;
        const S    pK = left ? L.p : R.p;
        const S    FK0 = left ? FL0 : FR0, FK1 = left ? FL1 : FR1, FK3 = left ? FL3 : FR3;
        const S    p_star = pK + K0 * (sK - unK) * (sM - unK);
        const S    inv = s_rcp(sK - sM);
        const S    st0 = (sM * (sK * K0 - FK0)) * inv;
        const S    st1 = (sM * (sK * (K0 * unK) - FK1) + sK * p_star) * inv;
        const S    st2 = utK * st0;
        const S    st3 = (sM * (sK * K3 - FK3) + sK * p_star * sM) * inv;
        const bool takeL = s_branch(sL) >= 0.0;
        const bool star  = left || s_branch(sR) >= 0.0;
        f0 = takeL ? FL0 : (star ? st0 : FR0);
        f1 = takeL ? FL1 : (star ? st1 : FR1);
        f2 = takeL ? FL2 : (star ? st2 : FR2);
        f3 = takeL ? FL3 : (star ? st3 : FR3);
    }
    Fs[0] = f0;
    Fs[1] = f1 * nx - f2 * ny;
    Fs[2] = f1 * ny + f2 * nx;
    Fs[3] = f3;
}

// ---- per-node records ----------------------------------------------------
// Primitive quantities of one 2D node, computed once per node and shared by every
// face that touches it: the reference recomputes them inside each flux and Riemann
// call (riemann_solver.hpp:29-66, 200-225, 260-283) with the same operations.
template <class S> struct NodePrim
{
    S rho_w, inv_rho, u, v, e, p, inv_covol;
};

// Products and multiply-adds with a fixed rounding: the compiler neither fuses pmul
// with a neighbouring addition nor splits pfma, so every inlined copy of the node
// primitives rounds alike (tile nodes and the halo nodes of a neighbouring tile give the
// same bits).  Complex: the textbook product with one explicit multiply-add per part.
__device__ __forceinline__ double pmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float pmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ cplx pmul(cplx a, cplx b)
{
    return {fma(a.re, b.re, -__dmul_rn(a.im, b.im)), fma(a.re, b.im, __dmul_rn(a.im, b.re))};
}
__device__ __forceinline__ double pfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float pfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ cplx pfma(cplx a, cplx b, cplx c) { return pmul(a, b) + c; }

template <int GAS, class S, class M = MathChecked>
__device__ __forceinline__ NodePrim<S> node_prim(const GasParams& g, S r0, S r1, S r2, S r3, const M& m = M{})
{
    NodePrim<S> q;
    q.rho_w   = s_wrap_positive(r0);
    if constexpr (GAS == FRSDG_GAS_IDEAL)
        q.inv_rho = m.rcp(q.rho_w);
    else
    {
        // 1/rho and 1/(1 - b rho) from one reciprocal of their product (a few ulps from
        // the two quotients; 2 % of the 1024^2 p = 5 residual's time).  At the gas law's
        // pole rho = 1/b this gives NaN where the quotients give an infinite pressure.
        const S covol = pfma(cs<S>(-g.b), q.rho_w, cs<S>(1.0));
        const S both = m.rcp(pmul(q.rho_w, covol));
        q.inv_rho = pmul(both, covol);
        q.inv_covol = pmul(both, q.rho_w);
    }
    q.u       = pmul(r1, q.inv_rho);
    q.v       = pmul(r2, q.inv_rho);
    const S E = s_wrap_positive(r3);
    // e = E / rho - (u^2 + v^2) / 2
    q.e       = pfma(E, q.inv_rho, pmul(cs<S>(-0.5), pfma(q.u, q.u, pmul(q.v, q.v))));
    const S gm1 = cs<S>(g.gamma) - cs<S>(1.0);
    if constexpr (GAS == FRSDG_GAS_IDEAL)
    {
        q.inv_covol = cs<S>(1.0);
        q.p         = pmul(pmul(gm1, q.rho_w), q.e);
    }
    else
    {
        // p = (gamma - 1) rho (e + a rho) / (1 - b rho) - a rho^2
        const S cvT = pfma(cs<S>(g.a), q.rho_w, q.e);
        q.p = pfma(pmul(pmul(gm1, q.rho_w), cvT), q.inv_covol, -pmul(pmul(cs<S>(g.a), q.rho_w), q.rho_w));
    }
    return q;
}

template <int GAS, class S, class M = MathChecked>
__device__ __forceinline__ S node_sound_speed(const GasParams& g, const NodePrim<S>& q, const M& m = M{})
{
    if constexpr (GAS == FRSDG_GAS_IDEAL)
        return m.sqrt(pmul(pmul(cs<S>(g.gamma), q.p), q.inv_rho));
    else
    {
        // c^2 = gamma (gamma - 1) (e + a rho) / (1 - b rho)^2
        //       + (gamma - 1) a rho (2 - b rho) / (1 - b rho)^2 - 2 a rho
        const S inv_dsq = pmul(q.inv_covol, q.inv_covol);
        const S thermal = pfma(cs<S>(g.a), q.rho_w, q.e);
        const S gm1     = cs<S>(g.gamma) - cs<S>(1.0);
        const S term1   = pmul(pmul(pmul(cs<S>(g.gamma), gm1), thermal), inv_dsq);
        const S term2   = pmul(pmul(pmul(pmul(gm1, cs<S>(g.a)), q.rho_w), pfma(cs<S>(-g.b), q.rho_w, cs<S>(2.0))), inv_dsq);
        const S term3   = pmul(pmul(cs<S>(2.0), cs<S>(g.a)), q.rho_w);
        return m.sqrt(term1 + term2 - term3);
    }
}

// Face record of a node: raw density and total energy, velocities, pressure and
// sound speed -- what a Riemann solve reads from each side of a face.
enum RecField : int
{
    RF_RHO = 0, RF_E = 1, RF_U = 2, RF_V = 3, RF_P = 4, RF_C = 5, RF_N = 6
};

// RiemannSolver2D (riemann_solver.hpp:189-349) on two face records.
template <int RIEM, class S, class M = MathChecked>
__device__ __forceinline__ void riemann_rec(const S L[RF_N], const S R[RF_N], double nx_, double ny_, S Fs[4],
                                            const M& m = M{})
{
    using real    = typename scalar_traits<S>::real;
    const real nx = static_cast<real>(nx_), ny = static_cast<real>(ny_);
    const S unL = L[RF_U] * nx + L[RF_V] * ny;
    const S utL = -L[RF_U] * ny + L[RF_V] * nx;
    const S unR = R[RF_U] * nx + R[RF_V] * ny;
    const S utR = -R[RF_U] * ny + R[RF_V] * nx;
    const S cL = L[RF_C], cR = R[RF_C], pL = L[RF_P], pR = R[RF_P];
    const S FL0 = L[RF_RHO] * unL, FL1 = L[RF_RHO] * unL * unL + pL, FL2 = L[RF_RHO] * unL * utL,
            FL3 = (L[RF_E] + pL) * unL;
    const S FR0 = R[RF_RHO] * unR, FR1 = R[RF_RHO] * unR * unR + pR, FR2 = R[RF_RHO] * unR * utR,
            FR3 = (R[RF_E] + pR) * unR;
    S f0, f1, f2, f3;
    if constexpr (RIEM == FRSDG_RUSANOV)
    {
        const S smax = smooth_max(smooth_abs(unL, m) + cL, smooth_abs(unR, m) + cR, m);
        const S h    = cs<S>(0.5);
        f0 = h * (FL0 + FR0) - h * smax * (R[RF_RHO] - L[RF_RHO]);
        f1 = h * (FL1 + FR1) - h * smax * (R[RF_RHO] * unR - L[RF_RHO] * unL);
        f2 = h * (FL2 + FR2) - h * smax * (R[RF_RHO] * utR - L[RF_RHO] * utL);
        f3 = h * (FL3 + FR3) - h * smax * (R[RF_E] - L[RF_E]);
    }
    else
    {
        const S sL = smooth_min(unL - cL, unR - cR, m);
        const S sR = smooth_max(unL + cL, unR + cR, m);
        const S rhoL_diff = L[RF_RHO] * (sL - unL);
        const S rhoR_diff = R[RF_RHO] * (sR - unR);
        const S sM = (pR - pL + unL * rhoL_diff - unR * rhoR_diff) * m.rcp(rhoL_diff - rhoR_diff);
        const bool left = s_branch(sM) >= 0.0;
        const S K0 = left ? L[RF_RHO] : R[RF_RHO];
        const S K3 = left ? L[RF_E] : R[RF_E];
        const S sK = left ? sL : sR;
        const S unK = left ? unL : unR;
        const S utK = left ? utL : utR;
        const S pK = left ? pL : pR;
        const S FK0 = left ? FL0 : FR0, FK1 = left ? FL1 : FR1, FK3 = left ? FL3 : FR3;
        const S p_star = pK + K0 * (sK - unK) * (sM - unK);
        const S inv = m.rcp(sK - sM);
        const S st0 = (sM * (sK * K0 - FK0)) * inv;
        const S st1 = (sM * (sK * (K0 * unK) - FK1) + sK * p_star) * inv;
        const S st2 = utK * st0;
        const S st3 = (sM * (sK * K3 - FK3) + sK * p_star * sM) * inv;
        const bool takeL = s_branch(sL) >= 0.0;
        const bool star  = left || s_branch(sR) >= 0.0;
        f0 = takeL ? FL0 : (star ? st0 : FR0);
        f1 = takeL ? FL1 : (star ? st1 : FR1);
        f2 = takeL ? FL2 : (star ? st2 : FR2);
        f3 = takeL ? FL3 : (star ? st3 : FR3);
    }
    Fs[0] = f0;
    Fs[1] = f1 * nx - f2 * ny;
    Fs[2] = f1 * ny + f2 * nx;
    Fs[3] = f3;
}

// ---- 1D ------------------------------------------------------------------
// make_state (riemann_solver.hpp:20-27) and euler_flux (39-46)
template <int GAS, class S>
__device__ __forceinline__ void flux1(const GasParams& g, const S U[3], S F[3], S& p_out, S& rho_w, S& e_out)
{
    const S rho = s_wrap_positive(U[0]);
    const S inv = s_rcp(rho);
    const S u   = U[1] * inv;
    const S E   = s_wrap_positive(U[2]);
    const S e   = E * inv - cs<S>(0.5) * u * u;
    const S p   = gas_pressure<GAS>(g, rho, e);
    F[0] = U[1];
    F[1] = U[1] * u + p;
    F[2] = (U[2] + p) * u;
    p_out = p;
    rho_w = rho;
    e_out = e;
}

// RiemannSolver<Rusanov> (riemann_solver.hpp:87-113) and <HLLC> (115-184).
// The 1D solvers divide by the unclamped density for the velocity.
template <int RIEM, int GAS, class S>
__device__ __forceinline__ void riemann1(const GasParams& g, const S UL[3], const S UR[3], S Fs[3])
{
    S FL[3], FR[3], pL, pR, rL, rR, eL, eR;
    flux1<GAS>(g, UL, FL, pL, rL, eL);
    flux1<GAS>(g, UR, FR, pR, rR, eR);
    const S aL = gas_sound_speed<GAS>(g, rL, s_rcp(rL), eL, pL);
    const S aR = gas_sound_speed<GAS>(g, rR, s_rcp(rR), eR, pR);
    const S uL = UL[1] / UL[0];
    const S uR = UR[1] / UR[0];
    if constexpr (RIEM == FRSDG_RUSANOV)
    {
        const S smax = smooth_max(smooth_abs(uL) + aL, smooth_abs(uR) + aR);
        const S h    = cs<S>(0.5);
        for (int q = 0; q < 3; ++q) Fs[q] = h * (FL[q] + FR[q]) - h * smax * (UR[q] - UL[q]);
    }
    else
    {
        const S ppL = FL[1] - uL * UL[1];
        const S ppR = FR[1] - uR * UR[1];
        const S sL = smooth_min(uL - aL, uR - aR);
        const S sR = smooth_max(uL + aL, uR + aR);
        const S rhoL_diff = UL[0] * (sL - uL);
        const S rhoR_diff = UR[0] * (sR - uR);
        const S sM = (ppR - ppL + uL * rhoL_diff - uR * rhoR_diff) * s_rcp(rhoL_diff - rhoR_diff);
        const bool left = s_branch(sM) >= 0.0;
        const S* UK = left ? UL : UR;
        const S* FK = left ? FL : FR;
        const S sK = left ? sL : sR, uK = left ? uL : uR, pK = left ? ppL : ppR;
        const S p_star = pK + UK[0] * (sK - uK) * (sM - uK);
        const S inv = s_rcp(sK - sM);
        S st[3];
        st[0] = (sM * (sK * UK[0] - FK[0])) * inv;
        st[1] = (sM * (sK * UK[1] - FK[1]) + sK * p_star) * inv;
        st[2] = (sM * (sK * UK[2] - FK[2]) + sK * p_star * sM) * inv;
        const bool takeL = s_branch(sL) >= 0.0;
        const bool star  = left || s_branch(sR) >= 0.0;
        for (int q = 0; q < 3; ++q) Fs[q] = takeL ? FL[q] : (star ? st[q] : FR[q]);
    }
}

// ---- boundary states ------------------------------------------------------
// Exact isentropic vortex (factory.hpp:311-352); gamma is fixed at 1.4 there.
__device__ __forceinline__ void exact_vortex_dev(double time, double x, double y, const double* vd, double out[4])
{
    const double u_0 = vd[0], v_0 = vd[1], beta = vd[2], r_v = vd[3], l = vd[4];
    const double gamma = 1.4;
    const double pi    = 3.14159265358979323846;
    double x_c = l / 2.0 + u_0 * time;
    double y_c = l / 2.0 + v_0 * time;
    x_c = x_c - l * floor(x_c / l);
    y_c = y_c - l * floor(y_c / l);
    const double dx = x - x_c, dy = y - y_c;
    const double r2 = dx * dx + dy * dy;
    const double f = 1.0 - (r2 / (r_v * r_v));
    const double exp_f = exp(f);
    const double rho = pow(1.0 - (beta * beta * (gamma - 1.0) * (exp_f * exp_f)) / (16.0 * gamma * pi * pi),
                           1.0 / (gamma - 1.0));
    const double u = u_0 - (beta * exp_f * dy) / (2.0 * pi * r_v);
    const double v = v_0 + (beta * exp_f * dx) / (2.0 * pi * r_v);
    const double p = pow(rho, gamma);
    out[0] = rho;
    out[1] = rho * u;
    out[2] = rho * v;
    out[3] = (p / (gamma - 1.0)) + 0.5 * rho * (u * u + v * v);
}

// Complex-step ghost of the user-lambda kinds that depend on the interior state,
// differentiated (the same formulas as below on complex scalars; pow as
// exp(y log x) on the principal branch).  Dirichlet and vortex ghosts do not
// depend on the state.
template <int GAS>
__device__ __forceinline__ bool bc_ghost2_exact(const BcDev& b, const GasParams& g, double nx, double ny,
                                                const cplx in[4], cplx o[4])
{
    switch (b.kind)
    {
        case FRSDG_BC_SLIP_WALL:
        {
            const cplx u_in = in[1] / in[0], v_in = in[2] / in[0];
            const cplx vn = u_in * nx + v_in * ny;
            o[0] = in[0];
            o[1] = in[0] * (u_in - 2.0 * vn * nx);
            o[2] = in[0] * (v_in - 2.0 * vn * ny);
            o[3] = in[3];
            return true;
        }
        case FRSDG_BC_SUBSONIC_INFLOW:
        {
            const double gm = g.gamma;
            const double p0 = b.params[0], T0 = b.params[1], Rg = b.params[2], ang = b.params[3];
            const cplx rho_w = s_wrap_positive(in[0]);
            const cplx E_w = s_wrap_positive(in[3]);
            const cplx uu = in[1] / rho_w, vv = in[2] / rho_w;
            const cplx e = E_w / rho_w - 0.5 * (uu * uu + vv * vv);
            cplx p = gas_pressure<GAS>(g, rho_w, e);
            if (p.re > p0) p = cplx(p0);
            const cplx M2 = (2.0 / (gm - 1.0)) * (s_exp(((gm - 1.0) / gm) * s_log(cplx(p0) / p)) - 1.0);
            const cplx T = cplx(T0) / (1.0 + 0.5 * (gm - 1.0) * M2);
            const cplx rho = p / (Rg * T);
            const cplx c = s_sqrt(gm * p / rho);
            const cplx vel = s_sqrt(M2) * c;
            const cplx u = vel * cos(ang), v = vel * sin(ang);
            o[0] = rho;
            o[1] = rho * u;
            o[2] = rho * v;
            o[3] = p / (gm - 1.0) + 0.5 * rho * (u * u + v * v);
            return true;
        }
        case FRSDG_BC_PRESSURE_OUTLET:
        {
            const cplx rho = in[0];
            const cplx u = in[1] / rho, v = in[2] / rho;
            const cplx vel2 = s_sqrt(u * u + v * v) * s_sqrt(u * u + v * v);
            const double pres = b.params[0];
            o[0] = in[0];
            o[1] = in[1];
            o[2] = in[2];
            if constexpr (GAS == FRSDG_GAS_IDEAL)
                o[3] = pres / (g.gamma - 1.0) + 0.5 * rho * vel2;
            else
            {
                const cplx covol = 1.0 - g.b * rho;
                const cplx arho2 = g.a * rho * rho;
                o[3] = ((pres + arho2) * covol) / (g.gamma - 1.0) - arho2 + 0.5 * rho * vel2;
            }
            return true;
        }
        default: return false;
    }
}

// Ghost state of a 2D boundary face point (BoundaryConditions<T,2>::evaluate_bc,
// boundary_conditions.hpp:239-248).  Native kinds act on the full scalar; the
// other kinds stand for user lambdas and see only the real part (276-293),
// unless `exact` asks for their complex-step derivative.
template <int GAS, class S>
__device__ __forceinline__ void bc_ghost2(const BcDev& b, int dir, const GasParams& g, double t, double x, double y, double nx, double ny, double Lx,
                                          double Ly, const S in[4], S out[4], bool exact = false)
{
    if constexpr (scalar_traits<S>::words == 2)
    {
        if (exact && bc_ghost2_exact<GAS>(b, g, nx, ny, in, out)) return;
    }
    switch (b.kind)
    {
        case FRSDG_BC_OUTFLOW:
        case FRSDG_BC_PERIODIC:
            for (int q = 0; q < 4; ++q) out[q] = in[q];
            return;
        case FRSDG_BC_WALL:
        {
            // the momentum component of the face axis flips (LEFT/RIGHT: x, TOP/BOTTOM: y)
            const bool xaxis = dir < 2;
            out[0] = in[0];
            out[1] = xaxis ? -in[1] : in[1];
            out[2] = xaxis ? in[2] : -in[2];
            out[3] = in[3];
            return;
        }
        default: break;
    }
    double r[4] = {s_re(in[0]), s_re(in[1]), s_re(in[2]), s_re(in[3])};
    double o[4] = {r[0], r[1], r[2], r[3]};
    switch (b.kind)
    {
        case FRSDG_BC_DIRICHLET:
            for (int q = 0; q < 4; ++q) o[q] = b.state[q];
            break;
        case FRSDG_BC_SLIP_WALL:
        {
            const double u_in = r[1] / r[0], v_in = r[2] / r[0];
            const double vn = u_in * nx + v_in * ny;
            o[1] = r[0] * (u_in - 2.0 * vn * nx);
            o[2] = r[0] * (v_in - 2.0 * vn * ny);
            break;
        }
        case FRSDG_BC_VORTEX:
        {
            if (dir == FRSDG_LEFT) exact_vortex_dev(t, 0.0, y, b.params, o);
            else if (dir == FRSDG_RIGHT) exact_vortex_dev(t, Lx, y, b.params, o);
            else if (dir == FRSDG_BOTTOM) exact_vortex_dev(t, x, 0.0, b.params, o);
            else exact_vortex_dev(t, x, Ly, b.params, o);
            break;
        }
        case FRSDG_BC_SUBSONIC_INFLOW:
        {
            const double gm = g.gamma;
            const double p0 = b.params[0], T0 = b.params[1], Rg = b.params[2], ang = b.params[3];
            const double rho_w = fmax(2.2250738585072014e-308, r[0]);
            const double E_w = fmax(2.2250738585072014e-308, r[3]);
            const double uu = r[1] / rho_w, vv = r[2] / rho_w;
            const double e = E_w / rho_w - 0.5 * (uu * uu + vv * vv);
            double p = gas_pressure<GAS>(g, rho_w, e);
            if (p > p0) p = p0;
            const double M2 = 2.0 / (gm - 1.0) * (pow(p0 / p, (gm - 1.0) / gm) - 1.0);
            const double T = T0 / (1.0 + 0.5 * (gm - 1.0) * M2);
            const double rho = p / (Rg * T);
            const double c = sqrt(gm * p / rho);
            const double vel = sqrt(M2) * c;
            const double u = vel * cos(ang), v = vel * sin(ang);
            o[0] = rho;
            o[1] = rho * u;
            o[2] = rho * v;
            o[3] = p / (gm - 1.0) + 0.5 * rho * (u * u + v * v);
            break;
        }
        case FRSDG_BC_PRESSURE_OUTLET:
        {
            const double rho = r[0];
            const double u = r[1] / rho, v = r[2] / rho;
            const double vel = sqrt(u * u + v * v);
            const double pres = b.params[0];
            if constexpr (GAS == FRSDG_GAS_IDEAL)
                o[3] = pres / (g.gamma - 1.0) + 0.5 * rho * vel * vel;
            else
            {
                const double covol = 1.0 - g.b * rho;
                const double arho2 = g.a * rho * rho;
                o[3] = ((pres + arho2) * covol) / (g.gamma - 1.0) - arho2 + 0.5 * rho * vel * vel;
            }
            break;
        }
        default: break;
    }
    for (int q = 0; q < 4; ++q) out[q] = S(o[q]);
}

} // namespace frsdg
