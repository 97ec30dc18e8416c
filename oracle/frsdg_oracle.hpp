// frsdg_oracle.hpp -- CPU restatement of fr_sdg's FR residual hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that tests/, the smoke()
// entry point and the CPU-baseline leg of bench.py compare the CUDA library
// against.  Nothing in fr_sdg_b200/ includes, links or calls it.
//
// It restates, operation by operation and in the same summation order, the
// reference's algorithm for the path (paths relative to the fr_sdg project):
//   include/macro_and_libc.hpp:80-138         smooth_abs/max/min, wrap_positive
//   include/gas_models.hpp:56-158              IdealGas, VanDerWaals
//   include/riemann_solver.hpp:20-349          make_state, fluxes, Rusanov/HLLC 1D and 2D
//   include/reference_element.hpp:50-147       GLL nodes (Golub-Welsch) and weights
//   include/cached_computations.hpp:37-137     VCJH dL/dR, differentiation matrix
//   include/filter.hpp:397-755                 spectral filter, WENO, shock sensor
//   include/geometry_models.hpp:72-195         Cartesian and de Laval geometry policies
//   tests/bump.cpp:13-171, tests/boundary_conforming.cpp:14-120  wall-profile geometries
//   include/boundary_conditions.hpp:214-323    2D boundary binders (+ 1D 37-211)
//   include/physics_evaluator.hpp:234-313      computational coordinates, composite metrics
//   include/physics_impl_2D.hpp:76-124, 126-154, 268-357, 646-902
//   include/physics_impl_1D.hpp:9-94, 96-121, 124-181, 183-205
//   include/problem_def.hpp:36-70              prim <-> cons change of variables
//   include/petsc_solver_impl.hpp:250-432, 626-670, 683-702  JVP, IFunction, RHS, post step
//
// The reference cannot be compiled here (it needs PETSc, MPI, Eigen, Boost.Math and a
// C++23 <print>).  Eigen's eigen-solver and LU and Boost's Legendre functions are
// replaced by an implicit-QL tridiagonal eigen-solver, partial-pivot LU and the
// three-term Legendre recurrence.  Parity pin: the reference's own known-answer
// checks (tests/sbp.cpp SBP identity, tests/filter_check.cpp filter eigenvalues,
// reference_element.hpp:41-45 sum of weights, factory.hpp:33-56 free-stream
// preservation) and closed-form GLL tables; the residual arithmetic itself has no
// golden vector in the reference, so residual parity against the reference binary
// is unpinned beyond those checks.
#pragma once

#include "../include/frsdg.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <limits>
#include <numbers>
#include <stdexcept>
#include <type_traits>
#include <vector>

namespace frsdg_oracle
{
using cplx = std::complex<double>;

template <class U> struct is_cplx : std::false_type {};
template <> struct is_cplx<cplx> : std::true_type {};

inline double re(double v) { return v; }
inline double re(const cplx& v) { return v.real(); }

// ---------------------------------------------------------------- scalar helpers
// macro_and_libc.hpp:80-91
template <class U> U smooth_abs(const U& val)
{
    const U eps{1e-7};
    return U{std::sqrt(val * val + eps * eps)} - eps;
}
// macro_and_libc.hpp:94-102
template <class U> U smooth_max(const U& a, const U& b) { return 0.5 * (a + b + smooth_abs(a - b)); }
// macro_and_libc.hpp:105-113
template <class U> U smooth_min(const U& a, const U& b) { return 0.5 * (a + b - smooth_abs(a - b)); }
// macro_and_libc.hpp:117-138
inline double wrap_positive(double rho) { return std::max(std::numeric_limits<double>::min(), rho); }
inline cplx wrap_positive(cplx rho)
{
    const double floor = std::numeric_limits<double>::min();
    if (std::real(rho) < floor) return cplx(floor, 0.0);
    return rho;
}
// riemann_solver.hpp:149-155 (HLLC branch test)
inline double branch_real(double v) { return v; }
inline double branch_real(const cplx& v) { return v.real() + v.imag(); }

// ---------------------------------------------------------------- gas models
struct Gas
{
    int    law{FRSDG_GAS_IDEAL};
    double gamma{1.4}, R{287.05}, a{0.0}, b{0.0};

    // gas_models.hpp:56-87 / 89-158
    template <class U> U pressure(const U& density, const U& energy) const
    {
        if (law == FRSDG_GAS_IDEAL) return (gamma - U{1.0}) * density * energy;
        U rho           = density;
        U covolume_term = U{1.0} - U{b} * rho;
        U cvT           = energy + U{a} * rho;
        U p_ideal       = ((U{gamma} - U{1.0}) * rho * cvT) / covolume_term;
        U p_attraction  = U{a} * rho * rho;
        return p_ideal - p_attraction;
    }
    template <class U> U sound_speed(const U& density, const U& energy) const
    {
        if (law == FRSDG_GAS_IDEAL) return std::sqrt(gamma * pressure(density, energy) / density);
        const U rho            = density;
        const U covolume_term  = U{1.0} - U{b} * rho;
        const U denom_sq       = covolume_term * covolume_term;
        const U thermal_energy = energy + U{a} * rho;
        const U term1          = (U{gamma} * (U{gamma} - U{1.0}) * thermal_energy) / denom_sq;
        const U term2 = ((U{gamma} - U{1.0}) * U{a} * rho * (U{2.0} - U{b} * rho)) / denom_sq;
        const U term3 = U{2.0} * U{a} * rho;
        return std::sqrt(term1 + term2 - term3);
    }
    double rhoE(double rho, double vel, double pres) const
    {
        if (law == FRSDG_GAS_IDEAL)
        {
            const double internal_energy = pres / (gamma - 1.0);
            const double kinetic_energy  = 0.5 * rho * vel * vel;
            return internal_energy + kinetic_energy;
        }
        double covolume_term = 1.0 - b * rho;
        double a_rho_sq      = a * rho * rho;
        double rho_e         = ((pres + a_rho_sq) * covolume_term) / (gamma - 1.0) - a_rho_sq;
        return rho_e + 0.5 * rho * vel * vel;
    }
};

template <class U> struct Thermo
{
    U density, energy;
};

// riemann_solver.hpp:20-27
template <class U> Thermo<U> make_state1(const U& rho_in, const U& rhoU, const U& rhoE_in)
{
    const U rho    = wrap_positive(rho_in);
    const U tot_en = wrap_positive(rhoE_in);
    const U u      = rhoU / rho;
    return {rho, (tot_en / rho - U(0.5) * u * u)};
}
// riemann_solver.hpp:29-37
template <class U> Thermo<U> make_state2(const std::array<U, 4>& s)
{
    const U rho    = wrap_positive(s[0]);
    const U tot_en = wrap_positive(s[3]);
    const U u      = s[1] / rho;
    const U v      = s[2] / rho;
    return {rho, (tot_en / rho - U(0.5) * (u * u + v * v))};
}
// riemann_solver.hpp:39-46
template <class U> std::array<U, 3> euler_flux1(const std::array<U, 3>& s, const Gas& g)
{
    const auto ts = make_state1(s[0], s[1], s[2]);
    const U    p  = g.pressure(ts.density, ts.energy);
    const U    u  = s[1] / wrap_positive(s[0]);
    return {s[1], s[1] * u + p, (s[2] + p) * u};
}
// riemann_solver.hpp:48-66
template <class U>
void euler_fluxes2(const std::array<U, 4>& s, const Gas& g, std::array<U, 4>& F, std::array<U, 4>& G,
                   U& pres)
{
    const U rho     = wrap_positive(s[0]);
    const U inv_rho = U(1.0) / rho;
    const U u       = s[1] * inv_rho;
    const U v       = s[2] * inv_rho;
    const auto ts   = make_state2(s);
    const U p       = g.pressure(ts.density, ts.energy);
    const U rEp     = s[3] + p;
    const U ruv     = s[1] * v;
    F               = {s[1], s[1] * u + p, ruv, u * rEp};
    G               = {s[2], ruv, s[2] * v + p, v * rEp};
    pres            = p;
}

// riemann_solver.hpp:87-113 and 115-184
template <class U>
std::array<U, 3> riemann1(int scheme, const std::array<U, 3>& UL, const std::array<U, 3>& UR, const Gas& g)
{
    const auto stateL = make_state1(UL[0], UL[1], UL[2]);
    const auto stateR = make_state1(UR[0], UR[1], UR[2]);
    if (scheme == FRSDG_RUSANOV)
    {
        const U sL   = smooth_abs(UL[1] / UL[0]) + g.sound_speed(stateL.density, stateL.energy);
        const U sR   = smooth_abs(UR[1] / UR[0]) + g.sound_speed(stateR.density, stateR.energy);
        const U smax = smooth_max(sL, sR);
        const auto FL = euler_flux1(UL, g);
        const auto FR = euler_flux1(UR, g);
        return {U(0.5) * (FL[0] + FR[0]) - U(0.5) * smax * (UR[0] - UL[0]),
                U(0.5) * (FL[1] + FR[1]) - U(0.5) * smax * (UR[1] - UL[1]),
                U(0.5) * (FL[2] + FR[2]) - U(0.5) * smax * (UR[2] - UL[2])};
    }
    const U uL = UL[1] / UL[0];
    const U uR = UR[1] / UR[0];
    const U aL = g.sound_speed(stateL.density, stateL.energy);
    const U aR = g.sound_speed(stateR.density, stateR.energy);
    const auto FL = euler_flux1(UL, g);
    const auto FR = euler_flux1(UR, g);
    const U pL = FL[1] - uL * UL[1];
    const U pR = FR[1] - uR * UR[1];
    const U sL = smooth_min(uL - aL, uR - aR);
    const U sR = smooth_max(uL + aL, uR + aR);
    const U rhoL_diff = UL[0] * (sL - uL);
    const U rhoR_diff = UR[0] * (sR - uR);
    const U sM = (pR - pL + uL * rhoL_diff - uR * rhoR_diff) / (rhoL_diff - rhoR_diff);
    if (branch_real(sL) >= 0.0) return FL;
    if (branch_real(sM) >= 0.0)
    {
        const U p_star = pL + UL[0] * (sL - uL) * (sM - uL);
        return {(sM * (sL * UL[0] - FL[0])) / (sL - sM),
                (sM * (sL * UL[1] - FL[1]) + sL * p_star) / (sL - sM),
                (sM * (sL * UL[2] - FL[2]) + sL * p_star * sM) / (sL - sM)};
    }
    if (branch_real(sR) >= 0.0)
    {
        const U p_star = pR + UR[0] * (sR - uR) * (sM - uR);
        return {(sM * (sR * UR[0] - FR[0])) / (sR - sM),
                (sM * (sR * UR[1] - FR[1]) + sR * p_star) / (sR - sM),
                (sM * (sR * UR[2] - FR[2]) + sR * p_star * sM) / (sR - sM)};
    }
    return FR;
}

// riemann_solver.hpp:189-247 and 249-349
template <class U>
std::array<U, 4> riemann2(int scheme, const std::array<U, 4>& UL, const std::array<U, 4>& UR, const Gas& g,
                          double nx, double ny)
{
    const U inv_rhoL = U(1.0) / wrap_positive(UL[0]);
    const U inv_rhoR = U(1.0) / wrap_positive(UR[0]);
    const U uL       = UL[1] * inv_rhoL;
    const U vL       = UL[2] * inv_rhoL;
    const U uR       = UR[1] * inv_rhoR;
    const U vR       = UR[2] * inv_rhoR;
    const U unL      = uL * nx + vL * ny;
    const U utL      = -uL * ny + vL * nx;
    const U unR      = uR * nx + vR * ny;
    const U utR      = -uR * ny + vR * nx;
    const auto thL   = make_state2(UL);
    const auto thR   = make_state2(UR);
    if (scheme == FRSDG_RUSANOV)
    {
        const U cL   = g.sound_speed(thL.density, thL.energy);
        const U cR   = g.sound_speed(thR.density, thR.energy);
        const U smax = smooth_max(smooth_abs(unL) + cL, smooth_abs(unR) + cR);
        const U pL   = g.pressure(thL.density, thL.energy);
        const U pR   = g.pressure(thR.density, thR.energy);
        std::array<U, 4> FLn = {UL[0] * unL, UL[0] * unL * unL + pL, UL[0] * unL * utL, (UL[3] + pL) * unL};
        std::array<U, 4> FRn = {UR[0] * unR, UR[0] * unR * unR + pR, UR[0] * unR * utR, (UR[3] + pR) * unR};
        U f_rho = 0.5 * (FLn[0] + FRn[0]) - 0.5 * smax * (UR[0] - UL[0]);
        U f_un  = 0.5 * (FLn[1] + FRn[1]) - 0.5 * smax * (UR[0] * unR - UL[0] * unL);
        U f_ut  = 0.5 * (FLn[2] + FRn[2]) - 0.5 * smax * (UR[0] * utR - UL[0] * utL);
        U f_E   = 0.5 * (FLn[3] + FRn[3]) - 0.5 * smax * (UR[3] - UL[3]);
        return {f_rho, f_un * nx - f_ut * ny, f_un * ny + f_ut * nx, f_E};
    }
    const U aL = g.sound_speed(thL.density, thL.energy);
    const U aR = g.sound_speed(thR.density, thR.energy);
    const U pL = g.pressure(thL.density, thL.energy);
    const U pR = g.pressure(thR.density, thR.energy);
    std::array<U, 4> FLn = {UL[0] * unL, UL[0] * unL * unL + pL, UL[0] * unL * utL, (UL[3] + pL) * unL};
    std::array<U, 4> FRn = {UR[0] * unR, UR[0] * unR * unR + pR, UR[0] * unR * utR, (UR[3] + pR) * unR};
    const U sL = smooth_min(unL - aL, unR - aR);
    const U sR = smooth_max(unL + aL, unR + aR);
    const U rhoL_diff = UL[0] * (sL - unL);
    const U rhoR_diff = UR[0] * (sR - unR);
    const U sM = (pR - pL + unL * rhoL_diff - unR * rhoR_diff) / (rhoL_diff - rhoR_diff);
    std::array<U, 4> fs;
    if (branch_real(sL) >= 0.0)
        fs = FLn;
    else if (branch_real(sM) >= 0.0)
    {
        const U p_star = pL + UL[0] * (sL - unL) * (sM - unL);
        fs[0] = (sM * (sL * UL[0] - FLn[0])) / (sL - sM);
        fs[1] = (sM * (sL * (UL[0] * unL) - FLn[1]) + sL * p_star) / (sL - sM);
        fs[2] = utL * fs[0];
        fs[3] = (sM * (sL * UL[3] - FLn[3]) + sL * p_star * sM) / (sL - sM);
    }
    else if (branch_real(sR) >= 0.0)
    {
        const U p_star = pR + UR[0] * (sR - unR) * (sM - unR);
        fs[0] = (sM * (sR * UR[0] - FRn[0])) / (sR - sM);
        fs[1] = (sM * (sR * (UR[0] * unR) - FRn[1]) + sR * p_star) / (sR - sM);
        fs[2] = utR * fs[0];
        fs[3] = (sM * (sR * UR[3] - FRn[3]) + sR * p_star * sM) / (sR - sM);
    }
    else
        fs = FRn;
    return {fs[0], fs[1] * nx - fs[2] * ny, fs[1] * ny + fs[2] * nx, fs[3]};
}

// ---------------------------------------------------------------- reference element
// Legendre P_n(x) and P'_n(x) by the three-term recurrence (Boost's legendre_p and
// legendre_p_prime in the reference).
inline void legendre(int n, double x, double& P, double& dP)
{
    if (n == 0) { P = 1.0; dP = 0.0; return; }
    double p0 = 1.0, p1 = x, d0 = 0.0, d1 = 1.0;
    for (int k = 1; k < n; ++k)
    {
        const double p2 = ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0);
        const double d2 = d0 + (2.0 * k + 1.0) * p1; // P'_{k+1} = P'_{k-1} + (2k+1) P_k
        p0 = p1; p1 = p2; d0 = d1; d1 = d2;
    }
    P = p1; dP = d1;
}
inline double legendre_p(int n, double x) { double P, dP; legendre(n, x, P, dP); return P; }
inline double legendre_p_prime(int n, double x)
{
    if (n < 0) return 0.0;
    double P, dP; legendre(n, x, P, dP); return dP;
}

// Eigenvalues of a symmetric tridiagonal matrix by the implicit QL method with
// Wilkinson shifts (Bowdler, Martin, Reinsch and Wilkinson, Numer. Math. 11, 1968),
// standing in for Eigen::SelfAdjointEigenSolver (reference_element.hpp:97).
inline std::vector<double> tridiag_eigenvalues(std::vector<double> d, std::vector<double> e)
{
    const int n = static_cast<int>(d.size());
    e.resize(n, 0.0);
    for (int l = 0; l < n; ++l)
    {
        for (int iter = 0; iter < 200; ++iter)
        {
            int m = l;
            for (; m < n - 1; ++m)
            {
                const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= std::numeric_limits<double>::epsilon() * dd) break;
            }
            if (m == l) break;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = std::hypot(g, 1.0);
            g        = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
            double s = 1.0, c = 1.0, p = 0.0;
            int    i = m - 1;
            bool   deflated = false;
            for (; i >= l; --i)
            {
                const double f = s * e[i];
                const double b = c * e[i];
                r              = std::hypot(f, g);
                e[i + 1]       = r;
                if (r == 0.0)
                {
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    deflated = true;
                    break;
                }
                s        = f / r;
                c        = g / r;
                g        = d[i + 1] - p;
                r        = (d[i] - g) * s + 2.0 * c * b;
                p        = s * r;
                d[i + 1] = g + p;
                g        = c * r - b;
            }
            if (deflated) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    std::sort(d.begin(), d.end());
    return d;
}

struct RefElement
{
    int                 p{}, n{};
    std::vector<double> csi, w, D, dL, dR; // D row-major n*n
};

// reference_element.hpp:50-147 and cached_computations.hpp:8-137
inline RefElement make_ref_element(int p, double c_rad)
{
    if (p < 1 || p > 9) throw std::invalid_argument("poly_deg must be in [1, 9]");
    RefElement r;
    r.p = p;
    r.n = p + 1;
    const int n = r.n;
    r.csi.assign(n, 0.0);
    r.w.assign(n, 0.0);
    if (p >= 2)
    {
        // compute_J_mat(p-1, alpha=1, beta=1)  (reference_element.hpp:118-147)
        const int    m = p - 1;
        const double alpha = 1.0, beta = 1.0;
        std::vector<double> diag(m), sub(m > 1 ? m - 1 : 0);
        for (int k = 0; k < m; ++k)
        {
            const double ab = alpha + beta, a2b2 = beta * beta - alpha * alpha;
            const double denom = (2.0 * k + ab) * (2.0 * k + ab + 2.0);
            diag[k] = (denom == 0.0) ? 0.0 : a2b2 / denom;
        }
        for (int k = 1; k < m; ++k)
        {
            const double ab  = alpha + beta;
            const double num = 4.0 * k * (k + alpha) * (k + beta) * (k + ab);
            const double dd  = (2.0 * k + ab) * (2.0 * k + ab);
            const double den = dd * (2.0 * k + ab - 1.0) * (2.0 * k + ab + 1.0);
            sub[k - 1]       = std::sqrt(num / den);
        }
        const auto vals = tridiag_eigenvalues(diag, sub);
        r.csi[0]     = -1.0;
        r.csi[n - 1] = 1.0;
        for (int k = 0; k < m; ++k) r.csi[1 + k] = vals[k];
        const double denominator_const = p * (p + 1);
        for (int k = 0; k < n; ++k)
        {
            const double p_n = std::legendre(static_cast<unsigned>(p), r.csi[k]);
            r.w[k]           = 2.0 / (denominator_const * p_n * p_n);
        }
    }
    else
    {
        r.csi = {-1.0, 1.0};
        r.w   = {1.0, 1.0};
    }
    // create_diff_matrix (cached_computations.hpp:107-137)
    r.D.assign(n * n, 0.0);
    std::vector<double> a(n, 1.0);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k)
            if (i != k) a[i] *= r.csi[i] - r.csi[k];
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            if (i != j)
                r.D[i * n + j] = a[i] / (a[j] * (r.csi[i] - r.csi[j]));
            else
            {
                double s = 0.0;
                for (int k = 0; k < n; ++k)
                    if (k != i) s += 1.0 / (r.csi[i] - r.csi[k]);
                r.D[i * n + i] = s;
            }
        }
    // build_Radaus_poly_deriv (cached_computations.hpp:37-105)
    r.dL.assign(n, 0.0);
    r.dR.assign(n, 0.0);
    const double sign = (p % 2 == 0) ? 1.0 : -1.0;
    auto factorial = [](int num) { double f = 1.0; for (int i = 2; i <= num; ++i) f *= double(i); return f; };
    const double p_fact    = factorial(p);
    const double ak        = factorial(2 * p) / (std::pow(2.0, p) * p_fact * p_fact);
    const double ak_fact_k = ak * p_fact;
    const double eta_k     = c_rad * double(2 * p + 1) * ak_fact_k * ak_fact_k / 2.0;
    for (int i = 0; i < n; ++i)
    {
        const double xi  = r.csi[i];
        const double dLp = legendre_p_prime(p, xi);
        const double dLm = legendre_p_prime(p - 1, xi);
        const double dLn = legendre_p_prime(p + 1, xi);
        const double term_ = (eta_k * dLm + dLn) / (1 + eta_k);
        r.dL[i] = sign * 0.5 * (dLp - term_);
        r.dR[i] = 0.5 * (dLp + term_);
    }
    return r;
}

// filter.hpp:451-484: V diag(sigma) V^-1 with an LU inverse (Eigen's PartialPivLU).
inline std::vector<double> make_filter_matrix(const RefElement& re, int n_cut_off, int strength, double alpha)
{
    const int n = re.n;
    auto sigma = [&](int i) -> double
    {
        if (i < n_cut_off) return 1.0;
        const double ratio = double(i - n_cut_off) / double((n - 1) - n_cut_off);
        return std::exp(-alpha * std::pow(ratio, double(strength)));
    };
    std::vector<double> V(n * n), Vinv(n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) V[i * n + j] = legendre_p(j, re.csi[i]);
    // LU with partial pivoting, then solve for the columns of the identity.
    std::vector<double> LU = V;
    std::vector<int>    piv(n);
    for (int i = 0; i < n; ++i) piv[i] = i;
    for (int k = 0; k < n; ++k)
    {
        int    pr = k;
        double mx = std::fabs(LU[k * n + k]);
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(LU[i * n + k]) > mx) { mx = std::fabs(LU[i * n + k]); pr = i; }
        if (pr != k)
        {
            for (int j = 0; j < n; ++j) std::swap(LU[k * n + j], LU[pr * n + j]);
            std::swap(piv[k], piv[pr]);
        }
        for (int i = k + 1; i < n; ++i)
        {
            LU[i * n + k] /= LU[k * n + k];
            for (int j = k + 1; j < n; ++j) LU[i * n + j] -= LU[i * n + k] * LU[k * n + j];
        }
    }
    for (int c = 0; c < n; ++c)
    {
        std::vector<double> y(n);
        for (int i = 0; i < n; ++i)
        {
            double s = (piv[i] == c) ? 1.0 : 0.0;
            for (int j = 0; j < i; ++j) s -= LU[i * n + j] * y[j];
            y[i] = s;
        }
        for (int i = n - 1; i >= 0; --i)
        {
            double s = y[i];
            for (int j = i + 1; j < n; ++j) s -= LU[i * n + j] * Vinv[j * n + c];
            Vinv[i * n + c] = s / LU[i * n + i];
        }
    }
    std::vector<double> F(n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += V[i * n + k] * sigma(k) * Vinv[k * n + j];
            F[i * n + j] = s;
        }
    return F;
}

// ---------------------------------------------------------------- geometry
struct GeomJac
{
    double dx_dcsi{1.0}, dy_dcsi{0.0}, dx_deta{0.0}, dy_deta{1.0};
};
struct VolMetrics
{
    double xi_x, xi_y, eta_x, eta_y, detJ;
    double norm_grad_xi() const { return std::sqrt(xi_x * xi_x + xi_y * xi_y); }
    double norm_grad_eta() const { return std::sqrt(eta_x * eta_x + eta_y * eta_y); }
};

struct Geometry
{
    int    kind{FRSDG_GEOM_CARTESIAN};
    int    profile{FRSDG_PROFILE_FLAT};
    double Lx{1.0}, Ly{1.0};
    double prm[4]{};

    // Wall profiles (h, dh/dx): tests/bump.cpp:29-119, tests/boundary_conforming.cpp:28-67.
    std::pair<double, double> wall(double x) const
    {
        const double m_L_x = Lx;
        if (profile == FRSDG_PROFILE_WEDGE_BUMP)
        {
            const double x_start = 0.15 * m_L_x, x_c_straight = 0.30 * m_L_x;
            const double x_e_start = 0.55 * m_L_x, x_e_end = 0.70 * m_L_x;
            const double compress_slope = 0.2, expand_slope = -0.2;
            const double A_c = compress_slope / (2.0 * (x_c_straight - x_start));
            const double dx_c = x_c_straight - x_start;
            const double h_c_end = A_c * dx_c * dx_c;
            if (x <= x_start) return {0.0, 0.0};
            if (x <= x_c_straight)
            {
                const double dx = x - x_start;
                return {-(A_c * dx * dx), -(2.0 * A_c * dx)};
            }
            if (x <= x_e_start)
            {
                const double dx = x - x_c_straight;
                return {-(h_c_end + compress_slope * dx), -compress_slope};
            }
            const double dx_run = x_e_start - x_c_straight;
            const double h_e_start = h_c_end + compress_slope * dx_run;
            const double dx_e = x_e_end - x_e_start;
            const double A_e = (expand_slope - compress_slope) / (2.0 * dx_e);
            if (x <= x_e_end)
            {
                const double dx = x - x_e_start;
                return {-(h_e_start + compress_slope * dx + A_e * dx * dx), -(compress_slope + 2.0 * A_e * dx)};
            }
            const double h_e_end = h_e_start + compress_slope * dx_e + A_e * dx_e * dx_e;
            const double dx = x - x_e_end;
            return {-(h_e_end + expand_slope * dx), -expand_slope};
        }
        if (profile == FRSDG_PROFILE_WEDGE_BC)
        {
            const double x_start = 0.3 * m_L_x, x_straight = 0.5 * m_L_x, wedge_slope = 0.2;
            const double A = wedge_slope / (2.0 * (x_straight - x_start));
            if (x <= x_start) return {0.0, 0.0};
            if (x <= x_straight)
            {
                const double dx = x - x_start;
                return {A * dx * dx, 2.0 * A * dx};
            }
            const double dx_trans = x_straight - x_start;
            const double h_base = A * dx_trans * dx_trans;
            const double dx = x - x_straight;
            return {h_base + wedge_slope * dx, wedge_slope};
        }
        if (profile == FRSDG_PROFILE_GAUSS_BUMP)
        {
            const double A = prm[1], k = prm[2];
            const double ex = std::exp(-k * x * x);
            return {A * ex, -2.0 * k * x * A * ex};
        }
        return {0.0, 0.0};
    }

    std::pair<double, double> coords(double csi, double eta) const
    {
        switch (kind)
        {
            case FRSDG_GEOM_DELAVAL:
            {
                const double x_phys = Lx * csi;
                const double h_x = 0.5;
                const double Y1 = -h_x, Y2 = h_x;
                return {x_phys, Y1 * (1.0 - eta) + Y2 * eta};
            }
            case FRSDG_GEOM_WALL_PROFILE:
            {
                const double x_phys = prm[0] + Lx * csi;
                const auto   hw = wall(x_phys);
                return {x_phys, hw.first * (1.0 - eta) + Ly * eta};
            }
            case FRSDG_GEOM_SINE_WARP:
            {
                const double two_pi = 2.0 * std::numbers::pi;
                const double d = prm[0] * std::sin(two_pi * csi) * std::sin(two_pi * eta);
                return {Lx * csi + d, Ly * eta + d};
            }
            default: return {Lx * csi, Ly * eta};
        }
    }

    GeomJac jac(double csi, double eta) const
    {
        switch (kind)
        {
            case FRSDG_GEOM_DELAVAL:
            {
                const double h_x = 0.5, dh_dx = 0.0;
                return {Lx, dh_dx * Lx * eta, 0.0, h_x};
            }
            case FRSDG_GEOM_WALL_PROFILE:
            {
                const double x_phys = prm[0] + Lx * csi;
                const auto   hw = wall(x_phys);
                return {Lx, hw.second * Lx * (1.0 - eta), 0.0, Ly - hw.first};
            }
            case FRSDG_GEOM_SINE_WARP:
            {
                const double two_pi = 2.0 * std::numbers::pi;
                const double A = prm[0];
                const double sc = std::sin(two_pi * csi), cc = std::cos(two_pi * csi);
                const double se = std::sin(two_pi * eta), ce = std::cos(two_pi * eta);
                const double d_dcsi = two_pi * A * cc * se;
                const double d_deta = two_pi * A * sc * ce;
                return {Lx + d_dcsi, d_dcsi, d_deta, Ly + d_deta};
            }
            default: return {Lx, 0.0, 0.0, Ly};
        }
    }

    std::pair<double, double> x_face(double csi, double eta) const
    {
        if (kind == FRSDG_GEOM_SINE_WARP)
        {
            const GeomJac g = jac(csi, eta);
            const double unx = g.dy_deta, uny = -g.dx_deta;
            const double inv = 1.0 / std::sqrt(unx * unx + uny * uny);
            return {unx * inv, uny * inv};
        }
        return {1.0, 0.0};
    }
    std::pair<double, double> y_face(double csi, double eta) const
    {
        switch (kind)
        {
            case FRSDG_GEOM_DELAVAL:
            {
                const double dh_dx = 0.0;
                double unx = -dh_dx * eta, uny = 1.0;
                double inv = 1.0 / std::sqrt(unx * unx + uny * uny);
                return {unx * inv, uny * inv};
            }
            case FRSDG_GEOM_WALL_PROFILE:
            {
                const double x_phys = prm[0] + Lx * csi;
                const double dh_dx = wall(x_phys).second;
                double unx = -dh_dx * Lx * (1.0 - eta), uny = Lx;
                double inv = 1.0 / std::sqrt(unx * unx + uny * uny);
                return {unx * inv, uny * inv};
            }
            case FRSDG_GEOM_SINE_WARP:
            {
                const GeomJac g = jac(csi, eta);
                const double unx = -g.dy_dcsi, uny = g.dx_dcsi;
                const double inv = 1.0 / std::sqrt(unx * unx + uny * uny);
                return {unx * inv, uny * inv};
            }
            default: return {0.0, 1.0};
        }
    }
};

// ---------------------------------------------------------------- the problem
struct Problem
{
    frsdg_config        cfg{};
    RefElement          re;
    Gas                 gas;
    Geometry            geom;
    std::vector<double> filt; // n*n
    int                 n{}, Nx{}, Ny{};
    bool                per_x{false}, per_y{false};
    int                 ndofs{};
    int                 nthreads{1};

    explicit Problem(const frsdg_config& c) : cfg(c)
    {
        re = make_ref_element(c.poly_deg, c.radau_corr);
        n  = re.n;
        gas.law = c.gas_law; gas.gamma = c.gamma; gas.R = c.R_spec; gas.a = c.vdw_a; gas.b = c.vdw_b;
        geom.kind = c.geometry; geom.profile = c.geom_profile;
        geom.Lx = c.box_length[0]; geom.Ly = c.box_length[1];
        for (int i = 0; i < 4; ++i) geom.prm[i] = c.geom_params[i];
        filt = make_filter_matrix(re, c.filt_cut_off, c.filt_strength, c.filt_alpha);
        Nx = c.n_elems[0];
        Ny = (c.dim == 2) ? c.n_elems[1] : 1;
        per_x = c.bc[FRSDG_LEFT].kind == FRSDG_BC_PERIODIC && c.bc[FRSDG_RIGHT].kind == FRSDG_BC_PERIODIC;
        per_y = c.bc[FRSDG_TOP].kind == FRSDG_BC_PERIODIC && c.bc[FRSDG_BOTTOM].kind == FRSDG_BC_PERIODIC;
        ndofs = (c.dim == 2) ? 4 * n * n : 3 * n;
    }
    int64_t n_total() const { return int64_t(Nx) * Ny * ndofs; }

    // physics_evaluator.hpp:235-246
    double comp_x(int i, int k) const
    {
        const double h_x = 1.0 / static_cast<double>(Nx);
        return h_x * (static_cast<double>(i) + 0.5 * (1.0 + re.csi[k]));
    }
    double comp_y(int j, int l) const
    {
        const double h_y = 1.0 / static_cast<double>(Ny);
        return h_y * (static_cast<double>(j) + 0.5 * (1.0 + re.csi[l]));
    }
    // physics_evaluator.hpp:282-305
    VolMetrics metrics(double cx, double cy) const
    {
        const GeomJac g      = geom.jac(cx, cy);
        const double dcsi_dr = 0.5 / static_cast<double>(Nx);
        const double deta_ds = 0.5 / static_cast<double>(Ny);
        const double dx_dr = g.dx_dcsi * dcsi_dr, dy_dr = g.dy_dcsi * dcsi_dr;
        const double dx_ds = g.dx_deta * deta_ds, dy_ds = g.dy_deta * deta_ds;
        const double detJ  = dx_dr * dy_ds - dx_ds * dy_dr;
        return {dy_ds / detJ, -dx_ds / detJ, -dy_dr / detJ, dx_dr / detJ, detJ};
    }
};

// ---------------------------------------------------------------- boundary conditions
// Exact isentropic vortex (factory.hpp:311-352).
inline std::array<double, 4> exact_vortex(double time, double x, double y, const double* vd)
{
    const double u_0 = vd[0], v_0 = vd[1], beta = vd[2], r_v = vd[3], l = vd[4];
    const auto gamma{1.4};
    const auto pi{std::numbers::pi_v<double>};
    double x_c = l / 2.0 + u_0 * time;
    double y_c = l / 2.0 + v_0 * time;
    x_c = x_c - l * std::floor(x_c / l);
    y_c = y_c - l * std::floor(y_c / l);
    const auto dx = x - x_c;
    const auto dy = y - y_c;
    const auto r2 = (dx * dx) + (dy * dy);
    const auto f = 1.0 - (r2 / (r_v * r_v));
    const auto exp_f = std::exp(f);
    const auto rho = std::pow(1.0 - (beta * beta * (gamma - 1.0) * (exp_f * exp_f)) / (16.0 * gamma * pi * pi),
                              1.0 / (gamma - 1.0));
    const auto u = u_0 - (beta * exp_f * dy) / (2.0 * pi * r_v);
    const auto v = v_0 + (beta * exp_f * dx) / (2.0 * pi * r_v);
    const auto p = std::pow(rho, gamma);
    const auto E = (p / (gamma - 1.0)) + 0.5 * rho * (u * u + v * v);
    return {rho, rho * u, rho * v, E};
}

// Real-valued custom boundary state (the "lambda" kinds).  nx, ny: face normal at
// the face point; x, y: physical face coordinates.
inline std::array<double, 4> custom_bc2(const Problem& P, int dir, double t, double x, double y, double nx,
                                        double ny, const std::array<double, 4>& in)
{
    const frsdg_bc& b = P.cfg.bc[dir];
    switch (b.kind)
    {
        case FRSDG_BC_DIRICHLET: return {b.state[0], b.state[1], b.state[2], b.state[3]};
        case FRSDG_BC_SLIP_WALL:
        {
            // tests/bump.cpp:250-272
            auto   ext = in;
            double u_in = in[1] / in[0];
            double v_in = in[2] / in[0];
            double vn_in = u_in * nx + v_in * ny;
            double u_out = u_in - 2.0 * vn_in * nx;
            double v_out = v_in - 2.0 * vn_in * ny;
            ext[1] = ext[0] * u_out;
            ext[2] = ext[0] * v_out;
            return ext;
        }
        case FRSDG_BC_VORTEX:
        {
            // factory.hpp:504-511 (left/right); the same pattern on bottom/top.
            if (dir == FRSDG_LEFT) return exact_vortex(t, 0.0, y, b.params);
            if (dir == FRSDG_RIGHT) return exact_vortex(t, P.cfg.box_length[0], y, b.params);
            if (dir == FRSDG_BOTTOM) return exact_vortex(t, x, 0.0, b.params);
            return exact_vortex(t, x, P.cfg.box_length[1], b.params);
        }
        case FRSDG_BC_SUBSONIC_INFLOW:
        {
            const double g = P.gas.gamma;
            const double p0 = b.params[0], T0 = b.params[1], Rg = b.params[2], ang = b.params[3];
            const auto   th = make_state2(in);
            double p = P.gas.pressure(th.density, th.energy);
            if (p > p0) p = p0;
            const double M2 = 2.0 / (g - 1.0) * (std::pow(p0 / p, (g - 1.0) / g) - 1.0);
            const double T = T0 / (1.0 + 0.5 * (g - 1.0) * M2);
            const double rho = p / (Rg * T);
            const double c = std::sqrt(g * p / rho);
            const double vel = std::sqrt(M2) * c;
            const double u = vel * std::cos(ang), v = vel * std::sin(ang);
            return {rho, rho * u, rho * v, p / (g - 1.0) + 0.5 * rho * (u * u + v * v)};
        }
        case FRSDG_BC_PRESSURE_OUTLET:
        {
            const double rho = in[0];
            const double u = in[1] / rho, v = in[2] / rho;
            const double vel2 = u * u + v * v;
            return {rho, in[1], in[2], P.gas.rhoE(rho, std::sqrt(vel2), b.params[0])};
        }
        default: return in;
    }
}

// BoundaryConditions<T,2>::evaluate_bc (boundary_conditions.hpp:239-248) for the
// real or complex scalar: native kinds act on the full scalar, lambda kinds see
// the real parts and return a real ghost (boundary_conditions.hpp:276-293).
template <class U>
std::array<U, 4> evaluate_bc2(const Problem& P, int dir, double t, double x, double y, double nx, double ny,
                              const std::array<U, 4>& in)
{
    const int kind = P.cfg.bc[dir].kind;
    if (kind == FRSDG_BC_OUTFLOW || kind == FRSDG_BC_PERIODIC) return in;
    if (kind == FRSDG_BC_WALL)
    {
        auto         r    = in;
        const size_t axis = static_cast<size_t>(dir) / 2;
        r[1 + axis]       = -r[1 + axis];
        return r;
    }
    std::array<double, 4> rin{re(in[0]), re(in[1]), re(in[2]), re(in[3])};
    const auto            o = custom_bc2(P, dir, t, x, y, nx, ny, rin);
    return {U(o[0]), U(o[1]), U(o[2]), U(o[3])};
}

// 1D: boundary_conditions.hpp:59-151
template <class U> std::array<U, 3> evaluate_bc1(const Problem& P, int dir, double /*t*/, const std::array<U, 3>& in)
{
    const frsdg_bc& b = P.cfg.bc[dir];
    if (b.kind == FRSDG_BC_OUTFLOW || b.kind == FRSDG_BC_PERIODIC) return in;
    if (b.kind == FRSDG_BC_WALL) { auto r = in; r[1] = -r[1]; return r; }
    if (b.kind == FRSDG_BC_DIRICHLET) return {U(b.state[0]), U(b.state[1]), U(b.state[2])};
    throw std::invalid_argument("unsupported 1D boundary kind");
}

// ---------------------------------------------------------------- 2D residual
// PhysicsEvaluator<Traits,2>::residual_kernel (physics_impl_2D.hpp:646-902) with
// compute_volume_term (268-357).  Vectors in DMDA natural order.
template <class U> void residual2d(const Problem& P, double time, const U* X, U* R)
{
    const int n = P.n, Nx = P.Nx, Ny = P.Ny, nd = P.ndofs;
    const auto& D = P.re.D;
    auto elem = [&](const U* base, int i, int j) -> const U*
    {
        i = (i % Nx + Nx) % Nx;
        j = (j % Ny + Ny) % Ny;
        return base + (int64_t(j) * Nx + i) * nd;
    };
    auto at = [n](const U* e, int eq, int k, int l) -> const U& { return e[(l * n + k) * 4 + eq]; };

    // ---- volume (physics_impl_2D.hpp:676-684, 268-357)
#pragma omp parallel for schedule(static) num_threads(P.nthreads)
    for (int j = 0; j < Ny; ++j)
    {
        std::vector<U> Fb(nd), Gb(nd);
        for (int i = 0; i < Nx; ++i)
        {
            const U* u  = elem(X, i, j);
            U*       rs = R + (int64_t(j) * Nx + i) * nd;
            for (int q = 0; q < nd; ++q) rs[q] = U{0.0};
            for (int l = 0; l < n; ++l)
                for (int k = 0; k < n; ++k)
                {
                    std::array<U, 4> s{at(u, 0, k, l), at(u, 1, k, l), at(u, 2, k, l), at(u, 3, k, l)};
                    std::array<U, 4> F, G;
                    U                p;
                    euler_fluxes2(s, P.gas, F, G, p);
                    for (int eq = 0; eq < 4; ++eq)
                    {
                        Fb[(l * n + k) * 4 + eq] = F[eq];
                        Gb[(l * n + k) * 4 + eq] = G[eq];
                    }
                }
            for (int l = 0; l < n; ++l)
                for (int k = 0; k < n; ++k)
                {
                    const auto m = P.metrics(P.comp_x(i, k), P.comp_y(j, l));
                    for (int eq = 0; eq < 4; ++eq)
                    {
                        U dF_dxi{0.0}, dG_dxi{0.0};
                        for (int mm = 0; mm < n; ++mm)
                        {
                            dG_dxi += D[k * n + mm] * Gb[(l * n + mm) * 4 + eq];
                            dF_dxi += D[k * n + mm] * Fb[(l * n + mm) * 4 + eq];
                        }
                        U dG_deta{0.0}, dF_deta{0.0};
                        for (int mm = 0; mm < n; ++mm)
                        {
                            dG_deta += D[l * n + mm] * Gb[(mm * n + k) * 4 + eq];
                            dF_deta += D[l * n + mm] * Fb[(mm * n + k) * 4 + eq];
                        }
                        const U px = m.xi_x * dF_dxi + m.eta_x * dF_deta;
                        const U py = m.xi_y * dG_dxi + m.eta_y * dG_deta;
                        rs[(l * n + k) * 4 + eq] += px + py;
                    }
                }
        }
    }

    // ---- x faces (physics_impl_2D.hpp:689-792)
    const auto& dLx = P.re.dL;
    const auto& dRx = P.re.dR;
    const bool phys_left = !P.per_x, phys_right = !P.per_x;
#pragma omp parallel for schedule(static) num_threads(P.nthreads)
    for (int j = 0; j < Ny; ++j)
    {
        for (int I = 0; I <= Nx; ++I)
        {
            const bool upd_L   = I > 0;
            const bool upd_R   = I < Nx;
            const bool bc_left = (I == 0) && phys_left;
            const bool bc_right = (I == Nx) && phys_right;
            const U* uL = elem(X, I - 1, j);
            const U* uR = elem(X, I, j);
            const double cx = P.comp_x(I, 0);
            for (int l = 0; l < n; ++l)
            {
                const double cy = P.comp_y(j, l);
                const auto   fn = P.geom.x_face(cx, cy);
                const auto   mt = P.metrics(cx, cy);
                const double nx = fn.first, ny = fn.second;
                const double scale = mt.norm_grad_xi();
                std::array<U, 4> UL, UR;
                if (!bc_right) UR = {at(uR, 0, 0, l), at(uR, 1, 0, l), at(uR, 2, 0, l), at(uR, 3, 0, l)};
                if (!bc_left) UL = {at(uL, 0, n - 1, l), at(uL, 1, n - 1, l), at(uL, 2, n - 1, l), at(uL, 3, n - 1, l)};
                if (bc_left)
                {
                    const auto xy = P.geom.coords(cx, cy);
                    UL = evaluate_bc2(P, FRSDG_LEFT, time, xy.first, xy.second, nx, ny, UR);
                }
                if (bc_right)
                {
                    const auto xy = P.geom.coords(cx, cy);
                    UR = evaluate_bc2(P, FRSDG_RIGHT, time, xy.first, xy.second, nx, ny, UL);
                }
                std::array<U, 4> FxL, FyL, FxR, FyR;
                U                pd;
                euler_fluxes2(UL, P.gas, FxL, FyL, pd);
                euler_fluxes2(UR, P.gas, FxR, FyR, pd);
                const auto Fs = riemann2(P.cfg.riemann, UL, UR, P.gas, nx, ny);
                for (int eq = 0; eq < 4; ++eq)
                {
                    if (upd_L)
                    {
                        U*      rL  = R + (int64_t(j) * Nx + (I - 1)) * nd;
                        const U nfL = FxL[eq] * nx + FyL[eq] * ny;
                        for (int k = 0; k < n; ++k) rL[(l * n + k) * 4 + eq] += scale * (Fs[eq] - nfL) * dRx[k];
                    }
                    if (upd_R)
                    {
                        U*      rR  = R + (int64_t(j) * Nx + I) * nd;
                        const U nfR = FxR[eq] * nx + FyR[eq] * ny;
                        for (int k = 0; k < n; ++k) rR[(l * n + k) * 4 + eq] += scale * (Fs[eq] - nfR) * dLx[k];
                    }
                }
            }
        }
    }

    // ---- y faces (physics_impl_2D.hpp:797-899)
    const bool phys_bot = !P.per_y, phys_top = !P.per_y;
#pragma omp parallel for schedule(static) num_threads(P.nthreads)
    for (int i = 0; i < Nx; ++i)
    {
        for (int J = 0; J <= Ny; ++J)
        {
            const bool upd_B  = J > 0;
            const bool upd_T  = J < Ny;
            const bool bc_bot = (J == 0) && phys_bot;
            const bool bc_top = (J == Ny) && phys_top;
            const U* uB = elem(X, i, J - 1);
            const U* uT = elem(X, i, J);
            const double cy = P.comp_y(J, 0);
            for (int k = 0; k < n; ++k)
            {
                const double cx = P.comp_x(i, k);
                const auto   fn = P.geom.y_face(cx, cy);
                const auto   mt = P.metrics(cx, cy);
                const double nx = fn.first, ny = fn.second;
                const double scale = mt.norm_grad_eta();
                std::array<U, 4> UB, UT;
                if (!bc_top) UT = {at(uT, 0, k, 0), at(uT, 1, k, 0), at(uT, 2, k, 0), at(uT, 3, k, 0)};
                if (!bc_bot) UB = {at(uB, 0, k, n - 1), at(uB, 1, k, n - 1), at(uB, 2, k, n - 1), at(uB, 3, k, n - 1)};
                if (bc_bot)
                {
                    const auto xy = P.geom.coords(cx, cy);
                    UB = evaluate_bc2(P, FRSDG_BOTTOM, time, xy.first, xy.second, nx, ny, UT);
                }
                if (bc_top)
                {
                    const auto xy = P.geom.coords(cx, cy);
                    UT = evaluate_bc2(P, FRSDG_TOP, time, xy.first, xy.second, nx, ny, UB);
                }
                std::array<U, 4> FxB, FyB, FxT, FyT;
                U                pd;
                euler_fluxes2(UB, P.gas, FxB, FyB, pd);
                euler_fluxes2(UT, P.gas, FxT, FyT, pd);
                const auto Gs = riemann2(P.cfg.riemann, UB, UT, P.gas, nx, ny);
                for (int eq = 0; eq < 4; ++eq)
                {
                    if (upd_B)
                    {
                        U*      rB  = R + (int64_t(J - 1) * Nx + i) * nd;
                        const U nfB = FxB[eq] * nx + FyB[eq] * ny;
                        for (int l = 0; l < n; ++l) rB[(l * n + k) * 4 + eq] += scale * (Gs[eq] - nfB) * dRx[l];
                    }
                    if (upd_T)
                    {
                        U*      rT  = R + (int64_t(J) * Nx + i) * nd;
                        const U nfT = FxT[eq] * nx + FyT[eq] * ny;
                        for (int l = 0; l < n; ++l) rT[(l * n + k) * 4 + eq] += scale * (Gs[eq] - nfT) * dLx[l];
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------- 1D residual
// PhysicsEvaluator<Traits,1>::residual_kernel and local_steady_res
// (physics_impl_1D.hpp:9-94, 124-181).
template <class U> void residual1d(const Problem& P, double time, const U* X, U* R)
{
    const int    n = P.n, N = P.Nx, nd = P.ndofs;
    const double h = P.cfg.box_length[0] / P.cfg.n_elems[0];
    const double inv_jac = 2.0 / h;
    const auto&  D = P.re.D;
    const auto&  dL = P.re.dL;
    const auto&  dR = P.re.dR;
    auto el   = [&](int e) -> const U* { e = (e % N + N) % N; return X + int64_t(e) * nd; };
    auto node = [n](const U* s, int k) { return std::array<U, 3>{s[0 * n + k], s[1 * n + k], s[2 * n + k]}; };

    auto local = [&](int e, const std::array<U, 3>& prev, const std::array<U, 3>& next)
    {
        const U* s   = el(e);
        U*       res = R + int64_t(e) * nd;
        for (int q = 0; q < nd; ++q) res[q] = U{};
        for (int j = 0; j < n; ++j)
        {
            const auto Fj = euler_flux1(node(s, j), P.gas);
            for (int i = 0; i < n; ++i)
            {
                const U D_ij = inv_jac * D[i * n + j];
                res[0 * n + i] += D_ij * Fj[0];
                res[1 * n + i] += D_ij * Fj[1];
                res[2 * n + i] += D_ij * Fj[2];
            }
        }
        const auto FdL = euler_flux1(node(s, 0), P.gas);
        const auto FdR = euler_flux1(node(s, n - 1), P.gas);
        const auto FsL = riemann1(P.cfg.riemann, prev, node(s, 0), P.gas);
        const auto FsR = riemann1(P.cfg.riemann, node(s, n - 1), next, P.gas);
        for (int eq = 0; eq < 3; ++eq)
        {
            const U delta_L = FsL[eq] - FdL[eq];
            const U delta_R = FsR[eq] - FdR[eq];
            for (int i = 0; i < n; ++i) res[eq * n + i] += inv_jac * (delta_L * dL[i] + delta_R * dR[i]);
        }
    };

    int first = 0, last = N;
    if (!P.per_x)
    {
        --last;
        {
            const int e = N - 1;
            local(e, node(el(e - 1), n - 1), evaluate_bc1(P, FRSDG_RIGHT, time, node(el(e), n - 1)));
        }
        ++first;
        {
            const int e = 0;
            local(e, evaluate_bc1(P, FRSDG_LEFT, time, node(el(e), 0)), node(el(e + 1), 0));
        }
    }
#pragma omp parallel for schedule(static) num_threads(P.nthreads)
    for (int e = first; e < last; ++e)
    {
        local(e, node(el(e - 1), n - 1), node(el(e + 1), 0));
        if (P.cfg.coord_sys == FRSDG_COORD_RADIAL)
        {
            const U* sp  = el(e);
            U*       res = R + int64_t(e) * nd;
            for (int k = 0; k < n; ++k)
            {
                const double r = (e + 0.5 * (P.re.csi[k] + 1.0)) * h;
                const double inv_r = (r > 1e-8) ? 1.0 / r : 0.0;
                const U& rho = sp[0 * n + k];
                const U& rhoU = sp[1 * n + k];
                const U& rhoE = sp[2 * n + k];
                const U vel = rhoU / rho;
                const U pres = P.gas.pressure(rho, rhoE / rho - U(0.5) * vel * vel);
                res[0 * n + k] += inv_r * rhoU;
                res[1 * n + k] += inv_r * rhoU * vel;
                res[2 * n + k] += inv_r * vel * (rhoE + pres);
            }
        }
    }
}

template <class U> void residual(const Problem& P, double t, const U* X, U* R)
{
    if (P.cfg.dim == 2) residual2d(P, t, X, R);
    else residual1d(P, t, X, R);
}

// ---------------------------------------------------------------- change of variables
// problem_def.hpp:36-51, called per node as in physics_impl_2D.hpp:126-154 and
// physics_impl_1D.hpp:183-205.
template <class U> void prim_to_cons(const Problem& P, const U* prim, U* cons)
{
    const int n = P.n;
    const int64_t nel = int64_t(P.Nx) * P.Ny;
    for (int64_t e = 0; e < nel; ++e)
    {
        const U* p = prim + e * P.ndofs;
        U*       c = cons + e * P.ndofs;
        if (P.cfg.dim == 2)
        {
            for (int q = 0; q < n * n; ++q)
            {
                const U rho_t = p[q * 4 + 0], u = p[q * 4 + 1], v = p[q * 4 + 2], e_t = p[q * 4 + 3];
                const U rho = std::exp(rho_t);
                const U sum_v_sq = (U{0.0} + u * u) + v * v;
                const U kin_en = U{0.5} * sum_v_sq;
                const U rhoE = rho * (std::exp(e_t) + kin_en);
                c[q * 4 + 0] = rho; c[q * 4 + 1] = rho * u; c[q * 4 + 2] = rho * v; c[q * 4 + 3] = rhoE;
            }
        }
        else
        {
            for (int k = 0; k < n; ++k)
            {
                const U rho_t = p[0 * n + k], vel = p[1 * n + k], ie = p[2 * n + k];
                const U rho = std::exp(rho_t);
                const U sum_v_sq = U{0.0} + vel * vel;
                const U rhoE = rho * (std::exp(ie) + U{0.5} * sum_v_sq);
                c[0 * n + k] = rho; c[1 * n + k] = rho * vel; c[2 * n + k] = rhoE;
            }
        }
    }
}

// rhs_func (petsc_solver_impl.hpp:657-670)
inline void rhs(const Problem& P, double t, const double* U, double* F)
{
    residual(P, t, U, F);
    for (int64_t q = 0; q < P.n_total(); ++q) F[q] *= -1.0;
}

// fun_implicit (petsc_solver_impl.hpp:626-655)
inline void ifunction(const Problem& P, double t, const double* U, const double* Udot, double* F)
{
    std::vector<double> cons;
    const double*       active = U;
    if (P.cfg.cond_sys)
    {
        cons.resize(P.n_total());
        prim_to_cons(P, U, cons.data());
        active = cons.data();
    }
    residual(P, t, active, F);
    for (int64_t q = 0; q < P.n_total(); ++q) F[q] = Udot[q] + 1.0 * F[q];
}

// ComplexStepJacobianStrategy::matmult_{1,2}d_impl (petsc_solver_impl.hpp:270-432)
inline void jvp(const Problem& P, double t, double sigma, const double* U, const double* V, double* JV)
{
    const int64_t     N = P.n_total();
    const double      h = P.cfg.csd_eps;
    const double      one_over_h = 1.0 / h;
    std::vector<cplx> uiv(N), f(N);
    if (!P.cfg.cond_sys)
        for (int64_t q = 0; q < N; ++q) uiv[q] = cplx(U[q], V[q] * h);
    else
    {
        std::vector<cplx> prim(N);
        for (int64_t q = 0; q < N; ++q) prim[q] = cplx(U[q], V[q] * h);
        prim_to_cons(P, prim.data(), uiv.data());
    }
    for (int64_t q = 0; q < N; ++q) JV[q] = sigma * std::imag(uiv[q]) * one_over_h;
    residual(P, t, uiv.data(), f.data());
    for (int64_t q = 0; q < N; ++q) JV[q] += std::imag(f[q]) * one_over_h;
}

// ---------------------------------------------------------------- stabilisation
// filter.hpp:486-755 on one strided line: in/out accessors take the node index.
struct Stab
{
    const Problem& P;
    double         one_over_norm{};
    std::array<double, 3> gammas{};
    explicit Stab(const Problem& p) : P(p)
    {
        const double g = P.cfg.weno_gamma;
        gammas = {(1 - g) * 0.5, g, (1 - g) * 0.5};
        const double d_min = *std::min_element(gammas.begin(), gammas.end());
        one_over_norm = 1.0 / (std::pow(std::abs(1.0 / d_min - 1.0), P.cfg.shock_theta) + gammas.size() - 1);
    }
    double cell_average(const double* v) const
    {
        double s = 0.0;
        for (int i = 0; i < P.n; ++i) s += P.re.w[i] * v[i];
        return 0.5 * s;
    }
    double smoothness(const double* v) const
    {
        const int n = P.n;
        double cur[16], nxt[16];
        for (int i = 0; i < n; ++i) cur[i] = v[i];
        double beta = 0.0, factor = 4.0;
        for (int s = 1; s <= n - 1; ++s)
        {
            for (int r = 0; r < n; ++r)
            {
                double acc = 0.0;
                for (int c = 0; c < n; ++c) acc += P.re.D[r * n + c] * cur[c];
                nxt[r] = acc;
            }
            for (int r = 0; r < n; ++r) cur[r] = nxt[r];
            double integ = 0.0;
            for (int i = 0; i < n; ++i) integ += P.re.w[i] * cur[i] * cur[i];
            beta += factor * (0.5 * integ);
            factor *= 4.0;
        }
        return beta;
    }
    void filter(const double* in, double* out) const
    {
        const int n = P.n;
        for (int r = 0; r < n; ++r)
        {
            double acc = 0.0;
            for (int c = 0; c < n; ++c) acc += P.filt[r * n + c] * in[c];
            out[r] = acc;
        }
    }
    // StabilizationTechniques::apply_element_stabilization (filter.hpp:716-755)
    void apply(const double* prev, const double* curr, const double* next, double* out) const
    {
        const int  n = P.n;
        const bool spec = P.cfg.apply_filter != 0, weno = P.cfg.apply_weno != 0;
        if (!spec && !weno) { for (int i = 0; i < n; ++i) out[i] = curr[i]; return; }
        if (weno)
        {
            std::array<double, 3> betas = {smoothness(prev), smoothness(curr), smoothness(next)};
            std::array<double, 3> cg = gammas;
            for (int i = 0; i < 3; ++i) cg[i] /= std::pow(1.0e-6 + betas[i], 2);
            const double w_sum = cg[0] + cg[1] + cg[2];
            for (auto& g : cg) g /= w_sum;
            double num = 0.0;
            for (int i = 0; i < 3; ++i) num += std::pow(std::abs(cg[i] / gammas[i] - 1.0), P.cfg.shock_theta);
            const double r_j = num * one_over_norm;
            if (std::abs(r_j) >= P.cfg.shock_threshold)
            {
                const double ap = cell_average(prev), ac = cell_average(curr), an = cell_average(next);
                for (int i = 0; i < n; ++i)
                    out[i] = cg[0] * (prev[i] - ap + ac) + cg[1] * curr[i] + cg[2] * (next[i] - an + ac);
                if (spec) filter(curr, out);
                return;
            }
        }
        if (spec) filter(curr, out);
        else for (int i = 0; i < n; ++i) out[i] = curr[i];
    }
};

// PetscSolver::apply_stabilization (petsc_solver_impl.hpp:683-702) with
// limit_solution (2D physics_impl_2D.hpp:76-124, 1D physics_impl_1D.hpp:96-121).
// Neighbours across a non-periodic boundary are the never-written DMDA ghost
// entries of a local vector, which PETSc zero-initialises.
inline void post_step(const Problem& P, double* U)
{
    const int64_t       N = P.n_total();
    std::vector<double> src(U, U + N);
    const int           n = P.n, Nx = P.Nx, Ny = P.Ny, nd = P.ndofs;
    Stab                st(P);
    std::vector<double> zeros(nd, 0.0);
    auto elem = [&](int i, int j) -> const double*
    {
        if (i < 0 || i >= Nx) { if (!P.per_x) return zeros.data(); i = (i % Nx + Nx) % Nx; }
        if (j < 0 || j >= Ny) { if (!P.per_y) return zeros.data(); j = (j % Ny + Ny) % Ny; }
        return src.data() + (int64_t(j) * Nx + i) * nd;
    };
    if (P.cfg.dim == 1)
    {
        for (int e = 0; e < Nx; ++e)
        {
            const double* sp = elem(e, 0);
            const double* pv = elem(e - 1, 0);
            const double* nx = elem(e + 1, 0);
            for (int eq = 0; eq < 3; ++eq)
                st.apply(pv + eq * n, sp + eq * n, nx + eq * n, U + int64_t(e) * nd + eq * n);
        }
        return;
    }
#pragma omp parallel for schedule(static) num_threads(P.nthreads)
    for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i)
        {
            const double* uL = elem(i - 1, j);
            const double* uC = elem(i, j);
            const double* uR = elem(i + 1, j);
            const double* uB = elem(i, j - 1);
            const double* uT = elem(i, j + 1);
            double*       out = U + (int64_t(j) * Nx + i) * nd;
            std::vector<double> scr(nd);
            double a[16], b[16], c[16], o[16];
            for (int eq = 0; eq < 4; ++eq)
                for (int l = 0; l < n; ++l)
                {
                    for (int k = 0; k < n; ++k)
                    {
                        a[k] = uL[(l * n + k) * 4 + eq];
                        b[k] = uC[(l * n + k) * 4 + eq];
                        c[k] = uR[(l * n + k) * 4 + eq];
                    }
                    st.apply(a, b, c, o);
                    for (int k = 0; k < n; ++k) scr[(l * n + k) * 4 + eq] = o[k];
                }
            for (int eq = 0; eq < 4; ++eq)
                for (int k = 0; k < n; ++k)
                {
                    for (int l = 0; l < n; ++l)
                    {
                        a[l] = uB[(l * n + k) * 4 + eq];
                        b[l] = uC[(l * n + k) * 4 + eq];
                        c[l] = uT[(l * n + k) * 4 + eq];
                    }
                    st.apply(a, b, c, o);
                    for (int l = 0; l < n; ++l) out[(l * n + k) * 4 + eq] = o[l];
                }
            for (int q = 0; q < nd; ++q) out[q] = 0.5 * (scr[q] + out[q]);
        }
}

// ---------------------------------------------------------------- positivity limiter
// The scaling limiter of Zhang and Shu (J. Comput. Phys. 229 (2010) 8918-8934,
// sec. 3): per element, with the cell average Ubar taken by GLL quadrature (weights
// w_k w_l detJ_kl in 2D, w_k in 1D) and eps = min(cfg.pp_eps, rho_bar, p_bar),
//   1. rho_min < eps:  rho <- rho_bar + theta1 (rho - rho_bar),
//                      theta1 = (rho_bar - eps) / (rho_bar - rho_min);
//   2. p(U_q) < eps at some node: U <- Ubar + theta2 (U - Ubar), theta2 = min_q t_q,
//      t_q in [0, 1) the point of the segment Ubar -> U_q where the pressure is eps,
//      found by 60 bisection steps (p(Ubar + t d) >= eps keeps the lower end).
// Elements whose average is itself inadmissible are left unchanged.  It has no
// counterpart in the reference (cfg.pp_limit turns it on); the time integrators apply
// it to every Runge-Kutta stage and after the post-step stabilisation.
inline double pp_pressure(const Gas& g, int nv, const double* u)
{
    double m2 = 0.0;
    for (int c = 1; c < nv - 1; ++c) m2 += u[c] * u[c];
    const double rho = u[0];
    const double e = (u[nv - 1] - 0.5 * m2 / rho) / rho;
    return g.pressure(rho, e);
}

inline double pp_segment_root(const Gas& g, int nv, const double* ub, const double* uq, double eps)
{
    double lo = 0.0, hi = 1.0, s[4];
    for (int it = 0; it < 60; ++it)
    {
        const double mid = 0.5 * (lo + hi);
        for (int c = 0; c < nv; ++c) s[c] = ub[c] + mid * (uq[c] - ub[c]);
        if (s[0] > 0.0 && pp_pressure(g, nv, s) >= eps) lo = mid;
        else hi = mid;
    }
    return lo;
}

// One element: nq nodes, value c of node q at u[q * sq + c * sc]; W[q] quadrature weights.
inline void pp_limit_element(const Gas& g, int nv, int nq, const double* W, double* u, int sq, int sc, double eps0)
{
    double wsum = 0.0, ub[4] = {0.0, 0.0, 0.0, 0.0};
    for (int q = 0; q < nq; ++q)
    {
        wsum += W[q];
        for (int c = 0; c < nv; ++c) ub[c] += W[q] * u[q * sq + c * sc];
    }
    for (int c = 0; c < nv; ++c) ub[c] /= wsum;
    const double pb = pp_pressure(g, nv, ub);
    if (!(ub[0] > 0.0) || !(pb > 0.0)) return;
    const double eps = std::min(eps0, std::min(ub[0], pb));
    double rmin = u[0];
    for (int q = 1; q < nq; ++q) rmin = std::min(rmin, u[q * sq]);
    if (rmin < eps)
    {
        const double th1 = (ub[0] - eps) / (ub[0] - rmin);
        for (int q = 0; q < nq; ++q) u[q * sq] = ub[0] + th1 * (u[q * sq] - ub[0]);
    }
    double th2 = 1.0, uq[4];
    for (int q = 0; q < nq; ++q)
    {
        for (int c = 0; c < nv; ++c) uq[c] = u[q * sq + c * sc];
        if (!(pp_pressure(g, nv, uq) >= eps)) th2 = std::min(th2, pp_segment_root(g, nv, ub, uq, eps));
    }
    if (th2 < 1.0)
        for (int q = 0; q < nq; ++q)
            for (int c = 0; c < nv; ++c) u[q * sq + c * sc] = ub[c] + th2 * (u[q * sq + c * sc] - ub[c]);
}

inline void pp_limit(const Problem& P, double* U)
{
    const int n = P.n, nd = P.ndofs;
    if (P.cfg.dim == 1)
    {
        for (int e = 0; e < P.Nx; ++e) pp_limit_element(P.gas, 3, n, P.re.w.data(), U + int64_t(e) * nd, 1, n, P.cfg.pp_eps);
        return;
    }
    const bool curved = P.cfg.geometry == FRSDG_GEOM_SINE_WARP || P.cfg.geometry == FRSDG_GEOM_WALL_PROFILE;
#pragma omp parallel for schedule(static) num_threads(P.nthreads)
    for (int j = 0; j < P.Ny; ++j)
    {
        std::vector<double> W(size_t(n) * n);
        for (int i = 0; i < P.Nx; ++i)
        {
            for (int l = 0; l < n; ++l)
                for (int k = 0; k < n; ++k)
                    W[size_t(l) * n + k] = P.re.w[k] * P.re.w[l] *
                                           (curved ? P.metrics(P.comp_x(i, k), P.comp_y(j, l)).detJ : 1.0);
            pp_limit_element(P.gas, 4, n * n, W.data(), U + (int64_t(j) * P.Nx + i) * nd, 4, 1, P.cfg.pp_eps);
        }
    }
}

// The post-step of this build: the reference's stabilisation, then (cfg.pp_limit) the
// positivity limiter.
inline void post_step_full(const Problem& P, double* U)
{
    if (P.cfg.apply_filter || P.cfg.apply_weno) post_step(P, U);
    if (P.cfg.pp_limit) pp_limit(P, U);
}

} // namespace frsdg_oracle
