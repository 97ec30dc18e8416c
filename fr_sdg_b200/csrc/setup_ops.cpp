// setup_ops.cpp -- reference element, spectral filter and geometry maps (host).
//
// GLL nodes: Newton iteration on q = P_{p+1} - P_{p-1} (whose interior roots are
// the GLL points), started from the Chebyshev-Gauss-Lobatto points and mirrored
// for exact symmetry (D. A. Kopriva, "Implementing Spectral Methods for PDEs",
// Springer 2009, Algorithm 25).  Weights 2 / (p (p+1) P_p(x)^2) as in
// reference_element.hpp:104-115.  Differentiation matrix and VCJH correction
// derivatives follow cached_computations.hpp:37-137 (Vincent, Castonguay and
// Jameson, J. Sci. Comput. 47, 2011).  The filter's inverse Vandermonde matrix
// is the discrete Legendre transform on the GLL points (exact for this node
// set), in place of the reference's LU inverse (filter.hpp:451-484).
#include "setup_ops.hpp"

#include <cmath>
#include <limits>
#include <stdexcept>

namespace frsdg
{
namespace
{
// P_k(x) and P'_k(x) for k = 0..n by the three-term recurrence.
void legendre_table(int n, double x, double* P, double* dP)
{
    P[0] = 1.0;
    dP[0] = 0.0;
    if (n == 0) return;
    P[1] = x;
    dP[1] = 1.0;
    for (int k = 1; k < n; ++k)
    {
        P[k + 1]  = ((2 * k + 1) * x * P[k] - k * P[k - 1]) / (k + 1);
        dP[k + 1] = dP[k - 1] + (2 * k + 1) * P[k];
    }
}
double legendre_p(int k, double x)
{
    double P[16], dP[16];
    legendre_table(k, x, P, dP);
    return P[k];
}
double legendre_dp(int k, double x)
{
    if (k < 0) return 0.0;
    double P[16], dP[16];
    legendre_table(k, x, P, dP);
    return dP[k];
}
} // namespace

void ref_element_into(int p, double c, double* X, double* W, double* Dm, double* DL, double* DR)
{
    if (p < 1 || p > 9) throw std::invalid_argument("poly_deg must be in [1, 9]");
    const int n = p + 1;
    for (int k = 0; k < n; ++k) X[k] = W[k] = 0.0;
    X[0] = -1.0;
    X[p] = 1.0;
    const double pi = 3.14159265358979323846;
    for (int j = 1; j <= (n + 1) / 2 - 1; ++j)
    {
        double x = -std::cos(pi * j / p);
        for (int it = 0; it < 100; ++it)
        {
            double P[16], dP[16];
            legendre_table(p + 1, x, P, dP);
            const double q  = P[p + 1] - P[p - 1];
            const double dq = (2 * p + 1) * P[p];
            const double dx = -q / dq;
            x += dx;
            if (std::fabs(dx) <= 4.0 * std::numeric_limits<double>::epsilon() * std::fabs(x)) break;
        }
        X[j]     = x;
        X[p - j] = -x;
    }
    if (p % 2 == 0) X[p / 2] = 0.0;
    for (int k = 0; k < n; ++k)
    {
        const double Pp = legendre_p(p, X[k]);
        W[k]            = 2.0 / (double(p) * (p + 1) * Pp * Pp);
    }
    // differentiation matrix
    double a[16];
    for (int i = 0; i < n; ++i)
    {
        a[i] = 1.0;
        for (int k = 0; k < n; ++k)
            if (k != i) a[i] *= X[i] - X[k];
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            if (i != j) Dm[i * n + j] = a[i] / (a[j] * (X[i] - X[j]));
            else
            {
                double sum = 0.0;
                for (int k = 0; k < n; ++k)
                    if (k != i) sum += 1.0 / (X[i] - X[k]);
                Dm[i * n + i] = sum;
            }
        }
    // VCJH: eta_p = c (2p+1) (a_p p!)^2 / 2 with a_p = (2p)! / (2^p (p!)^2)
    double pf = 1.0, p2f = 1.0;
    for (int i = 2; i <= p; ++i) pf *= i;
    for (int i = 2; i <= 2 * p; ++i) p2f *= i;
    const double ap   = p2f / (std::pow(2.0, p) * pf * pf);
    const double apf  = ap * pf;
    const double eta  = c * double(2 * p + 1) * apf * apf / 2.0;
    const double sign = (p % 2 == 0) ? 1.0 : -1.0;
    for (int i = 0; i < n; ++i)
    {
        const double d0 = legendre_dp(p, X[i]);
        const double dm = legendre_dp(p - 1, X[i]);
        const double dp = legendre_dp(p + 1, X[i]);
        const double t  = (eta * dm + dp) / (1.0 + eta);
        DL[i] = sign * 0.5 * (d0 - t);
        DR[i] = 0.5 * (d0 + t);
    }
}

RefElem build_ref_element(int p, double c)
{
    if (p < 1 || p > 9) throw std::invalid_argument("poly_deg must be in [1, 9]");
    RefElem r;
    r.p = p;
    r.n = p + 1;
    r.x.assign(r.n, 0.0);
    r.w.assign(r.n, 0.0);
    r.D.assign(r.n * r.n, 0.0);
    r.dL.assign(r.n, 0.0);
    r.dR.assign(r.n, 0.0);
    ref_element_into(p, c, r.x.data(), r.w.data(), r.D.data(), r.dL.data(), r.dR.data());
    return r;
}

void filter_matrix_into(int p, const double* X, const double* W, int nc, int s, double alpha, double* F)
{
    const int n = p + 1;
    double sigma[16], gam[16], V[16 * 16];
    for (int i = 0; i < n; ++i)
    {
        if (i < nc) sigma[i] = 1.0;
        else
        {
            const double ratio = double(i - nc) / double((n - 1) - nc);
            sigma[i]           = std::exp(-alpha * std::pow(ratio, double(s)));
        }
        gam[i] = (i < p) ? 2.0 / (2.0 * i + 1.0) : 2.0 / double(p);
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) V[i * n + j] = legendre_p(j, X[i]);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k)
        {
            double acc = 0.0;
            for (int j = 0; j < n; ++j) acc += V[i * n + j] * sigma[j] * W[k] * V[k * n + j] / gam[j];
            F[i * n + k] = acc;
        }
}

std::vector<double> build_filter_matrix(const RefElem& re, int nc, int s, double alpha)
{
    std::vector<double> F(re.n * re.n, 0.0);
    filter_matrix_into(re.p, re.x.data(), re.w.data(), nc, s, alpha, F.data());
    return F;
}

// ---------------------------------------------------------------- geometry
GeometryMap::GeometryMap(const frsdg_config& c)
    : kind_(c.geometry), profile_(c.geom_profile), Lx_(c.box_length[0]), Ly_(c.box_length[1])
{
    for (int i = 0; i < 4; ++i) prm_[i] = c.geom_params[i];
}

bool GeometryMap::affine() const { return kind_ == FRSDG_GEOM_CARTESIAN || kind_ == FRSDG_GEOM_DELAVAL; }

std::pair<double, double> GeometryMap::wall(double x) const
{
    switch (profile_)
    {
        case FRSDG_PROFILE_WEDGE_BUMP:
        {
            // flat, parabolic compression, straight ramp, parabolic expansion, straight ramp
            const double x1 = 0.15 * Lx_, x2 = 0.30 * Lx_, x3 = 0.55 * Lx_, x4 = 0.70 * Lx_;
            const double sc = 0.2, se = -0.2;
            const double Ac = sc / (2.0 * (x2 - x1));
            const double d12 = x2 - x1;
            const double h2 = Ac * d12 * d12;
            if (x <= x1) return {0.0, 0.0};
            if (x <= x2) { const double d = x - x1; return {-(Ac * d * d), -(2.0 * Ac * d)}; }
            if (x <= x3) { const double d = x - x2; return {-(h2 + sc * d), -sc}; }
            const double h3 = h2 + sc * (x3 - x2);
            const double d34 = x4 - x3;
            const double Ae = (se - sc) / (2.0 * d34);
            if (x <= x4) { const double d = x - x3; return {-(h3 + sc * d + Ae * d * d), -(sc + 2.0 * Ae * d)}; }
            const double h4 = h3 + sc * d34 + Ae * d34 * d34;
            const double d = x - x4;
            return {-(h4 + se * d), -se};
        }
        case FRSDG_PROFILE_WEDGE_BC:
        {
            const double x1 = 0.3 * Lx_, x2 = 0.5 * Lx_, sl = 0.2;
            const double A = sl / (2.0 * (x2 - x1));
            if (x <= x1) return {0.0, 0.0};
            if (x <= x2) { const double d = x - x1; return {A * d * d, 2.0 * A * d}; }
            const double d12 = x2 - x1;
            const double d = x - x2;
            return {A * d12 * d12 + sl * d, sl};
        }
        case FRSDG_PROFILE_GAUSS_BUMP:
        {
            const double A = prm_[1], k = prm_[2];
            const double ex = std::exp(-k * x * x);
            return {A * ex, -2.0 * k * x * A * ex};
        }
        default: return {0.0, 0.0};
    }
}

std::pair<double, double> GeometryMap::physical(double csi, double eta) const
{
    const double two_pi = 2.0 * 3.14159265358979323846;
    switch (kind_)
    {
        case FRSDG_GEOM_DELAVAL: return {Lx_ * csi, -0.5 * (1.0 - eta) + 0.5 * eta};
        case FRSDG_GEOM_WALL_PROFILE:
        {
            const double x = prm_[0] + Lx_ * csi;
            return {x, wall(x).first * (1.0 - eta) + Ly_ * eta};
        }
        case FRSDG_GEOM_SINE_WARP:
        {
            const double d = prm_[0] * std::sin(two_pi * csi) * std::sin(two_pi * eta);
            return {Lx_ * csi + d, Ly_ * eta + d};
        }
        default: return {Lx_ * csi, Ly_ * eta};
    }
}

GeomJacobian GeometryMap::jacobian(double csi, double eta) const
{
    const double two_pi = 2.0 * 3.14159265358979323846;
    switch (kind_)
    {
        case FRSDG_GEOM_DELAVAL: return {Lx_, 0.0 * Lx_ * eta, 0.0, 0.5};
        case FRSDG_GEOM_WALL_PROFILE:
        {
            const auto hw = wall(prm_[0] + Lx_ * csi);
            return {Lx_, hw.second * Lx_ * (1.0 - eta), 0.0, Ly_ - hw.first};
        }
        case FRSDG_GEOM_SINE_WARP:
        {
            const double A = prm_[0];
            const double dc = two_pi * A * std::cos(two_pi * csi) * std::sin(two_pi * eta);
            const double de = two_pi * A * std::sin(two_pi * csi) * std::cos(two_pi * eta);
            return {Lx_ + dc, dc, de, Ly_ + de};
        }
        default: return {Lx_, 0.0, 0.0, Ly_};
    }
}

std::pair<double, double> GeometryMap::x_face_normal(double csi, double eta) const
{
    if (kind_ == FRSDG_GEOM_SINE_WARP)
    {
        const GeomJacobian g = jacobian(csi, eta);
        const double       a = g.dy_deta, b = -g.dx_deta;
        const double       inv = 1.0 / std::sqrt(a * a + b * b);
        return {a * inv, b * inv};
    }
    return {1.0, 0.0};
}

std::pair<double, double> GeometryMap::y_face_normal(double csi, double eta) const
{
    switch (kind_)
    {
        case FRSDG_GEOM_WALL_PROFILE:
        {
            const double dh = wall(prm_[0] + Lx_ * csi).second;
            const double a = -dh * Lx_ * (1.0 - eta), b = Lx_;
            const double inv = 1.0 / std::sqrt(a * a + b * b);
            return {a * inv, b * inv};
        }
        case FRSDG_GEOM_SINE_WARP:
        {
            const GeomJacobian g = jacobian(csi, eta);
            const double       a = -g.dy_dcsi, b = g.dx_dcsi;
            const double       inv = 1.0 / std::sqrt(a * a + b * b);
            return {a * inv, b * inv};
        }
        default: return {0.0, 1.0};
    }
}

} // namespace frsdg
