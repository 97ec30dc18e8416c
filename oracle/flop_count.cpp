// flop_count.cpp -- floating-point operation count of the oracle's residual.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY: instantiates the oracle's residual (the
// restatement of the reference's algorithm) with a scalar type that counts its own
// arithmetic, so that the residual kernel's compute bound can be quoted in operations
// of the reference algorithm.  oracle/count_flops.py runs it and writes the figure to
// profiles/; nothing in fr_sdg_b200/ links it.
//
// Counted: additions and subtractions, multiplications, divisions and square roots
// are one operation each (no fused multiply-add credit); exp, log and pow are tallied
// separately; comparisons, min/max and absolute values are not counted.
#include <algorithm>
#include <cmath>
#include <cstdint>

namespace frsdg_count
{
struct Tally
{
    uint64_t add = 0, mul = 0, div = 0, sqrt = 0, other = 0;
};
inline Tally g_tally;

struct Counted
{
    double v;
    constexpr Counted() : v(0.0) {}
    constexpr Counted(double x) : v(x) {}
    explicit operator double() const { return v; }
    Counted& operator+=(const Counted& o) { ++g_tally.add; v += o.v; return *this; }
    Counted& operator-=(const Counted& o) { ++g_tally.add; v -= o.v; return *this; }
    Counted& operator*=(const Counted& o) { ++g_tally.mul; v *= o.v; return *this; }
    Counted& operator/=(const Counted& o) { ++g_tally.div; v /= o.v; return *this; }
};
inline Counted operator+(Counted a, Counted b) { ++g_tally.add; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++g_tally.add; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { ++g_tally.mul; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++g_tally.div; return Counted(a.v / b.v); }
inline Counted operator+(double a, Counted b) { return Counted(a) + b; }
inline Counted operator-(double a, Counted b) { return Counted(a) - b; }
inline Counted operator*(double a, Counted b) { return Counted(a) * b; }
inline Counted operator/(double a, Counted b) { return Counted(a) / b; }
inline Counted operator+(Counted a, double b) { return a + Counted(b); }
inline Counted operator-(Counted a, double b) { return a - Counted(b); }
inline Counted operator*(Counted a, double b) { return a * Counted(b); }
inline Counted operator/(Counted a, double b) { return a / Counted(b); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline Counted operator+(Counted a) { return a; }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { return a.v != b.v; }
inline bool operator<(Counted a, double b) { return a.v < b; }
inline bool operator>(Counted a, double b) { return a.v > b; }
inline bool operator<=(Counted a, double b) { return a.v <= b; }
inline bool operator>=(Counted a, double b) { return a.v >= b; }
inline bool operator<(double a, Counted b) { return a < b.v; }
inline bool operator>(double a, Counted b) { return a > b.v; }

// the oracle's scalar helpers, found by argument-dependent lookup
inline double re(const Counted& v) { return v.v; }
inline double branch_real(const Counted& v) { return v.v; }
inline Counted wrap_positive(Counted rho) { return Counted(std::max(std::numeric_limits<double>::min(), rho.v)); }
} // namespace frsdg_count

// The oracle calls the standard math functions by their qualified names; these
// overloads make them count for the counting scalar (measurement build only).
namespace std
{
inline frsdg_count::Counted sqrt(frsdg_count::Counted x)
{
    ++frsdg_count::g_tally.sqrt;
    return frsdg_count::Counted(std::sqrt(x.v));
}
inline frsdg_count::Counted exp(frsdg_count::Counted x)
{
    ++frsdg_count::g_tally.other;
    return frsdg_count::Counted(std::exp(x.v));
}
inline frsdg_count::Counted log(frsdg_count::Counted x)
{
    ++frsdg_count::g_tally.other;
    return frsdg_count::Counted(std::log(x.v));
}
inline frsdg_count::Counted pow(frsdg_count::Counted x, double y)
{
    ++frsdg_count::g_tally.other;
    return frsdg_count::Counted(std::pow(x.v, y));
}
inline frsdg_count::Counted abs(frsdg_count::Counted x) { return frsdg_count::Counted(std::abs(x.v)); }
inline frsdg_count::Counted fabs(frsdg_count::Counted x) { return frsdg_count::Counted(std::fabs(x.v)); }
inline frsdg_count::Counted max(frsdg_count::Counted a, frsdg_count::Counted b) { return a.v < b.v ? b : a; }
inline frsdg_count::Counted min(frsdg_count::Counted a, frsdg_count::Counted b) { return b.v < a.v ? b : a; }
} // namespace std

#include "frsdg_oracle.hpp"

#include <vector>

using frsdg_count::Counted;

extern "C" {

// Operation counts of one residual evaluation of problem h at (t, U): counts[0..4] =
// additions, multiplications, divisions, square roots, exp/log/pow.  Single-threaded.
int oracle_count_flops(void* h, double t, const double* U, uint64_t* counts)
{
    auto& P = *static_cast<frsdg_oracle::Problem*>(h);
    const int64_t n = P.n_total();
    std::vector<Counted> X(U, U + n), R(n);
    const int threads = P.nthreads;
    P.nthreads = 1;
    frsdg_count::g_tally = {};
    frsdg_oracle::residual(P, t, X.data(), R.data());
    P.nthreads = threads;
    const auto& g = frsdg_count::g_tally;
    counts[0] = g.add;
    counts[1] = g.mul;
    counts[2] = g.div;
    counts[3] = g.sqrt;
    counts[4] = g.other;
    return 0;
}

} // extern "C"
