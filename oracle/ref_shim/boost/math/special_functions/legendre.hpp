// Stand-in for boost/math/special_functions/legendre.hpp: the two functions the
// reference's operators call, written from the Legendre recurrences (test
// infrastructure of oracle/_ref).
//   P_0 = 1, P_1 = x, (n+1) P_{n+1} = (2n+1) x P_n - n P_{n-1}   (Bonnet)
//   P'_{n+1} = P'_{n-1} + (2n+1) P_n                              (derivative identity)
// with P_{-n-1} = P_n for negative degrees, as Boost.Math defines them.
#pragma once

namespace boost::math
{
template <class T> T legendre_p(int l, T x)
{
    if (l < 0) l = -l - 1;
    if (l == 0) return T(1);
    T p0 = T(1), p1 = x;
    for (int n = 1; n < l; ++n)
    {
        const T p2 = (T(2 * n + 1) * x * p1 - T(n) * p0) / T(n + 1);
        p0 = p1;
        p1 = p2;
    }
    return p1;
}

template <class T> T legendre_p_prime(int l, T x)
{
    if (l < 0) l = -l - 1;
    if (l == 0) return T(0);
    // d_{n+1} = d_{n-1} + (2n+1) P_n, starting from d_0 = 0, d_1 = 1
    T d_prev = T(0), d_curr = T(1);  // P'_0, P'_1
    T p0 = T(1), p1 = x;             // P_0, P_1
    for (int n = 1; n < l; ++n)
    {
        const T d_next = d_prev + T(2 * n + 1) * p1;
        const T p2     = (T(2 * n + 1) * x * p1 - T(n) * p0) / T(n + 1);
        d_prev = d_curr;
        d_curr = d_next;
        p0 = p1;
        p1 = p2;
    }
    return d_curr;
}
} // namespace boost::math
