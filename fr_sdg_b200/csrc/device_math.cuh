// device_math.cuh -- scalar types of the residual kernels.
//
// The residual is templated on its scalar S:
//   double  the FP64 residual (rhs_func / fun_implicit),
//   cplx    complex FP64 for the complex-step JVP (matmult of the reference),
//   float   the FP32 residual of the mixed-precision form.
// cplx follows std::complex<double> semantics for finite values: principal-branch
// sqrt, Smith's division (R. L. Smith, "Algorithm 116: Complex division",
// CACM 5(8), 1962) and the textbook product.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace frsdg
{

struct __align__(16) cplx
{
    double re, im;
    __host__ __device__ constexpr cplx() : re(0.0), im(0.0) {}
    __host__ __device__ constexpr cplx(double r) : re(r), im(0.0) {}
    __host__ __device__ constexpr cplx(double r, double i) : re(r), im(i) {}
};

__device__ __forceinline__ cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx operator-(cplx a) { return {-a.re, -a.im}; }
__device__ __forceinline__ cplx operator*(cplx a, cplx b)
{
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx operator*(double s, cplx a) { return {s * a.re, s * a.im}; }
__device__ __forceinline__ cplx operator*(cplx a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ cplx operator+(cplx a, double s) { return {a.re + s, a.im}; }
__device__ __forceinline__ cplx operator+(double s, cplx a) { return {s + a.re, a.im}; }
__device__ __forceinline__ cplx operator-(cplx a, double s) { return {a.re - s, a.im}; }
__device__ __forceinline__ cplx operator-(double s, cplx a) { return {s - a.re, -a.im}; }
__device__ __forceinline__ cplx operator/(cplx a, cplx b)
{
    // Smith's algorithm.
    if (fabs(b.re) >= fabs(b.im))
    {
        const double r   = b.im / b.re;
        const double den = b.re + b.im * r;
        return {(a.re + a.im * r) / den, (a.im - a.re * r) / den};
    }
    const double r   = b.re / b.im;
    const double den = b.re * r + b.im;
    return {(a.re * r + a.im) / den, (a.im * r - a.re) / den};
}
__device__ __forceinline__ cplx operator/(cplx a, double s) { return {a.re / s, a.im / s}; }
__device__ __forceinline__ cplx operator/(double s, cplx b) { return cplx(s) / b; }
__device__ __forceinline__ cplx& operator+=(cplx& a, cplx b) { a = a + b; return a; }
__device__ __forceinline__ cplx& operator-=(cplx& a, cplx b) { a = a - b; return a; }

// ---- generic scalar functions -------------------------------------------
// Exponent tests of the fast paths: |x| (or x, positive) in [2^-122, 2^123), well
// inside the range of normal floats, by the biased exponent with integer operations
// (zero, subnormals, inf and NaN fail them; so do negatives in the signed test).
__device__ __forceinline__ bool in_float_range(double x)
{
    const unsigned e = (static_cast<unsigned>(__double2hiint(x)) >> 20) & 0x7ffu;
    return e - (1023u - 122u) < 245u;
}
__device__ __forceinline__ bool positive_in_float_range(double x)
{
    return (static_cast<unsigned>(__double2hiint(x)) >> 20) - (1023u - 122u) < 245u;
}
// The IEEE operations for inputs outside that range, out of line so that the fast
// path does not carry them (measured on the 1024^2 p = 5 residual: 1.400 ms with the
// IEEE operations inline behind the branch, 1.366 ms out of line; selects instead of
// the branch, with exact power-of-two scaling of the outside inputs, 1.385 ms).
static __device__ __noinline__ double ieee_sqrt(double x) { return sqrt(x); }
static __device__ __noinline__ double ieee_rcp(double x) { return 1.0 / x; }

// sqrt in FP64: single-precision reciprocal square root seed, two Newton steps
// y <- y (3 - x y^2) / 2 for 1/sqrt(x), then s = x y with one Heron correction
// s <- s + (x - s^2) y / 2 (Karp and Markstein, ACM TOMS 23(4), 1997).  Inputs
// outside [2^-122, 2^123) (zero, negatives, subnormals, inf, NaN) take the IEEE
// square root.
__device__ __forceinline__ double sqrt_fast(double x)
{
    double y = static_cast<double>(rsqrtf(static_cast<float>(x)));
    y = y * fma(-0.5 * x, y * y, 1.5);
    y = y * fma(-0.5 * x, y * y, 1.5);
    const double s = x * y;
    return fma(fma(-s, s, x), 0.5 * y, s);
}
__device__ __forceinline__ double s_sqrt(double x)
{
    if (!positive_in_float_range(x)) return ieee_sqrt(x);
    return sqrt_fast(x);
}
__device__ __forceinline__ float s_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ cplx s_sqrt(cplx z)
{
    // principal branch, as C99 csqrt
    if (z.re == 0.0 && z.im == 0.0) return {0.0, z.im};
    const double t = sqrt(0.5 * (fabs(z.re) + hypot(z.re, z.im)));
    if (z.re >= 0.0) return {t, z.im / (2.0 * t)};
    return {fabs(z.im) / (2.0 * t), copysign(t, z.im)};
}
__device__ __forceinline__ double s_log(double x) { return log(x); }
__device__ __forceinline__ cplx s_log(cplx z) { return {log(hypot(z.re, z.im)), atan2(z.im, z.re)}; }
__device__ __forceinline__ double s_exp(double x) { return exp(x); }
__device__ __forceinline__ float s_exp(float x) { return expf(x); }
__device__ __forceinline__ cplx s_exp(cplx z)
{
    const double m = exp(z.re);
    double       s, c;
    sincos(z.im, &s, &c);
    return {m * c, m * s};
}

// reciprocal: 1/x.  In FP64 the hardware's approximate single-precision reciprocal
// (rcp.approx, at most one FP32 ulp off by the PTX ISA) seeds two Newton-Raphson
// steps r <- r + r (1 - x r) (error below 2^-90 before rounding, so within 2 ulp of the
// correctly rounded value; Markstein, IBM J. Res. Dev. 34(1), 1990).  Inputs outside
// [2^-122, 2^123) in magnitude take the IEEE division.  (Against a correctly rounded FP32
// seed: the same results on the 1024^2 p = 5 residual, 2.4 % less time.)
__device__ __forceinline__ double rcp_fast(double x)
{
    float sf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(sf) : "f"(static_cast<float>(x)));
    double r = static_cast<double>(sf);
    r = fma(r, fma(-x, r, 1.0), r);
    r = fma(r, fma(-x, r, 1.0), r);
    return r;
}
__device__ __forceinline__ double s_rcp(double x)
{
    if (!in_float_range(x)) return ieee_rcp(x);
    return rcp_fast(x);
}
__device__ __forceinline__ float s_rcp(float x) { return 1.0f / x; }
__device__ __forceinline__ cplx s_rcp(cplx z) { return cplx(1.0) / z; }

// Math policies of the physics helpers.  MathChecked: s_rcp and s_sqrt.  MathDeferred:
// in FP64 the fast paths alone, each recording in `bad` whether its input lay outside
// their range; a computation that ends with bad == 0 equals its MathChecked twin bit for
// bit, and one that does not is redone with MathChecked.  A node or face computation
// then carries one branch instead of one per reciprocal and square root (measured on the
// 1024^2 p = 5 residual: the per-operation branches cost 8 %).  Other scalars take the
// checked functions (bad stays 0).
struct MathChecked
{
    template <class S> __device__ __forceinline__ S rcp(S x) const { return s_rcp(x); }
    template <class S> __device__ __forceinline__ S sqrt(S x) const { return s_sqrt(x); }
};
struct MathDeferred
{
    unsigned& bad;
    __device__ __forceinline__ double rcp(double x) const
    {
        bad |= in_float_range(x) ? 0u : 1u;
        return rcp_fast(x);
    }
    __device__ __forceinline__ double sqrt(double x) const
    {
        bad |= positive_in_float_range(x) ? 0u : 1u;
        return sqrt_fast(x);
    }
    // FP32: the hardware approximations with one Newton step (within 2 ulp of the IEEE
    // results) for normal inputs whose results stay normal; zero, subnormals, huge values,
    // inf and NaN (exponent tests as above) take the redo with the IEEE operations
    __device__ __forceinline__ float rcp(float x) const
    {
        const unsigned e = (__float_as_uint(x) >> 23) & 0xffu;
        bad |= e - 2u < 250u ? 0u : 1u;  // 2^-125 <= |x| < 2^125
        float r;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
        return fmaf(r, fmaf(-x, r, 1.0f), r);
    }
    __device__ __forceinline__ float sqrt(float x) const
    {
        bad |= (__float_as_uint(x) >> 23) - 2u < 250u ? 0u : 1u;  // positive, 2^-125 <= x < 2^125
        float y;
        asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
        const float s = x * y;
        return fmaf(fmaf(-s, s, x), 0.5f * y, s);
    }
    __device__ __forceinline__ cplx rcp(cplx x) const { return s_rcp(x); }
    __device__ __forceinline__ cplx sqrt(cplx x) const { return s_sqrt(x); }
};

// real part, and the value the HLLC branch tests (riemann_solver.hpp:149-155:
// Re + Im for complex, the value itself for real scalars).
__device__ __forceinline__ double s_re(double x) { return x; }
__device__ __forceinline__ double s_re(float x) { return x; }
__device__ __forceinline__ double s_re(cplx z) { return z.re; }
__device__ __forceinline__ double s_im(cplx z) { return z.im; }
__device__ __forceinline__ double s_branch(double x) { return x; }
__device__ __forceinline__ double s_branch(float x) { return x; }
__device__ __forceinline__ double s_branch(cplx z) { return z.re + z.im; }

// wrap_positive (macro_and_libc.hpp:117-138): max(DBL_MIN, rho); for complex, the
// real part decides and a clamped value loses its imaginary part.
__device__ __forceinline__ double s_wrap_positive(double r)
{
    const double floor = 2.2250738585072014e-308; // DBL_MIN
    return fmax(floor, r);
}
__device__ __forceinline__ float s_wrap_positive(float r)
{
    const float floor = 1.17549435e-38f; // FLT_MIN
    return fmaxf(floor, r);
}
__device__ __forceinline__ cplx s_wrap_positive(cplx r)
{
    const double floor = 2.2250738585072014e-308;
    return (r.re < floor) ? cplx(floor, 0.0) : r;
}

template <class S> __device__ __forceinline__ S s_select(bool c, S a, S b) { return c ? a : b; }

// The health word's test of a density: positive and finite.  Positive finite doubles
// (subnormals included) are exactly the bit patterns 1 .. 0x7fefffffffffffff.
__device__ __forceinline__ bool density_ok(double rho)
{
    return static_cast<unsigned long long>(__double_as_longlong(rho)) - 1ull < 0x7fefffffffffffffull;
}

template <class S> struct scalar_traits;
template <> struct scalar_traits<double>
{
    using real = double;
    static constexpr int words = 1;
};
template <> struct scalar_traits<float>
{
    using real = float;
    static constexpr int words = 1;
};
template <> struct scalar_traits<cplx>
{
    using real = double;
    static constexpr int words = 2;
};

} // namespace frsdg
