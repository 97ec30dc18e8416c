// krylov.cu -- the Arnoldi step of restarted GMRES on the device.
//
// The implicit path solves every Newton system with right-preconditioned GMRES(m)
// (Saad, "Iterative Methods for Sparse Linear Systems", 2nd ed., algorithm 6.9 with
// Givens rotations, section 6.5.3); the reference hands this to PETSc's KSPGMRES
// (petsc_solver_impl.hpp:549-612).  One Arnoldi step here is, with no host round trip:
//   orthogonalisation  h = V_j^T w, w <- w - V_j h by classical Gram-Schmidt, repeated
//                      once when the first pass shrinks ||w|| below 1/sqrt(2) of its
//                      value (the criterion of Daniel, Gragg, Kaufman and Stewart,
//                      Math. Comp. 30, 1976); hn = ||w||;
//   Givens update      the new Hessenberg column takes the previous rotations, a new
//                      rotation zeroes its subdiagonal, and the residual vector g of the
//                      least-squares problem turns with it; 1/hn (0 at breakdown) scales
//                      the next basis vector;
//   back substitution  y = R^-1 g at the end of a cycle (R the rotated Hessenberg).
// Reductions are two-stage (per-block partial sums in a fixed order, then one block per
// sum), so repeated solves give identical bits.  Every kernel reads its sizes from the
// arguments; scratch is the caller's `work` array (frsdg_gmres_work_doubles).
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/frsdg.h"

namespace frsdg
{
int report(int code, const char* msg);
int report_cuda(cudaError_t e, const char* what);

constexpr int kKryThreads = 256;
constexpr int kKryPerThread = 8;                            // vector entries per thread
constexpr int kKryChunk = kKryThreads * kKryPerThread;      // entries per block
constexpr int kKryMaxBasis = 256;                           // Arnoldi vectors per cycle

static int64_t kry_blocks(int64_t n) { return (n + kKryChunk - 1) / kKryChunk; }

// work layout (doubles): part[(kKryMaxBasis + 1) * B] | h1[kKryMaxBasis] | h2[kKryMaxBasis] |
// scalars[4] (0: ||w||^2 before, 1: ||w||^2 after the first pass, 2: reorthogonalise
// flag as 0/1, 3: ||w||^2 after the second pass)
struct KryWork
{
    double* part;
    double* h1;
    double* h2;
    double* sc;
};

static KryWork kry_work(double* work, int64_t B)
{
    KryWork k;
    k.part = work;
    k.h1 = work + (kKryMaxBasis + 1) * B;
    k.h2 = k.h1 + kKryMaxBasis;
    k.sc = k.h2 + kKryMaxBasis;
    return k;
}

__device__ __forceinline__ double block_sum(double v, double* red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();  // red is reused by consecutive calls
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < kKryThreads / 32; ++q) s += red[q];
    return s;  // valid on thread 0
}

// Per-block partial dot products of w with V[0..nv) (and w.w when with_norm) into
// part[i * B + block]; skipped unless the flag (when given) is set.
__global__ void __launch_bounds__(kKryThreads) kry_dot_kernel(const double* V, int64_t ldv, int nv, const double* w,
                                                               int64_t n, double* part, int with_norm,
                                                               const double* flag)
{
    if (flag && *flag == 0.0) return;
    __shared__ double red[kKryThreads / 32];
    const int64_t base = int64_t(blockIdx.x) * kKryChunk + threadIdx.x;
    const int64_t B = gridDim.x;
    double wv[kKryPerThread];
#pragma unroll
    for (int k = 0; k < kKryPerThread; ++k)
    {
        const int64_t e = base + int64_t(k) * kKryThreads;
        wv[k] = e < n ? w[e] : 0.0;
    }
    if (with_norm)
    {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < kKryPerThread; ++k) s = fma(wv[k], wv[k], s);
        s = block_sum(s, red);
        if (threadIdx.x == 0) part[int64_t(nv) * B + blockIdx.x] = s;
    }
    for (int i = 0; i < nv; ++i)
    {
        const double* v = V + int64_t(i) * ldv;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < kKryPerThread; ++k)
        {
            const int64_t e = base + int64_t(k) * kKryThreads;
            if (e < n) s = fma(__ldg(v + e), wv[k], s);
        }
        s = block_sum(s, red);
        if (threadIdx.x == 0) part[int64_t(i) * B + blockIdx.x] = s;
    }
}

// w <- w - sum_i h[i] V[i]; per-block partial ||w||^2 into part[nv * B + block].
__global__ void __launch_bounds__(kKryThreads) kry_update_kernel(const double* V, int64_t ldv, int nv, double* w,
                                                                  int64_t n, const double* h, double* part,
                                                                  const double* flag)
{
    if (flag && *flag == 0.0) return;
    __shared__ double red[kKryThreads / 32];
    __shared__ double sh[kKryMaxBasis];
    for (int i = threadIdx.x; i < nv; i += kKryThreads) sh[i] = h[i];
    __syncthreads();
    const int64_t base = int64_t(blockIdx.x) * kKryChunk + threadIdx.x;
    const int64_t B = gridDim.x;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kKryPerThread; ++k)
    {
        const int64_t e = base + int64_t(k) * kKryThreads;
        if (e < n)
        {
            double acc = w[e];
            for (int i = 0; i < nv; ++i) acc = fma(-sh[i], __ldg(V + int64_t(i) * ldv + e), acc);
            w[e] = acc;
            s = fma(acc, acc, s);
        }
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) part[int64_t(nv) * B + blockIdx.x] = s;
}

// One block per sum: out[i] = sum_b part[i * B + b] for i in [0, count), in a fixed order.
__global__ void __launch_bounds__(kKryThreads) kry_reduce_kernel(const double* part, int64_t B, double* out,
                                                                  const double* flag)
{
    if (flag && *flag == 0.0) return;
    __shared__ double red[kKryThreads / 32];
    const double* p = part + int64_t(blockIdx.x) * B;
    double s = 0.0;
    for (int64_t b = threadIdx.x; b < B; b += kKryThreads) s += p[b];
    s = block_sum(s, red);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// After the first pass: reorthogonalise when ||w||^2 fell below half its value.
__global__ void kry_dgks_kernel(double* sc)
{
    sc[2] = sc[1] < 0.5 * sc[0] ? 1.0 : 0.0;
}

// The new Hessenberg column j: H[0..j][j] = h1 + h2 (h2 only after a second pass),
// H[j+1][j] = ||w||; the previous rotations, the new one, the residual vector g, and
// 1/||w|| (0 when w vanished) for the next basis vector.  H is row-major with leading
// dimension ldh.
__global__ void kry_givens_kernel(double* H, int ldh, double* cs, double* sn, double* g, const double* h1,
                                  const double* h2, const double* sc, int j, double* inv_hn)
{
    const bool second = sc[2] != 0.0;
    for (int i = 0; i <= j; ++i) H[int64_t(i) * ldh + j] = second ? h1[i] + h2[i] : h1[i];
    const double nrm2 = second ? sc[3] : sc[1];
    const double hn = sqrt(nrm2 > 0.0 ? nrm2 : 0.0);
    H[int64_t(j + 1) * ldh + j] = hn;
    for (int i = 0; i < j; ++i)
    {
        const double a = H[int64_t(i) * ldh + j], b = H[int64_t(i + 1) * ldh + j];
        H[int64_t(i) * ldh + j] = cs[i] * a + sn[i] * b;
        H[int64_t(i + 1) * ldh + j] = -sn[i] * a + cs[i] * b;
    }
    const double a = H[int64_t(j) * ldh + j], b = H[int64_t(j + 1) * ldh + j];
    const double den = hypot(a, b);
    const double c = den == 0.0 ? 1.0 : a / den, s = den == 0.0 ? 0.0 : b / den;
    cs[j] = c;
    sn[j] = s;
    H[int64_t(j) * ldh + j] = c * a + s * b;
    H[int64_t(j + 1) * ldh + j] = 0.0;
    g[j + 1] = -s * g[j];
    g[j] = c * g[j];
    *inv_hn = hn > 0.0 ? 1.0 / hn : 0.0;
}

// y = R^-1 g over the first k columns; a zero diagonal (columns after a breakdown)
// leaves y at zero there.
__global__ void kry_solve_kernel(const double* H, int ldh, const double* g, int k, double* y)
{
    for (int i = k - 1; i >= 0; --i)
    {
        double s = g[i];
        for (int l = i + 1; l < k; ++l) s -= H[int64_t(i) * ldh + l] * y[l];
        const double d = H[int64_t(i) * ldh + i];
        y[i] = d != 0.0 ? s / d : 0.0;
    }
}

} // namespace frsdg

using namespace frsdg;

extern "C" {

int64_t frsdg_gmres_work_doubles(int64_t n)
{
    if (n <= 0) return 0;
    return (kKryMaxBasis + 1) * kry_blocks(n) + 2 * kKryMaxBasis + 4;
}

int frsdg_gmres_arnoldi(const double* V, int64_t ldv, int32_t j, double* w, int64_t n, double* H, int32_t ldh,
                        double* cs, double* sn, double* g, double* inv_hn, double* work, void* stream)
{
    if (!V || !w || !H || !cs || !sn || !g || !inv_hn || !work || n <= 0 || j < 0 || j + 1 > kKryMaxBasis ||
        ldv < n || ldh < j + 1)
        return report(FRSDG_ERR_ARG, "frsdg_gmres_arnoldi: bad argument (at most 256 basis vectors)");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t B = kry_blocks(n);
    const KryWork k = kry_work(work, B);
    const int nv = j + 1;
    const unsigned grid = unsigned(B);
    // first pass: h1 = V^T w and ||w||^2 (sc[0]); w -= V h1 and ||w||^2 (sc[1])
    kry_dot_kernel<<<grid, kKryThreads, 0, s>>>(V, ldv, nv, w, n, k.part, 1, nullptr);
    kry_reduce_kernel<<<unsigned(nv), kKryThreads, 0, s>>>(k.part, B, k.h1, nullptr);
    kry_reduce_kernel<<<1, kKryThreads, 0, s>>>(k.part + int64_t(nv) * B, B, k.sc, nullptr);
    kry_update_kernel<<<grid, kKryThreads, 0, s>>>(V, ldv, nv, w, n, k.h1, k.part, nullptr);
    kry_reduce_kernel<<<1, kKryThreads, 0, s>>>(k.part + int64_t(nv) * B, B, k.sc + 1, nullptr);
    kry_dgks_kernel<<<1, 1, 0, s>>>(k.sc);
    // second pass when flagged: h2, w -= V h2, ||w||^2 (sc[3])
    kry_dot_kernel<<<grid, kKryThreads, 0, s>>>(V, ldv, nv, w, n, k.part, 0, k.sc + 2);
    kry_reduce_kernel<<<unsigned(nv), kKryThreads, 0, s>>>(k.part, B, k.h2, k.sc + 2);
    kry_update_kernel<<<grid, kKryThreads, 0, s>>>(V, ldv, nv, w, n, k.h2, k.part, k.sc + 2);
    kry_reduce_kernel<<<1, kKryThreads, 0, s>>>(k.part + int64_t(nv) * B, B, k.sc + 3, k.sc + 2);
    kry_givens_kernel<<<1, 1, 0, s>>>(H, ldh, cs, sn, g, k.h1, k.h2, k.sc, j, inv_hn);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FRSDG_OK : report_cuda(e, "frsdg_gmres_arnoldi launch");
}

int frsdg_gmres_solve(const double* H, int32_t ldh, const double* g, int32_t k, double* y, void* stream)
{
    if (!H || !g || !y || k < 0 || ldh < k) return report(FRSDG_ERR_ARG, "frsdg_gmres_solve: bad argument");
    if (k == 0) return FRSDG_OK;
    kry_solve_kernel<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(H, ldh, g, k, y);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? FRSDG_OK : report_cuda(e, "frsdg_gmres_solve launch");
}

} // extern "C"
