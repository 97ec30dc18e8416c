// jacobi.cu -- element block-Jacobi preconditioner of the implicit path.
//
// The reference preconditions its matrix-free Newton-Krylov solve with a
// finite-difference Jacobian assembled by DMDA colouring (MatFDColoringApply,
// include/petsc_solver_impl.hpp:72-95 and 223-248).  Here the preconditioner is
// the element-diagonal part of the same Jacobian, J_ee = sigma dM/dU + dR/dU,
// from the coloured complex-step launch of the residual kernel (MODE_JAC), each
// block inverted once per Newton step in FP64 and kept in FP32:
//   block_inverse_kernel  Gauss-Jordan elimination with partial pivoting of one
//                         column-major ND x ND block per CTA, in shared memory;
//   block_apply_kernel    z_e = inv(J_ee) r_e, one CTA per element, FP64 sums.
#include "jacobi.hpp"

namespace frsdg
{

namespace
{

constexpr int kInvThreads = 256;

// In-place inverse of the column-major n x n block A (a_ij at A[j n + i]) by
// Gauss-Jordan elimination with row pivoting; the row exchanges are undone as
// column exchanges at the end.  A zero pivot counts one singular block.
__global__ void __launch_bounds__(kInvThreads) block_inverse_kernel(const double* __restrict__ blocks, int64_t stride,
                                                                    float* __restrict__ inv, int n,
                                                                    unsigned long long* singular)
{
    extern __shared__ double sA[];  // n * n doubles, n doubles of column k, n ints of pivot rows
    double* fcol = sA + n * n;
    int* perm = reinterpret_cast<int*>(sA + n * n + n);
    __shared__ int s_piv;
    __shared__ double s_red_v[kInvThreads / 32];
    __shared__ int s_red_i[kInvThreads / 32];
    const int64_t base = int64_t(blockIdx.x) * n * n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int q = tid; q < n * n; q += kInvThreads) sA[q] = blocks[int64_t(blockIdx.x) * stride + q];
    __syncthreads();
    bool bad = false;
    for (int k = 0; k < n; ++k)
    {
        // pivot: largest |a_ik|, i >= k (lowest index among equals)
        double best = -1.0;
        int bi = k;
        for (int i = k + tid; i < n; i += kInvThreads)
        {
            const double v = fabs(sA[k * n + i]);
            if (v > best) { best = v; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1)
        {
            const double ov = __shfl_down_sync(0xffffffffu, best, o);
            const int oi = __shfl_down_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (lane == 0) { s_red_v[warp] = best; s_red_i[warp] = bi; }
        __syncthreads();
        if (tid == 0)
        {
            double b = s_red_v[0];
            int i0 = s_red_i[0];
            for (int w = 1; w < kInvThreads / 32; ++w)
                if (s_red_v[w] > b || (s_red_v[w] == b && s_red_i[w] < i0)) { b = s_red_v[w]; i0 = s_red_i[w]; }
            s_piv = b > 0.0 ? i0 : -1;
            perm[k] = b > 0.0 ? i0 : k;
        }
        __syncthreads();
        const int pr = s_piv;
        if (pr < 0)
        {
            bad = true;  // leave the block as it is; the caller reports the failure
            break;
        }
        // exchange rows k and pr
        if (pr != k)
            for (int j = tid; j < n; j += kInvThreads)
            {
                const double t = sA[j * n + k];
                sA[j * n + k] = sA[j * n + pr];
                sA[j * n + pr] = t;
            }
        __syncthreads();
        const double rp = 1.0 / sA[k * n + k];
        // scale row k (its pivot entry becomes 1/a_kk); keep column k's multipliers
        for (int j = tid; j < n; j += kInvThreads) sA[j * n + k] = (j == k ? 1.0 : sA[j * n + k]) * rp;
        for (int i = tid; i < n; i += kInvThreads) fcol[i] = sA[k * n + i];
        __syncthreads();
        // eliminate column k from every other row: a_ij -= a_ik a_kj (a_ik -> -a_ik / a_kk)
        for (int q = tid; q < n * n; q += kInvThreads)
        {
            const int j = q / n, i = q - j * n;
            if (i == k) continue;
            sA[q] = (j == k ? 0.0 : sA[q]) - fcol[i] * sA[j * n + k];
        }
        __syncthreads();
    }
    if (bad)
    {
        if (tid == 0 && singular) atomicAdd(singular, 1ull);
        return;
    }
    // undo the row exchanges as column exchanges, last first
    for (int k = n - 1; k >= 0; --k)
    {
        const int pr = perm[k];
        if (pr != k)
            for (int i = tid; i < n; i += kInvThreads)
            {
                const double t = sA[k * n + i];
                sA[k * n + i] = sA[pr * n + i];
                sA[pr * n + i] = t;
            }
        __syncthreads();
    }
    for (int q = tid; q < n * n; q += kInvThreads) inv[base + q] = static_cast<float>(sA[q]);
}

// Row i of B v for an n x n FP32 block stored column-major (entry (i, j) at j n + i):
// four partial sums, so four loads and four FMA chains are in flight per thread.
__device__ __forceinline__ double block_row(const float* __restrict__ B, const double* v, int n, int i)
{
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int j = 0;
    for (; j + 3 < n; j += 4)
    {
        a0 = fma(static_cast<double>(__ldg(B + int64_t(j) * n + i)), v[j], a0);
        a1 = fma(static_cast<double>(__ldg(B + int64_t(j + 1) * n + i)), v[j + 1], a1);
        a2 = fma(static_cast<double>(__ldg(B + int64_t(j + 2) * n + i)), v[j + 2], a2);
        a3 = fma(static_cast<double>(__ldg(B + int64_t(j + 3) * n + i)), v[j + 3], a3);
    }
    for (; j < n; ++j) a0 = fma(static_cast<double>(__ldg(B + int64_t(j) * n + i)), v[j], a0);
    return (a0 + a1) + (a2 + a3);
}

// z_e = inv_e r_e for every element e: one CTA per element, thread i owns row i.
__global__ void block_apply_kernel(const float* __restrict__ inv, const double* __restrict__ r, double* __restrict__ z, int n)
{
    extern __shared__ double sr[];
    const int64_t e = blockIdx.x;
    for (int j = threadIdx.x; j < n; j += blockDim.x) sr[j] = r[e * n + j];
    __syncthreads();
    const float* B = inv + e * int64_t(n) * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) z[e * n + i] = block_row(B, sr, n, i);
}

// Off-diagonal blocks (slots 1-4 of each element's five) to FP32, packed four per element.
__global__ void offdiag_to_f32_kernel(const double* __restrict__ blocks5, float* __restrict__ off, int64_t nel, int nn)
{
    const int64_t total = nel * 4 * nn;
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < total; q += int64_t(gridDim.x) * blockDim.x)
    {
        const int64_t e = q / (4 * nn), r = q - e * 4 * nn;  // r: (slot - 1) * nn + entry
        off[q] = static_cast<float>(blocks5[e * 5 * nn + nn + r]);
    }
}

// One colour half-sweep of the red-black block Gauss-Seidel preconditioner.  A CTA takes
// epc elements of the active colour (the k-th of a colour sits in row k / ceil(Nx/2)),
// n/4 threads per element; each thread owns four rows and reads the column-major FP32
// blocks with 16-byte loads (n is a multiple of 4), four columns in flight (the 256 x 64
// element bump, n = 64: 0.297 ms per sweep, 4.85 TB/s, against 0.309 ms with one row per
// thread and one CTA per element of either colour).  Neighbour slots: 0 right,
// 1 top, 2 bottom, 3 left (the off-diagonal blocks of slots 1-4).
//   phase 0 (red):   z_e = inv_e r_e
//   phase 1 (black): z_e = inv_e (r_e - sum_s J_es z_s)
//   phase 2 (red):   z_e = z_e - inv_e (sum_s J_es z_s)
constexpr int kGsThreads = 128;

__global__ void __launch_bounds__(kGsThreads) block_gs_kernel(const float* __restrict__ inv,
                                                              const float* __restrict__ off,
                                                              const double* __restrict__ r, double* __restrict__ z,
                                                              int n, int Nx, int Ny, int phase, int epc)
{
    extern __shared__ double sv[];  // per element slot: t[n], then the neighbour values nbv[4 n]
    const int tpe = n / 4;
    const int slot = threadIdx.x / tpe, li = threadIdx.x - slot * tpe;
    const int colour = phase == 1 ? 1 : 0;
    const int half = (Nx + 1) / 2;
    const int64_t k = int64_t(blockIdx.x) * epc + slot;
    const int gj = int(k / half), gi = 2 * int(k % half) + ((int(k / half) + colour) & 1);
    const bool active = slot < epc && gj < Ny && gi < Nx;
    const int64_t e = int64_t(gj) * Nx + gi;
    double* t = sv + size_t(slot < epc ? slot : 0) * 5 * n;
    double* nbv = t + n;
    const int64_t nbi[4] = {gi + 1 < Nx ? e + 1 : -1, gj + 1 < Ny ? e + Nx : -1, gj > 0 ? e - Nx : -1,
                            gi > 0 ? e - 1 : -1};
    const int64_t nn = int64_t(n) * n;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (phase > 0)
    {
        if (active)
            for (int q = li; q < 4 * n; q += tpe)
            {
                const int sl = q / n, j = q - sl * n;
                nbv[q] = nbi[sl] >= 0 ? z[nbi[sl] * n + j] : 0.0;
            }
        __syncthreads();
        if (active)
        {
            for (int sl = 0; sl < 4; ++sl)
            {
                if (nbi[sl] < 0) continue;
                const float4* B = reinterpret_cast<const float4*>(off + (e * 4 + sl) * nn) + li;  // column j at + j tpe
                const double* v = nbv + sl * n;
#pragma unroll 4
                for (int j = 0; j < n; ++j)
                {
                    const float4 b = __ldg(B + int64_t(j) * tpe);
                    const double vj = v[j];
                    acc[0] = fma(static_cast<double>(b.x), vj, acc[0]);
                    acc[1] = fma(static_cast<double>(b.y), vj, acc[1]);
                    acc[2] = fma(static_cast<double>(b.z), vj, acc[2]);
                    acc[3] = fma(static_cast<double>(b.w), vj, acc[3]);
                }
            }
        }
    }
    if (active)
    {
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            const int i = 4 * li + q;
            t[i] = phase == 0 ? r[e * n + i] : phase == 1 ? r[e * n + i] - acc[q] : acc[q];
        }
    }
    __syncthreads();
    if (!active) return;
    const float4* Bi = reinterpret_cast<const float4*>(inv + e * nn) + li;
    double o[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 4
    for (int j = 0; j < n; ++j)
    {
        const float4 b = __ldg(Bi + int64_t(j) * tpe);
        const double tj = t[j];
        o[0] = fma(static_cast<double>(b.x), tj, o[0]);
        o[1] = fma(static_cast<double>(b.y), tj, o[1]);
        o[2] = fma(static_cast<double>(b.z), tj, o[2]);
        o[3] = fma(static_cast<double>(b.w), tj, o[3]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        const int i = 4 * li + q;
        z[e * n + i] = phase == 2 ? z[e * n + i] - o[q] : o[q];
    }
}

} // namespace

size_t block_inverse_smem(int n) { return size_t(n) * (n + 1) * sizeof(double) + size_t(n) * sizeof(int); }

cudaError_t launch_block_inverse(const double* blocks, int64_t stride, float* inv, int n, int64_t n_blocks,
                                 unsigned long long* singular, cudaStream_t s)
{
    const size_t smem = block_inverse_smem(n);
    cudaError_t e = cudaFuncSetAttribute(block_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    block_inverse_kernel<<<unsigned(n_blocks), kInvThreads, smem, s>>>(blocks, stride, inv, n, singular);
    return cudaGetLastError();
}

cudaError_t launch_offdiag_to_f32(const double* blocks5, float* off, int n, int64_t nel, cudaStream_t s)
{
    offdiag_to_f32_kernel<<<1184, 256, 0, s>>>(blocks5, off, nel, n * n);
    return cudaGetLastError();
}

cudaError_t launch_block_gs(const float* inv, const float* off, const double* r, double* z, int n, int Nx, int Ny,
                            cudaStream_t s)
{
    if (n % 4 != 0 || n / 4 > kGsThreads) return cudaErrorInvalidValue;
    const int tpe = n / 4, epc = kGsThreads / tpe;
    const size_t smem = size_t(epc) * 5 * n * sizeof(double);  // at most 20.5 KB for n <= 144
    const int64_t slots = int64_t((Nx + 1) / 2) * Ny;            // element slots of one colour
    const unsigned grid = unsigned((slots + epc - 1) / epc);
    cudaError_t e;
    for (int phase = 0; phase < 3; ++phase)
    {
        block_gs_kernel<<<grid, kGsThreads, smem, s>>>(inv, off, r, z, n, Nx, Ny, phase, epc);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_block_apply(const float* inv, const double* r, double* z, int n, int64_t n_blocks, cudaStream_t s)
{
    const int threads = n <= 64 ? 64 : n <= 128 ? 128 : 160;
    block_apply_kernel<<<unsigned(n_blocks), threads, size_t(n) * sizeof(double), s>>>(inv, r, z, n);
    return cudaGetLastError();
}

} // namespace frsdg
