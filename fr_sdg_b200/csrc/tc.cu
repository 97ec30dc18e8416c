// tc.cu -- the split-precision tensor-core line contraction (tc_sm100.cuh) on its own,
// for validation: out[l][k] = sum_m D[k][m] v[l][m] for L lines of n values.
//
// One CTA of 192 threads takes 192 lines in two 128-line MMA tiles (the second tile's
// last 64 rows are zero), the same thread/lane arrangement the FP32 residual uses:
// warps 0-3 read tile 0 from TMEM lanes 0-127, warps 4-5 read tile 1 from lanes 0-63.
#include <cstdint>
#include <cuda_runtime.h>

#include "frsdg_internal.hpp"
#include "tc_sm100.cuh"

namespace frsdg
{

constexpr int kTcLinesCta = 192;

template <int N>
__global__ void __launch_bounds__(kTcLinesCta) tc_lines_kernel(const float* v, const double* D, float* out, int64_t L,
                                                               int* err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    unsigned char* a_hi = smem;
    unsigned char* a_lo = smem + 2 * tc::kTileBytes;
    unsigned char* b_hi = smem + 4 * tc::kTileBytes;
    unsigned char* b_lo = b_hi + tc::kBBytes;
    const int t = threadIdx.x;
    if (t < 32) tc::tmem_alloc(&tmem_base, 32);
    if (t == 32) tc::mbar_init(&bar, 1);

    const int64_t line = int64_t(blockIdx.x) * kTcLinesCta + t;
    float vals[N];
#pragma unroll
    for (int k = 0; k < N; ++k) vals[k] = line < L ? v[line * N + k] : 0.0f;
    tc::pack_line<N>(a_hi, a_lo, t, vals);
    if (t < 2 * tc::kTileLines - kTcLinesCta)
    {
        float z[N];
#pragma unroll
        for (int k = 0; k < N; ++k) z[k] = 0.0f;
        tc::pack_line<N>(a_hi, a_lo, kTcLinesCta + t, z);
    }
    else if (t >= 64 && t < 80)
        tc::pack_matrix_row<N>(b_hi, b_lo, t - 64, D);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tm = tmem_base;
    if (t == 0)
    {
        const uint32_t ah = tc::smem_u32(a_hi), al = tc::smem_u32(a_lo);
        const uint32_t bh = tc::smem_u32(b_hi), bl = tc::smem_u32(b_lo);
        tc::split_product(tm, 0, ah, al, bh, bl);
        tc::split_product(tm, tc::kCols, ah + tc::kTileBytes, al + tc::kTileBytes, bh, bl);
        tc::mma_commit(&bar);
    }
    const bool ok = tc::mbar_wait(&bar, 0, 1 << 22);
    tc::fence_after_sync();
    float o[8];
    tc::load8(tm, t < tc::kTileLines ? 0 : tc::kCols, o);  // warp-uniform column block
    if (!ok && t == 0) atomicExch(err, 1);
    if (ok && line < L)
    {
#pragma unroll
        for (int k = 0; k < N; ++k) out[line * N + k] = o[k];
    }
    tc::fence_before_sync();
    __syncthreads();
    if (t < 32)
    {
        tc::fence_after_sync();
        tc::tmem_free(tm, 32);
    }
}

cudaError_t launch_tc_lines(int n, const float* v, const double* D, float* out, int64_t L, int* err, cudaStream_t s)
{
    const unsigned grid = unsigned((L + kTcLinesCta - 1) / kTcLinesCta);
    const size_t smem = 4 * tc::kTileBytes + 2 * tc::kBBytes;
    switch (n)
    {
#define FRSDG_TC_CASE(NV)                                                                                          \
    case NV:                                                                                                        \
        tc_lines_kernel<NV><<<grid, kTcLinesCta, smem, s>>>(v, D, out, L, err);                                    \
        break;
        FRSDG_TC_CASE(2)
        FRSDG_TC_CASE(3)
        FRSDG_TC_CASE(4)
        FRSDG_TC_CASE(5)
        FRSDG_TC_CASE(6)
        FRSDG_TC_CASE(7)
        FRSDG_TC_CASE(8)
#undef FRSDG_TC_CASE
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

} // namespace frsdg
